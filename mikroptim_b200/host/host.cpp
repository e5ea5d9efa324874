// C++ host layer over the C ABI (see mikroptim_b200.hpp for the reference classes mirrored).
#include "mikroptim_b200.hpp"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <set>
#include <utility>

#include "gauss_legendre_table.hpp"

namespace mkb {

namespace {

constexpr int kMaxRings = detail::kMaxRings;

int sample_count(int rings, int spokes, PupilMode mode) {
    return mode == PupilMode::Axis ? rings : rings * spokes;
}

}  // namespace

// ---- BatchTopology / SystemBatchHost ---------------------------------------------------------

void BatchTopology::validate() const {
    if (surfaces < 2 || surfaces > MKB_MAX_SURFACES)
        throw std::invalid_argument("BatchTopology: surfaces must be in [2, 64]");
    if (wavelengths < 1 || wavelengths > MKB_MAX_WAVELENGTHS)
        throw std::invalid_argument("BatchTopology: wavelengths must be in [1, 16]");
    if (fields < 1 || fields > MKB_MAX_FIELDS)
        throw std::invalid_argument("BatchTopology: fields must be in [1, 16]");
    if (fields * wavelengths > MKB_MAX_TUPLES)
        throw std::invalid_argument("BatchTopology: fields * wavelengths must be <= 128");
    if (static_cast<int>(type.size()) != surfaces)
        throw std::invalid_argument("BatchTopology: type needs one entry per surface");
    if (type[0] != SurfaceKind::Stop)
        throw std::invalid_argument("BatchTopology: surface 0 must be the stop");
    int plates = 0, stops = 0;
    for (int s = 1; s < surfaces; ++s) {
        if (type[s] == SurfaceKind::GhostPlate) ++plates;
        else if (type[s] == SurfaceKind::ApertureStop) {
            if (++stops > 1 || s > surfaces - 2)
                throw std::invalid_argument("BatchTopology: at most one interior aperture stop, "
                                            "at 1 <= s <= S - 2");
        } else if (type[s] != SurfaceKind::Plane && type[s] != SurfaceKind::Sphere)
            throw std::invalid_argument("BatchTopology: unknown surface kind");
    }
    if (stops > 0 && (non_coaxial || plates > 0))
        throw std::logic_error("BatchTopology: an interior aperture stop is traced in coaxial "
                               "batches without ghost plates");
    if (plates != ghost_plates)
        throw std::invalid_argument("BatchTopology: ghost_plates must equal the number of "
                                    "GhostPlate surfaces");
    if (ghost_plates > MKB_MAX_GHOST_PLATES)
        throw std::logic_error("BatchTopology: too many ghost plates for this build");
    if (ghost_terms < 0 || ghost_terms > MKB_MAX_GHOST_TERMS || (ghost_plates > 0 && ghost_terms < 1))
        throw std::invalid_argument("BatchTopology: ghost_terms out of range");
    if (static_cast<int>(pupil_mode.size()) != fields)
        throw std::invalid_argument("BatchTopology: pupil_mode needs one entry per field");
    if (non_coaxial)
        for (PupilMode m : pupil_mode)
            if (m != PupilMode::Full)
                throw std::invalid_argument("BatchTopology: a non-coaxial batch needs the Full "
                                            "pupil in every field");
}

SystemBatchHost::SystemBatchHost(BatchTopology topology, int variants)
    : topology_(std::move(topology)), variants_(variants) {
    topology_.validate();
    if (variants < 0) throw std::invalid_argument("SystemBatchHost: variants must be >= 0");
    const size_t V = static_cast<size_t>(variants);
    const size_t S = topology_.surfaces, L = topology_.wavelengths, F = topology_.fields;
    type_.resize(S);
    for (size_t s = 0; s < S; ++s) type_[s] = static_cast<uint8_t>(topology_.type[s]);
    wavelength_weight.assign(L, 1.0);
    field_weight.assign(F, 1.0);
    curvature_.assign(V * S, 0.0);
    thickness_.assign(V * S, 0.0);
    index_.assign(V * S * L, 1.0);
    pupil_radius_.assign(V, 0.0);
    field_angle_.assign(V * F, 0.0);
    field_target_.assign(V * F, 0.0);
    if (topology_.non_coaxial) decenter_tilt_.assign(V * S * 4, 0.0);
    const size_t G = topology_.ghost_plates, K = topology_.ghost_terms;
    ghost_coeff_.assign(V * G * K, 0.0);
    ghost_index_.assign(V * G * L, 1.0);
    ghost_norm_radius_.assign(G, 1.0);
    buchdahl_coeff_.assign(V * S * 4, 0.0);
    wavelength_nm.assign(L, 0.0);
}

double& SystemBatchHost::buchdahl_coeff(int v, int s, int j) {
    if (j < 0 || j >= 4) throw std::out_of_range("SystemBatchHost: Buchdahl coefficient");
    return buchdahl_coeff_.at(index2(v, s, surfaces()) * 4 + j);
}

double SystemBatchHost::buchdahl_coeff(int v, int s, int j) const {
    if (j < 0 || j >= 4) throw std::out_of_range("SystemBatchHost: Buchdahl coefficient");
    return buchdahl_coeff_.at(index2(v, s, surfaces()) * 4 + j);
}

void SystemBatchHost::refresh_glass_index(int v, int s) {
    const double* b = buchdahl_coeff_.data() + index2(v, s, surfaces()) * 4;
    for (int l = 0; l < wavelengths(); ++l) {
        const double dl = wavelength_nm.at(static_cast<size_t>(l)) / 1000.0 - 0.546074;
        const double w = dl / (1.0 + 2.5 * dl);
        index(v, s, l) = b[0] + w * (b[1] + w * (b[2] + w * b[3]));
    }
}

double& SystemBatchHost::ghost_coeff(int v, int g, int k) {
    if (g < 0 || g >= topology_.ghost_plates || k < 0 || k >= topology_.ghost_terms)
        throw std::out_of_range("SystemBatchHost: ghost coefficient out of range");
    return ghost_coeff_.at((check_v(v) * topology_.ghost_plates + g) * topology_.ghost_terms + k);
}

double& SystemBatchHost::ghost_index(int v, int g, int l) {
    if (g < 0 || g >= topology_.ghost_plates || l < 0 || l >= wavelengths())
        throw std::out_of_range("SystemBatchHost: ghost index out of range");
    return ghost_index_.at((check_v(v) * topology_.ghost_plates + g) * wavelengths() + l);
}

double& SystemBatchHost::ghost_norm_radius(int g) {
    if (g < 0 || g >= topology_.ghost_plates)
        throw std::out_of_range("SystemBatchHost: ghost plate out of range");
    return ghost_norm_radius_.at(static_cast<size_t>(g));
}

int SystemBatchHost::ghost_surface(int g) const {
    if (g < 0 || g >= topology_.ghost_plates)
        throw std::out_of_range("SystemBatchHost: ghost plate out of range");
    for (int s = 1, n = 0; s < surfaces(); ++s)
        if (topology_.type[s] == SurfaceKind::GhostPlate && n++ == g) return s;
    return -1;
}

double& SystemBatchHost::decenter_tilt(int v, int s, int k) {
    if (!topology_.non_coaxial)
        throw std::invalid_argument("SystemBatchHost: decenter and tilt need a non-coaxial "
                                    "batch (make_non_coaxial)");
    if (k < 0 || k >= 4) throw std::out_of_range("SystemBatchHost: decenter_tilt component");
    return decenter_tilt_.at(index2(v, s, surfaces()) * 4 + k);
}

double SystemBatchHost::decenter_tilt(int v, int s, int k) const {
    if (k < 0 || k >= 4) throw std::out_of_range("SystemBatchHost: decenter_tilt component");
    const size_t i = index2(v, s, surfaces());
    return topology_.non_coaxial ? decenter_tilt_.at(i * 4 + k) : 0.0;
}

void SystemBatchHost::set_decenter_tilt(int v, int s, double dx, double dy, double alpha,
                                        double beta) {
    decenter_tilt(v, s, 0) = dx;
    decenter_tilt(v, s, 1) = dy;
    decenter_tilt(v, s, 2) = alpha;
    decenter_tilt(v, s, 3) = beta;
}

SystemBatchHost take_variants(const SystemBatchHost& batch, const std::vector<int>& variants) {
    SystemBatchHost out(batch.topology(), static_cast<int>(variants.size()));
    out.reference_wavelength_nm = batch.reference_wavelength_nm;
    out.wavelength_weight = batch.wavelength_weight;
    out.field_weight = batch.field_weight;
    out.ghost_norm_radius_ = batch.ghost_norm_radius_;
    auto copy = [&](const std::vector<double>& from, std::vector<double>& to, size_t n) {
        for (size_t j = 0; j < variants.size(); ++j) {
            const size_t i = batch.check_v(variants[j]);
            std::copy(from.begin() + i * n, from.begin() + (i + 1) * n, to.begin() + j * n);
        }
    };
    const size_t S = batch.surfaces(), L = batch.wavelengths(), F = batch.fields();
    const size_t G = batch.topology().ghost_plates, K = batch.topology().ghost_terms;
    copy(batch.curvature_, out.curvature_, S);
    copy(batch.thickness_, out.thickness_, S);
    copy(batch.index_, out.index_, S * L);
    copy(batch.pupil_radius_, out.pupil_radius_, 1);
    copy(batch.field_angle_, out.field_angle_, F);
    copy(batch.field_target_, out.field_target_, F);
    if (!batch.decenter_tilt_.empty()) copy(batch.decenter_tilt_, out.decenter_tilt_, S * 4);
    copy(batch.ghost_coeff_, out.ghost_coeff_, G * K);
    copy(batch.ghost_index_, out.ghost_index_, G * L);
    copy(batch.buchdahl_coeff_, out.buchdahl_coeff_, S * 4);
    out.wavelength_nm = batch.wavelength_nm;
    out.glass = batch.glass;
    return out;
}

SystemBatchHost make_non_coaxial(const SystemBatchHost& batch) {
    BatchTopology t = batch.topology();
    t.non_coaxial = true;
    t.pupil_mode.assign(static_cast<size_t>(t.fields), PupilMode::Full);
    SystemBatchHost out(t, batch.variants());
    out.reference_wavelength_nm = batch.reference_wavelength_nm;
    out.wavelength_weight = batch.wavelength_weight;
    out.field_weight = batch.field_weight;
    out.curvature_ = batch.curvature_;
    out.thickness_ = batch.thickness_;
    out.index_ = batch.index_;
    out.pupil_radius_ = batch.pupil_radius_;
    out.field_angle_ = batch.field_angle_;
    out.field_target_ = batch.field_target_;
    out.ghost_coeff_ = batch.ghost_coeff_;
    out.ghost_index_ = batch.ghost_index_;
    out.ghost_norm_radius_ = batch.ghost_norm_radius_;
    return out;
}

size_t SystemBatchHost::check_v(int v) const {
    if (v < 0 || v >= variants_) throw std::out_of_range("SystemBatchHost: variant out of range");
    return static_cast<size_t>(v);
}

size_t SystemBatchHost::index2(int v, int i, int n) const {
    if (i < 0 || i >= n) throw std::out_of_range("SystemBatchHost: index out of range");
    return check_v(v) * n + i;
}

double& SystemBatchHost::index(int v, int s, int l) {
    if (l < 0 || l >= wavelengths()) throw std::out_of_range("SystemBatchHost: wavelength");
    return index_.at(index2(v, s, surfaces()) * wavelengths() + l);
}

void SystemBatchHost::validate_values() const {
    auto finite = [](const std::vector<double>& a, const char* name) {
        for (double x : a)
            if (!std::isfinite(x))
                throw std::invalid_argument(std::string("SystemBatchHost: ") + name +
                                            " is not finite");
    };
    finite(curvature_, "curvature");
    finite(thickness_, "thickness");
    finite(index_, "index");
    finite(pupil_radius_, "pupil_radius");
    finite(field_angle_, "field_angle");
    finite(field_target_, "field_target");
    finite(wavelength_weight, "wavelength_weight");
    finite(field_weight, "field_weight");
    finite(decenter_tilt_, "decenter_tilt");
    finite(ghost_coeff_, "ghost_coeff");
    for (double x : ghost_index_)
        if (!(x > 0)) throw std::invalid_argument("SystemBatchHost: ghost index must be > 0");
    for (double x : ghost_norm_radius_)
        if (!(x > 0)) throw std::invalid_argument("SystemBatchHost: ghost radius must be > 0");
    for (size_t i = 2; i < decenter_tilt_.size(); i += 4)
        for (size_t k = i; k < i + 2; ++k)
            if (!(std::abs(decenter_tilt_[k]) < 1.5707963267948966))
                throw std::invalid_argument("SystemBatchHost: tilt angles must be in "
                                            "(-pi/2, pi/2)");
    for (double r : pupil_radius_)
        if (!(r > 0)) throw std::invalid_argument("SystemBatchHost: pupil radius must be > 0");
    for (double n : index_)
        if (!(n > 0)) throw std::invalid_argument("SystemBatchHost: refractive indices must be > 0");
    for (double w : wavelength_weight)
        if (w < 0) throw std::invalid_argument("SystemBatchHost: weights must be >= 0");
    for (double w : field_weight)
        if (w < 0) throw std::invalid_argument("SystemBatchHost: weights must be >= 0");
    if (!(reference_wavelength_nm > 0))
        throw std::invalid_argument("SystemBatchHost: reference wavelength must be > 0");
    for (int f = 0; f < fields(); ++f)
        if (topology_.pupil_mode[f] == PupilMode::Axis)
            for (int v = 0; v < variants_; ++v)
                if (field_angle_[static_cast<size_t>(v) * fields() + f] != 0.0)
                    throw std::invalid_argument("SystemBatchHost: an axis field has a non-zero "
                                                "field angle (check_pupil_modes)");
}

mkb_batch_view SystemBatchHost::view() const {
    if (static_cast<int>(wavelength_weight.size()) != wavelengths() ||
        static_cast<int>(field_weight.size()) != fields())
        throw std::invalid_argument("SystemBatchHost: weight arrays do not match the topology");
    mkb_batch_view v{};
    v.variants = variants_;
    v.surfaces = surfaces();
    v.wavelengths = wavelengths();
    v.fields = fields();
    v.reference_wavelength_nm = reference_wavelength_nm;
    v.type = type_.data();
    v.wavelength_weight = wavelength_weight.data();
    v.field_weight = field_weight.data();
    v.curvature = curvature_.data();
    v.thickness = thickness_.data();
    v.index = index_.data();
    v.pupil_radius = pupil_radius_.data();
    v.field_angle = field_angle_.data();
    v.field_target = field_target_.data();
    v.decenter_tilt = topology_.non_coaxial ? decenter_tilt_.data() : nullptr;
    if (glass) {
        if (static_cast<int>(wavelength_nm.size()) != wavelengths())
            throw std::invalid_argument("SystemBatchHost: wavelength_nm does not match");
        v.buchdahl_coeff = buchdahl_coeff_.data();
        v.wavelength_nm = wavelength_nm.data();
    }
    v.ghost_plates = topology_.ghost_plates;
    v.ghost_terms = topology_.ghost_terms;
    if (topology_.ghost_plates > 0) {
        v.ghost_coeff = ghost_coeff_.data();
        v.ghost_norm_radius = ghost_norm_radius_.data();
        v.ghost_index = ghost_index_.data();
    }
    return v;
}

// ---- ResidualLayout ---------------------------------------------------------------------------

ResidualLayout::ResidualLayout(const BatchTopology& topology, const ResidualSettings& settings)
    : topology_(topology), settings_(settings) {
    topology_.validate();
    if (settings.rings < 1 || settings.rings > kMaxRings)
        throw std::invalid_argument("ResidualLayout: rings must be in [1, 32]");
    if (settings.spokes < 1) throw std::invalid_argument("ResidualLayout: spokes must be >= 1");
    for (PupilMode m : topology.pupil_mode)
        if (m != PupilMode::Axis && settings.spokes > MKB_MAX_SPOKES)
            throw std::invalid_argument("ResidualLayout: spokes must be <= 64 in this build");
    if (!(settings.fail_weight >= 0 && std::isfinite(settings.fail_weight)))
        throw std::invalid_argument("ResidualLayout: fail_weight must be finite and >= 0");
    int64_t off = 0;
    for (int f = 0; f < topology.fields; ++f) {
        const int n = sample_count(settings.rings, settings.spokes, topology.pupil_mode[f]);
        samples_.push_back(n);
        field_offset_.push_back(off);
        off += static_cast<int64_t>(topology.wavelengths) * n;
    }
    rays_ = off;
}

int64_t ResidualLayout::trace_rows() const {
    return rays_ * (1 + (settings_.failure == FailureMode::Soft ? 1 : 0) +
                    (settings_.transverse_weight > 0.0 ? 2 : 0));
}

int64_t ResidualLayout::offset(int f, int l) const {
    if (f < 0 || f >= topology_.fields) throw std::out_of_range("ResidualLayout: field");
    if (l < 0 || l >= topology_.wavelengths) throw std::out_of_range("ResidualLayout: wavelength");
    return field_offset_[f] + static_cast<int64_t>(l) * samples_[f];
}

std::unique_ptr<ResidualPlan> ResidualLayout::plan(const SystemBatchHost& batch) const {
    if (batch.fields() != topology_.fields || batch.wavelengths() != topology_.wavelengths)
        throw std::invalid_argument("ResidualLayout: batch does not match the layout");
    return plan_from(batch.field_weight, batch.wavelength_weight, batch.reference_wavelength_nm);
}

std::unique_ptr<ResidualPlan> ResidualLayout::plan_for_sizing() const {
    return plan_from(std::vector<double>(topology_.fields, 1.0),
                     std::vector<double>(topology_.wavelengths, 1.0), 587.56);
}

std::unique_ptr<ResidualPlan> ResidualLayout::plan_from(
    const std::vector<double>& field_weight, const std::vector<double>& wavelength_weight,
    double reference_wavelength_nm) const {
    std::unique_ptr<ResidualPlan> p(new ResidualPlan());
    const int n = settings_.rings;
    for (int i = 0; i < n; ++i) {
        p->u_.push_back(detail::kGaussLegendre[n - 1][2 * i]);
        p->w_.push_back(detail::kGaussLegendre[n - 1][2 * i + 1]);
    }
    for (PupilMode m : topology_.pupil_mode) p->modes_.push_back(static_cast<uint8_t>(m));
    p->field_weight_ = field_weight;
    p->wavelength_weight_ = wavelength_weight;
    mkb_residual_plan& c = p->plan_;
    c.rings = n;
    c.spokes = settings_.spokes;
    c.failure = static_cast<int32_t>(settings_.failure);
    c.precision = static_cast<int32_t>(settings_.precision);
    c.fail_weight = settings_.fail_weight;
    c.transverse_weight = settings_.transverse_weight;
    c.reference_wavelength_nm = reference_wavelength_nm;
    c.fields = topology_.fields;
    c.wavelengths = topology_.wavelengths;
    c.pupil_mode = p->modes_.data();
    c.field_weight = p->field_weight_.data();
    c.wavelength_weight = p->wavelength_weight_.data();
    c.quad_u = p->u_.data();
    c.quad_w = p->w_.data();
    return p;
}

// ---- VariableSet / LmOptions ----------------------------------------------------------------

VariableSet::VariableSet(const BatchTopology& topology, std::vector<Variable> variables)
    : variables_(std::move(variables)) {
    const int S = topology.surfaces;
    if (variables_.size() > MKB_MAX_VARIABLES)
        throw std::invalid_argument("VariableSet: at most 64 variables");
    std::set<std::pair<int, int>> seen;
    for (size_t k = 0; k < variables_.size(); ++k) {
        Variable& v = variables_[k];
        if (v.type == VariableType::Curvature) {
            if (v.surface < 1 || v.surface >= S || topology.type[v.surface] != SurfaceKind::Sphere)
                throw std::invalid_argument("VariableSet: curvature variable needs a sphere");
        } else if (v.type == VariableType::Thickness) {
            if (v.surface < 0 || v.surface >= S - 1)
                throw std::invalid_argument("VariableSet: thickness surface out of range");
            if (v.surface == 0)
                for (int s = 1; s < S; ++s)
                    if (topology.type[s] == SurfaceKind::ApertureStop)
                        throw std::invalid_argument("VariableSet: thickness[0] follows the "
                                                    "interior stop's entrance pupil");
        } else if (v.type == VariableType::WorkingDistance) {
            v.surface = S - 1;
        } else if (v.type == VariableType::Glass) {
            if (v.surface < 0 || v.surface >= S || v.glass_component < 0 || v.glass_component > 2)
                throw std::invalid_argument("VariableSet: glass variable out of range");
        } else if (v.type == VariableType::GhostCoefficient) {
            if (v.ghost_plate < 0 || v.ghost_plate >= topology.ghost_plates ||
                v.ghost_order < 1 || v.ghost_order > topology.ghost_terms)
                throw std::invalid_argument("VariableSet: ghost coefficient out of range");
            for (int s = 1, n = 0; s < S; ++s)
                if (topology.type[s] == SurfaceKind::GhostPlate && n++ == v.ghost_plate)
                    v.surface = s;
        } else {
            throw std::logic_error("VariableSet: variable type not traced by this build");
        }
        const std::pair<int, int> key =
            v.type == VariableType::GhostCoefficient
                ? std::pair<int, int>{2 + v.ghost_plate, v.ghost_order}
            : v.type == VariableType::Glass
                ? std::pair<int, int>{100 + v.surface, v.glass_component}
                : std::pair<int, int>{v.type == VariableType::Curvature ? 1 : 0, v.surface};
        if (!seen.insert(key).second)
            throw std::invalid_argument("VariableSet: parameter already used by a variable");
        if (std::isnan(v.lower) || std::isnan(v.upper) || v.lower > v.upper)
            throw std::invalid_argument("VariableSet: invalid bounds");
        if (!(v.typical > 0 && std::isfinite(v.typical)))
            throw std::invalid_argument("VariableSet: typical size must be > 0");
        type_.push_back(static_cast<int32_t>(v.type));
        surface_.push_back(v.surface);
        ghost_plate_.push_back(v.ghost_plate);
        ghost_order_.push_back(v.ghost_order);
        glass_component_.push_back(v.glass_component);
        lower_.push_back(v.lower);
        upper_.push_back(v.upper);
        typical_.push_back(v.typical);
    }
}

std::vector<double> VariableSet::extract(const SystemBatchHost& batch, int v) const {
    std::vector<double> x;
    for (const Variable& var : variables_)
        x.push_back(var.type == VariableType::Curvature ? batch.curvature(v, var.surface)
                    : var.type == VariableType::Glass
                        ? batch.buchdahl_coeff(v, var.surface, var.glass_component)
                    : var.type == VariableType::GhostCoefficient
                        ? const_cast<SystemBatchHost&>(batch).ghost_coeff(v, var.ghost_plate,
                                                                          var.ghost_order - 1)
                        : batch.thickness(v, var.surface));
    return x;
}

void VariableSet::apply(SystemBatchHost& batch, int v, const double* x) const {
    for (size_t k = 0; k < variables_.size(); ++k) {
        const Variable& var = variables_[k];
        if (var.type == VariableType::Curvature) batch.curvature(v, var.surface) = x[k];
        else if (var.type == VariableType::GhostCoefficient)
            batch.ghost_coeff(v, var.ghost_plate, var.ghost_order - 1) = x[k];
        else if (var.type == VariableType::Glass)
            batch.buchdahl_coeff(v, var.surface, var.glass_component) = x[k];
        else batch.thickness(v, var.surface) = x[k];
    }
    std::set<int> glass_surfaces;
    for (const Variable& var : variables_)
        if (var.type == VariableType::Glass) glass_surfaces.insert(var.surface);
    for (int gs : glass_surfaces) batch.refresh_glass_index(v, gs);
}

mkb_variables VariableSet::c_struct() const {
    mkb_variables c{};
    c.count = size();
    c.type = type_.data();
    c.surface = surface_.data();
    c.lower = lower_.data();
    c.upper = upper_.data();
    c.typical = typical_.data();
    c.ghost_plate = ghost_plate_.data();
    c.ghost_order = ghost_order_.data();
    c.glass_component = glass_component_.data();
    return c;
}

mkb_lm_options LmOptions::c_struct(std::vector<mkb_paraxial_constraint>* storage) const {
    mkb_lm_options o{};
    o.max_iterations = max_iterations;
    o.reject_new_failures = reject_new_failures ? 1 : 0;
    o.ftol = ftol;
    o.xtol = xtol;
    o.gtol = gtol;
    o.initial_damping = initial_damping;
    o.max_damping = max_damping;
    o.diag_floor = diag_floor;
    o.jacobian = static_cast<int32_t>(jacobian);
    o.gram_exact = gram_exact ? 1 : 0;
    if (!paraxial.items.empty()) {
        if (storage == nullptr)
            throw std::invalid_argument("LmOptions: paraxial constraints need a storage vector");
        storage->clear();
        for (const ParaxialConstraint& c : paraxial.items)
            storage->push_back(mkb_paraxial_constraint{c.type, c.mode, c.weight, c.target,
                                                       c.reference_surface, 0, c.offset,
                                                       c.shift});
        o.paraxial_count = static_cast<int32_t>(storage->size());
        o.paraxial = storage->data();
        o.paraxial_column = paraxial.column;
        o.paraxial_derivative = paraxial.analytic ? MKB_PARAXIAL_ADJOINT : MKB_PARAXIAL_FD;
    }
    return o;
}

// ---- cuda ------------------------------------------------------------------------------------
namespace cuda {

void check(int status, const char* what) {
    if (status == MKB_OK) return;
    const std::string msg = std::string(what) + ": " + mkb_last_error();
    if (status == MKB_ERR_ARGUMENT) throw std::invalid_argument(msg);
    if (status == MKB_ERR_UNSUPPORTED) throw std::logic_error(msg);
    throw CudaError(msg);
}

namespace {

void cuda_check(cudaError_t err, const char* what) {
    if (err != cudaSuccess)
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(err));
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

template <class T>
void copy_out(std::vector<T>& dst, const DeviceBuffer& src, size_t count, void* stream) {
    dst.resize(count);
    if (count == 0) return;
    cuda_check(cudaMemcpyAsync(dst.data(), src.get(), count * sizeof(T), cudaMemcpyDeviceToHost,
                               as_stream(stream)),
               "download");
}

template <class T>
void* upload(DeviceBuffer& dst, const std::vector<T>& src, void* stream) {
    void* p = dst.reserve(src.size() * sizeof(T));
    if (!src.empty())
        cuda_check(cudaMemcpyAsync(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice,
                                   as_stream(stream)),
                   "upload");
    return p;
}

}  // namespace

DeviceBuffer::~DeviceBuffer() { release(); }

void* DeviceBuffer::reserve(size_t bytes) {
    if (bytes <= bytes_ && ptr_ != nullptr) return ptr_;
    release();
    if (bytes == 0) return nullptr;
    cuda_check(cudaMalloc(&ptr_, bytes), "cudaMalloc");
    bytes_ = bytes;
    return ptr_;
}

void DeviceBuffer::release() {
    if (ptr_ != nullptr) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
}

void DeviceSystemBatch::upload(const SystemBatchHost& batch, void* stream) {
    upload(batch, 0, batch.variants(), stream);
}

void DeviceSystemBatch::upload(const SystemBatchHost& batch, int first, int count,
                               void* stream) {
    batch.validate_values();
    if (first < 0 || count < 0 || first + count > batch.variants())
        throw std::out_of_range("DeviceSystemBatch: variant range outside the batch");
    mkb_batch_view view = batch.view();
    // the tranche's rows of every per-variant array; the shared arrays stay
    const int S = view.surfaces, L = view.wavelengths, F = view.fields;
    const int G = view.ghost_plates, K = view.ghost_terms;
    const size_t v0 = static_cast<size_t>(first);
    view.variants = count;
    view.curvature += v0 * S;
    view.thickness += v0 * S;
    view.index += v0 * S * L;
    view.pupil_radius += v0;
    view.field_angle += v0 * F;
    view.field_target += v0 * F;
    if (view.decenter_tilt != nullptr) view.decenter_tilt += v0 * S * 4;
    if (view.ghost_coeff != nullptr) view.ghost_coeff += v0 * G * K;
    if (view.ghost_index != nullptr) view.ghost_index += v0 * G * L;
    if (view.buchdahl_coeff != nullptr) view.buchdahl_coeff += v0 * S * 4;
    const int32_t non_coaxial = view.decenter_tilt != nullptr ? 1 : 0;
    const int32_t glass = view.buchdahl_coeff != nullptr ? 1 : 0;
    const int32_t stride = mkb_record_stride_ext(S, L, F, non_coaxial, G, K, glass);
    wavelength_nm_.assign(batch.wavelength_nm.begin(), batch.wavelength_nm.end());
    host_records_.assign(static_cast<size_t>(count) * stride, 0.0);
    check(mkb_pack_batch_host(&view, host_records_.data()), "pack batch");
    void* d = cuda::upload(records_, host_records_, stream);
    type_.assign(view.type, view.type + S);
    batch_ = mkb_device_batch{};
    batch_.variants = count;
    batch_.surfaces = S;
    batch_.wavelengths = L;
    batch_.fields = F;
    batch_.record_stride = stride;
    batch_.non_coaxial = non_coaxial;
    batch_.ghost_plates = G;
    batch_.ghost_terms = K;
    batch_.glass = glass;
    batch_.wavelength_nm = wavelength_nm_.data();
    batch_.records = static_cast<const double*>(d);
    batch_.type = type_.data();
}

const char* to_string(TraceMode mode) {
    return mode == TraceMode::Merit ? "MERIT" : "RESIDUALS";
}

TraceEngine::TraceEngine(int device, const EngineOptions& options)
    : device_(device), options_(options) {
    int count = 0;
    cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (count == 0) throw CudaError("TraceEngine: no CUDA device");
    if (device < 0 || device >= count)
        throw std::invalid_argument("TraceEngine: no such CUDA device");
    (void)usable_bytes(0);  // checks the reserve (std::invalid_argument)
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    device_name_ = prop.name;
    cudaStream_t s;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    stream_ = s;
}

TraceEngine::~TraceEngine() {
    release();
    if (stream_ != nullptr) cudaStreamDestroy(as_stream(stream_));
}

void TraceEngine::release() noexcept {
    batch_.release();
    out_.release();
    opd_.release();
    status_.release();
    merit_.release();
    failed_.release();
    hard_.release();
    workspace_.release();
    extra_.release();
    extrema_.release();
}

std::size_t TraceEngine::device_bytes() const {
    return batch_.capacity_bytes() + out_.bytes() + opd_.bytes() + status_.bytes() +
           merit_.bytes() + failed_.bytes() + hard_.bytes() + workspace_.bytes() +
           extra_.bytes() + extrema_.bytes();
}

void TraceEngine::synchronize() {
    cuda_check(cudaStreamSynchronize(as_stream(stream_)), "synchronize");
    check(mkb_device_status(), "device status");
}

std::size_t TraceEngine::available_bytes() const {
    size_t free_bytes = 0, total = 0;
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
    // the engine's own buffers count as available: a run reuses or frees them
    size_t available = free_bytes + device_bytes();
    if (options_.memory_limit_bytes) available = std::min(available, *options_.memory_limit_bytes);
    return available;
}

std::size_t TraceEngine::usable_bytes(std::size_t available) const {
    size_t usable = 0;
    if (mkb_usable_bytes(available, options_.reserve.min_bytes, options_.reserve.fraction,
                         &usable) != MKB_OK)
        throw std::invalid_argument("TraceEngine: reserve fraction must be in [0, 1]");
    return usable;
}

namespace {

void check_settings(const TraceSettings& settings) {
    if (settings.extra_residuals < 0)
        throw std::invalid_argument("TraceEngine: extra_residuals must be >= 0");
    if (settings.pack_rays < 1) throw std::invalid_argument("TraceEngine: pack_rays must be >= 1");
}

ResidualSettings quadrature_of(const TraceSettings& settings) {
    ResidualSettings q = settings.quadrature;
    if (settings.precision) q.precision = *settings.precision;
    return q;
}

mkb_device_batch shape_of(const BatchTopology& t, bool glass, std::vector<uint8_t>& type) {
    type.clear();
    for (SurfaceKind k : t.type) type.push_back(static_cast<uint8_t>(k));
    mkb_device_batch b{};
    b.surfaces = t.surfaces;
    b.wavelengths = t.wavelengths;
    b.fields = t.fields;
    b.non_coaxial = t.non_coaxial ? 1 : 0;
    b.ghost_plates = t.ghost_plates;
    b.ghost_terms = t.ghost_terms;
    b.glass = glass ? 1 : 0;
    b.record_stride = mkb_record_stride_ext(b.surfaces, b.wavelengths, b.fields, b.non_coaxial,
                                            b.ghost_plates, b.ghost_terms, b.glass);
    b.type = type.data();
    return b;
}

int64_t tranche_for(size_t usable, const mkb_device_batch& shape, const mkb_residual_plan* plan,
                    const TraceSettings& settings, bool merit, int granularity) {
    mkb_trace_options o{};
    o.pack_rays = settings.pack_rays;
    const int64_t n = mkb_trace_tranche_variants(
        usable, &shape, plan, &o, merit ? 1 : 0, settings.extra_residuals, settings.opd ? 1 : 0,
        merit && !settings.extra_merit.empty() ? 1 : 0, granularity);
    if (n < 0) check(static_cast<int>(n), "tranche plan");
    return n;
}

}  // namespace

int TraceEngine::max_variants(const BatchTopology& topology, TraceMode mode,
                              const TraceSettings& settings) const {
    check_settings(settings);
    const ResidualLayout layout(topology, quadrature_of(settings));
    const auto plan = layout.plan_for_sizing();
    std::vector<uint8_t> type;
    const mkb_device_batch shape = shape_of(topology, false, type);
    return static_cast<int>(tranche_for(usable_bytes(available_bytes()), shape, plan->get(),
                                        settings, mode == TraceMode::Merit, 1));
}

TraceEngine::TranchePlan TraceEngine::plan_tranches(const SystemBatchHost& batch, TraceMode mode,
                                                    const ResidualLayout& layout,
                                                    const TraceSettings& settings,
                                                    int granularity) {
    const bool merit = mode == TraceMode::Merit;
    const auto plan = layout.plan(batch);
    std::vector<uint8_t> type;
    const mkb_device_batch shape = shape_of(batch.topology(), batch.glass, type);
    // the other mode's buffers stay while the tranche does not shrink because of them
    const size_t other = merit ? out_.bytes() + opd_.bytes() + status_.bytes()
                               : merit_.bytes() + failed_.bytes() + hard_.bytes() +
                                     workspace_.bytes() + extra_.bytes();
    const size_t available = available_bytes();
    size_t usable = usable_bytes(available - std::min(other, available));
    int64_t tranche = tranche_for(usable, shape, plan->get(), settings, merit, granularity);
    if (other > 0 && tranche < batch.variants()) {
        const size_t usable_all = usable_bytes(available);
        const int64_t tranche_all =
            tranche_for(usable_all, shape, plan->get(), settings, merit, granularity);
        if (tranche_all > tranche) {
            if (merit) {
                out_.release();
                opd_.release();
                status_.release();
            } else {
                merit_.release();
                failed_.release();
                hard_.release();
                workspace_.release();
                extra_.release();
            }
            tranche = tranche_all;
            usable = usable_all;
        }
    }
    if (tranche < 1)
        throw CudaError("TraceEngine: not even " +
                        (granularity == 1 ? std::string("one variant fits")
                                          : std::to_string(granularity) +
                                                " variants that belong together fit") +
                        " into the device memory (available " + std::to_string(available) +
                        " B, after the reserve " + std::to_string(usable) + " B)");
    // buffers that are too small go before the new ones come (old and new never coexist)
    batch_.release();
    return TranchePlan{static_cast<int>(std::min<int64_t>(tranche, batch.variants())), usable};
}

DeviceTranche TraceEngine::residual_tranche(const SystemBatchHost& batch,
                                            const ResidualLayout& layout,
                                            const TraceSettings& settings, int first,
                                            int count) {
    const int64_t rays = layout.rays_per_variant();
    const int64_t stride = layout.trace_rows() + settings.extra_residuals;
    const size_t n = static_cast<size_t>(count);
    batch_.upload(batch, first, count, stream_);
    const mkb_device_batch b = batch_.c_struct();
    const auto plan = layout.plan(batch);
    auto* res = static_cast<double*>(out_.reserve(n * stride * sizeof(double)));
    auto* st = static_cast<uint8_t*>(status_.reserve(n * rays));
    double* opd = settings.opd ? static_cast<double*>(opd_.reserve(n * rays * sizeof(double)))
                               : nullptr;
    if (settings.extra_residuals > 0)
        cuda_check(cudaMemsetAsync(res, 0, n * stride * sizeof(double), as_stream(stream_)),
                   "clear residuals");
    mkb_trace_options o{};
    o.pack_rays = settings.pack_rays;
    o.variants_per_cta = settings.variants_per_cta;
    if (settings.extrema)
        o.extrema = static_cast<double*>(
            extrema_.reserve(n * static_cast<size_t>(batch.surfaces()) * 2 * sizeof(double)));
    check(mkb_residuals_ex_device(&b, plan->get(), &o, res, stride, opd, st, stream_),
          "residuals");
    synchronize();
    DeviceTranche t;
    t.first = first;
    t.count = count;
    t.rays_per_variant = rays;
    t.penalty_rows = settings.quadrature.failure == FailureMode::Soft ? rays : 0;
    t.stride = stride;
    t.residuals = res;
    t.status = st;
    t.opd = opd;
    return t;
}

TraceOutput TraceEngine::run(const SystemBatchHost& batch, TraceMode mode,
                             const TraceSettings& settings) {
    TraceOutput out;
    run(batch, mode, settings, out);
    return out;
}

void TraceEngine::run(const SystemBatchHost& batch, TraceMode mode,
                      const TraceSettings& settings, TraceOutput& out) {
    check_settings(settings);
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    const ResidualLayout layout(batch.topology(), quadrature_of(settings));
    batch.validate_values();
    const int V = batch.variants();
    const bool merit_mode = mode == TraceMode::Merit;
    if (merit_mode && !settings.extra_merit.empty() &&
        settings.extra_merit.size() != static_cast<size_t>(V))
        throw std::invalid_argument("TraceEngine: extra_merit must be empty or hold " +
                                    std::to_string(V) + " values");
    const int64_t rays = layout.rays_per_variant();
    const int64_t stride = layout.trace_rows() + settings.extra_residuals;
    const size_t rays_total = static_cast<size_t>(V) * rays;
    const size_t S2 = static_cast<size_t>(batch.surfaces()) * 2;
    out.mode = mode;
    out.info = TraceRunInfo{};
    out.info.variants = V;
    out.residuals = ResidualResult{};
    out.merit = MeritResult{};
    if (merit_mode) {
        out.merit.variants = V;
        out.merit.rays_per_variant = rays;
        out.merit.merit.resize(V);
        out.merit.failed.resize(V);
        out.merit.hard_failed.resize(V);
        if (settings.extrema) out.merit.extrema.resize(static_cast<size_t>(V) * S2);
    } else {
        out.residuals.variants = V;
        out.residuals.rays_per_variant = rays;
        out.residuals.penalty_rows = settings.quadrature.failure == FailureMode::Soft ? rays : 0;
        out.residuals.stride = stride;
        out.residuals.residuals.resize(static_cast<size_t>(V) * stride);
        out.residuals.opd.resize(settings.opd ? rays_total : 0);
        out.residuals.status.resize(settings.status ? rays_total : 0);
        if (settings.extrema) out.residuals.extrema.resize(static_cast<size_t>(V) * S2);
    }
    out.layout.emplace(layout);
    if (V == 0) {
        out.info.device_bytes = device_bytes();
        return;
    }
    const TranchePlan tp = plan_tranches(batch, mode, layout, settings, 1);
    const auto plan = layout.plan(batch);
    for (int first = 0; first < V; first += tp.tranche) {
        const int count = std::min(tp.tranche, V - first);
        const size_t v0 = static_cast<size_t>(first), n = static_cast<size_t>(count);
        auto down = [&](void* dst, const void* src, size_t bytes) {
            if (bytes > 0)
                cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost,
                                           as_stream(stream_)),
                           "download");
        };
        if (merit_mode) {
            batch_.upload(batch, first, count, stream_);
            const mkb_device_batch b = batch_.c_struct();
            workspace_.reserve(mkb_merit_workspace_bytes(count, plan->get()));
            auto* m = static_cast<double*>(merit_.reserve(n * sizeof(double)));
            auto* f = static_cast<int64_t*>(failed_.reserve(n * sizeof(int64_t)));
            auto* h = static_cast<int64_t*>(hard_.reserve(n * sizeof(int64_t)));
            mkb_trace_options o{};
            o.pack_rays = settings.pack_rays;
            o.variants_per_cta = settings.variants_per_cta;
            if (settings.extrema)
                o.extrema = static_cast<double*>(extrema_.reserve(
                    n * static_cast<size_t>(batch.surfaces()) * 2 * sizeof(double)));
            if (!settings.extra_merit.empty()) {
                void* e = extra_.reserve(n * sizeof(double));
                cuda_check(cudaMemcpyAsync(e, settings.extra_merit.data() + v0,
                                           n * sizeof(double), cudaMemcpyHostToDevice,
                                           as_stream(stream_)),
                           "upload extra_merit");
                o.extra_merit = static_cast<const double*>(e);
            }
            check(mkb_merit_ex_device(&b, plan->get(), &o, m, f, h, workspace_.get(),
                                      workspace_.bytes(), stream_),
                  "merit");
            down(out.merit.merit.data() + v0, m, n * sizeof(double));
            down(out.merit.failed.data() + v0, f, n * sizeof(int64_t));
            down(out.merit.hard_failed.data() + v0, h, n * sizeof(int64_t));
            if (settings.extrema)
                down(out.merit.extrema.data() + v0 * S2, extrema_.get(), n * S2 * sizeof(double));
            synchronize();
        } else {
            const DeviceTranche t = residual_tranche(batch, layout, settings, first, count);
            down(out.residuals.residuals.data() + v0 * stride, t.residuals,
                 n * stride * sizeof(double));
            if (settings.status)
                down(out.residuals.status.data() + v0 * rays, t.status, n * rays);
            if (settings.opd)
                down(out.residuals.opd.data() + v0 * rays, t.opd, n * rays * sizeof(double));
            if (settings.extrema)
                down(out.residuals.extrema.data() + v0 * S2, extrema_.get(),
                     n * S2 * sizeof(double));
            synchronize();
        }
        ++out.info.tranches;
    }
    out.info.tranche_variants = tp.tranche;
    out.info.budget_bytes = tp.usable;
    out.info.device_bytes = device_bytes();
}

TraceRunInfo TraceEngine::run_on_device(const SystemBatchHost& batch,
                                        const TraceSettings& settings, int granularity,
                                        const DeviceTrancheFn& consume) {
    check_settings(settings);
    if (granularity < 1) throw std::invalid_argument("TraceEngine: granularity must be >= 1");
    if (!consume) throw std::invalid_argument("TraceEngine: run_on_device without a callback");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    const ResidualLayout layout(batch.topology(), quadrature_of(settings));
    batch.validate_values();
    TraceRunInfo info;
    info.variants = batch.variants();
    if (info.variants == 0) {
        info.device_bytes = device_bytes();
        return info;
    }
    const TranchePlan tp =
        plan_tranches(batch, TraceMode::Residuals, layout, settings, granularity);
    for (int first = 0; first < info.variants; first += tp.tranche) {
        const int count = std::min(tp.tranche, info.variants - first);
        consume(residual_tranche(batch, layout, settings, first, count));
        cuda_check(cudaDeviceSynchronize(), "tranche callback");
        ++info.tranches;
    }
    info.tranche_variants = tp.tranche;
    info.budget_bytes = tp.usable;
    info.device_bytes = device_bytes();
    return info;
}

namespace {

int runs_of(const VariableSet& variables, const SystemBatchHost& base,
            const std::vector<double>& x0) {
    const int P = variables.size();
    if (P < 1) throw std::invalid_argument("variables: at least one variable");
    if (x0.size() % P != 0) throw std::invalid_argument("x0: size is not a multiple of P");
    const int runs = static_cast<int>(x0.size() / P);
    if (base.variants() != 1 && base.variants() != runs)
        throw std::invalid_argument("base batch must hold 1 variant or one per run");
    return runs;
}

}  // namespace

void DeviceFdJacobian::compute(TraceEngine& engine, const VariableSet& variables,
                               const SystemBatchHost& base, const std::vector<double>& x0,
                               const ResidualSettings& settings, JacobianResult& out) {
    cuda_check(cudaSetDevice(engine.device()), "cudaSetDevice");
    const int runs = runs_of(variables, base, x0);
    const int P = variables.size();
    const ResidualLayout layout(base.topology(), settings);
    const auto plan = layout.plan(base);
    templates_.upload(base, engine.stream());
    const mkb_device_batch t = templates_.c_struct();
    const mkb_variables v = variables.c_struct();
    const int64_t R = layout.trace_rows();
    const auto* x = static_cast<const double*>(upload(x0_, x0, engine.stream()));
    auto* J = static_cast<double*>(J_.reserve(sizeof(double) * runs * P * R));
    auto* r0 = static_cast<double*>(r0_.reserve(sizeof(double) * runs * R));
    const int chunk = runs < 64 ? runs : 64;
    const size_t ws = mkb_fd_jacobian_workspace_bytes(&t, plan->get(), P, runs, chunk);
    if (ws == 0) check(MKB_ERR_ARGUMENT, "fd jacobian workspace");
    workspace_.reserve(ws);
    check(mkb_fd_jacobian_device(&t, plan->get(), &v, x, runs, J, r0, nullptr, workspace_.get(),
                                 workspace_.bytes(), engine.stream()),
          "fd jacobian");
    out.runs = runs;
    out.P = P;
    out.rows = R;
    copy_out(out.J, J_, static_cast<size_t>(runs) * P * R, engine.stream());
    copy_out(out.r0, r0_, static_cast<size_t>(runs) * R, engine.stream());
    engine.synchronize();
}

void DeviceAdjointJacobian::compute(TraceEngine& engine, const VariableSet& variables,
                                    const SystemBatchHost& base, const std::vector<double>& x0,
                                    const ResidualSettings& settings, JacobianResult& out) {
    cuda_check(cudaSetDevice(engine.device()), "cudaSetDevice");
    const int runs = runs_of(variables, base, x0);
    const int P = variables.size();
    const ResidualLayout layout(base.topology(), settings);
    const auto plan = layout.plan(base);
    templates_.upload(base, engine.stream());
    const mkb_device_batch t = templates_.c_struct();
    const mkb_variables v = variables.c_struct();
    const int64_t R = layout.trace_rows();
    const auto* x = static_cast<const double*>(upload(x0_, x0, engine.stream()));
    auto* J = static_cast<double*>(J_.reserve(sizeof(double) * runs * P * R));
    auto* r0 = static_cast<double*>(r0_.reserve(sizeof(double) * runs * R));
    auto* st = static_cast<uint8_t*>(status_.reserve(static_cast<size_t>(runs) *
                                                     layout.rays_per_variant()));
    workspace_.reserve(mkb_adjoint_jacobian_workspace_bytes(&t, runs));
    check(mkb_adjoint_jacobian_device(&t, plan->get(), &v, x, runs, J, r0, st, workspace_.get(),
                                      workspace_.bytes(), engine.stream()),
          "adjoint jacobian");
    out.runs = runs;
    out.P = P;
    out.rows = R;
    copy_out(out.J, J_, static_cast<size_t>(runs) * P * R, engine.stream());
    copy_out(out.r0, r0_, static_cast<size_t>(runs) * R, engine.stream());
    engine.synchronize();
}

void DeviceNormalEquations::compute(TraceEngine& engine, const JacobianResult& jac, bool exact) {
    cuda_check(cudaSetDevice(engine.device()), "cudaSetDevice");
    if (jac.J.size() != static_cast<size_t>(jac.runs) * jac.P * jac.rows ||
        jac.r0.size() != static_cast<size_t>(jac.runs) * jac.rows)
        throw std::invalid_argument("normal equations: J / r0 sizes do not match");
    const auto* J = static_cast<const double*>(upload(J_, jac.J, engine.stream()));
    const auto* r = static_cast<const double*>(upload(r_, jac.r0, engine.stream()));
    const size_t n = static_cast<size_t>(jac.P) + 1;
    auto* g = static_cast<double*>(dgram_.reserve(sizeof(double) * jac.runs * n * n));
    check(mkb_normal_equations_device(J, r, jac.runs, jac.P, jac.rows, g, exact ? 1 : 0,
                                      engine.stream()),
          "normal equations");
    copy_out(gram_, dgram_, jac.runs * n * n, engine.stream());
    engine.synchronize();
    runs_ = jac.runs;
    P_ = jac.P;
}

void DeviceNormalEquations::download(std::vector<double>& a, std::vector<double>& g) const {
    const size_t P = P_, n = P + 1;
    a.assign(static_cast<size_t>(runs_) * P * P, 0.0);
    g.assign(static_cast<size_t>(runs_) * P, 0.0);
    for (size_t run = 0; run < static_cast<size_t>(runs_); ++run) {
        const double* G = gram_.data() + run * n * n;
        for (size_t q = 0; q < P; ++q) {
            for (size_t p = 0; p < P; ++p) a[run * P * P + q * P + p] = G[q * n + p];
            g[run * P + q] = G[q * n + P];
        }
    }
}

namespace {

// One LM pass of every run on the device.
// sum_e r_e^2 of run i at x (extra_merit_values, src/optim/levenberg_marquardt.cpp:659)
double extra_merit_at(const VariableSet& variables, SystemBatchHost& one,
                      const ExtraResiduals& extra, const double* x) {
    variables.apply(one, 0, x);
    std::vector<double> r(static_cast<size_t>(extra.count));
    extra.evaluate(one, 0, r);
    double s = 0.0;
    for (double e : r) s += e * e;
    return s;
}

SystemBatchHost run_template(const SystemBatchHost& base, int i) {
    return take_variants(base, {base.variants() == 1 ? 0 : i});
}

// The trace-dependent rows at the points (run i_j, y_j): one MERIT trace with extrema of all of
// them; values [points][Et].
std::vector<double> trace_rows_at(TraceEngine& engine, const VariableSet& variables,
                                  const SystemBatchHost& base, const ResidualSettings& settings,
                                  const TraceExtraResiduals& te, const std::vector<int>& runs,
                                  const std::vector<double>& ys) {
    const int P = variables.size(), n = static_cast<int>(runs.size()), Et = te.count;
    std::vector<int> tmpl;
    for (int i : runs) tmpl.push_back(base.variants() == 1 ? 0 : i);
    SystemBatchHost multi = take_variants(base, tmpl);
    for (int j = 0; j < n; ++j) variables.apply(multi, j, ys.data() + static_cast<size_t>(j) * P);
    TraceSettings ts(settings);
    ts.extrema = true;
    const TraceOutput out = engine.run(multi, TraceMode::Merit, ts);
    const size_t S2 = static_cast<size_t>(multi.surfaces()) * 2;
    std::vector<double> vals(static_cast<size_t>(n) * Et);
    for (int j = 0; j < n; ++j)
        te.evaluate(multi, j, std::span<const double>(out.merit.extrema.data() + j * S2, S2),
                    std::span<double>(vals.data() + static_cast<size_t>(j) * Et, Et));
    return vals;
}

double sum_squares(const double* v, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += v[i] * v[i];
    return s;
}

LmResult lm_pass(TraceEngine& engine, const VariableSet& variables, const SystemBatchHost& base,
                 const std::vector<double>& x0, const LmOptions& options,
                 const ResidualSettings& settings, LmGpuStats* stats) {
    cuda_check(cudaSetDevice(engine.device()), "cudaSetDevice");
    const int runs = runs_of(variables, base, x0);
    const int P = variables.size();
    for (int r = 0; r < runs; ++r)  // the reference rejects start values outside the bounds
        for (int k = 0; k < P; ++k) {
            const double x = x0[static_cast<size_t>(r) * P + k];
            const Variable& v = variables.variables()[k];
            if (!(x >= v.lower && x <= v.upper))
                throw std::invalid_argument("optimize_lm_gpu: start value of variable " +
                                            std::to_string(k) + " of run " +
                                            std::to_string(r) + " outside its bounds");
        }
    const ResidualLayout layout(base.topology(), settings);
    const auto plan = layout.plan(base);
    DeviceSystemBatch templates;
    templates.upload(base, engine.stream());
    const mkb_device_batch t = templates.c_struct();
    const mkb_variables v = variables.c_struct();
    std::vector<mkb_paraxial_constraint> paraxial_storage;
    const mkb_lm_options o = options.c_struct(&paraxial_storage);
    DeviceBuffer dx0, ws;
    const auto* x = static_cast<const double*>(upload(dx0, x0, engine.stream()));
    const size_t bytes = mkb_lm_workspace_bytes(&t, plan->get(), &v, &o, runs);
    if (bytes == 0) check(MKB_ERR_ARGUMENT, "lm workspace");
    ws.reserve(bytes);
    const int E0 = options.extra.count, Et = options.trace_extra.count, E = E0 + Et;
    if (E0 < 0 || (E0 > 0 && !options.extra.evaluate) || Et < 0 ||
        (Et > 0 && !options.trace_extra.evaluate))
        throw std::invalid_argument("optimize_lm_gpu: extra rows need a count >= 0 and a function");
    DeviceBuffer dtrace;
    std::vector<SystemBatchHost> work;  // one-variant working copies of the run templates
    DeviceBuffer dextra, dje, dre;
    std::vector<double> em(static_cast<size_t>(runs), 0.0);
    if (E > 0) {
        for (int i = 0; i < runs; ++i) work.push_back(run_template(base, i));
        if (E0 > 0)
            for (int i = 0; i < runs; ++i)
                em[i] = extra_merit_at(variables, work[i], options.extra,
                                       x0.data() + static_cast<size_t>(i) * P);
        upload(dextra, em, engine.stream());
    }
    if (Et > 0) {
        std::vector<int> all(static_cast<size_t>(runs));
        for (int i = 0; i < runs; ++i) all[i] = i;
        const std::vector<double> vals =
            trace_rows_at(engine, variables, base, settings, options.trace_extra, all, x0);
        std::vector<double> tm(static_cast<size_t>(runs));
        for (int i = 0; i < runs; ++i) tm[i] = sum_squares(vals.data() + static_cast<size_t>(i) * Et, Et);
        upload(dtrace, tm, engine.stream());
    }
    check(mkb_lm_start_ex_device(&t, plan->get(), &v, &o, x,
                                 E0 > 0 ? static_cast<const double*>(dextra.get()) : nullptr,
                                 Et > 0 ? static_cast<const double*>(dtrace.get()) : nullptr,
                                 runs, ws.get(), ws.bytes(), engine.stream()),
          "lm start");
    int32_t running = runs;
    int cycles = 0;
    while (running > 0 && cycles <= options.max_iterations) {
        if (E == 0) {
            check(mkb_lm_cycle_device(&t, plan->get(), &v, &o, runs, ws.get(), ws.bytes(),
                                      engine.stream()),
                  "lm cycle");
        } else {
            // phases: trace-row normal equations, the caller's rows at the points that got
            // them, step, trial merit with the extra merit at the trial points, acceptance
            check(mkb_lm_cycle_jacobian_device(&t, plan->get(), &v, &o, runs, ws.get(),
                                               ws.bytes(), engine.stream()),
                  "lm cycle (Jacobian)");
            std::vector<int32_t> flags(static_cast<size_t>(runs));
            std::vector<double> pts(static_cast<size_t>(runs) * P);
            check(mkb_lm_points_device(&t, plan->get(), &v, &o, runs, ws.get(), flags.data(),
                                       pts.data(), nullptr, nullptr, engine.stream()),
                  "lm points");
            engine.synchronize();
            std::vector<double> je(static_cast<size_t>(runs) * P * E, 0.0),
                re(static_cast<size_t>(runs) * E, 0.0);
            for (int i = 0; i < runs; ++i) {
                if (!flags[i]) continue;
                std::vector<double> xi(pts.begin() + static_cast<ptrdiff_t>(i) * P,
                                       pts.begin() + static_cast<ptrdiff_t>(i + 1) * P);
                double* Ji = je.data() + static_cast<size_t>(i) * P * E;
                double* ri = re.data() + static_cast<size_t>(i) * E;
                if (E0 > 0) {
                    std::vector<double> J1, r1;
                    extra_rows_host(variables, work[i], xi, options.extra, J1, r1);
                    for (int k = 0; k < P; ++k)
                        for (int e = 0; e < E0; ++e) Ji[k * E + e] = J1[k * E0 + e];
                    for (int e = 0; e < E0; ++e) ri[e] = r1[e];
                }
                if (Et > 0) {  // FD points of run i traced with their extrema
                    std::vector<double> xp(P), xm(P), dp(P), dm(P);
                    std::vector<int32_t> st(P);
                    const mkb_variables vc = variables.c_struct();
                    check(mkb_fd_pattern_host(&vc, xi.data(), 1, xp.data(), xm.data(), dp.data(),
                                              dm.data(), st.data()),
                          "fd pattern");
                    std::vector<int> who(static_cast<size_t>(2 * P + 1), i);
                    std::vector<double> ys;
                    ys.insert(ys.end(), xi.begin(), xi.end());
                    for (int k = 0; k < P; ++k)
                        for (double val : {xp[k], xm[k]}) {
                            std::vector<double> y = xi;
                            y[k] = val;
                            ys.insert(ys.end(), y.begin(), y.end());
                        }
                    const std::vector<double> vals = trace_rows_at(
                        engine, variables, base, settings, options.trace_extra, who, ys);
                    std::vector<double> col(static_cast<size_t>(Et));
                    for (int k = 0; k < P; ++k) {
                        check(mkb_fd_derivative_host(
                                  st[k], dp[k], dm[k], Et, vals.data(),
                                  vals.data() + static_cast<size_t>(1 + 2 * k) * Et,
                                  vals.data() + static_cast<size_t>(2 + 2 * k) * Et, col.data()),
                              "fd derivative");
                        for (int e = 0; e < Et; ++e) Ji[k * E + E0 + e] = col[e];
                    }
                    for (int e = 0; e < Et; ++e) ri[E0 + e] = vals[e];
                }
            }
            const auto* dj = static_cast<const double*>(upload(dje, je, engine.stream()));
            const auto* dr = static_cast<const double*>(upload(dre, re, engine.stream()));
            check(mkb_lm_extra_rows_device(&t, plan->get(), &v, &o, runs, ws.get(), ws.bytes(),
                                           dj, dr, E, engine.stream()),
                  "lm extra rows");
            check(mkb_lm_cycle_step_device(&t, plan->get(), &v, &o, runs, ws.get(), ws.bytes(),
                                           engine.stream()),
                  "lm cycle (step)");
            check(mkb_lm_points_device(&t, plan->get(), &v, &o, runs, ws.get(), nullptr, nullptr,
                                       flags.data(), pts.data(), engine.stream()),
                  "lm points");
            engine.synchronize();
            for (int i = 0; i < runs; ++i)
                em[i] = flags[i] && E0 > 0
                            ? extra_merit_at(variables, work[i], options.extra,
                                             pts.data() + static_cast<size_t>(i) * P)
                            : 0.0;
            const auto* de = static_cast<const double*>(upload(dextra, em, engine.stream()));
            if (Et == 0) {
                check(mkb_lm_cycle_accept_device(&t, plan->get(), &v, &o, runs, ws.get(),
                                                 ws.bytes(), de, engine.stream()),
                      "lm cycle (acceptance)");
            } else {  // trial MERIT, then the trial points' extrema rows, then acceptance
                check(mkb_lm_cycle_trial_device(&t, plan->get(), &v, &o, runs, ws.get(),
                                                ws.bytes(), de, nullptr, engine.stream()),
                      "lm cycle (trial merit)");
                std::vector<int> who;
                std::vector<double> ys;
                for (int i = 0; i < runs; ++i)
                    if (flags[i]) {
                        who.push_back(i);
                        ys.insert(ys.end(), pts.begin() + static_cast<ptrdiff_t>(i) * P,
                                  pts.begin() + static_cast<ptrdiff_t>(i + 1) * P);
                    }
                std::vector<double> tm(static_cast<size_t>(runs), 0.0);
                if (!who.empty()) {
                    const std::vector<double> vals = trace_rows_at(
                        engine, variables, base, settings, options.trace_extra, who, ys);
                    for (size_t j = 0; j < who.size(); ++j)
                        tm[who[j]] = sum_squares(vals.data() + j * Et, Et);
                }
                const auto* dt = static_cast<const double*>(upload(dtrace, tm, engine.stream()));
                check(mkb_lm_cycle_decide_device(&t, plan->get(), &v, &o, runs, ws.get(),
                                                 ws.bytes(), dt, engine.stream()),
                      "lm cycle (acceptance)");
            }
        }
        ++cycles;
        check(mkb_lm_results_device(&t, plan->get(), &v, &o, runs, ws.get(), nullptr, nullptr,
                                    nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    nullptr, &running, engine.stream()),
              "lm results");
        engine.synchronize();
    }
    LmResult r;
    const size_t R = static_cast<size_t>(runs), H = static_cast<size_t>(options.max_iterations) + 1;
    r.x.resize(R * P);
    r.merit.resize(R);
    r.damping.resize(R);
    r.history.resize(R * H);
    r.status.resize(R);
    r.iterations.resize(R);
    r.accepted.resize(R);
    r.jacobians.resize(R);
    r.failed.resize(R);
    r.hard_failed.resize(R);
    check(mkb_lm_results_device(&t, plan->get(), &v, &o, runs, ws.get(), r.x.data(),
                                r.merit.data(), r.status.data(), r.iterations.data(),
                                r.accepted.data(), r.jacobians.data(), r.damping.data(),
                                r.history.data(), r.failed.data(), r.hard_failed.data(), nullptr,
                                engine.stream()),
          "lm results");
    engine.synchronize();
    r.history_width = static_cast<int>(H);
    r.fail_weight.assign(R, settings.fail_weight);
    r.penalty_rounds.assign(R, 1);
    if (stats != nullptr) stats->cycles += cycles;
    return r;
}

}  // namespace

void extra_rows_host(const VariableSet& variables, const SystemBatchHost& base,
                     const std::vector<double>& x0, const ExtraResiduals& extra,
                     std::vector<double>& jacobian, std::vector<double>& residuals) {
    const int P = variables.size(), E = extra.count;
    const int runs = runs_of(variables, base, x0);
    if (E < 0 || (E > 0 && !extra.evaluate))
        throw std::invalid_argument("extra rows: count >= 0 and an evaluate function needed");
    jacobian.assign(static_cast<size_t>(runs) * P * E, 0.0);
    residuals.assign(static_cast<size_t>(runs) * E, 0.0);
    const mkb_variables vc = variables.c_struct();
    std::vector<double> xp(P), xm(P), dp(P), dm(P), y(P), r0(E), ra(E), rb(E), col(E);
    std::vector<int32_t> st(P);
    for (int i = 0; i < runs; ++i) {
        SystemBatchHost one = run_template(base, i);
        const double* x = x0.data() + static_cast<size_t>(i) * P;
        check(mkb_fd_pattern_host(&vc, x, 1, xp.data(), xm.data(), dp.data(), dm.data(),
                                  st.data()),
              "fd pattern");
        auto evaluate = [&](std::vector<double>& out) {
            variables.apply(one, 0, y.data());
            extra.evaluate(one, 0, out);
        };
        y.assign(x, x + P);
        evaluate(r0);
        std::copy(r0.begin(), r0.end(), residuals.begin() + static_cast<ptrdiff_t>(i) * E);
        for (int k = 0; k < P; ++k) {
            y[k] = xp[k];
            evaluate(ra);
            y[k] = xm[k];
            evaluate(rb);
            y[k] = x[k];
            check(mkb_fd_derivative_host(st[k], dp[k], dm[k], E, r0.data(), ra.data(), rb.data(),
                                         col.data()),
                  "fd derivative");
            std::copy(col.begin(), col.end(),
                      jacobian.begin() + (static_cast<ptrdiff_t>(i) * P + k) * E);
        }
    }
}

PrefilterResult TraceEngine::prefilter_variants(const SystemBatchHost& batch,
                                                const PrefilterSettings& settings) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    batch.validate_values();
    const ResidualLayout layout(batch.topology(), settings.quadrature);
    const auto plan = layout.plan(batch);
    const int V = batch.variants();
    const mkb_prefilter_options o{settings.options.criteria.max_failed_fraction,
                                  settings.options.criteria.max_merit,
                                  settings.options.criteria.max_merit_factor,
                                  settings.options.margins.boundary,
                                  settings.options.margins.opl_error_factor,
                                  settings.options.margins.merit_relative};
    if (!settings.extra_merit.empty() && settings.extra_merit.size() != static_cast<size_t>(V))
        throw std::invalid_argument("prefilter: extra_merit must be empty or hold one value per "
                                    "variant");
    PrefilterResult r;
    PrefilterStats& st = r.stats;
    st.variants = V;
    st.rays_per_variant = layout.rays_per_variant();
    const size_t n = static_cast<size_t>(V);
    st.merit.assign(n, 0.0);
    st.optical_length.assign(n, 0.0);
    st.failed.assign(n, 0);
    st.uncertain_ok.assign(n, 0);
    st.uncertain_failed.assign(n, 0);
    if (V > 0) {
        batch_.upload(batch, stream_);
        const mkb_device_batch b = batch_.c_struct();
        const mkb_batch_view view = batch.view();
        std::vector<float> trig(n * static_cast<size_t>(batch.fields()) * 2);
        check(mkb_prefilter_field_trig_host(&view, trig.data()), "prefilter field table");
        DeviceBuffer dtrig, dout, ws;
        void* t = dtrig.reserve(trig.size() * sizeof(float));
        cuda_check(cudaMemcpyAsync(t, trig.data(), trig.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream_)),
                   "prefilter upload");
        char* out = static_cast<char*>(dout.reserve(5 * n * 8));
        void* w = ws.reserve(mkb_prefilter_workspace_bytes(V, plan->get()));
        check(mkb_prefilter_device(&b, plan->get(), static_cast<const float*>(t),
                                   o.boundary, reinterpret_cast<double*>(out),
                                   reinterpret_cast<double*>(out + 8 * n),
                                   reinterpret_cast<int64_t*>(out + 16 * n),
                                   reinterpret_cast<int64_t*>(out + 24 * n),
                                   reinterpret_cast<int64_t*>(out + 32 * n), w, ws.bytes(),
                                   stream_),
              "prefilter");
        void* dst[5] = {st.merit.data(), st.optical_length.data(), st.failed.data(),
                        st.uncertain_ok.data(), st.uncertain_failed.data()};
        for (int k = 0; k < 5; ++k)
            cuda_check(cudaMemcpyAsync(dst[k], out + k * 8 * n, 8 * n, cudaMemcpyDeviceToHost,
                                       static_cast<cudaStream_t>(stream_)),
                       "prefilter download");
        synchronize();
    }
    r.merit_lower.assign(n, 0.0);
    r.merit_upper.assign(n, 0.0);
    r.reject.assign(n, 0);
    int32_t ref_v = -1, kept = 0;
    check(mkb_prefilter_decide_host(plan->get(), &o, V, st.merit.data(), st.optical_length.data(),
                                    st.failed.data(), st.uncertain_ok.data(),
                                    st.uncertain_failed.data(),
                                    settings.extra_merit.empty() ? nullptr
                                                                 : settings.extra_merit.data(),
                                    r.merit_lower.data(), r.merit_upper.data(), r.reject.data(),
                                    &r.reference_merit, &ref_v, &kept),
          "prefilter decide");
    r.reference_variant = ref_v;
    r.kept = kept;
    return r;
}

EvalResult TraceEngine::evaluate(const SystemBatchHost& batch, const EvalSettings& settings) {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    batch.validate_values();
    if (settings.half_pupil && !batch.coaxial())
        throw std::invalid_argument("EVAL: half pupil only for coaxial systems");
    EvalResult r;
    r.variants = batch.variants();
    r.fields = batch.fields();
    r.wavelengths = batch.wavelengths();
    r.grid_size = settings.grid;
    r.half_pupil = settings.half_pupil;
    r.field_ray_offset = settings.field_ray_offset;
    int64_t n = 0;
    check(mkb_eval_grid_host(settings.grid, settings.half_pupil ? 1 : 0, nullptr, &n),
          "eval grid");
    r.samples = n;
    r.grid.resize(static_cast<size_t>(3 * n));
    check(mkb_eval_grid_host(settings.grid, settings.half_pupil ? 1 : 0, r.grid.data(), &n),
          "eval grid");
    const size_t V = static_cast<size_t>(r.variants), F = static_cast<size_t>(r.fields);
    r.reference_curvature.assign(V * F, 0.0);
    r.exit_pupil_position.assign(V, 0.0);
    const mkb_batch_view view = batch.view();
    check(mkb_eval_reference_host(&view, static_cast<int32_t>(settings.reference),
                                  settings.paraxial_column, r.reference_curvature.data(),
                                  r.exit_pupil_position.data()),
          "eval reference");
    const size_t T = V * F * static_cast<size_t>(r.wavelengths);
    const size_t rays = T * static_cast<size_t>(n);
    r.opd.resize(rays);
    r.spot_x.resize(rays);
    r.spot_y.resize(rays);
    r.status.resize(rays);
    r.field_rays.resize(T * 20);
    r.field_status.resize(T * 4);
    if (V == 0) return r;
    batch_.upload(batch, stream_);
    const mkb_device_batch b = batch_.c_struct();
    const cudaStream_t s = static_cast<cudaStream_t>(stream_);
    DeviceBuffer dgrid, dkappa, dout, ws;
    void* g = dgrid.reserve(r.grid.size() * sizeof(double));
    void* k = dkappa.reserve(r.reference_curvature.size() * sizeof(double));
    cuda_check(cudaMemcpyAsync(g, r.grid.data(), r.grid.size() * sizeof(double),
                               cudaMemcpyHostToDevice, s), "eval upload");
    cuda_check(cudaMemcpyAsync(k, r.reference_curvature.data(),
                               r.reference_curvature.size() * sizeof(double),
                               cudaMemcpyHostToDevice, s), "eval upload");
    char* out = static_cast<char*>(dout.reserve(rays * 25 + T * 164 + 64));
    double* opd = reinterpret_cast<double*>(out);
    double* sx = opd + rays;
    double* sy = sx + rays;
    double* fr = sy + rays;
    uint8_t* st = reinterpret_cast<uint8_t*>(fr + T * 20);
    uint8_t* fs = st + rays;
    void* w = ws.reserve(mkb_eval_workspace_bytes(&b));
    check(mkb_eval_device(&b, static_cast<int32_t>(settings.reference),
                          settings.field_ray_offset, static_cast<int32_t>(settings.precision),
                          static_cast<const double*>(g), n, static_cast<const double*>(k), opd,
                          sx, sy, st, fr, fs, w, ws.bytes(), stream_),
          "eval");
    struct Copy {
        void* dst;
        const void* src;
        size_t bytes;
    } copies[] = {{r.opd.data(), opd, rays * 8},         {r.spot_x.data(), sx, rays * 8},
                  {r.spot_y.data(), sy, rays * 8},       {r.status.data(), st, rays},
                  {r.field_rays.data(), fr, T * 160},    {r.field_status.data(), fs, T * 4}};
    for (const Copy& c : copies)
        cuda_check(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, s),
                   "eval download");
    synchronize();
    return r;
}

LmResult optimize_lm_gpu(TraceEngine& engine, const VariableSet& variables,
                         const SystemBatchHost& base, const std::vector<double>& x0,
                         const LmOptions& options, const ResidualSettings& settings,
                         LmGpuStats* stats) {
    if (stats != nullptr) stats->cycles = 0;
    LmResult r = lm_pass(engine, variables, base, x0, options, settings, stats);
    const int P = variables.size();
    const size_t R = r.merit.size();
    // the merit history of every round, joined per run
    std::vector<std::vector<double>> hist(R);
    auto add_history = [](std::vector<double>& to, const double* h, int width) {
        for (int k = 0; k < width && !std::isnan(h[k]); ++k) to.push_back(h[k]);
    };
    for (size_t i = 0; i < R; ++i)
        add_history(hist[i], r.history.data() + i * r.history_width, r.history_width);
    double weight = settings.fail_weight;
    if (settings.failure == FailureMode::Soft && options.fail_weight_factor > 1.0 &&
        weight > 0.0) {
        for (;;) {
            weight *= options.fail_weight_factor;
            if (!(weight <= options.max_fail_weight)) break;
            std::vector<int> again;
            std::vector<double> xs;
            for (size_t i = 0; i < R; ++i)
                if (r.failed[i] > 0 && r.status[i] != static_cast<int32_t>(LmStatus::NumericalError)) {
                    again.push_back(static_cast<int>(i));
                    xs.insert(xs.end(), r.x.begin() + i * P, r.x.begin() + (i + 1) * P);
                }
            if (again.empty()) break;
            ResidualSettings round = settings;
            round.fail_weight = weight;
            const LmResult q = base.variants() == 1
                                   ? lm_pass(engine, variables, base, xs, options, round, stats)
                                   : lm_pass(engine, variables, take_variants(base, again), xs,
                                             options, round, stats);
            for (size_t j = 0; j < again.size(); ++j) {
                const size_t i = static_cast<size_t>(again[j]);
                std::copy(q.x.begin() + j * P, q.x.begin() + (j + 1) * P, r.x.begin() + i * P);
                r.merit[i] = q.merit[j];
                r.failed[i] = q.failed[j];
                r.hard_failed[i] = q.hard_failed[j];
                r.status[i] = q.status[j];
                r.damping[i] = q.damping[j];
                r.iterations[i] += q.iterations[j];
                r.accepted[i] += q.accepted[j];
                r.jacobians[i] += q.jacobians[j];
                add_history(hist[i], q.history.data() + j * q.history_width, q.history_width);
                r.fail_weight[i] = weight;
                ++r.penalty_rounds[i];
            }
        }
    }
    size_t width = static_cast<size_t>(r.history_width);
    for (const auto& h : hist) width = std::max(width, h.size());
    r.history.assign(R * width, std::numeric_limits<double>::quiet_NaN());
    for (size_t i = 0; i < R; ++i) std::copy(hist[i].begin(), hist[i].end(), r.history.begin() + i * width);
    r.history_width = static_cast<int>(width);
    return r;
}


// ---- scalar PSF and MTF ---------------------------------------------------------------------

int psf_fft_size(int grid, double padding) {
    int32_t m = 0;
    check(mkb_psf_fft_size_host(grid, padding, &m), "psf_fft_size");
    return m;
}

namespace {

// column i and row j of grid point k (x = (2i + 1 - N) / N) and the points of the full pupil
void grid_cells(const EvalResult& r, std::vector<int32_t>& col, std::vector<int32_t>& row,
                int& full) {
    const int n = r.grid_size;
    if (n < 1) throw std::invalid_argument("PSF: the EVAL result carries no grid edge");
    col.resize(static_cast<size_t>(r.samples));
    row.resize(static_cast<size_t>(r.samples));
    for (int64_t k = 0; k < r.samples; ++k) {
        col[static_cast<size_t>(k)] =
            static_cast<int32_t>(std::lround((r.grid[3 * k] * n + n - 1) / 2.0));
        row[static_cast<size_t>(k)] =
            static_cast<int32_t>(std::lround((r.grid[3 * k + 1] * n + n - 1) / 2.0));
    }
    full = 0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int64_t a = 2 * i + 1 - n, b = 2 * j + 1 - n;
            full += a * a + b * b <= int64_t(n) * n ? 1 : 0;
        }
}

}  // namespace

std::vector<double> eval_opd_map(const EvalResult& r, int v, int f, int l) {
    if (v < 0 || v >= r.variants || f < 0 || f >= r.fields || l < 0 || l >= r.wavelengths)
        throw std::out_of_range("EVAL: tuple does not exist");
    std::vector<int32_t> col, row;
    int full = 0;
    grid_cells(r, col, row, full);
    const size_t n = static_cast<size_t>(r.grid_size);
    std::vector<double> map(n * n, std::numeric_limits<double>::quiet_NaN());
    const size_t t = (static_cast<size_t>(v) * r.fields + f) * r.wavelengths + l;
    const size_t k0 = t * static_cast<size_t>(r.samples);
    for (int64_t k = 0; k < r.samples; ++k) {
        if (r.status[k0 + k] != MKB_STATUS_OK) continue;
        const size_t c = static_cast<size_t>(col[k]), j = static_cast<size_t>(row[k]);
        map[j * n + c] = r.opd[k0 + k];
        if (r.half_pupil) map[j * n + (n - 1 - c)] = r.opd[k0 + k];
    }
    return map;
}

PsfPupil make_psf_pupil(const SystemBatchHost& batch, const EvalResult& r, int v, int f, int l,
                        const PsfSettings& settings) {
    if (!(settings.padding >= 2.0) || !std::isfinite(settings.padding))
        throw std::invalid_argument("PSF: zero-padding factor must be >= 2");
    if (batch.variants() != r.variants || batch.fields() != r.fields ||
        batch.wavelengths() != r.wavelengths)
        throw std::invalid_argument("PSF: batch does not match the EVAL result");
    PsfPupil p;
    p.field = f;
    p.wavelength = l;
    p.grid = r.grid_size;
    p.opd = eval_opd_map(r, v, f, l);
    std::vector<int32_t> col, row;
    grid_cells(r, col, row, p.full_count);
    p.wavelength_nm = batch.wavelength_nm.at(static_cast<size_t>(l));
    const mkb_batch_view view = batch.view();
    const int S = batch.surfaces(), L = batch.wavelengths();
    const double n_image = view.index[(static_cast<size_t>(v) * S + S - 1) * L + l];
    const size_t t = (static_cast<size_t>(v) * r.fields + f) * r.wavelengths + l;
    int32_t fx = 0, fy = 0;
    check(mkb_psf_aperture_host(r.field_rays.data() + 20 * t, r.field_status.data() + 4 * t,
                                      n_image, r.field_ray_offset, settings.numerical_aperture,
                                      &p.na_x, &p.na_y, &fx, &fy),
                "psf aperture");
    p.flip_x = fx != 0;
    p.flip_y = fy != 0;
    return p;
}

std::vector<PsfPupil> make_psf_pupils(const SystemBatchHost& batch, const EvalResult& r, int v,
                                      const PsfSettings& settings) {
    std::vector<PsfPupil> out;
    for (int f = 0; f < r.fields; ++f)
        for (int l = 0; l < r.wavelengths; ++l)
            out.push_back(make_psf_pupil(batch, r, v, f, l, settings));
    return out;
}

PsfEngine::PsfEngine(int device, const EngineOptions& options)
    : device_(device), options_(options) {
    int count = 0;
    cuda_check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (count == 0) throw CudaError("PsfEngine: no CUDA device");
    if (device < 0 || device >= count) throw std::invalid_argument("PsfEngine: no such device");
    size_t usable = 0;
    if (mkb_usable_bytes(0, options_.reserve.min_bytes, options_.reserve.fraction, &usable) !=
        MKB_OK)
        throw std::invalid_argument("PsfEngine: reserve fraction must be in [0, 1]");
}

size_t PsfEngine::device_bytes() const {
    return maps_.bytes() + params_.bytes() + psf_.bytes() + mtf_.bytes() + work_.bytes();
}

void PsfEngine::release() {
    maps_.release();
    params_.release();
    psf_.release();
    mtf_.release();
    work_.release();
}

std::vector<PsfResult> PsfEngine::compute(const SystemBatchHost& batch, const EvalResult& result,
                                          int v, const PsfSettings& settings) {
    const std::vector<PsfPupil> pupils = make_psf_pupils(batch, result, v, settings);
    return compute(pupils, psf_fft_size(result.grid_size, settings.padding));
}

std::vector<PsfResult> PsfEngine::compute(std::span<const PsfPupil> pupils, int fft_size) {
    std::vector<PsfResult> out;
    info_ = PsfRunInfo{};
    info_.pupils = static_cast<int>(pupils.size());
    for (const PsfPupil& p : pupils) {  // every check before any device work
        if (p.grid != pupils.front().grid)
            throw std::invalid_argument("PsfEngine: every pupil needs the same grid edge");
        if (fft_size < 2 * p.grid || fft_size > MKB_MAX_PSF_FFT || (fft_size & (fft_size - 1)))
            throw std::invalid_argument("PSF: FFT size must be a power of two in [2N, 8192]");
        if (p.opd.size() != static_cast<size_t>(p.grid) * p.grid || p.full_count < 1 ||
            !(p.wavelength_nm > 0.0) || !(p.na_x > 0.0) || !(p.na_y > 0.0))
            throw std::invalid_argument("PSF: incomplete pupil");
        PsfResult r;
        r.field = p.field;
        r.wavelength = p.wavelength;
        r.grid = p.grid;
        r.fft_size = fft_size;
        r.wavelength_nm = p.wavelength_nm;
        r.na_x = p.na_x;
        r.na_y = p.na_y;
        out.push_back(std::move(r));
    }
    if (pupils.empty()) return out;
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    const int n = pupils.front().grid, m = fft_size, count = static_cast<int>(pupils.size());
    const size_t n2 = static_cast<size_t>(n) * n, m2 = static_cast<size_t>(m) * m;
    const size_t per_mtf = 2 * (static_cast<size_t>(n) + 1);
    auto tranche_bytes = [&](int t) {
        return static_cast<size_t>(t) * (n2 * 8 + sizeof(mkb_psf_pupil_params) + m2 * 8 +
                                         per_mtf * 8) +
               mkb_psf_workspace_bytes(t, n, m);
    };
    size_t free_bytes = 0, total = 0;
    cuda_check(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
    size_t available = free_bytes + device_bytes();
    if (options_.memory_limit_bytes) available = std::min(available, *options_.memory_limit_bytes);
    size_t usable = 0;
    check(mkb_usable_bytes(available, options_.reserve.min_bytes, options_.reserve.fraction,
                           &usable),
          "psf reserve");
    int tranche = count;
    while (tranche >= 1 && tranche_bytes(tranche) > usable)
        tranche = tranche > 1 ? std::max(1, tranche * 3 / 4) : 0;
    if (tranche < 1) throw CudaError("PsfEngine: not one pupil fits the device memory");
    auto* maps = static_cast<double*>(maps_.reserve(tranche * n2 * 8));
    auto* params = static_cast<mkb_psf_pupil_params*>(
        params_.reserve(tranche * sizeof(mkb_psf_pupil_params)));
    auto* psf = static_cast<double*>(psf_.reserve(tranche * m2 * 8));
    auto* mtf = static_cast<double*>(mtf_.reserve(tranche * per_mtf * 8));
    const size_t wbytes = mkb_psf_workspace_bytes(tranche, n, m);
    void* work = work_.reserve(wbytes);
    std::vector<double> stage(static_cast<size_t>(tranche) * n2), mtf_h(tranche * per_mtf);
    std::vector<mkb_psf_pupil_params> ph(static_cast<size_t>(tranche));
    for (int first = 0; first < count; first += tranche) {
        const int used = std::min(tranche, count - first);
        for (int t = 0; t < used; ++t) {
            const PsfPupil& p = pupils[static_cast<size_t>(first + t)];
            std::copy(p.opd.begin(), p.opd.end(), stage.begin() + t * n2);
            const double full = static_cast<double>(p.full_count);
            ph[t] = {p.wavelength_mm(), 1.0 / (full * full), p.flip_x ? -1 : 1,
                     p.flip_y ? -1 : 1};
        }
        cuda_check(cudaMemcpy(maps, stage.data(), used * n2 * 8, cudaMemcpyHostToDevice),
                   "psf upload");
        cuda_check(cudaMemcpy(params, ph.data(), used * sizeof(mkb_psf_pupil_params),
                              cudaMemcpyHostToDevice),
                   "psf upload");
        check(mkb_psf_device(used, n, m, maps, params, psf, mtf, work, wbytes, nullptr), "psf");
        cuda_check(cudaDeviceSynchronize(), "psf");
        cuda_check(cudaMemcpy(mtf_h.data(), mtf, used * per_mtf * 8, cudaMemcpyDeviceToHost),
                   "psf download");
        for (int t = 0; t < used; ++t) {
            PsfResult& r = out[static_cast<size_t>(first + t)];
            const PsfPupil& p = pupils[static_cast<size_t>(first + t)];
            r.psf.resize(m2);
            cuda_check(cudaMemcpy(r.psf.data(), psf + t * m2, m2 * 8, cudaMemcpyDeviceToHost),
                       "psf download");
            const double* mt = mtf_h.data() + t * per_mtf;
            r.mtf_sagittal.assign(mt, mt + n + 1);
            r.mtf_tangential.assign(mt + n + 1, mt + 2 * (n + 1));
            mkb_psf_metrics q{};
            check(mkb_psf_finish_host(n, m, p.opd.data(), p.full_count, p.wavelength_nm, p.na_x,
                                      p.na_y, p.flip_x ? 1 : 0, p.flip_y ? 1 : 0, r.psf.data(),
                                      &q),
                  "psf finish");
            r.transmitted = q.transmitted;
            r.energy = q.energy;
            r.strehl_fft = q.strehl_fft;
            r.strehl_origin = q.strehl_origin;
            r.strehl = q.strehl;
            r.reference_x = q.reference_x;
            r.reference_y = q.reference_y;
            r.peak = q.peak;
            r.peak_x = q.peak_x;
            r.peak_y = q.peak_y;
            r.dx = q.dx;
            r.dy = q.dy;
            r.airy_radius = q.airy_radius;
        }
        ++info_.tranches;
    }
    info_.tranche = tranche;
    info_.work_bytes = wbytes;
    info_.device_bytes = device_bytes();
    info_.budget_bytes = usable;
    return out;
}

}  // namespace cuda
}  // namespace mkb
