// Test infrastructure (the oracle), not product code.
//
// C-ABI driver around the reference's own CPU implementation of the trace-and-optimise path,
// compiled from the reference sources where they lie (oracle/Makefile) into
// oracle/_ref/libmko_ref.so. It turns the flat mkb_batch_view / mkb_residual_plan /
// mkb_variables structs of include/mikroptim_b200.h into the reference's SystemBatchHost,
// ResidualLayout and VariableSet and calls:
//   residuals_cpu          src/batch/batch_residuals.cpp:272
//   merit_cpu              src/batch/batch_merit.cpp:61
//   fd_jacobian_cpu        src/optim/fd_jacobian.cpp:182
//   adjoint_jacobian_cpu   src/optim/adjoint_jacobian.cpp:370
//   normal_equations_host  include/mikroptim/optim/normal_equations.hpp:33
//   optimize_lm_cpu        src/optim/levenberg_marquardt.cpp:972
//   paraxial_residuals     src/optim/paraxial_residuals.cpp:353 (extra residual rows)
//   prefilter_stats_cpu, prefilter_decide, prefilter_decide_exact, prefilter_rays_cpu
//                          src/batch/batch_prefilter.cpp (FP32 multistart prefilter)
//   eval_cpu               src/eval/eval.cpp:307 (EVAL on the dense pupil grid)
//   make_psf_pupils, psf_cpu, finish_psf
//                          src/eval/psf.cpp:196,330,290 (scalar PSF and MTF, own radix-2 FFT)
// Only tests/, the golden-fixture script and bench.py's CPU legs load this library.

#include "mikroptim_b200.h"

#include "mikroptim/batch/batch_extrema.hpp"
#include "mikroptim/batch/batch_merit.hpp"
#include "mikroptim/batch/batch_prefilter.hpp"
#include "mikroptim/eval/eval.hpp"
#include "mikroptim/eval/psf.hpp"
#include "mikroptim/batch/batch_residuals.hpp"
#include "mikroptim/batch/system_batch.hpp"
#include "mikroptim/model/system.hpp"
#include "mikroptim/optim/adjoint_jacobian.hpp"
#include "mikroptim/optim/fd_jacobian.hpp"
#include "mikroptim/optim/levenberg_marquardt.hpp"
#include "mikroptim/optim/normal_equations.hpp"
#include "mikroptim/optim/paraxial_residuals.hpp"
#include "mikroptim/optim/trace_extra_residuals.hpp"
#include "mikroptim/optim/variable_set.hpp"
#include "optim/parallel_variants.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <limits>
#include <string>
#include <vector>

namespace {

thread_local std::string g_error;

int fail(const std::exception& e) {
    g_error = e.what();
    return -1;
}

mko::BatchTopology topology_of_view(const mkb_batch_view& v, const mkb_residual_plan& plan) {
    mko::BatchTopology t;
    t.surfaces = v.surfaces;
    t.wavelengths = v.wavelengths;
    t.fields = v.fields;
    t.ghost_plates = v.ghost_plates;
    t.ghost_terms = v.ghost_terms;
    t.non_coaxial = v.decenter_tilt != nullptr;
    t.source = mko::SourceKind::Collimated;
    for (int s = 0; s < v.surfaces; ++s) {
        t.type.push_back(static_cast<mko::SurfaceKind>(v.type[s]));
    }
    for (int f = 0; f < v.fields; ++f) {
        t.pupil_mode.push_back(static_cast<mko::PupilMode>(plan.pupil_mode[f]));
    }
    return t;
}

mko::SystemBatchHost batch_of_view(const mkb_batch_view& v, const mkb_residual_plan& plan) {
    mko::SystemBatchHost b(topology_of_view(v, plan), v.variants);
    const int S = v.surfaces, L = v.wavelengths, F = v.fields;
    b.reference_wavelength_nm = v.reference_wavelength_nm;
    for (int l = 0; l < L; ++l) {
        b.wavelength_weight(l) = v.wavelength_weight[l];
        // the trace reads the indices directly; the wavelengths matter to EVAL's PSF only
        b.wavelength_nm(l) = v.wavelength_nm != nullptr ? v.wavelength_nm[l] : 500.0 + l;
    }
    for (int f = 0; f < F; ++f) {
        b.field_weight(f) = v.field_weight[f];
    }
    for (int i = 0; i < v.variants; ++i) {
        for (int s = 0; s < S; ++s) {
            b.curvature(i, s) = v.curvature[i * S + s];
            b.thickness(i, s) = v.thickness[i * S + s];
            for (int l = 0; l < L; ++l) {
                b.index(i, s, l) = v.index[(static_cast<std::size_t>(i) * S + s) * L + l];
            }
            b.paraxial_index(i, s) = v.index[(static_cast<std::size_t>(i) * S + s) * L];
        }
        b.pupil_radius(i) = v.pupil_radius[i];
        for (int f = 0; f < F; ++f) {
            b.field_angle(i, f) = v.field_angle[i * F + f];
            b.field_target(i, f) = v.field_target[i * F + f];
        }
        for (int g = 0; g < v.ghost_plates; ++g) {
            for (int k = 0; k < v.ghost_terms; ++k)
                b.ghost_coeff(i, g, k) =
                    v.ghost_coeff[(static_cast<std::size_t>(i) * v.ghost_plates + g) *
                                      v.ghost_terms + k];
            for (int l = 0; l < L; ++l)
                b.ghost_index(i, g, l) =
                    v.ghost_index[(static_cast<std::size_t>(i) * v.ghost_plates + g) * L + l];
            // the plate's paraxial glass index: column 0, like paraxial_index
            b.paraxial_ghost_index(i, g) =
                v.ghost_index[(static_cast<std::size_t>(i) * v.ghost_plates + g) * L];
        }
        if (v.decenter_tilt != nullptr)
            for (int s = 0; s < S; ++s)
                for (int k = 0; k < 4; ++k)
                    b.decenter_tilt(i, s, k) =
                        v.decenter_tilt[(static_cast<std::size_t>(i) * S + s) * 4 + k];
    }
    for (int g = 0; g < v.ghost_plates; ++g) b.ghost_norm_radius(g) = v.ghost_norm_radius[g];
    if (v.buchdahl_coeff != nullptr) {
        for (int l = 0; l < L; ++l) b.wavelength_nm(l) = v.wavelength_nm[l];
        for (int i = 0; i < v.variants; ++i)
            for (int s = 0; s < S; ++s)
                for (int j = 0; j < 4; ++j)
                    b.buchdahl_coeff(i, s, j) =
                        v.buchdahl_coeff[(static_cast<std::size_t>(i) * S + s) * 4 + j];
    }
    return b;
}

mko::ResidualSettings settings_of(const mkb_residual_plan& plan) {
    mko::ResidualSettings s;
    s.rings = plan.rings;
    s.spokes = plan.spokes;
    s.failure = plan.failure == MKB_FAILURE_HARD ? mko::FailureMode::Hard : mko::FailureMode::Soft;
    s.fail_weight = plan.fail_weight;
    return s;
}

// A file-model description whose surfaces match the batch (variant 0 values), with one
// variable item per entry of `vars`. Only used to build the reference VariableSet.
mko::SystemDescription description_of(const mko::SystemBatchHost& b, const mkb_variables& vars,
                                       const double* x0) {
    mko::SystemDescription d;
    d.name = "oracle";
    d.spectrum.reference_nm = b.reference_wavelength_nm;
    for (int l = 0; l < b.wavelengths(); ++l) {
        d.spectrum.wavelengths_nm.push_back(b.wavelength_nm(l));
        d.spectrum.weights.push_back(b.wavelength_weight(l));
    }
    d.source.type = mko::SourceType::Collimated;
    for (int f = 0; f < b.fields(); ++f) {
        d.source.field_angles_deg.push_back(b.field_angle(0, f) * 180.0 / M_PI);
        d.source.field_weights.push_back(b.field_weight(f));
    }
    // file surfaces are the table's non-ghost surfaces; a gap with ghost plates is one file
    // thickness (the sum of its table pieces), each plate at its distance from the gap's
    // first vertex (make_surface_map, src/model/system.cpp:361)
    const int S = b.surfaces();
    std::vector<int> file_of_table(static_cast<std::size_t>(S), -1);
    std::vector<int> plate_of_table(static_cast<std::size_t>(S), -1);
    int files = 0, plates = 0;
    for (int s = 0; s < S; ++s) {
        if (b.type(s) == mko::SurfaceKind::GhostPlate) plate_of_table[s] = plates++;
        else file_of_table[s] = files++;
    }
    for (int s = 0; s < S; ++s) {
        if (file_of_table[s] < 0) continue;
        mko::Surface surf;
        const auto kind = b.type(s);
        surf.type = kind == mko::SurfaceKind::Stop    ? mko::SurfaceType::Stop
                    : kind == mko::SurfaceKind::Plane ? mko::SurfaceType::Plane
                                                      : mko::SurfaceType::Sphere;
        surf.curvature = b.curvature(0, s);
        double gap = b.thickness(0, s);
        for (int q = s + 1; q < S && plate_of_table[q] >= 0; ++q) {
            mko::GhostPlate gp;
            gp.after_surface = file_of_table[s];
            gp.distance = gap;
            gp.glass.kind = mko::MaterialKind::Constant;
            gp.glass.n = b.ghost_index(0, plate_of_table[q], 0);
            gp.norm_radius = b.ghost_norm_radius(plate_of_table[q]);
            for (int k = 0; k < b.ghost_terms(); ++k)
                gp.coefficients.push_back(b.ghost_coeff(0, plate_of_table[q], k));
            d.ghost_plates.push_back(gp);
            gap += b.thickness(0, q);
        }
        surf.thickness = gap;
        const double n = b.index(0, s, 0);
        bool glass_var = false;
        for (int k = 0; k < vars.count; ++k)
            glass_var = glass_var || (vars.type[k] == MKB_VAR_GLASS && vars.surface[k] == s);
        if (glass_var) {  // Buchdahl glass (the material of a glass variable)
            surf.material.kind = mko::MaterialKind::Buchdahl;
            surf.material.n0 = b.buchdahl_coeff(0, s, 0);
            for (int j = 0; j < 3; ++j) surf.material.nu[j] = b.buchdahl_coeff(0, s, j + 1);
        } else if (n == 1.0) {
            surf.material.kind = mko::MaterialKind::Air;
        } else {
            surf.material.kind = mko::MaterialKind::Constant;
            surf.material.n = n;
        }
        surf.semi_diameter = s == 0 ? b.pupil_radius(0) : 100.0;
        d.surfaces.push_back(surf);
    }
    // start values of the description = x0 of run 0 (resolve_variables checks the bounds);
    // variables of this driver sit on gaps without plates, so table and file values agree
    mko::Variables items;
    for (int k = 0; k < vars.count; ++k) {
        mko::VariableSpec spec;
        const int s = vars.surface[k];
        if (vars.type[k] == MKB_VAR_CURVATURE) {
            spec.type = mko::VariableType::Curvature;
            spec.selection = mko::SurfaceSelection::One;
            spec.surfaces = {file_of_table[s]};
            d.surfaces[file_of_table[s]].curvature = x0[k];
        } else if (vars.type[k] == MKB_VAR_THICKNESS) {
            spec.type = mko::VariableType::Thickness;
            spec.selection = mko::SurfaceSelection::One;
            spec.surfaces = {file_of_table[s]};
            d.surfaces[file_of_table[s]].thickness = x0[k];
        } else if (vars.type[k] == MKB_VAR_GLASS) {
            // one item for the three components n0, nu1, nu2 (listed in that order, no bounds,
            // the reference's typical sizes)
            if (vars.glass_component[k] != 0) continue;
            spec.type = mko::VariableType::Glass;
            spec.selection = mko::SurfaceSelection::One;
            spec.surfaces = {file_of_table[s]};
            auto& mat = d.surfaces[file_of_table[s]].material;
            mat.n0 = x0[k];
            mat.nu[0] = x0[k + 1];
            mat.nu[1] = x0[k + 2];
            items.items.push_back(spec);
            continue;
        } else if (vars.type[k] == MKB_VAR_GHOST_COEFFICIENT) {
            spec.type = mko::VariableType::GhostCoefficient;
            spec.selection = mko::SurfaceSelection::None;
            spec.plate_selection = mko::SurfaceSelection::One;
            spec.plates = {vars.ghost_plate[k]};
            spec.order_selection = mko::SurfaceSelection::One;
            spec.orders = {vars.ghost_order[k]};
            d.ghost_plates[static_cast<std::size_t>(vars.ghost_plate[k])]
                .coefficients[static_cast<std::size_t>(vars.ghost_order[k] - 1)] = x0[k];
        } else {
            spec.type = mko::VariableType::WorkingDistance;
            spec.selection = mko::SurfaceSelection::None;
            d.surfaces[static_cast<std::size_t>(files - 1)].thickness = x0[k];
        }
        if (std::isfinite(vars.lower[k])) {
            spec.min = vars.lower[k];
        }
        if (std::isfinite(vars.upper[k])) {
            spec.max = vars.upper[k];
        }
        spec.typical = vars.typical[k];
        items.items.push_back(spec);
    }
    d.variables = items;
    return d;
}

// Paraxial constraints from flat arrays: type (ConstraintType order: 0 FocalLength,
// 1 ParfocalLength, 2 WorkingDistance, 3 ParaxialFocus, 4 Petzval), mode (0 Equal, 1 Min,
// 2 Max), weight, target.
mko::ParaxialConstraints constraints_of(int n, const int32_t* type, const int32_t* mode,
                                        const double* weight, const double* target) {
    mko::ParaxialConstraints c;
    for (int i = 0; i < n; ++i) {
        mko::ParaxialConstraint k;
        k.type = static_cast<mko::ConstraintType>(type[i]);
        k.mode = static_cast<mko::ConstraintMode>(mode[i]);
        k.weight = weight[i];
        k.target = target[i];
        c.items.push_back(k);
    }
    return c;
}

} // namespace

extern "C" {

const char* mko_ref_last_error(void) {
    return g_error.c_str();
}

int64_t mko_ref_rays_per_variant(const mkb_batch_view* view, const mkb_residual_plan* plan) {
    try {
        const mko::ResidualLayout layout(topology_of_view(*view, *plan), settings_of(*plan));
        return layout.rays_per_variant();
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// residuals [V][trace_rows], opd [V][rays], status [V][rays]; variants split over `threads`
// host threads with the reference's own parallel_for_variants.
int mko_ref_residuals(const mkb_batch_view* view, const mkb_residual_plan* plan, double* residuals,
                      double* opd, uint8_t* status, int threads) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::ResidualLayout layout(b.topology(), settings_of(*plan));
        const std::int64_t rows = layout.trace_rows();
        const std::int64_t rays = layout.rays_per_variant();
        mko::detail::parallel_for_variants(0, b.variants(), threads, [&](int v) {
            const mko::ResidualResult r = mko::residuals_cpu(b, v, layout);
            std::memcpy(residuals + v * rows, r.residuals.data(), sizeof(double) * rows);
            if (opd != nullptr) {
                std::memcpy(opd + v * rays, r.opd.data(), sizeof(double) * rays);
            }
            if (status != nullptr) {
                std::memcpy(status + v * rays, r.status.data(), rays);
            }
        });
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int mko_ref_merit(const mkb_batch_view* view, const mkb_residual_plan* plan, double* merit,
                  int64_t* failed, int64_t* hard_failed, int threads) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::ResidualLayout layout(b.topology(), settings_of(*plan));
        mko::detail::parallel_for_variants(0, b.variants(), threads, [&](int v) {
            const mko::MeritResult r = mko::merit_cpu(b, v, layout, false);
            merit[v] = r.merit[0];
            failed[v] = r.failed[0];
            hard_failed[v] = r.hard_failed[0];
        });
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// surface_extrema_cpu (src/batch/batch_extrema.cpp, hard maxima): out [V][S][2].
int mko_ref_surface_extrema(const mkb_batch_view* view, const mkb_residual_plan* plan,
                            double* out) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::ResidualLayout layout(b.topology(), settings_of(*plan));
        const mko::SurfaceExtremaResult r = mko::surface_extrema_cpu(b, layout);
        std::memcpy(out, r.values.data(), sizeof(double) * r.values.size());
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// FP32 prefilter, the reference's CPU path: per-variant raw results (prefilter_stats_cpu) and
// the decision (prefilter_decide) with the criteria and margins of `o`; extra [V] or null.
// Outputs [V]: merit, optical_length, failed, uncertain_ok, uncertain_failed, lower, upper,
// reject; reference merit / variant and kept count.
int mko_ref_prefilter(const mkb_batch_view* view, const mkb_residual_plan* plan,
                      const mkb_prefilter_options* o, const double* extra, double* merit,
                      double* optical_length, int64_t* failed, int64_t* uncertain_ok,
                      int64_t* uncertain_failed, double* lower, double* upper, uint8_t* reject,
                      double* reference_merit, int32_t* reference_variant, int32_t* kept) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::ResidualLayout layout(b.topology(), settings_of(*plan));
        mko::PrefilterOptions opt;
        opt.criteria.max_failed_fraction = o->max_failed_fraction;
        opt.criteria.max_merit = o->max_merit;
        opt.criteria.max_merit_factor = o->max_merit_factor;
        opt.margins.boundary = o->boundary;
        opt.margins.opl_error_factor = o->opl_error_factor;
        opt.margins.merit_relative = o->merit_relative;
        const std::size_t V = static_cast<std::size_t>(b.variants());
        const mko::PrefilterResult r = mko::prefilter_cpu(
            b, layout, opt,
            extra != nullptr ? std::span<const double>(extra, V) : std::span<const double>());
        for (std::size_t v = 0; v < V; ++v) {
            merit[v] = r.stats.merit[v];
            optical_length[v] = r.stats.optical_length[v];
            failed[v] = r.stats.failed[v];
            uncertain_ok[v] = r.stats.uncertain_ok[v];
            uncertain_failed[v] = r.stats.uncertain_failed[v];
            lower[v] = r.merit_lower[v];
            upper[v] = r.merit_upper[v];
            reject[v] = r.reject[v];
        }
        *reference_merit = r.reference_merit;
        *reference_variant = r.reference_variant;
        *kept = r.kept;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// The decision rule on FP64 merits (prefilter_decide_exact).
int mko_ref_prefilter_decide_exact(const mkb_prefilter_options* o, int32_t V, int64_t rays,
                                   const double* merit, const int64_t* failed,
                                   const double* extra, uint8_t* reject) {
    try {
        mko::MeritResult m;
        m.variants = V;
        m.rays_per_variant = rays;
        m.merit.assign(merit, merit + V);
        m.failed.assign(failed, failed + V);
        m.hard_failed.assign(static_cast<std::size_t>(V), 0);
        mko::PrefilterCriteria c;
        c.max_failed_fraction = o->max_failed_fraction;
        c.max_merit = o->max_merit;
        c.max_merit_factor = o->max_merit_factor;
        const std::vector<std::uint8_t> r = mko::prefilter_decide_exact(
            m, c,
            extra != nullptr ? std::span<const double>(extra, static_cast<std::size_t>(V))
                             : std::span<const double>());
        std::copy(r.begin(), r.end(), reject);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Per-ray prefilter data of variant v (prefilter_rays_cpu): status, margin, certain [rays].
int mko_ref_prefilter_rays(const mkb_batch_view* view, const mkb_residual_plan* plan, int v,
                           double boundary, uint8_t* status, double* margin, uint8_t* certain) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::ResidualLayout layout(b.topology(), settings_of(*plan));
        const mko::PrefilterRayData d = mko::prefilter_rays_cpu(b, v, layout, boundary);
        std::copy(d.status.begin(), d.status.end(), status);
        std::copy(d.margin.begin(), d.margin.end(), margin);
        std::copy(d.certain.begin(), d.certain.end(), certain);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// eval_cpu: grid points n (out), then the arrays in the reference's layout when `opd` is not
// null (call twice: sizes first). reference: 0 ExitPupil, 1 Vertex, 2 Infinite.
int mko_ref_eval(const mkb_batch_view* view, const mkb_residual_plan* plan, int grid, int half,
                 int reference, double delta, int64_t* n, double* opd, double* spot_x,
                 double* spot_y, uint8_t* status, double* field_rays, uint8_t* field_status,
                 double* kappa, double* exit_pupil) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        mko::EvalSettings s;
        s.grid = grid;
        s.half_pupil = half != 0;
        s.reference = static_cast<mko::EvalReference>(reference);
        s.field_ray_offset = delta;
        if (opd == nullptr) {
            *n = mko::make_eval_grid(grid, half != 0).samples();
            return 0;
        }
        const mko::EvalResult r = mko::eval_cpu(b, s);
        *n = r.samples();
        std::copy(r.opd.begin(), r.opd.end(), opd);
        std::copy(r.spot_x.begin(), r.spot_x.end(), spot_x);
        std::copy(r.spot_y.begin(), r.spot_y.end(), spot_y);
        std::copy(r.status.begin(), r.status.end(), status);
        std::copy(r.field_rays.begin(), r.field_rays.end(), field_rays);
        std::copy(r.field_status.begin(), r.field_status.end(), field_status);
        std::copy(r.reference_curvature.begin(), r.reference_curvature.end(), kappa);
        std::copy(r.exit_pupil_position.begin(), r.exit_pupil_position.end(), exit_pupil);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Scalar PSF of variant v: EVAL (grid, half, reference, delta) then make_psf_pupils and
// psf_cpu with (padding, na). Per tuple t = f L + l: maps [T][N][N], na [T][2], flips [T][2],
// psf [T][M][M], mtf [T][2][N + 1], metrics [T][13] in mkb_psf_metrics order (transmitted as
// a double); *fft_size and *full_count out. With psf == nullptr only the sizes are returned.
int mko_ref_psf(const mkb_batch_view* view, const mkb_residual_plan* plan, int grid, int half,
                int reference, double delta, int v, double padding, double na, int* fft_size,
                int* full_count, double* maps, double* na_out, int* flips, double* psf,
                double* mtf, double* metrics) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        mko::EvalSettings es;
        es.grid = grid;
        es.half_pupil = half != 0;
        es.reference = static_cast<mko::EvalReference>(reference);
        es.field_ray_offset = delta;
        mko::PsfSettings ps;
        ps.padding = padding;
        ps.numerical_aperture = na;
        *fft_size = mko::psf_fft_size(grid, padding);
        *full_count = mko::make_eval_grid(grid, half != 0).full_count;
        if (psf == nullptr) return 0;
        const mko::EvalResult r = mko::eval_cpu(b, es);
        const std::vector<mko::PsfPupil> pupils = mko::make_psf_pupils(b, r, v, ps);
        const size_t n2 = size_t(grid) * grid, m2 = size_t(*fft_size) * (*fft_size);
        for (size_t t = 0; t < pupils.size(); ++t) {
            const mko::PsfPupil& p = pupils[t];
            const mko::PsfResult q = mko::psf_cpu(p, *fft_size);
            std::copy(p.opd.begin(), p.opd.end(), maps + t * n2);
            na_out[2 * t] = p.na_x;
            na_out[2 * t + 1] = p.na_y;
            flips[2 * t] = p.flip_x ? 1 : 0;
            flips[2 * t + 1] = p.flip_y ? 1 : 0;
            std::copy(q.psf.begin(), q.psf.end(), psf + t * m2);
            const size_t per = size_t(grid) + 1;
            std::copy(q.mtf_sagittal.begin(), q.mtf_sagittal.end(), mtf + t * 2 * per);
            std::copy(q.mtf_tangential.begin(), q.mtf_tangential.end(), mtf + t * 2 * per + per);
            const double m[13] = {static_cast<double>(q.transmitted), q.energy, q.strehl_fft,
                                  q.strehl_origin, q.strehl, q.reference_x, q.reference_y,
                                  q.peak, q.peak_x, q.peak_y, q.dx, q.dy, q.airy_radius};
            std::copy(m, m + 13, metrics + t * 13);
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// psf_cpu of one given pupil (map [N][N], NaN: no transmission): psf [M][M], mtf [2][N + 1],
// metrics [13].
int mko_ref_psf_pupil(int grid, int fft_size, const double* map, int full_count,
                      double wavelength_nm, double na_x, double na_y, int flip_x, int flip_y,
                      double* psf, double* mtf, double* metrics) {
    try {
        mko::PsfPupil p;
        p.grid = grid;
        p.full_count = full_count;
        p.wavelength_nm = wavelength_nm;
        p.na_x = na_x;
        p.na_y = na_y;
        p.flip_x = flip_x != 0;
        p.flip_y = flip_y != 0;
        p.opd.assign(map, map + size_t(grid) * grid);
        const mko::PsfResult q = mko::psf_cpu(p, fft_size);
        std::copy(q.psf.begin(), q.psf.end(), psf);
        std::copy(q.mtf_sagittal.begin(), q.mtf_sagittal.end(), mtf);
        std::copy(q.mtf_tangential.begin(), q.mtf_tangential.end(), mtf + grid + 1);
        const double m[13] = {static_cast<double>(q.transmitted), q.energy, q.strehl_fft,
                              q.strehl_origin, q.strehl, q.reference_x, q.reference_y, q.peak,
                              q.peak_x, q.peak_y, q.dx, q.dy, q.airy_radius};
        std::copy(m, m + 13, metrics);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// finish_psf (and prepare_psf_result's geometry) on a given PSF [M][M] of a pupil map.
int mko_ref_psf_finish(int grid, int fft_size, const double* map, int full_count,
                       double wavelength_nm, double na_x, double na_y, int flip_x, int flip_y,
                       const double* psf, double* metrics) {
    try {
        mko::PsfPupil p;
        p.grid = grid;
        p.full_count = full_count;
        p.wavelength_nm = wavelength_nm;
        p.na_x = na_x;
        p.na_y = na_y;
        p.flip_x = flip_x != 0;
        p.flip_y = flip_y != 0;
        p.opd.assign(map, map + size_t(grid) * grid);
        mko::PsfResult q = mko::prepare_psf_result(p, fft_size);
        std::copy(psf, psf + size_t(fft_size) * fft_size, q.psf.begin());
        mko::finish_psf(q, p);
        const double m[13] = {static_cast<double>(q.transmitted), q.energy, q.strehl_fft,
                              q.strehl_origin, q.strehl, q.reference_x, q.reference_y, q.peak,
                              q.peak_x, q.peak_y, q.dx, q.dy, q.airy_radius};
        std::copy(m, m + 13, metrics);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// FD Jacobian (central scheme) of `runs` runs; base has 1 variant or one per run.
// J [runs][P][R], r0 [runs][R], status_changes [runs][P], R = trace_rows.
int mko_ref_fd_jacobian(const mkb_batch_view* view, const mkb_residual_plan* plan,
                        const mkb_variables* vars, const double* x0, int runs, double* J,
                        double* r0, int64_t* status_changes) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::SystemDescription d = description_of(b, *vars, x0);
        const mko::VariableSet set(d, b.topology());
        mko::FdJacobianOptions opt;
        opt.quadrature = settings_of(*plan);
        const auto P = static_cast<std::size_t>(vars->count);
        const mko::FdJacobian fd = mko::fd_jacobian_cpu(
            set, b, std::span<const double>(x0, P * static_cast<std::size_t>(runs)), opt);
        std::memcpy(J, fd.jacobian.data(), sizeof(double) * fd.jacobian.size());
        std::memcpy(r0, fd.residuals.data(), sizeof(double) * fd.residuals.size());
        if (status_changes != nullptr) {
            std::memcpy(status_changes, fd.status_changes.data(),
                        sizeof(int64_t) * fd.status_changes.size());
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Adjoint Jacobian of `runs` runs (one variant per run at x0). Same layout as the FD one,
// status [runs][rays].
int mko_ref_adjoint_jacobian(const mkb_batch_view* view, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const double* x0, int runs, double* J,
                             double* r0, uint8_t* status, int threads) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::SystemDescription d = description_of(b, *vars, x0);
        const mko::VariableSet set(d, b.topology());
        mko::AdjointJacobianOptions opt;
        opt.quadrature = settings_of(*plan);
        opt.threads = threads;
        const auto P = static_cast<std::size_t>(vars->count);
        const mko::AdjointJacobian aj = mko::adjoint_jacobian_cpu(
            set, b, std::span<const double>(x0, P * static_cast<std::size_t>(runs)), opt);
        std::memcpy(J, aj.jacobian.data(), sizeof(double) * aj.jacobian.size());
        std::memcpy(r0, aj.residuals.data(), sizeof(double) * aj.residuals.size());
        if (status != nullptr) {
            std::memcpy(status, aj.status.data(), aj.status.size());
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// extra_rows_cpu (src/optim/adjoint_jacobian.cpp:300) with paraxial constraints as the extra
// rows: J [runs][P][E], r [runs][E].
int mko_ref_extra_rows(const mkb_batch_view* view, const mkb_residual_plan* plan,
                       const mkb_variables* vars, const double* x0, int runs, int n,
                       const int32_t* type, const int32_t* mode, const double* weight,
                       const double* target, double* J, double* r) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::SystemDescription d = description_of(b, *vars, x0);
        const mko::VariableSet set(d, b.topology());
        const mko::ParaxialConstraints c = constraints_of(n, type, mode, weight, target);
        mko::check_paraxial_constraints(c, b.topology());
        mko::AdjointJacobianOptions opt;
        opt.quadrature = settings_of(*plan);
        opt.extra = mko::make_paraxial_residuals(c);
        const auto P = static_cast<std::size_t>(vars->count);
        const mko::ExtraRowsJacobian e = mko::extra_rows_cpu(
            set, b, std::span<const double>(x0, P * static_cast<std::size_t>(runs)), opt);
        std::memcpy(J, e.jacobian.data(), sizeof(double) * e.jacobian.size());
        std::memcpy(r, e.residuals.data(), sizeof(double) * e.residuals.size());
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int mko_ref_normal_equations(const double* J, const double* r, int P, int64_t R, double* A,
                             double* g) {
    try {
        const auto n = static_cast<std::size_t>(P);
        const auto rows = static_cast<std::size_t>(R);
        mko::normal_equations_host(std::span<const double>(J, n * rows),
                                   std::span<const double>(r, rows), P,
                                   std::span<double>(A, n * n), std::span<double>(g, n));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// paraxial_residuals of variant v (the reference's ExtraResidualFn for paraxial constraints).
int mko_ref_paraxial_residuals(const mkb_batch_view* view, const mkb_residual_plan* plan, int v,
                               int n, const int32_t* type, const int32_t* mode,
                               const double* weight, const double* target, double* out) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::ParaxialConstraints c = constraints_of(n, type, mode, weight, target);
        mko::check_paraxial_constraints(c, b.topology());
        mko::paraxial_residuals(c, b, v, std::span<double>(out, static_cast<std::size_t>(n)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Batched LM on the CPU (optimize_lm_cpu) for `runs` runs. method 0 = FD, 1 = adjoint.
// Outputs per run: x [runs][P], merit, status (LmStatus value), iterations, accepted and the
// merit history [runs][max_iterations + 1] padded with NaN (first penalty round only).
// With n_constraints > 0 the paraxial constraints join as extra residual rows
// (make_paraxial_residuals, LmOptions::jacobian.extra).
int mko_ref_optimize_lm(const mkb_batch_view* view, const mkb_residual_plan* plan,
                        const mkb_variables* vars, const double* x0, int runs, int max_iterations,
                        int method, int penalty_rounds, int threads, double* x_out,
                        double* merit_out, int32_t* status_out, int32_t* iterations_out,
                        int32_t* accepted_out, double* history_out, int n_constraints,
                        const int32_t* c_type, const int32_t* c_mode, const double* c_weight,
                        const double* c_target, int n_trace, const int32_t* t_surface,
                        const int32_t* t_kind, const double* t_weight, const double* t_limit) {
    try {
        const mko::SystemBatchHost b = batch_of_view(*view, *plan);
        const mko::SystemDescription d = description_of(b, *vars, x0);
        const mko::VariableSet set(d, b.topology());
        mko::LmOptions opt;
        opt.max_iterations = max_iterations;
        opt.jacobian.quadrature = settings_of(*plan);
        opt.jacobian_method = method == 1 ? mko::JacobianMethod::Adjoint
                                          : mko::JacobianMethod::FiniteDifferences;
        opt.threads = threads;
        opt.jacobian.extra_threads = threads;
        if (penalty_rounds <= 1) {
            opt.fail_weight_factor = 1.0; // one pass, no outer penalty rounds
        }
        if (n_constraints > 0) {
            const mko::ParaxialConstraints c =
                constraints_of(n_constraints, c_type, c_mode, c_weight, c_target);
            mko::check_paraxial_constraints(c, b.topology());
            opt.jacobian.extra = mko::make_paraxial_residuals(c);
        }
        if (n_trace > 0) {
            // trace-dependent rows from the extrema: kind 0 sqrt(w) max(0, h_s - limit) (a
            // semi-diameter), kind 1 sqrt(w) max(0, limit - cos I_s) (an incidence angle)
            std::vector<int32_t> ts(t_surface, t_surface + n_trace), tk(t_kind, t_kind + n_trace);
            std::vector<double> tw(t_weight, t_weight + n_trace), tl(t_limit, t_limit + n_trace);
            mko::TraceExtraResiduals te;
            te.count = n_trace;
            te.evaluate = [ts, tk, tw, tl](const mko::SystemBatchHost&, int,
                                           const mko::VariantExtrema& e, std::span<double> out) {
                for (std::size_t i = 0; i < ts.size(); ++i) {
                    const double q = tk[i] == 0 ? e.max_height(ts[i]) - tl[i]
                                                : tl[i] - e.min_cos_incidence(ts[i]);
                    out[i] = std::sqrt(tw[i]) * std::max(0.0, q);
                }
            };
            opt.jacobian.trace_extra = te;
        }
        const auto P = static_cast<std::size_t>(vars->count);
        const mko::LmResult res = mko::optimize_lm_cpu(
            set, b, std::span<const double>(x0, P * static_cast<std::size_t>(runs)), opt);
        const auto H = static_cast<std::size_t>(max_iterations) + 1;
        for (int i = 0; i < runs; ++i) {
            const mko::LmRunResult& r = res.runs[static_cast<std::size_t>(i)];
            std::memcpy(x_out + i * P, r.x.data(), sizeof(double) * P);
            merit_out[i] = r.merit;
            status_out[i] = static_cast<int32_t>(r.status);
            iterations_out[i] = r.iterations;
            accepted_out[i] = r.accepted;
            if (history_out != nullptr) {
                for (std::size_t h = 0; h < H; ++h) {
                    history_out[i * H + h] = h < r.history.size()
                                                 ? r.history[h]
                                                 : std::numeric_limits<double>::quiet_NaN();
                }
            }
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

} // extern "C"
