// C ABI entry points (include/mikroptim_b200.h): argument checks, parameter blocks, pack
// plans, error reporting. Every check runs on the host before anything is enqueued.
#include "launch.cuh"

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <string>

namespace mkb {

namespace {
thread_local std::string g_error;
std::atomic<int64_t> g_launches{0};
}  // namespace

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

int cuda_status(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return MKB_OK;
    set_error("%s: %s", what, cudaGetErrorString(err));
    return MKB_ERR_CUDA;
}

namespace {

int sample_count(const mkb_residual_plan* plan, int f) {
    return plan->pupil_mode[f] == MKB_PUPIL_AXIS ? plan->rings : plan->rings * plan->spokes;
}

// tuple_weight, residual_scale, penalty_scale (reference merit/ray_residual.hpp:98,127,186):
// same operations and order as the CPU reference, so the factors are bit-identical.
double tuple_weight(const mkb_residual_plan* p, int f, int l) {
    const double wf = p->field_weight[f];
    const double wl = p->wavelength_weight[l];
    if (!(wf > 0.0) || !(wl > 0.0)) return 0.0;
    double sum_f = 0.0, sum_l = 0.0;
    for (int i = 0; i < p->fields; ++i) sum_f += p->field_weight[i];
    for (int i = 0; i < p->wavelengths; ++i) sum_l += p->wavelength_weight[i];
    return (wf / sum_f) * (wl / sum_l);
}

int check_plan(const mkb_residual_plan* plan) {
    if (plan == nullptr) {
        set_error("residual plan is null");
        return MKB_ERR_ARGUMENT;
    }
    if (plan->rings < 1 || plan->rings > kMaxRings) {
        set_error("rings must be in [1, %d], got %d", kMaxRings, plan->rings);
        return MKB_ERR_ARGUMENT;
    }
    if (plan->spokes < 1 || plan->spokes > kMaxSpokes) {
        set_error("spokes must be in [1, %d], got %d", kMaxSpokes, plan->spokes);
        return MKB_ERR_ARGUMENT;
    }
    if (plan->fields < 1 || plan->fields > kMaxFields || plan->wavelengths < 1 ||
        plan->wavelengths > MKB_MAX_WAVELENGTHS ||
        plan->fields * plan->wavelengths > kMaxTuples) {
        set_error("fields (%d) or wavelengths (%d) out of range", plan->fields,
                  plan->wavelengths);
        return MKB_ERR_ARGUMENT;
    }
    if (plan->failure != MKB_FAILURE_SOFT && plan->failure != MKB_FAILURE_HARD) {
        set_error("unknown failure mode %d", plan->failure);
        return MKB_ERR_ARGUMENT;
    }
    if (!(plan->fail_weight >= 0.0) || !std::isfinite(plan->fail_weight)) {
        set_error("fail_weight must be finite and >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (!(plan->transverse_weight >= 0.0) || !std::isfinite(plan->transverse_weight)) {
        set_error("transverse_weight must be finite and >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (!(plan->reference_wavelength_nm > 0.0) || !std::isfinite(plan->reference_wavelength_nm)) {
        set_error("reference wavelength must be > 0");
        return MKB_ERR_ARGUMENT;
    }
    if (!plan->pupil_mode || !plan->field_weight || !plan->wavelength_weight || !plan->quad_u ||
        !plan->quad_w) {
        set_error("residual plan has a null array");
        return MKB_ERR_ARGUMENT;
    }
    for (int f = 0; f < plan->fields; ++f) {
        const int m = plan->pupil_mode[f];
        if (m != MKB_PUPIL_HALF && m != MKB_PUPIL_FULL && m != MKB_PUPIL_AXIS) {
            set_error("unknown pupil mode %d of field %d", m, f);
            return MKB_ERR_ARGUMENT;
        }
        if (!(plan->field_weight[f] >= 0.0)) {
            set_error("field weight %d must be >= 0", f);
            return MKB_ERR_ARGUMENT;
        }
    }
    for (int l = 0; l < plan->wavelengths; ++l)
        if (!(plan->wavelength_weight[l] >= 0.0)) {
            set_error("wavelength weight %d must be >= 0", l);
            return MKB_ERR_ARGUMENT;
        }
    return MKB_OK;
}

}  // namespace

int64_t trace_rows_of(const mkb_residual_plan* plan, int64_t rays) {
    return rays * (1 + (plan->failure == MKB_FAILURE_SOFT ? 1 : 0) +
                   (plan->transverse_weight > 0.0 ? 2 : 0));
}

int residual_scales(const mkb_residual_plan* plan, double* scale) {
    const int rc = check_plan(plan);
    if (rc != MKB_OK) return rc;
    const double lambda_ref_mm = plan->reference_wavelength_nm * 1e-6;
    for (int f = 0; f < plan->fields; ++f)
        for (int l = 0; l < plan->wavelengths; ++l) {
            const double w = tuple_weight(plan, f, l);
            scale[f * plan->wavelengths + l] = w > 0.0 ? std::sqrt(w) / lambda_ref_mm : 0.0;
        }
    return MKB_OK;
}

int make_trace_params(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                      int pack_rays, TraceParams* out) {
    if (batch == nullptr) {
        set_error("batch is null");
        return MKB_ERR_ARGUMENT;
    }
    int rc = check_plan(plan);
    if (rc != MKB_OK) return rc;
    const int S = batch->surfaces, L = batch->wavelengths, F = batch->fields;
    if (S < 2 || S > kMaxSurfaces) {
        set_error("surfaces must be in [2, %d], got %d", kMaxSurfaces, S);
        return MKB_ERR_ARGUMENT;
    }
    if (L != plan->wavelengths || F != plan->fields) {
        set_error("plan (F=%d, L=%d) does not match the batch (F=%d, L=%d)", plan->fields,
                  plan->wavelengths, F, L);
        return MKB_ERR_ARGUMENT;
    }
    if (batch->variants < 0) {
        set_error("variants must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (batch->non_coaxial != 0 && batch->non_coaxial != 1) {
        set_error("non_coaxial must be 0 or 1");
        return MKB_ERR_ARGUMENT;
    }
    if (batch->ghost_plates < 0 || batch->ghost_terms < 0 ||
        batch->ghost_plates > kMaxGhostPlates || batch->ghost_terms > kMaxGhostTerms) {
        set_error("ghost plates (G=%d, K=%d) out of range [0, %d] x [0, %d]",
                  batch->ghost_plates, batch->ghost_terms, kMaxGhostPlates, kMaxGhostTerms);
        return MKB_ERR_ARGUMENT;
    }
    const RecordLayout lay = record_layout(S, L, F, batch->non_coaxial, batch->ghost_plates,
                                           batch->ghost_terms, batch->glass ? 1 : 0);
    if (batch->record_stride != lay.stride) {
        set_error("record_stride %d does not match the shape (expected %d)",
                  batch->record_stride, lay.stride);
        return MKB_ERR_ARGUMENT;
    }
    if (batch->non_coaxial)
        for (int f = 0; f < F; ++f)
            if (plan->pupil_mode[f] != MKB_PUPIL_FULL) {
                set_error("a non-coaxial batch traces Full pupils only (field %d)", f);
                return MKB_ERR_ARGUMENT;
            }
    if (batch->variants > 0 && (batch->records == nullptr ||
                                (reinterpret_cast<uintptr_t>(batch->records) & 15u) != 0)) {
        set_error("records must be a 16-byte aligned device pointer");
        return MKB_ERR_ARGUMENT;
    }
    if (batch->type == nullptr) {
        set_error("type array is null");
        return MKB_ERR_ARGUMENT;
    }
    if (batch->type[0] != MKB_SURFACE_STOP) {
        set_error("surface 0 must be the stop");
        return MKB_ERR_ARGUMENT;
    }
    int plates = 0, stop = 0;
    for (int s = 1; s < S; ++s) {
        const int t = batch->type[s];
        if (t == MKB_SURFACE_GHOST_PLATE) {
            ++plates;
            continue;
        }
        if (t == MKB_SURFACE_APERTURE_STOP) {
            if (stop != 0 || s > S - 2) {
                set_error("an interior aperture stop lies at 1 <= s <= S - 2, at most one "
                          "per table (surface %d)", s);
                return MKB_ERR_ARGUMENT;
            }
            stop = s;
            continue;
        }
        if (t != MKB_SURFACE_PLANE && t != MKB_SURFACE_SPHERE) {
            set_error("surface %d has unknown kind %d", s, t);
            return MKB_ERR_ARGUMENT;
        }
    }
    if (stop > 0 && (batch->non_coaxial || plates > 0 || batch->variant_surfaces != nullptr)) {
        set_error("an interior aperture stop is traced in coaxial batches of one table without "
                  "ghost plates");
        return MKB_ERR_UNSUPPORTED;
    }
    if (plates != batch->ghost_plates) {
        set_error("the table has %d ghost-plate surfaces but the batch carries %d plates",
                  plates, batch->ghost_plates);
        return MKB_ERR_ARGUMENT;
    }
    if (plates > kMaxGhostPlates) {
        set_error("%d ghost plates; this build traces at most %d", plates, kMaxGhostPlates);
        return MKB_ERR_UNSUPPORTED;
    }
    TraceParams& p = *out;
    std::memset(&p, 0, sizeof(p));
    p.V = batch->variants;
    p.S = S;
    p.non_coaxial = batch->non_coaxial;
    p.G = batch->ghost_plates;
    p.K = batch->ghost_terms;
    p.glass = batch->glass ? 1 : 0;
    p.vsurf = batch->variant_surfaces;
    p.order = nullptr;
    p.stop = stop;
    p.spheres = 0;
    for (int s = 0; s < S && s < 64; ++s)
        if (batch->type[s] == MKB_SURFACE_SPHERE) p.spheres |= uint64_t(1) << s;
    p.L = L;
    p.F = F;
    p.stride = lay.stride;
    p.failure = plan->failure;
    p.rings = plan->rings;
    p.spokes = plan->spokes;
    for (int s = 0, g = 0; s < kMaxSurfaces; ++s) {
        p.ghost_of[s] = -1;
        if (s >= S) continue;
        p.type[s] = batch->type[s];
        if (s > 0 && batch->type[s] == MKB_SURFACE_GHOST_PLATE) p.ghost_of[s] = static_cast<int8_t>(g++);
    }
    int offset = 0;
    for (int f = 0; f < F; ++f) {
        p.pupil_mode[f] = plan->pupil_mode[f];
        p.sample_count[f] = sample_count(plan, f);
        p.field_offset[f] = offset;
        offset += L * p.sample_count[f];
    }
    p.rays = offset;
    // pupil tables (pupil/quadrature.hpp:71): rho = sqrt(u), weight = W / M, phi per mode
    const double pi = 3.14159265358979323846264338327950288;
    for (int i = 0; i < plan->rings; ++i) {
        p.rho[i] = std::sqrt(plan->quad_u[i]);
        p.w_axis[i] = plan->quad_w[i] / 1.0;
        p.rw_axis[i] = std::sqrt(p.w_axis[i]);
        p.w_spoke[i] = plan->quad_w[i] / static_cast<double>(plan->spokes);
        p.rw_spoke[i] = std::sqrt(p.w_spoke[i]);
    }
    for (int j = 0; j < plan->spokes; ++j) {
        const double half = static_cast<double>(2 * j + 1) * pi / static_cast<double>(2 * plan->spokes);
        const double full = static_cast<double>(2 * j + 1) * pi / static_cast<double>(plan->spokes);
        p.sin_half[j] = std::sin(half);
        p.cos_half[j] = std::cos(half);
        p.sin_full[j] = std::sin(full);
        p.cos_full[j] = std::cos(full);
    }
    p.n_tuples = F * L;
    const double lambda_ref_mm = plan->reference_wavelength_nm * 1e-6;
    for (int f = 0; f < F; ++f)
        for (int l = 0; l < L; ++l) {
            const double w = tuple_weight(plan, f, l);
            p.scale[f * L + l] = w > 0.0 ? std::sqrt(w) / lambda_ref_mm : 0.0;
            p.pscale[f * L + l] = w > 0.0 ? std::sqrt(plan->fail_weight * w) : 0.0;
            p.tscale[f * L + l] = w > 0.0 ? std::sqrt(plan->transverse_weight * w) : 0.0;
        }
    p.transverse = plan->transverse_weight > 0.0 ? 1 : 0;
    // pack plan: consecutive tuples until pack_rays rays or kMaxPackTuples tuples; a tuple
    // with more rays than pack_rays (fine pupils) gets a pack of its own
    for (int t = 0; t < p.n_tuples; ++t)
        if (p.sample_count[t / L] > pack_rays) pack_rays = p.sample_count[t / L];
    int packs = 0;
    int t = 0;
    while (t < p.n_tuples) {
        const int n0 = p.sample_count[t / L];
        if (packs >= kMaxPacks) {
            set_error("too many packs (%d tuples)", p.n_tuples);
            return MKB_ERR_ARGUMENT;
        }
        Pack& pk = p.packs[packs];
        pk.first_tuple = static_cast<int16_t>(t);
        pk.first_ray = p.field_offset[t / L] + (t % L) * n0;
        int rays = 0, tuples = 0;
        while (t < p.n_tuples && tuples < kMaxPackTuples) {
            const int n = p.sample_count[t / L];
            if (tuples > 0 && rays + n > pack_rays) break;
            rays += n;
            ++tuples;
            ++t;
        }
        pk.tuples = static_cast<int16_t>(tuples);
        pk.rays = rays;
        ++packs;
    }
    p.n_packs = packs;
    p.vpc = 1;
    p.pack_max = 0;
    for (int k = 0; k < packs; ++k)
        if (p.packs[k].rays > p.pack_max) p.pack_max = p.packs[k].rays;
    return MKB_OK;
}

int sweep_floor_of(const mkb_variables* vars, int S, const uint8_t* type) {
    int plate_surface[kMaxGhostPlates];
    int plates = 0;
    for (int s = 1; s < S; ++s)
        if (type[s] == MKB_SURFACE_GHOST_PLATE && plates < kMaxGhostPlates)
            plate_surface[plates++] = s;
    int floor = kMaxSurfaces;
    for (int k = 0; k < vars->count; ++k) {
        const int t = vars->type[k];
        int s = vars->surface[k], c;
        if (t == MKB_VAR_WORKING_DISTANCE) {
            c = S - 1;
        } else if (t == MKB_VAR_THICKNESS) {
            c = s;
        } else {
            if (t == MKB_VAR_GHOST_COEFFICIENT) {
                const int g = vars->ghost_plate ? vars->ghost_plate[k] : 0;
                s = g >= 0 && g < plates ? plate_surface[g] : 1;
            }
            c = s > 0 ? s - 1 : 0;
        }
        if (c < floor) floor = c;
    }
    return floor;
}

int make_var_params(const mkb_variables* vars, int S, const uint8_t* type, VarParams* out,
                    int ghost_terms, int L, const double* wavelength_nm, int glass) {
    if (vars == nullptr || vars->count < 1 || vars->count > MKB_MAX_VARIABLES) {
        set_error("variables: count must be in [1, %d]", MKB_MAX_VARIABLES);
        return MKB_ERR_ARGUMENT;
    }
    if (!vars->type || !vars->surface || !vars->lower || !vars->upper || !vars->typical) {
        set_error("variables: null array");
        return MKB_ERR_ARGUMENT;
    }
    VarParams& v = *out;
    std::memset(&v, 0, sizeof(v));
    v.P = vars->count;
    for (int s = 0; s < kMaxSurfaces; ++s) v.col_curvature[s] = v.col_thickness[s] = -1;
    std::memset(v.col_ghost, -1, sizeof(v.col_ghost));
    std::memset(v.col_glass, -1, sizeof(v.col_glass));
    v.L = L;
    // table surface of every ghost plate (plates are numbered in table order)
    int plate_surface[kMaxGhostPlates];
    int plates = 0;
    for (int s = 1; s < S; ++s)
        if (type[s] == MKB_SURFACE_GHOST_PLATE && plates < kMaxGhostPlates)
            plate_surface[plates++] = s;
    for (int k = 0; k < v.P; ++k) {
        const int t = vars->type[k];
        int s = vars->surface[k];
        if (t == MKB_VAR_WORKING_DISTANCE) s = S - 1;
        if (t != MKB_VAR_CURVATURE && t != MKB_VAR_THICKNESS && t != MKB_VAR_WORKING_DISTANCE &&
            t != MKB_VAR_GHOST_COEFFICIENT && t != MKB_VAR_GLASS) {
            set_error("variable %d: unknown type %d (curvature, thickness, working distance, "
                      "ghost coefficient, glass)", k, t);
            return MKB_ERR_UNSUPPORTED;
        }
        int8_t* slot;
        if (t == MKB_VAR_GLASS) {
            const int c = vars->glass_component ? vars->glass_component[k] : -1;
            if (!glass || wavelength_nm == nullptr || L < 1 || L > MKB_MAX_WAVELENGTHS) {
                set_error("variable %d: a glass variable needs the batch's Buchdahl "
                          "coefficients and wavelengths", k);
                return MKB_ERR_ARGUMENT;
            }
            if (s < 0 || s >= S || c < 0 || c > 2) {
                set_error("variable %d: glass of surface %d, component %d out of range", k, s, c);
                return MKB_ERR_ARGUMENT;
            }
            v.glass_component[k] = static_cast<int8_t>(c);
            v.has_glass = 1;
            slot = &v.col_glass[s][c];
        } else if (t == MKB_VAR_GHOST_COEFFICIENT) {
            const int g = vars->ghost_plate ? vars->ghost_plate[k] : -1;
            const int order = vars->ghost_order ? vars->ghost_order[k] : 0;
            if (g < 0 || g >= plates || order < 1 || order > ghost_terms) {
                set_error("variable %d: ghost coefficient a_%d of plate %d out of range "
                          "(%d plates, %d terms)", k, order, g, plates, ghost_terms);
                return MKB_ERR_ARGUMENT;
            }
            s = plate_surface[g];
            v.ghost_plate[k] = static_cast<int8_t>(g);
            v.ghost_order[k] = static_cast<int8_t>(order);
            slot = &v.col_ghost[g][order - 1];
        } else {
            if (s < 0 || s >= S || (t == MKB_VAR_THICKNESS && s == S - 1)) {
                set_error("variable %d: surface %d out of range", k, s);
                return MKB_ERR_ARGUMENT;
            }
            if (t == MKB_VAR_CURVATURE && type[s] != MKB_SURFACE_SPHERE) {
                set_error("variable %d: curvature of surface %d, which is not a sphere", k, s);
                return MKB_ERR_ARGUMENT;
            }
            if (t == MKB_VAR_THICKNESS && s == 0) {
                bool stop = false;
                for (int u = 1; u < S; ++u) stop = stop || type[u] == MKB_SURFACE_APERTURE_STOP;
                if (stop) {
                    set_error("variable %d: thickness[0] follows the interior stop's entrance "
                              "pupil and is no variable", k);
                    return MKB_ERR_ARGUMENT;
                }
            }
            slot = t == MKB_VAR_CURVATURE ? &v.col_curvature[s] : &v.col_thickness[s];
        }
        if (*slot >= 0) {
            set_error("variable %d: its parameter already belongs to variable %d", k, *slot);
            return MKB_ERR_ARGUMENT;
        }
        *slot = static_cast<int8_t>(k);
        v.type[k] = static_cast<int8_t>(t == MKB_VAR_WORKING_DISTANCE ? MKB_VAR_THICKNESS : t);
        v.surface[k] = static_cast<int8_t>(s);
        v.lower[k] = vars->lower[k];
        v.upper[k] = vars->upper[k];
        v.typical[k] = vars->typical[k];
        if (std::isnan(v.lower[k]) || std::isnan(v.upper[k]) || v.lower[k] > v.upper[k]) {
            set_error("variable %d: invalid bounds", k);
            return MKB_ERR_ARGUMENT;
        }
        if (!(v.typical[k] > 0.0) || !std::isfinite(v.typical[k])) {
            set_error("variable %d: typical size must be > 0", k);
            return MKB_ERR_ARGUMENT;
        }
    }
    // the reverse step onto surface c + 1 writes the columns of curvature[c + 1] and of plate
    // c + 1's coefficients, of thickness[c] (the working distance in the image step, c = S - 1)
    // and of the media c and c + 1 (medium 0 in the step onto surface 1)
    v.sweep_floor = kMaxSurfaces;
    for (int k = 0; k < v.P; ++k) {
        const int s = v.surface[k];
        const int c = v.type[k] == MKB_VAR_THICKNESS ? s : (s > 0 ? s - 1 : 0);
        if (c < v.sweep_floor) v.sweep_floor = c;
    }
    if (v.has_glass) {
        // Buchdahl coordinate w = dl / (1 + 2.5 dl), dl = lambda [um] - 0.546074 um
        // (buchdahl_omega, glass/dispersion.hpp:87; nm_to_um divides by 1000)
        for (int l = 0; l < L; ++l) {
            const double dl = wavelength_nm[l] / 1000.0 - 0.546074;
            const double den = 1.0 + 2.5 * dl;
            if (!(den > 0.0)) {
                set_error("glass variables: the Buchdahl coordinate of %g nm is undefined",
                          wavelength_nm[l]);
                return MKB_ERR_ARGUMENT;
            }
            v.omega[l] = dl / den;
        }
    }
    return MKB_OK;
}

}  // namespace mkb

using namespace mkb;

extern "C" {

const char* mkb_last_error(void) { return g_error.c_str(); }
const char* mkb_version(void) { return "mikroptim_b200 0.1 (sm_100a)"; }
int64_t mkb_launch_count(void) { return g_launches.load(); }

int mkb_device_status(void) {
    int (*readers[])() = {trace_device_error, gram_device_error, adjoint_device_error,
                              jacobian_device_error, lm_device_error, prefilter_device_error};
    int status = MKB_OK;
    for (auto read : readers) {
        const int v = read();
        if (v != MKB_OK && status == MKB_OK) status = v;
    }
    if (status != MKB_OK) set_error("a bounded device-side wait gave up (status %d)", status);
    return status;
}

int mkb_set_wait_limit(uint32_t polls) {
    int (*setters[])(uint32_t) = {trace_device_error_wait_limit, gram_device_error_wait_limit,
                                  adjoint_device_error_wait_limit,
                                  jacobian_device_error_wait_limit, lm_device_error_wait_limit,
                                  prefilter_device_error_wait_limit};
    for (auto set : setters) {
        const int rc = set(polls);
        if (rc != MKB_OK) {
            set_error("mkb_set_wait_limit: cudaMemcpyToSymbol failed");
            return rc;
        }
    }
    return MKB_OK;
}

int32_t mkb_record_stride(int32_t surfaces, int32_t wavelengths, int32_t fields) {
    return record_layout(surfaces, wavelengths, fields).stride;
}

int32_t mkb_record_stride_ext(int32_t surfaces, int32_t wavelengths, int32_t fields,
                              int32_t non_coaxial, int32_t ghost_plates, int32_t ghost_terms,
                              int32_t glass) {
    return record_layout(surfaces, wavelengths, fields, non_coaxial ? 1 : 0,
                         ghost_plates > 0 ? ghost_plates : 0,
                         ghost_plates > 0 && ghost_terms > 0 ? ghost_terms : 0,
                         glass ? 1 : 0).stride;
}

int mkb_pack_batch_host(const mkb_batch_view* v, double* records) {
    if (v == nullptr || records == nullptr) {
        set_error("pack: null argument");
        return MKB_ERR_ARGUMENT;
    }
    const int S = v->surfaces, L = v->wavelengths, F = v->fields;
    if (S < 2 || S > kMaxSurfaces || L < 1 || L > MKB_MAX_WAVELENGTHS || F < 1 ||
        F > kMaxFields || v->variants < 0) {
        set_error("pack: shape out of range (S=%d, L=%d, F=%d)", S, L, F);
        return MKB_ERR_ARGUMENT;
    }
    const int G = v->ghost_plates, K = v->ghost_terms;
    if (G < 0 || K < 0 || G > kMaxGhostPlates || K > kMaxGhostTerms ||
        (G > 0 && (!v->ghost_coeff || !v->ghost_norm_radius || !v->ghost_index))) {
        set_error("pack: ghost plates (G=%d, K=%d) out of range or without data", G, K);
        return MKB_ERR_ARGUMENT;
    }
    const int non_coaxial = v->decenter_tilt != nullptr ? 1 : 0;
    const int glass = v->buchdahl_coeff != nullptr ? 1 : 0;
    if (v->type == nullptr) {
        set_error("pack: type array is null");
        return MKB_ERR_ARGUMENT;
    }
    const RecordLayout lay = with_stop(record_layout(S, L, F, non_coaxial, G, K, glass), v->type, S);
    for (int64_t i = 0; i < v->variants; ++i) {
        double* r = records + i * lay.stride;
        std::memset(r, 0, sizeof(double) * lay.stride);
        for (int s = 0; s < S; ++s) {
            r[lay.curvature + s] = v->curvature[i * S + s];
            r[lay.thickness + s] = v->thickness[i * S + s];
            for (int l = 0; l < L; ++l)
                r[lay.index + s * L + l] = v->index[(i * S + s) * L + l];
        }
        r[lay.pupil] = v->pupil_radius[i];
        for (int f = 0; f < F; ++f) {
            const double th = v->field_angle[i * F + f];
            r[lay.sin_theta + f] = std::sin(th);
            r[lay.cos_theta + f] = std::cos(th);
            r[lay.target + f] = v->field_target[i * F + f];
        }
        // surface transforms (surface_transform_of, trace/surface_transform.hpp:99): a surface
        // whose four values are all zero is traced coaxially; otherwise the tilt sines and
        // cosines are taken with the host libm, as the CPU tracer takes them
        for (int s = 0; non_coaxial && s < S; ++s) {
            const double* t = v->decenter_tilt + (i * S + s) * 4;
            double* x = r + lay.xf + s * kXfValues;
            auto zero = [](double a) { return !(a > 0.0) && !(a < 0.0); };
            const bool moved = !(zero(t[0]) && zero(t[1]) && zero(t[2]) && zero(t[3]));
            x[0] = moved ? t[0] : 0.0;
            x[1] = moved ? t[1] : 0.0;
            x[2] = moved ? std::cos(t[2]) : 1.0;
            x[3] = moved ? std::sin(t[2]) : 0.0;
            x[4] = moved ? std::cos(t[3]) : 1.0;
            x[5] = moved ? std::sin(t[3]) : 0.0;
            x[6] = moved ? 1.0 : 0.0;
            x[7] = 0.0;
        }
        for (int s = 0; glass && s < S; ++s)
            for (int c = 0; c < 4; ++c)
                r[lay.glass + s * 4 + c] = v->buchdahl_coeff[(i * S + s) * 4 + c];
        for (int g = 0; g < G; ++g) {
            for (int k = 0; k < K; ++k)
                r[lay.ghost_coeff + g * K + k] = v->ghost_coeff[(i * G + g) * K + k];
            r[lay.ghost_radius + g] = v->ghost_norm_radius[g];
            for (int l = 0; l < L; ++l)
                r[lay.ghost_index + g * L + l] = v->ghost_index[(i * G + g) * L + l];
        }
        // an interior stop: the entrance pupil from paraxial ray aiming
        if (lay.stop > 0 && !aim_record(lay, r)) {
            set_error("pack: variant %lld: the interior stop's paraxial image is at infinity "
                      "or not finite", static_cast<long long>(i));
            return MKB_ERR_ARGUMENT;
        }
    }
    return MKB_OK;
}

int mkb_apply_variables_device(const mkb_device_batch* templates, const mkb_variables* vars,
                               const double* x, int32_t runs, double* records_out,
                               void* stream) {
    if (templates == nullptr || runs < 0 ||
        (templates->variants != 1 && templates->variants != runs)) {
        set_error("apply: templates must hold 1 variant or one per run");
        return MKB_ERR_ARGUMENT;
    }
    if (runs == 0) return MKB_OK;
    if (x == nullptr || records_out == nullptr || templates->records == nullptr ||
        templates->type == nullptr) {
        set_error("apply: null pointer");
        return MKB_ERR_ARGUMENT;
    }
    const int S = templates->surfaces, L = templates->wavelengths, F = templates->fields;
    if (S < 2 || S > kMaxSurfaces || L < 1 || L > MKB_MAX_WAVELENGTHS || F < 1 || F > kMaxFields) {
        set_error("apply: shape out of range (S=%d, L=%d, F=%d)", S, L, F);
        return MKB_ERR_ARGUMENT;
    }
    const RecordLayout lay = with_stop(record_layout(S, L, F, templates->non_coaxial != 0,
                                                     templates->ghost_plates,
                                                     templates->ghost_terms,
                                                     templates->glass ? 1 : 0),
                                       templates->type, S);
    if (templates->record_stride != lay.stride ||
        (reinterpret_cast<uintptr_t>(records_out) & 15u) != 0) {
        set_error("apply: record stride %d (expected %d) or unaligned output",
                  templates->record_stride, lay.stride);
        return MKB_ERR_ARGUMENT;
    }
    VarParams vp;
    const int rc = make_var_params(vars, S, templates->type, &vp, templates->ghost_terms,
                         templates->wavelengths, templates->wavelength_nm,
                         templates->glass);
    if (rc != MKB_OK) return rc;
    return launch_apply(vp, lay, templates->records, templates->variants, x, records_out, runs,
                        static_cast<cudaStream_t>(stream));
}

int64_t mkb_rays_per_variant(const mkb_residual_plan* plan) {
    if (check_plan(plan) != MKB_OK) return MKB_ERR_ARGUMENT;
    int64_t n = 0;
    for (int f = 0; f < plan->fields; ++f) n += static_cast<int64_t>(plan->wavelengths) * sample_count(plan, f);
    return n;
}

int64_t mkb_trace_rows(const mkb_residual_plan* plan) {
    const int64_t r = mkb_rays_per_variant(plan);
    if (r < 0) return r;
    return trace_rows_of(plan, r);
}

namespace {

// pack_rays of the options (0 or no options: the default), clamped to what the kernels stage
int options_pack_rays(const mkb_trace_options* options, int* pack_rays) {
    int v = options != nullptr ? options->pack_rays : 0;
    if (v < 0) {
        set_error("pack_rays must be >= 1 (0 = default), got %d", v);
        return MKB_ERR_ARGUMENT;
    }
    if (v == 0) v = pack_rays_default();
    *pack_rays = v < kMaxPackRaysOption ? v : kMaxPackRaysOption;
    return MKB_OK;
}

// variants_per_cta of the options (0 or no options: 1); with extrema it must be 1
int options_vpc(const mkb_trace_options* options, TraceParams* p) {
    const int v = options != nullptr ? options->variants_per_cta : 0;
    if (v < 0 || v > kMaxVariantsPerCta) {
        set_error("variants_per_cta must be in [1, %d] (0 = 1), got %d", kMaxVariantsPerCta, v);
        return MKB_ERR_ARGUMENT;
    }
    p->vpc = v == 0 ? 1 : v;
    if (p->vpc > 1 && options->extrema != nullptr) {
        set_error("variants_per_cta > 1 is not available with extrema");
        return MKB_ERR_UNSUPPORTED;
    }
    return MKB_OK;
}

int check_trace_precision(int precision, const char* what) {
    if (precision != MKB_PRECISION_FP64 && precision != MKB_PRECISION_FP64_FMA &&
        precision != MKB_PRECISION_MIXED && precision != MKB_PRECISION_DF64 &&
        precision != MKB_PRECISION_FP32_BULK) {
        set_error("%s: precision %d not available", what, precision);
        return MKB_ERR_UNSUPPORTED;
    }
    return MKB_OK;
}

}  // namespace

int mkb_residuals_ex_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                            const mkb_trace_options* options, double* residuals, int64_t stride,
                            double* opd, uint8_t* status, void* stream) {
    int pack_rays = 0;
    int rc = options_pack_rays(options, &pack_rays);
    if (rc != MKB_OK) return rc;
    TraceParams p;
    rc = make_trace_params(batch, plan, pack_rays, &p);
    if (rc != MKB_OK) return rc;
    rc = options_vpc(options, &p);
    if (rc != MKB_OK) return rc;
    rc = check_trace_precision(plan->precision, "residuals");
    if (rc != MKB_OK) return rc;
    const int64_t rows = trace_rows_of(plan, p.rays);
    if (stride < rows) {
        set_error("residuals: stride %lld < trace rows %lld", static_cast<long long>(stride),
                  static_cast<long long>(rows));
        return MKB_ERR_ARGUMENT;
    }
    if (p.V == 0) return MKB_OK;
    if (residuals == nullptr) {
        set_error("residuals: output is null");
        return MKB_ERR_ARGUMENT;
    }
    return launch_residuals(p, batch->records, residuals, stride, opd, status, plan->precision,
                            static_cast<cudaStream_t>(stream), {},
                            options != nullptr ? options->extrema : nullptr);
}

int mkb_residuals_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                         double* residuals, int64_t stride, double* opd, uint8_t* status,
                         void* stream) {
    return mkb_residuals_ex_device(batch, plan, nullptr, residuals, stride, opd, status, stream);
}

size_t mkb_merit_workspace_bytes(int32_t variants, const mkb_residual_plan* plan) {
    if (check_plan(plan) != MKB_OK || variants < 0) return 0;
    return merit_workspace_bytes(variants, plan->fields * plan->wavelengths);
}

int mkb_merit_ex_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                        const mkb_trace_options* options, double* merit, int64_t* failed,
                        int64_t* hard_failed, void* workspace, size_t workspace_bytes,
                        void* stream) {
    int pack_rays = 0;
    int rc = options_pack_rays(options, &pack_rays);
    if (rc != MKB_OK) return rc;
    TraceParams p;
    rc = make_trace_params(batch, plan, pack_rays, &p);
    if (rc != MKB_OK) return rc;
    rc = options_vpc(options, &p);
    if (rc != MKB_OK) return rc;
    rc = check_trace_precision(plan->precision, "merit");
    if (rc != MKB_OK) return rc;
    if (p.V == 0) return MKB_OK;
    if (!merit || !failed || !hard_failed) {
        set_error("merit: output is null");
        return MKB_ERR_ARGUMENT;
    }
    return launch_merit(p, batch->records, merit, failed, hard_failed, workspace,
                        workspace_bytes, plan->precision, static_cast<cudaStream_t>(stream), {},
                        options != nullptr ? options->extra_merit : nullptr,
                        options != nullptr ? options->extrema : nullptr);
}

int mkb_merit_device(const mkb_device_batch* batch, const mkb_residual_plan* plan, double* merit,
                     int64_t* failed, int64_t* hard_failed, void* workspace,
                     size_t workspace_bytes, void* stream) {
    return mkb_merit_ex_device(batch, plan, nullptr, merit, failed, hard_failed, workspace,
                               workspace_bytes, stream);
}

// ---- device memory of a TraceEngine run ----------------------------------------------------
int mkb_usable_bytes(size_t free_bytes, size_t reserve_min_bytes, double reserve_fraction,
                     size_t* usable) {
    if (usable == nullptr || !(reserve_fraction >= 0.0 && reserve_fraction <= 1.0)) {
        set_error("memory reserve: fraction must be in [0, 1]");
        return MKB_ERR_ARGUMENT;
    }
    const double part = reserve_fraction * static_cast<double>(free_bytes);
    size_t reserve = part >= static_cast<double>(SIZE_MAX) ? SIZE_MAX : static_cast<size_t>(part);
    if (reserve < reserve_min_bytes) reserve = reserve_min_bytes;
    *usable = free_bytes > reserve ? free_bytes - reserve : 0;
    return MKB_OK;
}

namespace {

// the trace parameters of a batch shape (its variants and records are not read)
int shape_params(const mkb_device_batch* shape, const mkb_residual_plan* plan, int pack_rays,
                 TraceParams* p) {
    if (shape == nullptr) {
        set_error("batch shape is null");
        return MKB_ERR_ARGUMENT;
    }
    mkb_device_batch s = *shape;
    s.variants = 0;
    s.records = nullptr;
    return make_trace_params(&s, plan, pack_rays, p);
}

// one buffer's worth of allocation granularity for each buffer a run holds (records, variant
// surface counts, up to three outputs, scratch, extra merit)
constexpr size_t kRunBuffers = 7;
constexpr size_t kBufferSlack = size_t(2) << 20;

int run_bytes(const TraceParams& p, const mkb_device_batch* shape, const mkb_residual_plan* plan,
              int merit_mode, int64_t extra_residuals, int opd, int extra_merit,
              size_t* per_variant, size_t* fixed) {
    if (extra_residuals < 0) {
        set_error("extra_residuals must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    const size_t rays = static_cast<size_t>(p.rays);
    size_t per = static_cast<size_t>(p.stride) * sizeof(double);
    if (shape->variant_surfaces != nullptr) per += 1;
    if (merit_mode) {
        per += 3 * sizeof(double) + merit_workspace_bytes(1, p.n_tuples);
        if (extra_merit) per += sizeof(double);
    } else {
        const size_t rows = static_cast<size_t>(trace_rows_of(plan, p.rays)) +
                            static_cast<size_t>(extra_residuals);
        per += rows * sizeof(double) + rays;  // residual rows and the status bytes
        if (opd) per += rays * sizeof(double);
    }
    *per_variant = per;
    *fixed = kRunBuffers * kBufferSlack;
    return MKB_OK;
}

}  // namespace

int mkb_trace_run_bytes(const mkb_device_batch* shape, const mkb_residual_plan* plan,
                        int32_t merit_mode, int64_t extra_residuals, int32_t opd,
                        int32_t extra_merit, size_t* per_variant, size_t* fixed) {
    if (per_variant == nullptr || fixed == nullptr) {
        set_error("run bytes: null output");
        return MKB_ERR_ARGUMENT;
    }
    TraceParams p;
    int rc = shape_params(shape, plan, pack_rays_default(), &p);
    if (rc != MKB_OK) return rc;
    return run_bytes(p, shape, plan, merit_mode, extra_residuals, opd, extra_merit, per_variant,
                     fixed);
}

int64_t mkb_trace_tranche_variants(size_t usable, const mkb_device_batch* shape,
                                   const mkb_residual_plan* plan,
                                   const mkb_trace_options* options, int32_t merit_mode,
                                   int64_t extra_residuals, int32_t opd, int32_t extra_merit,
                                   int32_t granularity) {
    if (granularity < 1) {
        set_error("granularity must be >= 1");
        return MKB_ERR_ARGUMENT;
    }
    int pack_rays = 0;
    int rc = options_pack_rays(options, &pack_rays);
    if (rc != MKB_OK) return rc;
    TraceParams p;
    rc = shape_params(shape, plan, pack_rays, &p);
    if (rc != MKB_OK) return rc;
    size_t per = 0, fixed = 0;
    rc = run_bytes(p, shape, plan, merit_mode, extra_residuals, opd, extra_merit, &per, &fixed);
    if (rc != MKB_OK) return rc;
    if (usable <= fixed) return 0;
    int64_t cap = static_cast<int64_t>((usable - fixed) / per);
    const int64_t grid_cap = static_cast<int64_t>(INT32_MAX) / (p.n_packs > 0 ? p.n_packs : 1);
    if (cap > grid_cap) cap = grid_cap;
    if (cap > INT32_MAX) cap = INT32_MAX;
    cap = cap / granularity * granularity;
    return cap;
}

}  // extern "C"
