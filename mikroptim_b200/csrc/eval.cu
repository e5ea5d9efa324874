// EVAL: evaluation of every variant on a dense Cartesian pupil grid, for sm_100a.
//
// Per tuple (variant, field, wavelength): the chief ray and three neighbours (field rays), then
// every grid point traced to the image plane (spot) and to the reference sphere (OPL), the
// piston over the grid weights and the OPD. Every failure is hard.
//   eval_field_kernel   one thread per (tuple, field ray); the chief ray's OPL is the tuple's
//                       OPL offset
//   eval_grid_kernel    grid-stride over (tuple, point): status, spot, OPL - offset (kept in
//                       the OPD output until the piston is known)
//   eval_piston_kernel  one warp per tuple: weight and weighted OPL sums in ascending point
//                       order (opd_statistics, include/mikroptim/merit/opd.hpp:43)
//   eval_opd_kernel     grid-stride: OPD = (OPL - offset) - piston, NaN for failed rays
// Arithmetic in Exact64 in the reference's order: bit-identical to eval_cpu
// (src/eval/eval.cpp:307; eval_ray, exit_pupil_sphere_step, eval_source_ray,
// include/mikroptim/eval/eval_ray.hpp:60-190; make_eval_grid and eval_reference_geometry,
// src/eval/eval.cpp:186,232).
#include "launch.cuh"

#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

namespace mkb {

namespace {

constexpr int kFieldRays = 4;

template <class T>
struct NumTag {
    using type = T;
};
constexpr int kFieldValues = 5;

struct EvalParams {
    TraceParams t;       // record layout, surface kinds, plates (V, S, L, F, stride, ...)
    int reference;       // MKB_EVAL_*
    double delta;        // field-ray offset
    int64_t n;           // grid points per tuple
};

struct EvalRayOut {
    int status;
    double opl, ix, iy, dx, dy, dz;
};

// exit_pupil_sphere_step (eval_ray.hpp:104): s + sigma R = b - kappa t / (sqrt(1 + kappa^2 t)
// + 1) with q = p - M, b = -q.d, t = -|q x d|^2; only the OPL moves.
template <class N>
__device__ inline int exit_pupil_step(RayT<N>& r, N h, N w, N kappa, N n_image) {
    const N qx = r.px - N(0.0), qy = r.py - h, qz = r.pz - w;
    const N b = -(qx * r.dx + qy * r.dy + qz * r.dz);
    const N cx = qy * r.dz - qz * r.dy;
    const N cy = qz * r.dx - qx * r.dz;
    const N cz = qx * r.dy - qy * r.dx;
    const N t = -(cx * cx + cy * cy + cz * cz);
    const N disc = N(1.0) + kappa * kappa * t;
    if (!(value_of(disc) >= 0.0)) return kMissed;
    const N step = b - kappa * t / (nsqrt(disc) + N(1.0));
    if (!(value_of(step) == value_of(step))) return kMissed;
    r.opl += n_image * step;
    return kOk;
}

// eval_ray (eval_ray.hpp:152) of pupil point (x, y) of variant v, field f, wavelength l, in
// number type N (Exact64: the reference's arithmetic; double: contracted, for the precision
// sweep's intercept errors)
template <class N, int kFeat>
__device__ inline EvalRayOut eval_ray(const EvalParams& e, const double* rec, int v, int f,
                                      int l, double x, double y, double kappa) {
    const TraceParams& p = e.t;
    const RecordLayout lay = layout_of(p);
    const int S = surfaces_of(p, v);
    const int L = p.L;
    EvalRayOut out{};
    const N a = N(rec[lay.pupil]);
    RayT<N> r;
    r.px = a * N(x);
    r.py = a * N(y);
    r.pz = N(0.0);
    r.dx = N(0.0);
    r.dy = N(rec[lay.sin_theta + f]);
    r.dz = N(rec[lay.cos_theta + f]);
    r.opl = (r.px * r.dx + r.py * r.dy) + r.pz * r.dz;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    N n_before = N(idx[l]);
    int st = kOk;
    for (int s = 1; s < S; ++s) {
        const N n_after = N(idx[s * L + l]);
        const N c = p.type[s] == MKB_SURFACE_SPHERE ? N(curv[s]) : N(0.0);
        GhostData gd;
        const bool plate = ghost_at<(kFeat & 2) != 0>(p, rec, lay, s, l, gd);
        int branch;
        st = step_surface_xf<N>(r, N(thick[s - 1]), c, n_before, n_before / n_after,
                                xf_at<(kFeat & 1) != 0>(rec, lay, s), nullptr, branch, nullptr,
                                plate ? &gd : nullptr, n_after);
        if (st != kOk) break;
        n_before = n_after;
    }
    if (st == kOk && !(value_of(r.dz) > 0.0)) st = kBackward;
    if (st == kOk) {
        // transfer_to_image_plane on a copy
        const N z = r.pz - N(thick[S - 1]);
        const N s0 = -z / r.dz;
        out.ix = value_of(r.px + s0 * r.dx);
        out.iy = value_of(r.py + s0 * r.dy);
        out.dx = value_of(r.dx);
        out.dy = value_of(r.dy);
        out.dz = value_of(r.dz);
        const N h = N(rec[lay.target + f]);
        const N w = N(thick[S - 1]);
        int branch;
        st = e.reference == MKB_EVAL_VERTEX
                 ? reference_step<N>(r, h, w, n_before, nullptr, branch)
                 : exit_pupil_step<N>(r, h, w, N(kappa), n_before);
    }
    out.status = st;
    out.opl = value_of(r.opl);
    return out;
}

template <class N, int kFeat>
__global__ void eval_field_kernel(const __grid_constant__ EvalParams e,
                                  const double* __restrict__ records,
                                  const double* __restrict__ kappa, double* __restrict__ fr,
                                  uint8_t* __restrict__ fs, double* __restrict__ offset) {
    const int64_t id = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    const int64_t tuples = int64_t(e.t.V) * e.t.F * e.t.L;
    if (id >= tuples * kFieldRays) return;
    const int64_t t = id / kFieldRays;
    const int j = static_cast<int>(id - t * kFieldRays);
    const int v = static_cast<int>(t / (int64_t(e.t.F) * e.t.L));
    const int fl = static_cast<int>(t - int64_t(v) * e.t.F * e.t.L);
    const int f = fl / e.t.L, l = fl - f * e.t.L;
    // eval_field_ray_point: chief (0, 0), (0, +d), (0, -d), (+d, 0)
    const double x = j == 3 ? e.delta : 0.0;
    const double y = j == 1 ? e.delta : (j == 2 ? -e.delta : 0.0);
    const double* rec = records + static_cast<int64_t>(v) * e.t.stride;
    const EvalRayOut r =
        eval_ray<N, kFeat>(e, rec, v, f, l, x, y, kappa[int64_t(v) * e.t.F + f]);
    const bool ok = r.status == kOk;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    const double h = rec[layout_of(e.t).target + f];
    double* o = fr + id * kFieldValues;
    o[0] = ok ? __dsub_rn(r.ix, 0.0) : nan;
    o[1] = ok ? __dsub_rn(r.iy, h) : nan;
    o[2] = ok ? r.dx : nan;
    o[3] = ok ? r.dy : nan;
    o[4] = ok ? r.dz : nan;
    fs[id] = static_cast<uint8_t>(r.status);
    if (j == 0) offset[t] = ok ? r.opl : 0.0;
}

template <class N, int kFeat>
__global__ void eval_grid_kernel(const __grid_constant__ EvalParams e,
                                 const double* __restrict__ records,
                                 const double* __restrict__ grid,
                                 const double* __restrict__ kappa,
                                 const double* __restrict__ offset, double* __restrict__ opl_out,
                                 double* __restrict__ sx, double* __restrict__ sy,
                                 uint8_t* __restrict__ status) {
    const int64_t total = int64_t(e.t.V) * e.t.F * e.t.L * e.n;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    for (int64_t id = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; id < total;
         id += int64_t(gridDim.x) * blockDim.x) {
        const int64_t t = id / e.n;
        const int64_t k = id - t * e.n;
        const int v = static_cast<int>(t / (int64_t(e.t.F) * e.t.L));
        const int fl = static_cast<int>(t - int64_t(v) * e.t.F * e.t.L);
        const int f = fl / e.t.L, l = fl - f * e.t.L;
        const double* rec = records + static_cast<int64_t>(v) * e.t.stride;
        const EvalRayOut r = eval_ray<N, kFeat>(e, rec, v, f, l, grid[3 * k], grid[3 * k + 1],
                                             kappa[int64_t(v) * e.t.F + f]);
        const bool ok = r.status == kOk;
        const double h = rec[layout_of(e.t).target + f];
        status[id] = static_cast<uint8_t>(r.status);
        opl_out[id] = __dsub_rn(r.opl, offset[t]);
        sx[id] = ok ? __dsub_rn(r.ix, 0.0) : nan;
        sy[id] = ok ? __dsub_rn(r.iy, h) : nan;
    }
}

// One warp per tuple: the lanes load 32 consecutive points at a time (coalesced) and form the
// terms w and w * OPL (each one rounded product, as in the sequential loop); lane 0 then adds
// them in ascending point order from shared memory, so the two sums keep the reference's
// order and bits while the loads of the next 32 points are already in flight.
constexpr int kPistonWarps = 8;

__global__ void __launch_bounds__(32 * kPistonWarps)
eval_piston_kernel(int64_t tuples, int64_t n, const double* __restrict__ grid,
                   const double* __restrict__ opl, const uint8_t* __restrict__ status,
                   double* __restrict__ piston) {
    __shared__ double ws[kPistonWarps][32], ts[kPistonWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t t = blockIdx.x * int64_t(kPistonWarps) + warp;
    if (t >= tuples) return;  // warp-uniform
    double wsum = 0.0, sum = 0.0;
    for (int64_t k0 = 0; k0 < n; k0 += 32) {
        const int64_t k = k0 + lane;
        const bool ok = k < n && status[t * n + k] == kOk;  // hard failure: in piston = Ok
        const double w = ok ? grid[3 * k + 2] : 0.0;
        ws[warp][lane] = w;
        ts[warp][lane] = ok ? __dmul_rn(w, opl[t * n + k]) : 0.0;
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        __syncwarp();
        if (lane == 0) {
            for (int j = 0; j < 32; ++j) {
                if (!((mask >> j) & 1u)) continue;
                wsum = __dadd_rn(wsum, ws[warp][j]);
                sum = __dadd_rn(sum, ts[warp][j]);
            }
        }
        __syncwarp();
    }
    // piston, and NaN as the mark of a tuple without a valid ray
    if (lane == 0)
        piston[t] = wsum > 0.0 ? __ddiv_rn(sum, wsum) : __longlong_as_double(0x7ff8000000000000ll);
}

__global__ void eval_opd_kernel(int64_t total, int64_t n, const double* __restrict__ piston,
                                const uint8_t* __restrict__ status, double* __restrict__ opd) {
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    for (int64_t id = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; id < total;
         id += int64_t(gridDim.x) * blockDim.x) {
        const double pst = piston[id / n];
        opd[id] = (pst == pst && status[id] == kOk) ? __dsub_rn(opd[id], pst) : nan;
    }
}

}  // namespace

}  // namespace mkb

using namespace mkb;

extern "C" {

int mkb_eval_grid_host(int32_t size, int32_t half_pupil, double* points, int64_t* count) {
    if (size < 1 || size > MKB_MAX_EVAL_GRID || count == nullptr) {
        set_error("eval grid: size must be in [1, %d]", MKB_MAX_EVAL_GRID);
        return MKB_ERR_ARGUMENT;
    }
    const int64_t N = size;
    auto inside = [N](int64_t i, int64_t j) {
        const int64_t a = 2 * i + 1 - N, b = 2 * j + 1 - N;
        return a * a + b * b <= N * N;
    };
    int64_t full = 0;
    for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i) full += inside(i, j) ? 1 : 0;
    int64_t n = 0;
    for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i) {
            if (!inside(i, j)) continue;
            const int64_t a = 2 * i + 1 - N;
            if (half_pupil && a < 0) continue;
            if (points != nullptr) {
                points[3 * n] = static_cast<double>(a) / static_cast<double>(N);
                points[3 * n + 1] = static_cast<double>(2 * j + 1 - N) / static_cast<double>(N);
                points[3 * n + 2] = (half_pupil && a > 0 ? 2.0 : 1.0) / static_cast<double>(full);
            }
            ++n;
        }
    *count = n;
    return MKB_OK;
}

int mkb_eval_reference_host(const mkb_batch_view* view, int32_t reference,
                            int32_t paraxial_column, double* kappa, double* exit_pupil) {
    if (view == nullptr || kappa == nullptr || exit_pupil == nullptr ||
        (view->variants > 0 && (!view->curvature || !view->thickness || !view->index ||
                                !view->field_target))) {
        set_error("eval reference: null argument");
        return MKB_ERR_ARGUMENT;
    }
    if (reference < MKB_EVAL_EXIT_PUPIL || reference > MKB_EVAL_INFINITE) {
        set_error("eval reference: unknown kind %d", reference);
        return MKB_ERR_ARGUMENT;
    }
    if (paraxial_column < 0 || paraxial_column >= view->wavelengths) {
        set_error("eval reference: paraxial column %d outside [0, %d)", paraxial_column,
                  view->wavelengths);
        return MKB_ERR_ARGUMENT;
    }
    if (reference == MKB_EVAL_EXIT_PUPIL && view->ghost_plates > 0 &&
        (view->type == nullptr || view->ghost_coeff == nullptr ||
         view->ghost_norm_radius == nullptr || view->ghost_index == nullptr)) {
        set_error("eval reference: ghost plates without their data");
        return MKB_ERR_ARGUMENT;
    }
    const int V = view->variants, S = view->surfaces, L = view->wavelengths, F = view->fields;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int v = 0; v < V; ++v) {
        const double w = view->thickness[int64_t(v) * S + S - 1];
        double z_ap = 0.0;
        bool infinite = reference == MKB_EVAL_INFINITE;
        exit_pupil[v] = nan;
        if (reference == MKB_EVAL_EXIT_PUPIL) {
            // the paraxial chief ray (y0 = 0, u0 = 1) of compute_paraxial
            // (src/paraxial/paraxial.cpp:130): exit pupil at -y / u' after the last surface
            // a ghost plate is a thin element in the medium of its gap (batch_paraxial,
            // src/batch/system_batch.cpp:980): power -2 (n_G - n_m) t2 joins the surface's
            const int G = view->ghost_plates, K = view->ghost_terms;
            double y = 0.0, u = 1.0, nb = 1.0;
            for (int s = 0, g = 0; s < S; ++s) {
                const double c = view->curvature[int64_t(v) * S + s];
                const double n = view->index[(int64_t(v) * S + s) * L + paraxial_column];
                if (s > 0) y += view->thickness[int64_t(v) * S + s - 1] * u;
                double phi = c * (n - nb);
                double power = 0.0;
                if (s > 0 && G > 0 && view->type[s] == MKB_SURFACE_GHOST_PLATE && g < G) {
                    // ghost_profile_t2 and ghost_plate_power (trace/ghost_plate.hpp:95,107)
                    const double* a = view->ghost_coeff + (int64_t(v) * G + g) * K;
                    double sum = 0.0;
                    for (int k = 1; k <= K; ++k) {
                        const double term = a[k - 1] * static_cast<double>(k * (k + 1));
                        sum += (k % 2 == 1) ? term : -term;
                    }
                    const double r = view->ghost_norm_radius[g];
                    const double t2 = sum / (r * r);
                    const double n_glass =
                        view->ghost_index[(int64_t(v) * G + g) * L + paraxial_column];
                    power = -2.0 * (n_glass - n) * t2;
                    ++g;
                }
                phi += power;
                u = (nb * u - y * phi) / n;
                nb = n;
            }
            const double D = nb * u;
            infinite = D == 0.0;
            if (!infinite) {
                z_ap = -y / u;
                if (!std::isfinite(z_ap)) {
                    set_error("eval reference: exit pupil of variant %d not finite", v);
                    return MKB_ERR_ARGUMENT;
                }
                exit_pupil[v] = z_ap;
            }
        }
        for (int f = 0; f < F; ++f) {
            const double h = view->field_target[int64_t(v) * F + f];
            double k = 0.0;
            if (!infinite) {
                const double dz = w - z_ap;
                const double radius = std::hypot(h, dz);
                if (!(radius > 0.0) || !std::isfinite(radius)) {
                    if (reference == MKB_EVAL_EXIT_PUPIL) {
                        set_error("eval reference: image point in the exit pupil (variant %d, "
                                  "field %d)", v, f);
                        return MKB_ERR_ARGUMENT;
                    }
                    k = nan;
                } else {
                    k = (dz >= 0.0 ? 1.0 : -1.0) / radius;
                }
            }
            kappa[int64_t(v) * F + f] = k;
        }
    }
    return MKB_OK;
}

size_t mkb_eval_workspace_bytes(const mkb_device_batch* batch) {
    if (batch == nullptr || batch->variants < 0) return 0;
    const size_t tuples = size_t(batch->variants) * batch->fields * batch->wavelengths;
    return 2 * tuples * sizeof(double) + 256;
}

int mkb_eval_device(const mkb_device_batch* batch, int32_t reference, double field_ray_offset,
                    int32_t precision, const double* grid, int64_t n, const double* kappa,
                    double* opd, double* spot_x, double* spot_y, uint8_t* status,
                    double* field_rays, uint8_t* field_status, void* workspace,
                    size_t workspace_bytes, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    if (batch == nullptr) {
        set_error("eval: batch is null");
        return MKB_ERR_ARGUMENT;
    }
    if (reference < MKB_EVAL_EXIT_PUPIL || reference > MKB_EVAL_INFINITE) {
        set_error("eval: unknown reference %d", reference);
        return MKB_ERR_ARGUMENT;
    }
    if (precision != MKB_PRECISION_FP64 && precision != MKB_PRECISION_FP64_FMA) {
        set_error("eval: precision %d not available (FP64 or FP64_FMA)", precision);
        return MKB_ERR_UNSUPPORTED;
    }
    if (batch->variant_surfaces != nullptr) {
        set_error("eval: batches of uneven surface counts are not built (one table per batch)");
        return MKB_ERR_UNSUPPORTED;
    }
    if (!(field_ray_offset > 0.0) || !(field_ray_offset <= 0.5)) {
        set_error("eval: field ray offset must lie in (0, 0.5]");
        return MKB_ERR_ARGUMENT;
    }
    // the trace parameters of the batch: a plan with one ring, only the record layout, the
    // surface kinds and the plates are used
    const uint8_t mode = MKB_PUPIL_FULL;
    const double one = 1.0, u = 0.5, wq = 1.0;
    std::vector<uint8_t> modes(static_cast<size_t>(batch->fields > 0 ? batch->fields : 1), mode);
    std::vector<double> fw(modes.size(), one), lw(static_cast<size_t>(
                                                     batch->wavelengths > 0 ? batch->wavelengths
                                                                            : 1), one);
    const mkb_residual_plan plan{1, 1, MKB_FAILURE_HARD, MKB_PRECISION_FP64, 0.0, 500.0,
                                 batch->fields, batch->wavelengths, modes.data(), fw.data(),
                                 lw.data(), &u, &wq};
    EvalParams e;
    std::memset(&e, 0, sizeof(e));
    int rc = make_trace_params(batch, &plan, 512, &e.t);
    if (rc != MKB_OK) return rc;
    e.reference = reference;
    e.delta = field_ray_offset;
    e.n = n;
    if (e.t.V == 0) return MKB_OK;
    if (n < 1 || !grid || !kappa || !opd || !spot_x || !spot_y || !status || !field_rays ||
        !field_status) {
        set_error("eval: null output or empty grid");
        return MKB_ERR_ARGUMENT;
    }
    const int64_t tuples = int64_t(e.t.V) * e.t.F * e.t.L;
    if (workspace == nullptr || workspace_bytes < mkb_eval_workspace_bytes(batch)) {
        set_error("eval: workspace of %zu bytes needed", mkb_eval_workspace_bytes(batch));
        return MKB_ERR_WORKSPACE;
    }
    double* offset = static_cast<double*>(workspace);
    double* piston = offset + tuples;
    const int feat = (e.t.non_coaxial ? 1 : 0) | (e.t.G > 0 ? 2 : 0);
    const int64_t nf = tuples * kFieldRays;
    const unsigned fb = static_cast<unsigned>((nf + 127) / 128);
    auto launch = [&](auto feat_tag, auto num_tag) {
        constexpr int F_ = decltype(feat_tag)::value;
        using N = typename decltype(num_tag)::type;
        eval_field_kernel<N, F_><<<fb, 128, 0, stream>>>(e, batch->records, kappa, field_rays,
                                                          field_status, offset);
        eval_grid_kernel<N, F_><<<148 * 16, 128, 0, stream>>>(
            e, batch->records, grid, kappa, offset, opd, spot_x, spot_y, status);
    };
    auto by_feat = [&](auto num_tag) {
        if (feat == 0) launch(std::integral_constant<int, 0>{}, num_tag);
        else if (feat == 1) launch(std::integral_constant<int, 1>{}, num_tag);
        else if (feat == 2) launch(std::integral_constant<int, 2>{}, num_tag);
        else launch(std::integral_constant<int, 3>{}, num_tag);
    };
    if (precision == MKB_PRECISION_FP64) by_feat(NumTag<Exact64>{});
    else by_feat(NumTag<double>{});
    count_launch(2);
    eval_piston_kernel<<<static_cast<unsigned>((tuples + kPistonWarps - 1) / kPistonWarps),
                         32 * kPistonWarps, 0, stream>>>(tuples, n, grid, opd, status, piston);
    eval_opd_kernel<<<148 * 16, 256, 0, stream>>>(tuples * n, n, piston, status, opd);
    count_launch(2);
    return cuda_status(cudaGetLastError(), "eval launch");
}

}  // extern "C"
