// RESIDUALS and MERIT forward trace for sm_100a.
//
// Work decomposition: one CTA per (variant, pack). A pack is a run of consecutive tuples
// (field f, wavelength l) of one variant with at most kPackRays rays in total, fixed for the
// whole batch (the topology fixes the layout). The CTA stages its variant's record (surface
// table, indices, pupil radius, field data) into shared memory with one bulk copy, traces its
// rays (thread t takes pack rays t, t + T, ...), keeps OPL / status / penalty in shared
// memory, and then one warp per tuple reduces the piston and writes the residual rows
// (RESIDUALS) or the tuple's sum of squares (MERIT) in a fixed order: lane-strided partial
// sums in ascending sample order, then a fixed xor-shuffle tree. Results are bit-identical
// across runs, batch positions and tranches.
//
// Reference behaviour restated: residuals_kernel / merit_kernel + merit_finalize_kernel
// (src/cuda/residuals.cu:57, src/cuda/merit.cu:62,206), batch_ray_opl (merit/ray_residual.hpp:69),
// opd_statistics (merit/opd.hpp:37), ray_residual / ray_penalty (merit/ray_residual.hpp:131,199).
#include "df64.cuh"
#include "launch.cuh"
#include "pupil.cuh"

#include <cstdio>
#include <mutex>
#include <type_traits>

namespace mkb {

namespace {

constexpr int kThreads = 128;
constexpr int kRaysPerThread = 4;
constexpr int kPackRays = kThreads * kRaysPerThread;
// resident CTAs per SM the register budget is sized for (56 registers, no spills); the shared
// memory of the workloads' tables fits as many. The variants with surface transforms or ghost
// plates (feature bits 1, 2) carry more state per step and take 64 registers at 8 CTAs.
constexpr int kTraceBlocksPerSm = 9;
template <int kFeat>
constexpr int trace_blocks_per_sm = (kFeat & 3) != 0 ? 8 : kTraceBlocksPerSm;

// The variant's record (the bulk-copy destination, 16-byte aligned), the mu table and the
// pack's per-ray OPL, penalty and status live in dynamic shared memory sized for the batch
// (trace_smem): record [stride] | mu [S][L] | opl [pack_max] | pen [pack_max] |
// [FP64: piston terms w [pack_max] | w * opl [pack_max]] | status.
struct alignas(16) SharedTrace {
    uint64_t bar;
    SharedTables tab;
    int tuple_start[kMaxPackTuples + 1];
    int vs[kMaxVariantsPerCta];  // the CTA's variants (-1: not traced in this launch)
    int any;
};
static_assert(offsetof(SharedTrace, bar) % 8 == 0, "mbarrier alignment");

// Trace of one ray to the reference sphere in number type N (trace_to_reference_sphere,
// reference_sphere.hpp:181, with batch_ray_opl and collimated_ray, merit/ray_residual.hpp:69,
// trace/trace.hpp:109): returns the status, the OPL and the soft penalty.
// mu_tab[s * L + l] = n_before / n_after of the step onto surface s (divided in N).
// kExtrema: hsq[s] / cosi[s] get the squared ray height x^2 + y^2 at surface
// s and cos I = d . N (d before the refraction, N = (-c x, -c y, 1 - c z), c = 0 off spheres)
// for every surface the ray passed; surface 0 is the start point and cos I = d_z there
// (RaySurfaceRecord, trace/surface_extrema.hpp; observer calls in trace/trace.hpp:316,346).
// kImage: img gets the ray's intersection (x, y) with the image plane, thickness[S - 1] behind
// the last vertex (transfer_to_image_plane, trace/trace.hpp:402, on a copy), for rays in the
// piston.
template <class N, int kFeat, bool kExtrema = false, bool kImage = false>
__device__ inline int trace_ray(const TraceParams& p, const double* rec, const double* mu_tab,
                                const RecordLayout& lay, int S, int f, int l, const Sample& smp,
                                bool soft_mode, double& opl, double& penalty,
                                double* hsq = nullptr, double* cosi = nullptr,
                                double* img = nullptr) {
    const int L = p.L;
    const N zero(0.0);
    const N a = rec[lay.pupil];
    const N st = rec[lay.sin_theta + f];
    const N ct = rec[lay.cos_theta + f];
    const N r0 = a * N(smp.rho);
    RayT<N> r;
    r.px = r0 * N(smp.sin_phi);
    r.py = r0 * N(smp.cos_phi);
    r.pz = zero;
    r.dx = zero;
    r.dy = st;
    r.dz = ct;
    r.opl = r.py * st;  // p . d with p_z = d_x = 0
    SoftT<N> soft{zero, kOk};
    SoftT<N>* sp = soft_mode ? &soft : nullptr;
    int status = kOk;
    if constexpr (kExtrema) {
        hsq[0] = value_of(r.px * r.px + r.py * r.py);
        cosi[0] = value_of(r.dz);
    }
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    N n_before = idx[l];
    for (int s = 1; s < S; ++s) {
        const N n_after = idx[s * L + l];
        const N c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        int branch;
        GhostData gd;
        const bool plate = ghost_at<(kFeat & 2) != 0>(p, rec, lay, s, l, gd);
        const N dbx = r.dx, dby = r.dy, dbz = r.dz;  // direction before the refraction
        status = step_surface_xf<N>(r, N(thick[s - 1]), c, n_before, N(mu_tab[s * L + l]),
                                    xf_at<(kFeat & 1) != 0>(rec, lay, s), sp, branch, nullptr,
                                    plate ? &gd : nullptr, n_after);
        if (status != kOk) break;
        if constexpr (kExtrema) {
            const double* xs = xf_at<(kFeat & 1) != 0>(rec, lay, s);
            if (xs != nullptr && xs[6] > 0.0) {
                // a decentered or tilted surface: height and incidence in its own frame -- the
                // state taken back into it and the direction before the step rotated into it
                // (trace_segment's observer, trace/trace.hpp:330)
                const Transform<N> tr = transform_at<N>(xs);
                RayT<N> loc = r;
                ray_to_surface(loc, tr);
                N ux = dbx, uy = dby, uz = dbz;
                rotate_to(tr, ux, uy, uz);
                hsq[s] = value_of(loc.px * loc.px + loc.py * loc.py);
                const N nx = -c * loc.px, ny = -c * loc.py, nz = N(1.0) - c * loc.pz;
                cosi[s] = value_of(ux * nx + uy * ny + uz * nz);
            } else {
                hsq[s] = value_of(r.px * r.px + r.py * r.py);
                const N nx = -c * r.px, ny = -c * r.py, nz = N(1.0) - c * r.pz;
                cosi[s] = value_of(dbx * nx + dby * ny + dbz * nz);
            }
        }
        n_before = n_after;
    }
    if (status == kOk && soft_mode) status = soft.first;
    if (in_piston(status)) {
        if (!(r.dz > zero)) {
            status = kBackward;
        } else {
            if constexpr (kImage) {
                const N z = r.pz - N(thick[S - 1]);
                const N s0 = -z / r.dz;
                img[0] = value_of(r.px + s0 * r.dx);
                img[1] = value_of(r.py + s0 * r.dy);
            }
            int branch;
            const int rst = reference_step<N>(r, N(rec[lay.target + f]), N(thick[S - 1]),
                                              n_before, sp, branch);
            if (!in_piston(rst)) status = rst;
            else if (status == kOk) status = rst;
        }
    }
    opl = value_of(r.opl);
    penalty = value_of(soft.penalty);
    return status;
}

// trace_ray in MKB_PRECISION_FP32_BULK (coaxial, no ghost plates): the start ray and the
// surface loop with step_surface_bulk, the reference sphere in FP64.
__device__ inline int trace_ray_bulk(const TraceParams& p, const double* rec, const double* mu_tab,
                                     const RecordLayout& lay, int S, int f, int l,
                                     const Sample& smp, bool soft_mode, double& opl,
                                     double& penalty) {
    const int L = p.L;
    const double a = rec[lay.pupil];
    const double st = rec[lay.sin_theta + f];
    const double ct = rec[lay.cos_theta + f];
    const double r0 = a * smp.rho;
    RayBulk r;
    r.px = r0 * smp.sin_phi;
    r.py = r0 * smp.cos_phi;
    r.pz = 0.0;
    r.dx = 0.0f;
    r.dy = static_cast<float>(st);
    r.dz = static_cast<float>(ct);
    r.opl = r.py * st;  // p . d with p_z = d_x = 0 (the exact start direction)
    SoftT<double> soft{0.0, kOk};
    SoftT<double>* sp = soft_mode ? &soft : nullptr;
    int status = kOk;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    double n_before = idx[l];
    for (int s = 1; s < S; ++s) {
        const double c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        int branch;
        status = step_surface_bulk(r, thick[s - 1], c, n_before,
                                   static_cast<float>(mu_tab[s * L + l]), sp, branch);
        if (status != kOk) break;
        n_before = idx[s * L + l];
    }
    if (status == kOk && soft_mode) status = soft.first;
    if (in_piston(status)) {
        if (!(r.dz > 0.0f)) {
            status = kBackward;
        } else {
            int branch;
            const int rst = reference_step_bulk(r, rec[lay.target + f], thick[S - 1], n_before,
                                                sp, branch);
            if (!in_piston(rst)) status = rst;
            else if (status == kOk) status = rst;
        }
    }
    opl = r.opl;
    penalty = soft.penalty;
    return status;
}

__device__ inline double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ inline int warp_sum_int(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct TupleOut {
    double* residuals;  // RESIDUALS: [V][stride]
    int64_t stride;
    double* opd;        // [V][rays] or null
    uint8_t* status;    // [V][rays] or null
    double* part;       // MERIT: [V][n_tuples] tuple sums
    int* part_failed;   // MERIT: [V][n_tuples]
    int* part_hard;     // MERIT: [V][n_tuples]
    RunMask mask;       // variants to trace
    unsigned long long* extrema;  // [V][S][2] order-preserving keys of (x^2 + y^2, cos I), or null
};

// Order-preserving keys: a larger key is a larger double (bits of a non-negative value, all
// bits flipped for a negative one), so the maximum and minimum over rays are integer atomics
// and do not depend on their order, as extremum_max / extremum_min do not.
__device__ inline unsigned long long order_key(double x) {
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ inline double key_value(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double(static_cast<long long>(b));
}

// kExact: per-ray arithmetic in Exact64 and every tuple sum sequential in ascending sample
// order (opd_statistics, merit/opd.hpp:37; variant_merit, src/batch/batch_merit.cpp:12), so
// RESIDUALS and MERIT equal the reference CPU results bit for bit. Otherwise contracted FP64
// with lane-strided sums and a fixed shuffle tree (deterministic, not bit-identical to CPU).
// kMulti: the CTA takes p.vpc variants side by side (built for coaxial batches without ghost
// plates); otherwise one variant, with the leaner indexing of that case.
template <bool kResiduals, int kPrecision, int kFeat, bool kExtrema = false, bool kMulti = false>
__global__ void __launch_bounds__(kThreads, trace_blocks_per_sm<kFeat>)
trace_kernel(const __grid_constant__ TraceParams p, const double* __restrict__ records,
             TupleOut out) {
    constexpr bool kExact = kPrecision == MKB_PRECISION_FP64;
    using N = typename std::conditional<
        kExact, Exact64,
        typename std::conditional<kPrecision == MKB_PRECISION_DF64, Df64, double>::type>::type;
    __shared__ SharedTrace sh;
    // this CTA: pack pk of the variants in queue slots group * vpc .. + nv - 1
    const int vpc = kMulti ? p.vpc : 1;
    const int group = blockIdx.x / p.n_packs;
    const int pk = blockIdx.x - group * p.n_packs;
    const int slot0 = group * vpc;
    const int nv = kMulti ? (p.V - slot0 < vpc ? p.V - slot0 : vpc) : 1;
    int* vs = sh.vs;
    if (threadIdx.x == 0) {
        int any = 0;
        for (int j = 0; j < nv; ++j) {
            const int slot = slot0 + j;
            int v = p.order != nullptr ? p.order[slot] : slot;
            if (!run_active(out.mask, v)) v = -1;
            vs[j] = v;
            any |= v >= 0;
        }
        sh.any = any;
    }
    __syncthreads();
    if (!sh.any) return;
    const Pack pack = p.packs[pk];
    const RecordLayout lay = layout_of(p);
    if (threadIdx.x <= pack.tuples) {
        int start = 0;
        for (int t = 0; t < static_cast<int>(threadIdx.x); ++t) {
            const int tu = pack.first_tuple + t;
            start += p.sample_count[tu / p.L];
        }
        sh.tuple_start[threadIdx.x] = start;
    }
    copy_tables(p, sh.tab);
    // dynamic shared memory: per variant of the CTA its record and mu table (rec_sh doubles),
    // then the per-ray arrays of all its packs (nv * pack.rays entries each)
    extern __shared__ __align__(16) double dyn[];
    const int rec_sh = p.stride + ((p.S * p.L + 1) & ~1);
    const int span = vpc * p.pack_max;
    double* opl_sh = dyn + vpc * rec_sh;     // [span]
    double* pen_sh = opl_sh + span;          // [span]
    double* w_sh = pen_sh + span;            // FP64 only: [span] piston weights
    double* ws_sh = w_sh + (kExact ? span : 0);  // FP64 only: [span] w * opl
    uint8_t* status_sh = reinterpret_cast<uint8_t*>(kExact ? ws_sh + span : w_sh);
    if constexpr (kMulti) {
        const double* src[kMaxVariantsPerCta];
        for (int j = 0; j < nv; ++j)
            src[j] = vs[j] >= 0 ? records + static_cast<int64_t>(vs[j]) * p.stride : nullptr;
        if (!stage_records(dyn, rec_sh, src, nv,
                           static_cast<uint32_t>(p.stride * sizeof(double)), &sh.bar))
            return;
    } else {
        if (!stage_to_shared(dyn, records + static_cast<int64_t>(vs[0]) * p.stride,
                             static_cast<uint32_t>(p.stride * sizeof(double)), &sh.bar))
            return;
    }
    const int S0 = surfaces_of(p, vs[0] >= 0 ? vs[0] : 0);
    const bool soft_mode = p.failure == MKB_FAILURE_SOFT;
    // mu of every step and wavelength, divided once per CTA as the step would divide it
    for (int i = threadIdx.x; i < nv * p.S * p.L; i += kThreads) {
        const int j = i / (p.S * p.L), sl = i - j * p.S * p.L;
        const int s = sl / p.L, l = sl - s * p.L;
        if (vs[j] < 0) continue;
        const double* record = dyn + j * rec_sh;
        dyn[j * rec_sh + p.stride + sl] = s >= 1 && s < (kMulti ? surfaces_of(p, vs[j]) : S0)
                                    ? value_of(N(record[lay.index + (s - 1) * p.L + l]) /
                                               N(record[lay.index + s * p.L + l]))
                                    : 0.0;
    }
    __syncthreads();

    // per-CTA extrema of the pack's valid rays (keys; surface s at [2s], [2s + 1])
    unsigned long long* ext_sh = nullptr;
    if constexpr (kExtrema) {
        __shared__ unsigned long long ext_keys[2 * kMaxSurfaces];
        ext_sh = ext_keys;
        for (int i = threadIdx.x; i < p.S; i += kThreads) {
            ext_keys[2 * i] = order_key(0.0);      // height^2 0 (neutral_height_sq)
            ext_keys[2 * i + 1] = order_key(1.0);  // cos I = 1 (neutral_cos_incidence)
        }
        __syncthreads();
    }

    // ---- phase 1: trace (ray ii = variant j's pack ray i) -------------------------------
    auto trace_one = [&](int j, int i, int ii) {
        const int S = kMulti ? surfaces_of(p, vs[j]) : S0;
        const double* record = dyn + j * rec_sh;
        const double* mu_tab = record + p.stride;
        int t = 0;
        while (t + 1 < pack.tuples && i >= sh.tuple_start[t + 1]) ++t;
        const int tu = pack.first_tuple + t;
        const int f = tu / p.L;
        const int l = tu - f * p.L;
        const int k = i - sh.tuple_start[t];
        const Sample smp = pupil_sample(p, sh.tab, f, k);
        double opl, pen;
        int st;
        if constexpr (kExtrema) {
            double hsq[kMaxSurfaces], cosi[kMaxSurfaces];
            st = trace_ray<N, kFeat, true>(p, record, mu_tab, lay, S, f, l, smp, soft_mode, opl,
                                           pen, hsq, cosi);
            if (st == kOk)  // only valid rays count (SurfaceExtrema::add_ray)
                for (int q = 0; q < S; ++q) {
                    if (hsq[q] == hsq[q]) atomicMax(&ext_sh[2 * q], order_key(hsq[q]));
                    if (cosi[q] == cosi[q]) atomicMin(&ext_sh[2 * q + 1], order_key(cosi[q]));
                }
        } else if constexpr (kPrecision == MKB_PRECISION_FP32_BULK) {
            st = trace_ray_bulk(p, record, mu_tab, lay, S, f, l, smp, soft_mode, opl, pen);
        } else {
            st = trace_ray<N, kFeat>(p, record, mu_tab, lay, S, f, l, smp, soft_mode, opl, pen);
        }
        opl_sh[ii] = opl;
        pen_sh[ii] = pen;
        status_sh[ii] = static_cast<uint8_t>(st);
    };
    if constexpr (kMulti) {
        // (j, i) advanced without a division per ray
        int j = static_cast<int>(threadIdx.x) / pack.rays;
        int i = static_cast<int>(threadIdx.x) - j * pack.rays;
        for (int ii = threadIdx.x; ii < nv * pack.rays; ii += kThreads) {
            const int jj = j, ir = i;
            i += kThreads;
            while (i >= pack.rays) {
                i -= pack.rays;
                ++j;
            }
            if (vs[jj] >= 0) trace_one(jj, ir, ii);
        }
    } else {
        for (int i = threadIdx.x; i < pack.rays; i += kThreads) trace_one(0, i, i);
    }
    __syncthreads();

    if constexpr (kExtrema) {
        const int S = surfaces_of(p, vs[0]);
        unsigned long long* g = out.extrema + static_cast<int64_t>(vs[0]) * p.S * 2;
        for (int q = threadIdx.x; q < S; q += kThreads) {
            atomicMax(&g[2 * q], ext_sh[2 * q]);
            atomicMin(&g[2 * q + 1], ext_sh[2 * q + 1]);
        }
    }

    // ---- phase 2: one warp per (variant, tuple) ------------------------------------------
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int v0 = vs[0];
    for (int tt = warp; tt < nv * pack.tuples; tt += kThreads / 32) {
        const int j = kMulti ? tt / pack.tuples : 0;
        const int t = tt - j * pack.tuples;
        const int v = kMulti ? vs[j] : v0;
        if (kMulti && v < 0) continue;
        const int tu = pack.first_tuple + t;
        const int f = tu / p.L;
        const int l = tu - f * p.L;
        const int n = p.sample_count[f];
        const int base = j * pack.rays + sh.tuple_start[t];
        const int64_t row0 = p.field_offset[f] + static_cast<int64_t>(l) * n;  // in the variant
        // piston: valid weight and weighted OPL sum over the rays in the piston
        double vw = 0.0, vs_ = 0.0;
        if (kExact) {
            // Every lane forms its samples' terms w_k and w_k * OPL_k (one rounded product, as
            // the sequential loop forms it; +0 for rays outside the piston, which leaves the
            // sums' bits unchanged: both start at +0 and never become -0), then lane 0 adds
            // them in ascending k: the dependent additions are all it executes alone.
            for (int k = lane; k < n; k += 32) {
                const bool in = in_piston(status_sh[base + k]);
                const N w = in ? N(pupil_sample(p, sh.tab, f, k).weight) : N(0.0);
                w_sh[base + k] = value_of(w);
                ws_sh[base + k] = in ? value_of(w * N(opl_sh[base + k])) : 0.0;
            }
            __syncwarp();
            if (lane == 0) {
                N w_acc(0.0), s_acc(0.0);
                for (int k = 0; k < n; ++k) {
                    w_acc += N(w_sh[base + k]);
                    s_acc += N(ws_sh[base + k]);
                }
                vw = value_of(w_acc);
                vs_ = value_of(s_acc);
            }
            vw = __shfl_sync(0xffffffffu, vw, 0);
            vs_ = __shfl_sync(0xffffffffu, vs_, 0);
        } else {
            for (int k = lane; k < n; k += 32) {
                if (in_piston(status_sh[base + k])) {
                    const Sample smp = pupil_sample(p, sh.tab, f, k);
                    vw += smp.weight;
                    vs_ += smp.weight * opl_sh[base + k];
                }
            }
            vw = warp_sum(vw);
            vs_ = warp_sum(vs_);
        }
        const bool valid = vw > 0.0;
        const N piston = valid ? value_of(N(vs_) / N(vw)) : 0.0;
        const N scale = p.scale[tu];
        const N pscale = p.pscale[tu];
        double sq = 0.0, psq = 0.0;
        int failed = 0, hard = 0;
        for (int k = lane; k < n; k += 32) {
            const int st = status_sh[base + k];
            const Sample smp = pupil_sample(p, sh.tab, f, k);
            const N e = (valid && in_piston(st)) ? N(opl_sh[base + k]) - piston : N(0.0);
            const N rw = smp.root_weight;
            const N r = scale * rw * e;
            N pr(0.0);
            if (soft_mode) {
                const N fp = st == kOk ? N(0.0)
                             : is_soft(st) ? N(pen_sh[base + k])
                                           : N(pen_sh[base + k]) + N(1.0);
                pr = pscale * rw * fp;
            }
            failed += st != kOk;
            hard += !in_piston(st);
            if (kResiduals) {
                const int64_t row = static_cast<int64_t>(v) * out.stride + row0 + k;
                out.residuals[row] = value_of(r);
                if (soft_mode) out.residuals[row + p.rays] = value_of(pr);
                const int64_t ray = static_cast<int64_t>(v) * p.rays + row0 + k;
                if (out.opd) out.opd[ray] = value_of(e);
                if (out.status) out.status[ray] = static_cast<uint8_t>(st);
            } else if (kExact) {
                // each lane rewrites only its own samples, with the rounded squares
                opl_sh[base + k] = value_of(r * r);
                pen_sh[base + k] = value_of(pr * pr);
            } else {
                sq += value_of(r * r);
                psq += value_of(pr * pr);
            }
        }
        if (!kResiduals) {
            if (kExact) {
                __syncwarp();
                if (lane == 0) {  // sum_k r_k^2, then sum_k p_k^2, in ascending k
                    N tuple(0.0), pen(0.0);
                    for (int k = 0; k < n; ++k) tuple += N(opl_sh[base + k]);
                    if (soft_mode) {
                        for (int k = 0; k < n; ++k) pen += N(pen_sh[base + k]);
                        tuple += pen;
                    }
                    sq = value_of(tuple);
                }
            } else {
                sq = warp_sum(sq);
                psq = warp_sum(psq);
                sq += psq;
            }
            failed = warp_sum_int(failed);
            hard = warp_sum_int(hard);
            if (lane == 0) {
                const int64_t slot = static_cast<int64_t>(v) * p.n_tuples + tu;
                out.part[slot] = sq;
                out.part_failed[slot] = failed;
                out.part_hard[slot] = hard;
            }
        }
    }
}

// Transverse ray-error rows (plan transverse_weight > 0): one CTA per (variant, tuple) traces
// the tuple's rays again with their image-plane intersection and writes the rows
// r_x = t_s sqrt(W) (x - 0), r_y = t_s sqrt(W) (y - h_f) (0 for rays that failed hard) after
// the ray and penalty rows (RESIDUALS), or adds sum_k r_x^2, then sum_k r_y^2, in ascending k
// to the tuple's MERIT partial sum. The arithmetic and the status of every ray are those of
// trace_kernel.
template <int kPrecision, int kFeat, bool kResiduals>
__global__ void __launch_bounds__(kThreads)
transverse_kernel(const __grid_constant__ TraceParams p, const double* __restrict__ records,
                  TupleOut out) {
    constexpr bool kExact = kPrecision == MKB_PRECISION_FP64;
    using N = typename std::conditional<kExact, Exact64, double>::type;
    __shared__ SharedTables tab;
    const int slot = blockIdx.x / p.n_tuples;
    const int tu = blockIdx.x - slot * p.n_tuples;
    const int v = p.order != nullptr ? p.order[slot] : slot;
    if (!run_active(out.mask, v)) return;
    copy_tables(p, tab);
    extern __shared__ __align__(16) double dyn[];
    double* mu_tab = dyn;                              // [S][L]
    double* sq = dyn + ((p.S * p.L + 1) & ~1);         // MERIT: [2 n] squares
    const int S = surfaces_of(p, v);
    const RecordLayout lay = layout_of(p);
    const double* rec = records + static_cast<int64_t>(v) * p.stride;
    for (int i = threadIdx.x; i < S * p.L; i += kThreads) {
        const int s = i / p.L, l = i - s * p.L;
        mu_tab[i] = s >= 1 ? value_of(N(rec[lay.index + (s - 1) * p.L + l]) /
                                      N(rec[lay.index + s * p.L + l]))
                           : 0.0;
    }
    __syncthreads();
    const int f = tu / p.L, l = tu - f * p.L;
    const int n = p.sample_count[f];
    const int64_t row0 = p.field_offset[f] + static_cast<int64_t>(l) * n;
    const bool soft_mode = p.failure == MKB_FAILURE_SOFT;
    const int64_t base = static_cast<int64_t>(p.rays) * (soft_mode ? 2 : 1);
    const N ts = p.tscale[tu];
    const N h = rec[lay.target + f];
    for (int k = threadIdx.x; k < n; k += kThreads) {
        const Sample smp = pupil_sample(p, tab, f, k);
        double opl, pen, img[2] = {0.0, 0.0};
        const int st = trace_ray<N, kFeat, false, true>(p, rec, mu_tab, lay, S, f, l, smp,
                                                        soft_mode, opl, pen, nullptr, nullptr,
                                                        img);
        const bool in = in_piston(st);
        const N ex = in ? N(img[0]) - N(0.0) : N(0.0);
        const N ey = in ? N(img[1]) - h : N(0.0);
        const N rw = smp.root_weight;
        const N rx = ts * rw * ex, ry = ts * rw * ey;
        if constexpr (kResiduals) {
            const int64_t row = static_cast<int64_t>(v) * out.stride + base + row0 + k;
            out.residuals[row] = value_of(rx);
            out.residuals[row + p.rays] = value_of(ry);
        } else {
            sq[k] = value_of(rx * rx);
            sq[n + k] = value_of(ry * ry);
        }
    }
    if constexpr (!kResiduals) {
        __syncthreads();
        if (threadIdx.x == 0) {
            N tx(0.0), ty(0.0);
            for (int k = 0; k < n; ++k) tx += N(sq[k]);
            for (int k = 0; k < n; ++k) ty += N(sq[n + k]);
            const int64_t slot_t = static_cast<int64_t>(v) * p.n_tuples + tu;
            N part = out.part[slot_t];
            part += tx;
            part += ty;
            out.part[slot_t] = value_of(part);
        }
    }
}

template <bool kResiduals>
int launch_transverse(const TraceParams& p, const double* records, const TupleOut& out,
                      int precision, cudaStream_t stream) {
    if (!p.transverse || p.V == 0) return MKB_OK;
    if (precision == MKB_PRECISION_DF64 || precision == MKB_PRECISION_FP32_BULK) {
        set_error("transverse rows: not built for DF64 or FP32_BULK");
        return MKB_ERR_UNSUPPORTED;
    }
    int max_n = 0;
    for (int f = 0; f < p.F; ++f) max_n = p.sample_count[f] > max_n ? p.sample_count[f] : max_n;
    const size_t smem = (static_cast<size_t>((p.S * p.L + 1) & ~1) +
                         (kResiduals ? 0 : 2 * static_cast<size_t>(max_n))) * sizeof(double);
    const int feat = (p.non_coaxial ? 1 : 0) | (p.G > 0 ? 2 : 0);
    constexpr int E = MKB_PRECISION_FP64, F = MKB_PRECISION_FP64_FMA;
    auto kernel = precision == MKB_PRECISION_FP64
                      ? (feat == 0   ? transverse_kernel<E, 0, kResiduals>
                         : feat == 1 ? transverse_kernel<E, 1, kResiduals>
                         : feat == 2 ? transverse_kernel<E, 2, kResiduals>
                                     : transverse_kernel<E, 3, kResiduals>)
                      : (feat == 0   ? transverse_kernel<F, 0, kResiduals>
                         : feat == 1 ? transverse_kernel<F, 1, kResiduals>
                         : feat == 2 ? transverse_kernel<F, 2, kResiduals>
                                     : transverse_kernel<F, 3, kResiduals>);
    if (smem > 48 * 1024) {
        const int rc = cuda_status(cudaFuncSetAttribute(
                                       kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)),
                                   "transverse rows: shared memory attribute");
        if (rc != MKB_OK) return rc;
    }
    const unsigned blocks = static_cast<unsigned>(static_cast<int64_t>(p.V) * p.n_tuples);
    kernel<<<blocks, kThreads, smem, stream>>>(p, records, out);
    count_launch();
    return cuda_status(cudaGetLastError(), "transverse rows launch");
}

// merit[v] = sum over tuples in order (f-major, then l); counts likewise.
// Extrema output [V][S][2]: neutral keys before the trace, then the values (sqrt of the largest
// height^2, smallest cos I) in place.
__global__ void extrema_init_kernel(unsigned long long* keys, int64_t n, RunMask mask, int S) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        if (!run_active(mask, static_cast<int>(i / (2 * S)))) continue;
        keys[i] = (i & 1) ? order_key(1.0) : order_key(0.0);
    }
}

__global__ void extrema_finalize_kernel(unsigned long long* keys, int64_t n, RunMask mask,
                                        int S) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        if (!run_active(mask, static_cast<int>(i / (2 * S)))) continue;
        const double x = key_value(keys[i]);
        reinterpret_cast<double*>(keys)[i] = (i & 1) ? x : __dsqrt_rn(x);
    }
}

// extra [V] (or null): added after the tuple sums (MeritRunOptions::extra_merit,
// src/cuda/merit.cu:222).
__global__ void merit_finalize_kernel(int V, int n_tuples, const double* part,
                                      const int* part_failed, const int* part_hard,
                                      double* merit, int64_t* failed, int64_t* hard,
                                      RunMask mask, const double* extra) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V || !run_active(mask, v)) return;
    double sum = 0.0;
    int64_t nf = 0, nh = 0;
    const int64_t o = static_cast<int64_t>(v) * n_tuples;
    for (int t = 0; t < n_tuples; ++t) {
        sum = __dadd_rn(sum, part[o + t]);
        nf += part_failed[o + t];
        nh += part_hard[o + t];
    }
    if (extra != nullptr) sum = __dadd_rn(sum, extra[v]);
    merit[v] = sum;
    failed[v] = nf;
    hard[v] = nh;
}

// dynamic shared memory of trace_kernel: the record (stride is even), the mu table and the
// pack's per-ray OPL, penalty and status
size_t trace_smem(const TraceParams& p, bool exact) {
    const size_t rec_sh =
        static_cast<size_t>(p.stride) + ((static_cast<size_t>(p.S) * p.L + 1) & ~size_t(1));
    const size_t span = static_cast<size_t>(p.vpc) * p.pack_max;
    return (p.vpc * rec_sh + (exact ? 4 : 2) * span) * sizeof(double) + ((span + 15) & ~size_t(15));
}

// Launches trace_kernel<kResiduals, precision> (MIXED traces in FP64 with contraction; its FP32
// part is the reverse sweep) with the dynamic shared memory the batch needs.
template <bool kResiduals>
int launch_trace(const TraceParams& p_in, const double* records, const TupleOut& out,
                 int precision, cudaStream_t stream) {
    TraceParams p = p_in;
    // several variants per CTA: built for coaxial batches without ghost plates in FP64; the
    // others trace one variant per CTA (the option only shapes the launch)
    if (p.non_coaxial || p.G > 0 || precision == MKB_PRECISION_DF64 ||
        precision == MKB_PRECISION_FP32_BULK)
        p.vpc = 1;
    const int64_t groups = (static_cast<int64_t>(p.V) + p.vpc - 1) / p.vpc;
    const unsigned blocks = static_cast<unsigned>(groups * p.n_packs);
    const size_t smem = trace_smem(p, precision == MKB_PRECISION_FP64);
    // kernel variant per precision and features (1: surface transforms, 2: ghost plates)
    const int feat = (p.non_coaxial ? 1 : 0) | (p.G > 0 ? 2 : 0);
    constexpr int E = MKB_PRECISION_FP64, F = MKB_PRECISION_FP64_FMA;
    constexpr int D = MKB_PRECISION_DF64;
    constexpr int B = MKB_PRECISION_FP32_BULK;
    if (precision == B && (feat != 0 || out.extrema != nullptr)) {
        set_error("trace: FP32_BULK is built for coaxial batches without ghost plates or "
                  "extrema");
        return MKB_ERR_UNSUPPORTED;
    }
    auto kernel = precision == B ? trace_kernel<kResiduals, B, 0>
                  : p.vpc > 1 ? (precision == MKB_PRECISION_FP64
                                   ? trace_kernel<kResiduals, E, 0, false, true>
                                   : trace_kernel<kResiduals, F, 0, false, true>)
                  : precision == MKB_PRECISION_DF64
                      ? (feat == 0   ? trace_kernel<kResiduals, D, 0>
                         : feat == 1 ? trace_kernel<kResiduals, D, 1>
                         : feat == 2 ? trace_kernel<kResiduals, D, 2>
                                     : trace_kernel<kResiduals, D, 3>)
                  : precision == MKB_PRECISION_FP64
                      ? (feat == 0   ? trace_kernel<kResiduals, E, 0>
                         : feat == 1 ? trace_kernel<kResiduals, E, 1>
                         : feat == 2 ? trace_kernel<kResiduals, E, 2>
                                     : trace_kernel<kResiduals, E, 3>)
                      : (feat == 0   ? trace_kernel<kResiduals, F, 0>
                         : feat == 1 ? trace_kernel<kResiduals, F, 1>
                         : feat == 2 ? trace_kernel<kResiduals, F, 2>
                                     : trace_kernel<kResiduals, F, 3>);
    const int64_t n_ext = static_cast<int64_t>(p.V) * p.S * 2;
    if (out.extrema != nullptr) {
        // per-surface extrema: one variant per CTA, FP64 / FP64_FMA / DF64 (a decentered or
        // tilted surface's in its own frame)
        if (p.vpc != 1) {
            set_error("trace: extrema need one variant per CTA");
            return MKB_ERR_UNSUPPORTED;
        }
        kernel = precision == MKB_PRECISION_FP64
                     ? (feat == 0   ? trace_kernel<kResiduals, E, 0, true>
                        : feat == 1 ? trace_kernel<kResiduals, E, 1, true>
                        : feat == 2 ? trace_kernel<kResiduals, E, 2, true>
                                    : trace_kernel<kResiduals, E, 3, true>)
                 : precision == MKB_PRECISION_DF64
                     ? (feat == 0   ? trace_kernel<kResiduals, D, 0, true>
                        : feat == 1 ? trace_kernel<kResiduals, D, 1, true>
                        : feat == 2 ? trace_kernel<kResiduals, D, 2, true>
                                    : trace_kernel<kResiduals, D, 3, true>)
                     : (feat == 0   ? trace_kernel<kResiduals, F, 0, true>
                        : feat == 1 ? trace_kernel<kResiduals, F, 1, true>
                        : feat == 2 ? trace_kernel<kResiduals, F, 2, true>
                                    : trace_kernel<kResiduals, F, 3, true>);
        extrema_init_kernel<<<592, 256, 0, stream>>>(out.extrema, n_ext, out.mask, p.S);
        count_launch();
    }
    if (p.vpc > 1) {  // the caller's choice must fit: larger ones are refused, not clamped
        int dev = 0, optin = 0;
        int rc = cuda_status(cudaGetDevice(&dev), "trace: cudaGetDevice");
        if (rc == MKB_OK)
            rc = cuda_status(cudaDeviceGetAttribute(&optin,
                                                    cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                             "trace: shared memory limit");
        if (rc != MKB_OK) return rc;
        if (smem + sizeof(SharedTrace) > static_cast<size_t>(optin)) {
            set_error("trace: %d variants per CTA need %zu bytes of shared memory, the device "
                      "has %d per block", p.vpc, smem, optin);
            return MKB_ERR_ARGUMENT;
        }
    }
    if (smem > 48 * 1024) {
        const cudaError_t err = cudaFuncSetAttribute(
            kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (err != cudaSuccess) return cuda_status(err, "trace: shared memory attribute");
    }
    kernel<<<blocks, kThreads, smem, stream>>>(p, records, out);
    count_launch();
    if (out.extrema != nullptr) {
        extrema_finalize_kernel<<<592, 256, 0, stream>>>(out.extrema, n_ext, out.mask, p.S);
        count_launch();
    }
    return cuda_status(cudaGetLastError(), kResiduals ? "residuals kernel launch"
                                                      : "merit kernel launch");
}

size_t merit_workspace(int V, int n_tuples) {
    const size_t slots = static_cast<size_t>(V) * n_tuples;
    return slots * (sizeof(double) + 2 * sizeof(int)) + 256;
}

}  // namespace

int launch_residuals(const TraceParams& p, const double* records, double* residuals,
                     int64_t stride, double* opd, uint8_t* status, int precision,
                     cudaStream_t stream, RunMask mask, double* extrema) {
    TupleOut out{residuals, stride, opd, status, nullptr, nullptr, nullptr, mask,
                 reinterpret_cast<unsigned long long*>(extrema)};
    const int rc = launch_trace<true>(p, records, out, precision, stream);
    if (rc != MKB_OK) return rc;
    return launch_transverse<true>(p, records, out, precision, stream);
}

int launch_merit(const TraceParams& p, const double* records, double* merit, int64_t* failed,
                 int64_t* hard, void* workspace, size_t ws_bytes, int precision,
                 cudaStream_t stream, RunMask mask, const double* extra, double* extrema) {
    const size_t need = merit_workspace(p.V, p.n_tuples);
    if (workspace == nullptr || ws_bytes < need) {
        set_error("merit: workspace of %zu bytes needed, %zu given", need, ws_bytes);
        return MKB_ERR_WORKSPACE;
    }
    const size_t slots = static_cast<size_t>(p.V) * p.n_tuples;
    char* ws = static_cast<char*>(workspace);
    TupleOut out{nullptr, 0, nullptr, nullptr, reinterpret_cast<double*>(ws),
                 reinterpret_cast<int*>(ws + slots * sizeof(double)),
                 reinterpret_cast<int*>(ws + slots * (sizeof(double) + sizeof(int))), mask,
                 reinterpret_cast<unsigned long long*>(extrema)};
    int rc = launch_trace<false>(p, records, out, precision, stream);
    if (rc != MKB_OK) return rc;
    rc = launch_transverse<false>(p, records, out, precision, stream);
    if (rc != MKB_OK) return rc;
    merit_finalize_kernel<<<(p.V + 255) / 256, 256, 0, stream>>>(
        p.V, p.n_tuples, out.part, out.part_failed, out.part_hard, merit, failed, hard, mask,
        extra);
    count_launch();
    return cuda_status(cudaGetLastError(), "merit finalize launch");
}

size_t merit_workspace_bytes(int V, int n_tuples) { return merit_workspace(V, n_tuples); }

// ---- MERIT without a caller workspace --------------------------------------------------------
// Some callers cannot allocate device memory: a host application that hands the library a
// fixed pool at start-up and owns every other byte of the GPU, or a tight optimisation loop
// that must never stall in cudaMalloc. For them MERIT keeps its per-tuple partial sums in this
// array, which lives in the library's own device image: every GPU that loads the library holds
// it (4 MiB + 256 B) until the process exits. All calls share it, so two calls that overlap on
// the GPU (different streams, or different host threads on one device) race; the caller runs
// one at a time per device. Nothing in it needs to start at zero: each call writes every
// partial sum before the finalize kernel reads it.
constexpr int64_t kNoAllocMeritSlots = MKB_NOALLOC_MERIT_MAX_SLOTS;
constexpr size_t kNoAllocScratchBytes =
    static_cast<size_t>(kNoAllocMeritSlots) * (sizeof(double) + 2 * sizeof(int)) + 256;
static __device__ __align__(256) unsigned char g_noalloc_merit_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_address[kMaxDevices] = {};
}  // namespace

// Device address of the scratch array in the current context. In host code the array's name
// is only a host-side stand-in, so the address is looked up with the device current. The array
// lives in the module loaded into each CUDA context, so an address found once is not kept for
// good: every call made outside a stream capture looks it up again (the lookup allocates
// nothing), which also covers a caller that switches to a non-primary context or resets the
// device between calls. A call made while `stream` is being captured cannot look anything up
// and uses the address that the last call outside a capture found on this device.
int noalloc_merit_scratch(cudaStream_t stream, void** out) {
    int dev = 0;
    int rc = cuda_status(cudaGetDevice(&dev), "no-allocation MERIT: cudaGetDevice");
    if (rc != MKB_OK) return rc;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("no-allocation MERIT: device %d out of range", dev);
        return MKB_ERR_ARGUMENT;
    }
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    rc = cuda_status(cudaStreamIsCapturing(stream, &capture),
                     "no-allocation MERIT: cudaStreamIsCapturing");
    if (rc != MKB_OK) return rc;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (capture == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        rc = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_merit_scratch),
                         "no-allocation MERIT: cudaGetSymbolAddress");
        if (rc != MKB_OK) return rc;
        g_noalloc_address[dev] = p;
    } else if (g_noalloc_address[dev] == nullptr) {
        set_error("no-allocation MERIT: first call on device %d made during a stream capture; "
                  "make one call outside the capture first", dev);
        return MKB_ERR_ARGUMENT;
    }
    *out = g_noalloc_address[dev];
    return MKB_OK;
}

int pack_rays_default() { return kPackRays; }

MKB_DEFINE_ERROR_READER(trace_device_error)

}  // namespace mkb

// No counterpart in the reference: MERIT for callers that cannot allocate device memory.
extern "C" int mkb_merit_noalloc_device(const mkb_device_batch* batch,
                                        const mkb_residual_plan* plan, double* merit,
                                        int64_t* failed, int64_t* hard_failed, void* stream) {
    using namespace mkb;
    TraceParams p;
    int rc = make_trace_params(batch, plan, pack_rays_default(), &p);
    if (rc != MKB_OK) return rc;
    if (plan->precision != MKB_PRECISION_FP64 && plan->precision != MKB_PRECISION_FP64_FMA &&
        plan->precision != MKB_PRECISION_MIXED) {
        set_error("no-allocation MERIT: precision %d not available", plan->precision);
        return MKB_ERR_UNSUPPORTED;
    }
    if (p.V == 0) return MKB_OK;
    if (!merit || !failed || !hard_failed) {
        set_error("no-allocation MERIT: output is null");
        return MKB_ERR_ARGUMENT;
    }
    const int64_t slots = static_cast<int64_t>(p.V) * p.n_tuples;
    if (slots > kNoAllocMeritSlots) {
        set_error("no-allocation MERIT: %d variants x %d tuples = %lld partial sums exceed the "
                  "built-in limit of %lld; split the batch or use mkb_merit_device",
                  p.V, p.n_tuples, static_cast<long long>(slots),
                  static_cast<long long>(kNoAllocMeritSlots));
        return MKB_ERR_ARGUMENT;
    }
    void* scratch = nullptr;
    rc = noalloc_merit_scratch(static_cast<cudaStream_t>(stream), &scratch);
    if (rc != MKB_OK) return rc;
    return launch_merit(p, batch->records, merit, failed, hard_failed, scratch,
                        kNoAllocScratchBytes, plan->precision,
                        static_cast<cudaStream_t>(stream));
}
