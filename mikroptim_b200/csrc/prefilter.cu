// FP32 prefilter of multistart variants for sm_100a: a float trace with per-ray margins, the
// per-variant sums of the certainly valid rays, and the conservative keep / reject decision.
//
// Work decomposition as the FP64 trace (trace.cu): one CTA per (variant, pack of tuples), the
// variant's record staged into shared memory by one bulk copy, thread t tracing pack rays t,
// t + 128, ... Every ray is traced in Exact32 (separately rounded float operations, correctly
// rounded division and square root) in the reference's order of operations, with the margin
// observer of its trace; then one warp per tuple forms the per-ray terms and lane 0 adds them
// in ascending sample order, as the reference's CPU loop does. A finalize kernel adds the
// tuples of a variant in (field, wavelength) order. The per-variant results therefore equal
// prefilter_stats_cpu bit for bit.
//
// Reference behaviour restated: prefilter_ray, PrefilterMarginObserver, prefilter_surface_failure,
// prefilter_opl_offset (include/mikroptim/merit/prefilter_ray.hpp:37-259), variant_stats,
// prefilter_decide, prefilter_decide_exact (src/batch/batch_prefilter.cpp:140-360), the kernel
// of src/cuda/prefilter.cu:87 and its finalize at :193.
//
// The prefilter's values only select variants for an FP64 evaluation; they never enter a
// merit, a residual, a Jacobian or the optimiser.
#include "launch.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

namespace mkb {

namespace {

constexpr int kThreads = 128;
constexpr int kPackRays = 512;

// Ray classes (src/cuda/prefilter.cu:44)
enum : uint8_t { kCertainOk = 0, kCertainFailed = 1, kUncertainOk = 2, kUncertainFailed = 3 };

// Float pupil tables, formed on the host as the reference's float quadrature forms them
// (sample, pupil/quadrature.hpp:71, with R = float: rho = sqrtf(u), weight = w / M,
// phi = (2j + 1) pi / (2M) or / M, and sinf / cosf of phi).
struct PrefilterTables {
    float rho[kMaxRings];
    float w_axis[kMaxRings], rw_axis[kMaxRings];
    float w_spoke[kMaxRings], rw_spoke[kMaxRings];
    float sin_half[kMaxSpokes], cos_half[kMaxSpokes];
    float sin_full[kMaxSpokes], cos_full[kMaxSpokes];
    float scale[kMaxTuples];  // residual_scale rounded to float
    float eta;                // boundary
};

struct PrefilterOut {
    double* part_sum;   // [V][n_tuples] float tuple sums (as double)
    float* part_len;    // [V][n_tuples] largest optical length of a certainly valid ray
    int* part_count;    // [V][n_tuples][3] certainly failed, uncertain valid, uncertain failed
};

struct SampleF {
    float rho, weight, root_weight, sin_phi, cos_phi;
};

__device__ inline SampleF sample_f(const TraceParams& p, const PrefilterTables& q, int f, int k) {
    SampleF s;
    const int mode = p.pupil_mode[f];
    if (mode == MKB_PUPIL_AXIS) {
        s.rho = q.rho[k];
        s.weight = q.w_axis[k];
        s.root_weight = q.rw_axis[k];
        s.sin_phi = 0.0f;  // sinf(0), cosf(0)
        s.cos_phi = 1.0f;
    } else {
        const int i = k / p.spokes;
        const int j = k - i * p.spokes;
        s.rho = q.rho[i];
        s.weight = q.w_spoke[i];
        s.root_weight = q.rw_spoke[i];
        s.sin_phi = mode == MKB_PUPIL_HALF ? q.sin_half[j] : q.sin_full[j];
        s.cos_phi = mode == MKB_PUPIL_HALF ? q.cos_half[j] : q.cos_full[j];
    }
    return s;
}

// prefilter_min_margin: the smaller value; NaN gives 0 ("uncertain")
__device__ __forceinline__ Exact32 min_margin(Exact32 acc, Exact32 x) {
    if (x.v < acc.v) return x;
    return x.v >= acc.v ? acc : Exact32(0.0f);
}
// prefilter_failure_linear / prefilter_failure_root (NaN gives 0)
__device__ __forceinline__ Exact32 failure_linear(Exact32 x) {
    return -x.v > 0.0f ? Exact32(-x.v) : Exact32(0.0f);
}
__device__ __forceinline__ Exact32 failure_root(Exact32 q) {
    return -q.v > 0.0f ? nsqrt(Exact32(-q.v)) : Exact32(0.0f);
}
__device__ __forceinline__ Exact32 larger(Exact32 a, Exact32 b) { return a.v > b.v ? a : b; }

// prefilter_surface_failure: the size of the violated test at surface fs from the state the
// trace returned in (Backward before the transfer, Missed in the tangent plane, TIR at the
// intersection point with the direction before the refraction, or in a ghost plate's plane).
template <int kFeat>
__device__ inline Exact32 surface_failure(const TraceParams& p, const double* rec,
                                          const RecordLayout& lay, int l, int fs, int st,
                                          const RayT<Exact32>& r) {
    using N = Exact32;
    const N one(1.0f);
    const int L = p.L;
    if (st == kBackward) return failure_linear(r.dz);
    const N c = p.type[fs] == MKB_SURFACE_SPHERE ? N(rec[lay.curvature + fs]) : N(0.0f);
    if (st == kMissed) {
        const N H = c * (r.px * r.px + r.py * r.py);
        const N B = r.dz - c * (r.px * r.dx + r.py * r.dy);
        const N D = B * B - c * H;
        return larger(failure_root(D), failure_linear(B));
    }
    if (st == kTir) {
        const N n_before = N(rec[lay.index + (fs - 1) * L + l]);
        const N n_after = N(rec[lay.index + fs * L + l]);
        GhostData gd;
        if (ghost_at<(kFeat & 2) != 0>(p, rec, lay, fs, l, gd)) {
            const N radius = gd.radius;
            const N inv_r2 = one / (radius * radius);
            const N u = (r.px * r.px + r.py * r.py) * inv_r2;
            N prof_t, dt_du;
            ghost_profile<N>(gd, u, prof_t, dt_du);
            const N dn = N(gd.n_glass) - n_before;
            const N radial = dn * dt_du * N(2.0f) * inv_r2;
            const N dx = (n_before * r.dx + radial * r.px) / n_after;
            const N dy = (n_before * r.dy + radial * r.py) / n_after;
            return failure_root(one - dx * dx - dy * dy);
        }
        const N nx = -c * r.px, ny = -c * r.py, nz = one - c * r.pz;
        const N cos_i = r.dx * nx + r.dy * ny + r.dz * nz;
        const N mu = n_before / n_after;
        return failure_root(one - mu * mu * (one - cos_i * cos_i));
    }
    return one;  // Unsupported depends on the topology only
}

// prefilter_ray: the collimated start ray, the trace with the margin observer (hard failure),
// d_z > 0 after the last refraction, and the step onto the reference sphere about
// (0, h_f, w) with its own margins. Returns the status; opl is OPL - offset (valid for Ok).
template <int kFeat>
__device__ inline int prefilter_trace(const TraceParams& p, const double* rec,
                                      const float* mu_tab, const RecordLayout& lay, int S, int f,
                                      int l, const SampleF& smp, float sin_t, float cos_t,
                                      float offset, float& opl, float& margin_out) {
    using N = Exact32;
    const N zero(0.0f), one(1.0f), two(2.0f);
    const int L = p.L;
    const N a = N(rec[lay.pupil]);
    const N r0 = a * N(smp.rho);
    RayT<N> r;
    r.px = r0 * N(smp.sin_phi);
    r.py = r0 * N(smp.cos_phi);
    r.pz = zero;
    r.dx = zero;
    r.dy = N(sin_t);
    r.dz = N(cos_t);
    r.opl = (r.px * r.dx + r.py * r.dy) + r.pz * r.dz;  // dot(p, d)
    r.opl -= N(offset);
    N margin = one;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    N n_before = N(idx[l]);
    int status = kOk, fs = -1;
    for (int s = 1; s < S; ++s) {
        const N n_after = N(idx[s * L + l]);
        const N c = p.type[s] == MKB_SURFACE_SPHERE ? N(curv[s]) : zero;
        GhostData gd;
        const bool plate = ghost_at<(kFeat & 2) != 0>(p, rec, lay, s, l, gd);
        const double* xf = xf_at<(kFeat & 1) != 0>(rec, lay, s);
        N ex = r.dx, ey = r.dy, ez = r.dz;  // direction before the step
        int branch;
        status = step_surface_xf<N>(r, N(thick[s - 1]), c, n_before, N(mu_tab[s * L + l]), xf,
                                    nullptr, branch, nullptr, plate ? &gd : nullptr, n_after);
        if (status != kOk) {
            fs = s;
            break;
        }
        // PrefilterMarginObserver::surface in the surface's own frame
        RayT<N> loc = r;
        if constexpr ((kFeat & 1) != 0) {
            if (xf[6] > 0.0) {
                const Transform<N> tr = transform_at<N>(xf);
                ray_to_surface(loc, tr);
                rotate_to(tr, ex, ey, ez);
            }
        }
        const N nx = -c * loc.px, ny = -c * loc.py, nz = one - c * loc.pz;
        margin = min_margin(margin, ez);
        margin = min_margin(margin, ex * nx + ey * ny + ez * nz);
        margin = min_margin(margin, loc.dx * nx + loc.dy * ny + loc.dz * nz);
        n_before = n_after;
    }
    opl = 0.0f;
    if (status != kOk) {
        margin_out = value_of(surface_failure<kFeat>(p, rec, lay, l, fs, status, r));
        return status;
    }
    if (!(r.dz > zero)) {
        margin_out = value_of(failure_linear(r.dz));
        return kBackward;
    }
    margin = min_margin(margin, r.dz);
    // the reference sphere's tests (the expressions of reference_sphere_step)
    const N h = N(rec[lay.target + f]);
    const N w = N(thick[S - 1]);
    const N r2 = (zero * zero + h * h) + w * w;
    const N inv_r = r2 > zero ? one / nsqrt(r2) : one;
    const N qx = r.px - zero, qy = r.py - h, qz = r.pz - w;
    const N bq = -(qx * r.dx + qy * r.dy + qz * r.dz);
    const N g = r.px * (r.px - two * zero) + r.py * (r.py - two * h) + r.pz * (r.pz - two * w);
    const N disc = bq * bq - g;
    const N sigma = w >= zero ? one : N(-1.0f);
    const N root = disc > zero ? nsqrt(disc) : zero;
    const N denom = sigma * (bq + sigma * root) * inv_r;
    int branch;
    const int rst = reference_step<N>(r, h, w, n_before, nullptr, branch);
    if (rst != kOk) {
        const N ma = failure_root(disc * inv_r * inv_r);
        const N mc = disc >= zero ? failure_linear(denom) : zero;
        margin_out = value_of(larger(ma, mc));
        return rst;
    }
    margin = min_margin(margin, root * inv_r);
    margin = min_margin(margin, denom);
    opl = value_of(r.opl);
    margin_out = value_of(margin);
    return kOk;
}

template <int kFeat>
__global__ void __launch_bounds__(kThreads)
prefilter_kernel(const __grid_constant__ TraceParams p, const __grid_constant__ PrefilterTables q,
                 const double* __restrict__ records, const float* __restrict__ field_trig,
                 PrefilterOut out) {
    __shared__ __align__(8) uint64_t bar;
    __shared__ int tuple_start[kMaxPackTuples + 1];
    const int v = blockIdx.x / p.n_packs;
    const int pk = blockIdx.x - v * p.n_packs;
    const int S = surfaces_of(p, v);
    const Pack pack = p.packs[pk];
    const RecordLayout lay = layout_of(p);
    if (threadIdx.x <= pack.tuples) {
        int start = 0;
        for (int t = 0; t < static_cast<int>(threadIdx.x); ++t)
            start += p.sample_count[(pack.first_tuple + t) / p.L];
        tuple_start[threadIdx.x] = start;
    }
    extern __shared__ __align__(16) double dyn[];
    double* record = dyn;                                      // [stride]
    float* mu_tab = reinterpret_cast<float*>(dyn + p.stride);  // [S][L]
    float* offset = mu_tab + p.S * p.L;                        // [L]
    float* opl_sh = offset + p.L;                              // [pack_max]
    float* t1_sh = opl_sh + p.pack_max;                        // [pack_max] terms
    float* t2_sh = t1_sh + p.pack_max;                         // [pack_max] terms
    uint8_t* cls_sh = reinterpret_cast<uint8_t*>(t2_sh + p.pack_max);
    if (!stage_to_shared(record, records + static_cast<int64_t>(v) * p.stride,
                         static_cast<uint32_t>(p.stride * sizeof(double)), &bar))
        return;
    for (int i = threadIdx.x; i < S * p.L; i += kThreads) {
        const int s = i / p.L, l = i - s * p.L;
        mu_tab[i] = s >= 1 ? value_of(Exact32(record[lay.index + (s - 1) * p.L + l]) /
                                      Exact32(record[lay.index + s * p.L + l]))
                           : 0.0f;
    }
    // prefilter_opl_offset: sum_{s <= S-2} n_s t_s in ascending s, per wavelength
    for (int l = threadIdx.x; l < p.L; l += kThreads) {
        Exact32 sum(0.0f);
        for (int s = 0; s + 1 < S; ++s)
            sum += Exact32(record[lay.index + s * p.L + l]) * Exact32(record[lay.thickness + s]);
        offset[l] = value_of(sum);
    }
    __syncthreads();
    const float eta = q.eta;

    // ---- phase 1: trace every ray of the pack -----------------------------------------------
    for (int i = threadIdx.x; i < pack.rays; i += kThreads) {
        int t = 0;
        while (t + 1 < pack.tuples && i >= tuple_start[t + 1]) ++t;
        const int tu = pack.first_tuple + t;
        const int f = tu / p.L;
        const int l = tu - f * p.L;
        const int k = i - tuple_start[t];
        const SampleF smp = sample_f(p, q, f, k);
        const float* trig = field_trig + (static_cast<int64_t>(v) * p.F + f) * 2;
        float opl, margin;
        const int st = prefilter_trace<kFeat>(p, record, mu_tab, lay, S, f, l, smp, trig[0],
                                              trig[1], offset[l], opl, margin);
        const bool certain = margin > eta;
        cls_sh[i] = st == kOk ? (certain ? kCertainOk : kUncertainOk)
                              : (certain ? kCertainFailed : kUncertainFailed);
        opl_sh[i] = opl;
    }
    __syncthreads();

    // ---- phase 2: one warp per tuple ------------------------------------------------------
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    for (int t = warp; t < pack.tuples; t += kThreads / 32) {
        const int tu = pack.first_tuple + t;
        const int f = tu / p.L;
        const int l = tu - f * p.L;
        const int n = p.sample_count[f];
        const int base = tuple_start[t];
        const Exact32 off_abs(fabsf(offset[l]));
        // terms of the piston sums (0 for rays outside the set: the sums start at +0 and the
        // additions of +0 leave them unchanged), the optical length and the counts
        float len_max = 0.0f;
        int c_failed = 0, c_uok = 0, c_ufail = 0;
        for (int k = lane; k < n; k += 32) {
            const uint8_t c = cls_sh[base + k];
            const float w = sample_f(p, q, f, k).weight;
            const float o = opl_sh[base + k];
            t1_sh[base + k] = c == kCertainOk ? w : 0.0f;
            t2_sh[base + k] = c == kCertainOk ? value_of(Exact32(w) * Exact32(o)) : 0.0f;
            if (c == kCertainOk) {
                const float len = value_of(off_abs + Exact32(fabsf(o)));
                len_max = len > len_max ? len : len_max;
            }
            c_failed += c == kCertainFailed;
            c_uok += c == kUncertainOk;
            c_ufail += c == kUncertainFailed;
        }
        __syncwarp();
        float w_ok = 0.0f, w_opl = 0.0f;
        if (lane == 0) {
            Exact32 a(0.0f), b(0.0f);
            for (int k = 0; k < n; ++k) {
                a += Exact32(t1_sh[base + k]);
                b += Exact32(t2_sh[base + k]);
            }
            w_ok = value_of(a);
            w_opl = value_of(b);
        }
        w_ok = __shfl_sync(0xffffffffu, w_ok, 0);
        w_opl = __shfl_sync(0xffffffffu, w_opl, 0);
        const bool valid = w_ok > 0.0f;
        const Exact32 piston = valid ? Exact32(w_opl) / Exact32(w_ok) : Exact32(0.0f);
        const Exact32 scale(q.scale[tu]);
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            const bool ok = valid && cls_sh[base + k] == kCertainOk;
            const Exact32 e = ok ? Exact32(opl_sh[base + k]) - piston : Exact32(0.0f);
            const Exact32 r = scale * Exact32(sample_f(p, q, f, k).root_weight) * e;
            t1_sh[base + k] = value_of(r * r);
        }
        __syncwarp();
        float sum = 0.0f;
        if (lane == 0) {
            Exact32 acc(0.0f);
            for (int k = 0; k < n; ++k) acc += Exact32(t1_sh[base + k]);
            sum = value_of(acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float other = __shfl_xor_sync(0xffffffffu, len_max, o);
            len_max = other > len_max ? other : len_max;
            c_failed += __shfl_xor_sync(0xffffffffu, c_failed, o);
            c_uok += __shfl_xor_sync(0xffffffffu, c_uok, o);
            c_ufail += __shfl_xor_sync(0xffffffffu, c_ufail, o);
        }
        if (lane == 0) {
            const int64_t slot = static_cast<int64_t>(v) * p.n_tuples + tu;
            out.part_sum[slot] = static_cast<double>(sum);
            out.part_len[slot] = len_max;
            out.part_count[3 * slot] = c_failed;
            out.part_count[3 * slot + 1] = c_uok;
            out.part_count[3 * slot + 2] = c_ufail;
        }
        __syncwarp();
    }
}

// Per variant: merit = sum of the tuple sums in (f, l) order (double), the largest optical
// length, and the counts (variant_stats, src/batch/batch_prefilter.cpp:140).
__global__ void prefilter_finalize_kernel(int V, int n_tuples, PrefilterOut in, double* merit,
                                          double* optical, int64_t* failed, int64_t* uok,
                                          int64_t* ufail) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int64_t o = static_cast<int64_t>(v) * n_tuples;
    double sum = 0.0;
    float len = 0.0f;
    int64_t a = 0, b = 0, c = 0;
    for (int t = 0; t < n_tuples; ++t) {
        sum = __dadd_rn(sum, in.part_sum[o + t]);
        const float x = in.part_len[o + t];
        len = x > len ? x : len;
        a += in.part_count[3 * (o + t)];
        b += in.part_count[3 * (o + t) + 1];
        c += in.part_count[3 * (o + t) + 2];
    }
    merit[v] = sum;
    optical[v] = static_cast<double>(len);
    failed[v] = a;
    uok[v] = b;
    ufail[v] = c;
}

size_t prefilter_smem(const TraceParams& p) {
    return static_cast<size_t>(p.stride) * sizeof(double) +
           (static_cast<size_t>(p.S) * p.L + p.L + 3 * static_cast<size_t>(p.pack_max)) *
               sizeof(float) +
           ((static_cast<size_t>(p.pack_max) + 15) & ~size_t(15));
}

size_t prefilter_workspace(int V, int n_tuples) {
    const size_t slots = static_cast<size_t>(V) * n_tuples;
    return slots * (sizeof(double) + sizeof(float) + 3 * sizeof(int)) + 256;
}

int tuples_of(const mkb_residual_plan* plan) {
    return plan != nullptr ? plan->fields * plan->wavelengths : 0;
}

}  // namespace

MKB_DEFINE_ERROR_READER(prefilter_device_error)

}  // namespace mkb

using namespace mkb;

extern "C" {

size_t mkb_prefilter_workspace_bytes(int32_t variants, const mkb_residual_plan* plan) {
    if (variants < 0 || plan == nullptr) return 0;
    return prefilter_workspace(variants, tuples_of(plan));
}

int mkb_prefilter_field_trig_host(const mkb_batch_view* view, float* field_trig) {
    if (view == nullptr || field_trig == nullptr || (view->variants > 0 && !view->field_angle)) {
        set_error("prefilter field trig: null argument");
        return MKB_ERR_ARGUMENT;
    }
    const int64_t n = static_cast<int64_t>(view->variants) * view->fields;
    for (int64_t i = 0; i < n; ++i) {
        const float theta = static_cast<float>(view->field_angle[i]);
        field_trig[2 * i] = std::sin(theta);  // the float overloads: sinf, cosf
        field_trig[2 * i + 1] = std::cos(theta);
    }
    return MKB_OK;
}

int mkb_prefilter_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                         const float* field_trig, double boundary, double* merit,
                         double* optical_length, int64_t* failed, int64_t* uncertain_ok,
                         int64_t* uncertain_failed, void* workspace, size_t workspace_bytes,
                         void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    TraceParams p;
    int rc = make_trace_params(batch, plan, kPackRays, &p);
    if (rc != MKB_OK) return rc;
    if (!(boundary >= 0.0) || !std::isfinite(boundary)) {
        set_error("prefilter: boundary must be finite and >= 0, got %g", boundary);
        return MKB_ERR_ARGUMENT;
    }
    if (p.V == 0) return MKB_OK;
    if (!field_trig || !merit || !optical_length || !failed || !uncertain_ok ||
        !uncertain_failed) {
        set_error("prefilter: null output or field table");
        return MKB_ERR_ARGUMENT;
    }
    const size_t need = prefilter_workspace(p.V, p.n_tuples);
    if (workspace == nullptr || workspace_bytes < need) {
        set_error("prefilter: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
        return MKB_ERR_WORKSPACE;
    }
    PrefilterTables q;
    std::memset(&q, 0, sizeof(q));
    const float pi = static_cast<float>(3.14159265358979323846264338327950288);
    for (int i = 0; i < plan->rings; ++i) {
        const float u = static_cast<float>(plan->quad_u[i]);
        const float w = static_cast<float>(plan->quad_w[i]);
        q.rho[i] = std::sqrt(u);
        q.w_axis[i] = w / 1.0f;
        q.rw_axis[i] = std::sqrt(q.w_axis[i]);
        q.w_spoke[i] = w / static_cast<float>(plan->spokes);
        q.rw_spoke[i] = std::sqrt(q.w_spoke[i]);
    }
    for (int j = 0; j < plan->spokes; ++j) {
        const float half = static_cast<float>(2 * j + 1) * pi / static_cast<float>(2 * plan->spokes);
        const float full = static_cast<float>(2 * j + 1) * pi / static_cast<float>(plan->spokes);
        q.sin_half[j] = std::sin(half);
        q.cos_half[j] = std::cos(half);
        q.sin_full[j] = std::sin(full);
        q.cos_full[j] = std::cos(full);
    }
    for (int t = 0; t < p.n_tuples; ++t) q.scale[t] = static_cast<float>(p.scale[t]);
    q.eta = static_cast<float>(boundary);
    const size_t slots = static_cast<size_t>(p.V) * p.n_tuples;
    char* ws = static_cast<char*>(workspace);
    PrefilterOut out{reinterpret_cast<double*>(ws),
                     reinterpret_cast<float*>(ws + slots * sizeof(double)),
                     reinterpret_cast<int*>(ws + slots * (sizeof(double) + sizeof(float)))};
    const int feat = (p.non_coaxial ? 1 : 0) | (p.G > 0 ? 2 : 0);
    auto kernel = feat == 0   ? prefilter_kernel<0>
                  : feat == 1 ? prefilter_kernel<1>
                  : feat == 2 ? prefilter_kernel<2>
                              : prefilter_kernel<3>;
    const size_t smem = prefilter_smem(p);
    if (smem > 48 * 1024) {
        rc = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)),
                         "prefilter: shared memory attribute");
        if (rc != MKB_OK) return rc;
    }
    const unsigned blocks = static_cast<unsigned>(static_cast<int64_t>(p.V) * p.n_packs);
    kernel<<<blocks, kThreads, smem, stream>>>(p, q, batch->records, field_trig, out);
    count_launch();
    rc = cuda_status(cudaGetLastError(), "prefilter kernel launch");
    if (rc != MKB_OK) return rc;
    prefilter_finalize_kernel<<<(p.V + 255) / 256, 256, 0, stream>>>(
        p.V, p.n_tuples, out, merit, optical_length, failed, uncertain_ok, uncertain_failed);
    count_launch();
    return cuda_status(cudaGetLastError(), "prefilter finalize launch");
}

void mkb_prefilter_default_options(mkb_prefilter_options* o) {
    if (o == nullptr) return;
    o->max_failed_fraction = 0.5;
    o->max_merit = std::numeric_limits<double>::infinity();
    o->max_merit_factor = std::numeric_limits<double>::infinity();
    o->boundary = 0.15;
    o->opl_error_factor = 32.0;
    o->merit_relative = 0.01;
}

namespace {

// check_prefilter_options (src/batch/batch_prefilter.cpp:40-60)
int check_criteria(const mkb_prefilter_options* o) {
    if (o == nullptr) {
        set_error("prefilter: options are null");
        return MKB_ERR_ARGUMENT;
    }
    if (!(o->max_failed_fraction >= 0.0) || !(o->max_merit >= 0.0) ||
        !(o->max_merit_factor >= 0.0)) {
        set_error("prefilter: max_failed_fraction, max_merit and max_merit_factor must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    return MKB_OK;
}

int check_margins(const mkb_prefilter_options* o) {
    if (!(o->boundary >= 0.0) || !std::isfinite(o->boundary)) {
        set_error("prefilter: boundary must be finite and >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (!(o->opl_error_factor >= 0.0) || !std::isfinite(o->opl_error_factor)) {
        set_error("prefilter: opl_error_factor must be finite and >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (!(o->merit_relative >= 0.0 && o->merit_relative < 1.0)) {
        set_error("prefilter: merit_relative must lie in [0, 1)");
        return MKB_ERR_ARGUMENT;
    }
    return MKB_OK;
}

bool too_many_failed(int64_t failed, int64_t rays, double fraction) {
    return static_cast<double>(failed) > fraction * static_cast<double>(rays);
}

}  // namespace

int mkb_prefilter_decide_host(const mkb_residual_plan* plan, const mkb_prefilter_options* o,
                              int32_t V, const double* merit, const double* optical_length,
                              const int64_t* failed, const int64_t* uncertain_ok,
                              const int64_t* uncertain_failed, const double* extra_merit,
                              double* merit_lower, double* merit_upper, uint8_t* reject,
                              double* reference_merit, int32_t* reference_variant,
                              int32_t* kept) {
    int rc = check_criteria(o);
    if (rc == MKB_OK) rc = check_margins(o);
    if (rc != MKB_OK) return rc;
    double scale[kMaxTuples];
    rc = residual_scales(plan, scale);
    if (rc != MKB_OK) return rc;
    if (V < 0 || (V > 0 && (!merit || !optical_length || !failed || !uncertain_ok ||
                            !uncertain_failed || !merit_lower || !merit_upper || !reject)) ||
        !reference_merit || !reference_variant || !kept) {
        set_error("prefilter decide: null argument");
        return MKB_ERR_ARGUMENT;
    }
    int64_t R = 0;
    for (int f = 0; f < plan->fields; ++f)
        R += static_cast<int64_t>(plan->wavelengths) *
             (plan->pupil_mode[f] == MKB_PUPIL_AXIS ? plan->rings : plan->rings * plan->spokes);
    // sqrt(sum_(f,l) s^2) in (f, l) order
    double scale_sq = 0.0;
    for (int t = 0; t < plan->fields * plan->wavelengths; ++t) scale_sq += scale[t] * scale[t];
    const double scale_norm = std::sqrt(scale_sq);
    const double inf = std::numeric_limits<double>::infinity();
    const bool soft = plan->failure == MKB_FAILURE_SOFT;
    constexpr double kUnitRoundoff = 0x1p-24;
    for (int v = 0; v < V; ++v) {
        const double root = std::sqrt(std::max(merit[v], 0.0));
        const double delta = o->opl_error_factor * kUnitRoundoff * optical_length[v] * scale_norm;
        const double lower = std::max(0.0, root - delta) / (1.0 + o->merit_relative);
        const double upper = (root + delta) / (1.0 - o->merit_relative);
        const double extra = extra_merit != nullptr ? extra_merit[v] : 0.0;
        merit_lower[v] = lower * lower + extra;
        const bool finite = std::isfinite(root) && std::isfinite(delta);
        const bool penalties = soft && failed[v] > 0;
        const bool uncertain = uncertain_ok[v] + uncertain_failed[v] != 0;
        merit_upper[v] = !uncertain && finite && !penalties ? upper * upper + extra : inf;
        if (!finite) merit_lower[v] = extra;
        reject[v] = MKB_PREFILTER_KEEP;
        if (too_many_failed(failed[v], R, o->max_failed_fraction))
            reject[v] |= MKB_PREFILTER_FAILED_RAYS;
        if (merit_lower[v] > o->max_merit) reject[v] |= MKB_PREFILTER_MERIT_ABSOLUTE;
    }
    *reference_merit = inf;
    *reference_variant = -1;
    if (std::isfinite(o->max_merit_factor)) {
        for (int v = 0; v < V; ++v) {
            if (uncertain_ok[v] + uncertain_failed[v] != 0 ||
                (reject[v] & MKB_PREFILTER_FAILED_RAYS) != 0 || failed[v] >= R)
                continue;
            if (merit_upper[v] < *reference_merit) {
                *reference_merit = merit_upper[v];
                *reference_variant = v;
            }
        }
        if (*reference_variant >= 0) {
            const double limit = o->max_merit_factor * *reference_merit;
            for (int v = 0; v < V; ++v)
                if (merit_lower[v] > limit) reject[v] |= MKB_PREFILTER_MERIT_RELATIVE;
        }
    }
    int32_t n = 0;
    for (int v = 0; v < V; ++v) n += reject[v] == MKB_PREFILTER_KEEP;
    *kept = n;
    return MKB_OK;
}

int mkb_prefilter_decide_exact_host(const mkb_prefilter_options* o, int32_t V,
                                    int64_t rays_per_variant, const double* merit,
                                    const int64_t* failed, const double* extra_merit,
                                    uint8_t* reject) {
    const int rc = check_criteria(o);
    if (rc != MKB_OK) return rc;
    if (V < 0 || (V > 0 && (!merit || !failed || !reject))) {
        set_error("prefilter decide exact: null argument");
        return MKB_ERR_ARGUMENT;
    }
    const int64_t R = rays_per_variant;
    double best = std::numeric_limits<double>::infinity();
    for (int v = 0; v < V; ++v) {
        const double m = merit[v] + (extra_merit != nullptr ? extra_merit[v] : 0.0);
        const bool too_many = too_many_failed(failed[v], R, o->max_failed_fraction);
        reject[v] = MKB_PREFILTER_KEEP;
        if (too_many) reject[v] |= MKB_PREFILTER_FAILED_RAYS;
        if (m > o->max_merit) reject[v] |= MKB_PREFILTER_MERIT_ABSOLUTE;
        if (!too_many && failed[v] < R && m < best) best = m;
    }
    if (std::isfinite(o->max_merit_factor) && std::isfinite(best)) {
        const double limit = o->max_merit_factor * best;
        for (int v = 0; v < V; ++v)
            if (merit[v] + (extra_merit != nullptr ? extra_merit[v] : 0.0) > limit)
                reject[v] |= MKB_PREFILTER_MERIT_RELATIVE;
    }
    return MKB_OK;
}

}  // extern "C"
