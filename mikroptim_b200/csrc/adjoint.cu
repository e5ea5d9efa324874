// Adjoint Jacobian of the trace rows for sm_100a (materialised J).
//
// Per ray (one thread): a forward trace that keeps only checkpoints -- the ray state (p, d)
// after every K-th surface -- and a 2-bit soft-failure branch code per surface; then a
// reverse sweep that, segment by segment from the last, replays the K surfaces of the segment
// from its checkpoint (same arithmetic, so the same states bit for bit) and back-propagates
// through them, writing dOPL/dx (seed opl = 1) and, for rays with a soft event, the scaled
// d(penalty)/dx (seed penalty = 1) into the run's Jacobian columns. A second kernel applies the
// piston projection per tuple and variable:
//     J_k = s sqrt(W_k) (g_k - sum_j W_j g_j / W_ok)   (rays in the piston, ascending j)
// Reference: adjoint_jacobian_kernel (src/cuda/adjoint_jacobian.cu:118), backward_ray and
// ray_gradient_rows (trace/adjoint_backward.hpp:495, merit/ray_jacobian.hpp:92), projection in
// adjoint_jacobian_cpu (src/optim/adjoint_jacobian.cpp:449). The reference keeps the full
// per-surface record in local memory (49 B per surface and ray); here only every K-th state
// is kept and the rest is recomputed (checkpointing).
#include "adjoint.cuh"
#include "pupil.cuh"

#include <type_traits>

namespace mkb {

namespace {

constexpr int kAdjThreads = 128;
constexpr int kInterval = 4;                               // K, surfaces per checkpoint segment
constexpr int kMaxCheckpoints = kMaxSurfaces / kInterval + 1;

struct AdjointParams {
    TraceParams t;
    VarParams v;
    int64_t rows;  // R = trace rows per run (J column length)
};

struct alignas(16) SharedAdj {
    double record[2 * kMaxSurfaces + kMaxSurfaces * MKB_MAX_WAVELENGTHS + 1 + 3 * kMaxFields + 1];
    uint64_t bar;
    SharedTables tab;
    int tuple_start[kMaxPackTuples + 1];
};
static_assert(offsetof(SharedAdj, record) % 16 == 0, "bulk-copy destination alignment");

// Forward record of one ray: checkpoints of (p, d) after surfaces 0, K, 2K, ... and the
// branch code of every surface (2 bits, 64 surfaces in 128 bits).
template <class N>
struct Record {
    Vec<N> p[kMaxCheckpoints];
    Vec<N> d[kMaxCheckpoints];
    uint64_t branch_lo, branch_hi;
    int count;         // states 0 .. count-1 passed (count = S when every surface was passed)
    int image_branch;  // branch of the reference-sphere step
    __device__ void set_branch(int s, int b) {
        if (s < 32) branch_lo |= static_cast<uint64_t>(b) << (2 * s);
        else branch_hi |= static_cast<uint64_t>(b) << (2 * (s - 32));
    }
    __device__ int branch(int s) const {
        return s < 32 ? static_cast<int>((branch_lo >> (2 * s)) & 3u)
                      : static_cast<int>((branch_hi >> (2 * (s - 32))) & 3u);
    }
};

// Forward pass with recording: the trace of trace_ray (trace.cu) with checkpoints. Returns the
// status; soft_first = first soft event (kOk without one).
template <class N>
__device__ int forward_record(const TraceParams& p, const double* rec, const RecordLayout& lay,
                              int f, int l, const Sample& smp, bool soft_mode, Record<N>& out,
                              int& soft_first) {
    const int S = p.S, L = p.L;
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
    r.opl = r.py * st;
    SoftT<N> soft{zero, kOk};
    SoftT<N>* sp = soft_mode ? &soft : nullptr;
    out.p[0] = {r.px, r.py, r.pz};
    out.d[0] = {r.dx, r.dy, r.dz};
    out.branch_lo = out.branch_hi = 0;
    out.count = 1;
    out.image_branch = kBranchRegular;
    int status = kOk;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    N n_before = idx[l];
    for (int s = 1; s < S; ++s) {
        const N n_after = idx[s * L + l];
        const N c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        int branch;
        status = step_surface<N>(r, N(thick[s - 1]), c, n_before, n_after, sp, branch);
        if (status != kOk) break;
        out.count = s + 1;
        out.set_branch(s, branch);
        if (s % kInterval == 0) {
            out.p[s / kInterval] = {r.px, r.py, r.pz};
            out.d[s / kInterval] = {r.dx, r.dy, r.dz};
        }
        n_before = n_after;
    }
    if (status == kOk && soft_mode) status = soft.first;
    if (in_piston(status)) {
        if (!(r.dz > zero)) {
            status = kBackward;
        } else {
            int branch;
            const int rst = reference_step<N>(r, N(rec[lay.target + f]), N(thick[S - 1]),
                                              n_before, sp, branch);
            if (!in_piston(rst)) {
                status = rst;
            } else {
                out.image_branch = branch;
                if (status == kOk) status = rst;
            }
        }
    }
    soft_first = soft.first;
    return status;
}

// Reverse sweep of one seed (backward_ray): writes factor * dPhi/dx into row `row` of the
// run's columns col0[c * R + row] for every variable whose parameter is reached.
template <class N>
__device__ void backward_sweep(const TraceParams& p, const VarParams& v, const double* rec,
                               const RecordLayout& lay, int f, int l, const Record<N>& ck,
                               bool reached_image, bool soft_mode, N seed_opl, N seed_pen,
                               N factor, double* col0, int64_t R, int64_t row) {
    const int S = p.S, L = p.L;
    const N zero(0.0);
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    const int count = ck.count;
    RayAdj<N> adj{{zero, zero, zero}, {zero, zero, zero}};
    int next_branch = kBranchRegular;
    const Vec<N> center{zero, N(rec[lay.target + f]), N(thick[S - 1])};
    auto write = [&](int col, N value) {
        if (col >= 0) col0[static_cast<int64_t>(col) * R + row] = value_of(factor * value);
    };
    for (int c = (count - 1) / kInterval; c >= 0; --c) {
        const int first = c * kInterval;
        const int n = (count - first) < kInterval ? (count - first) : kInterval;
        // replay the segment from its checkpoint
        Vec<N> sp[kInterval], sd[kInterval];
        sp[0] = ck.p[c];
        sd[0] = ck.d[c];
        RayT<N> r{sp[0].x, sp[0].y, sp[0].z, sd[0].x, sd[0].y, sd[0].z, zero};
        SoftT<N> dummy{zero, kOk};
#pragma unroll
        for (int i = 1; i < kInterval; ++i) {
            if (i < n) {
                const int s = first + i;
                const N cs = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
                int branch;
                step_surface<N>(r, N(thick[s - 1]), cs, N(idx[(s - 1) * L + l]),
                                N(idx[s * L + l]), soft_mode ? &dummy : nullptr, branch);
                sp[i] = {r.px, r.py, r.pz};
                sd[i] = {r.dx, r.dy, r.dz};
            }
        }
        // back-propagate through the segment's states, last first
#pragma unroll
        for (int i = kInterval - 1; i >= 0; --i) {
            if (i < n) {
                const int s = first + i;
                if (s == count - 1) {
                    if (reached_image && count == S) {
                        Vec<N> center_adj{zero, zero, zero};
                        N n_image_adj = zero;
                        reference_step_backward<N>(sp[i], sd[i], center,
                                                   N(idx[(S - 1) * L + l]), ck.image_branch,
                                                   seed_opl, seed_pen, adj, center_adj,
                                                   n_image_adj);
                        write(v.col_thickness[S - 1], center_adj.z);
                    }
                } else {
                    const int j = s + 1;
                    const bool sphere = p.type[j] == MKB_SURFACE_SPHERE;
                    const N cj = sphere ? curv[j] : 0.0;
                    StepAdj<N> par{zero, zero, zero, zero};
                    refracting_step_backward<N>(sp[i], sd[i], N(thick[s]), cj,
                                                N(idx[s * L + l]), N(idx[j * L + l]),
                                                next_branch, seed_opl, seed_pen, adj, par);
                    if (sphere) write(v.col_curvature[j], par.curvature);
                    write(v.col_thickness[s], par.thickness);
                }
                next_branch = ck.branch(s);
            }
        }
    }
}

template <bool kExact>
__global__ void __launch_bounds__(kAdjThreads)
adjoint_rows_kernel(const __grid_constant__ AdjointParams ap, const double* __restrict__ records,
                    double* __restrict__ J) {
    using N = typename std::conditional<kExact, Exact64, double>::type;
    const TraceParams& p = ap.t;
    __shared__ SharedAdj sh;
    const int v = blockIdx.x / p.n_packs;
    const int pk = blockIdx.x - v * p.n_packs;
    const Pack pack = p.packs[pk];
    const RecordLayout lay = record_layout(p.S, p.L, p.F);
    if (threadIdx.x <= pack.tuples) {
        int start = 0;
        for (int t = 0; t < static_cast<int>(threadIdx.x); ++t)
            start += p.sample_count[(pack.first_tuple + t) / p.L];
        sh.tuple_start[threadIdx.x] = start;
    }
    copy_tables(p, sh.tab);
    if (!stage_to_shared(sh.record, records + static_cast<int64_t>(v) * p.stride,
                         static_cast<uint32_t>(p.stride * sizeof(double)), &sh.bar))
        return;
    const bool soft_mode = p.failure == MKB_FAILURE_SOFT;
    double* col0 = J + static_cast<int64_t>(v) * ap.v.P * ap.rows;
    for (int i = threadIdx.x; i < pack.rays; i += kAdjThreads) {
        int t = 0;
        while (t + 1 < pack.tuples && i >= sh.tuple_start[t + 1]) ++t;
        const int tu = pack.first_tuple + t;
        const int f = tu / p.L;
        const int l = tu - f * p.L;
        const int k = i - sh.tuple_start[t];
        const Sample smp = pupil_sample(p, sh.tab, f, k);
        Record<N> ck;
        int soft_first;
        const int st = forward_record<N>(p, sh.record, lay, f, l, smp, soft_mode, ck, soft_first);
        const int64_t row = p.field_offset[f] + static_cast<int64_t>(l) * p.sample_count[f] + k;
        const bool reached = in_piston(st);
        if (reached)
            backward_sweep<N>(p, ap.v, sh.record, lay, f, l, ck, true, soft_mode, N(1.0), N(0.0),
                              N(1.0), col0, ap.rows, row);
        if (soft_mode && soft_first != kOk) {
            const N factor = N(p.pscale[tu]) * N(smp.root_weight);
            backward_sweep<N>(p, ap.v, sh.record, lay, f, l, ck, reached, soft_mode, N(0.0),
                              N(1.0), factor, col0, ap.rows, p.rays + row);
        }
    }
}

// Piston projection of the raw dOPL/dx rows, one thread per (run, tuple, variable):
// col_k = s sqrt(W_k) (col_k - mean) for rays in the piston, 0 otherwise, mean over the piston
// rays in ascending sample order (adjoint_jacobian_cpu, src/optim/adjoint_jacobian.cpp:449).
template <bool kExact>
__global__ void projection_kernel(const __grid_constant__ AdjointParams ap,
                                  const uint8_t* __restrict__ status, double* __restrict__ J,
                                  int64_t total) {
    using N = typename std::conditional<kExact, Exact64, double>::type;
    const TraceParams& p = ap.t;
    const int64_t id = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= total) return;
    const int P = ap.v.P;
    const int var = static_cast<int>(id % P);
    const int64_t rt = id / P;
    const int tu = static_cast<int>(rt % p.n_tuples);
    const int64_t run = rt / p.n_tuples;
    const int f = tu / p.L;
    const int l = tu - f * p.L;
    const int n = p.sample_count[f];
    const int64_t row0 = p.field_offset[f] + static_cast<int64_t>(l) * n;
    const uint8_t* st = status + run * p.rays + row0;
    double* col = J + (run * P + var) * ap.rows + row0;
    const int mode = p.pupil_mode[f];
    const int M = mode == MKB_PUPIL_AXIS ? 1 : p.spokes;
    const double* w_tab = mode == MKB_PUPIL_AXIS ? p.w_axis : p.w_spoke;
    const double* rw_tab = mode == MKB_PUPIL_AXIS ? p.rw_axis : p.rw_spoke;
    N w_ok(0.0), sum(0.0);
    for (int k = 0; k < n; ++k)
        if (in_piston(st[k])) w_ok += N(w_tab[k / M]);
    const N scale = p.scale[tu];
    if (!(value_of(w_ok) > 0.0)) {
        for (int k = 0; k < n; ++k) col[k] = 0.0;
        return;
    }
    for (int k = 0; k < n; ++k)
        if (in_piston(st[k])) sum += N(w_tab[k / M]) * N(col[k]);
    const N mean = sum / w_ok;
    for (int k = 0; k < n; ++k)
        col[k] = in_piston(st[k]) ? value_of(scale * N(rw_tab[k / M]) * (N(col[k]) - mean)) : 0.0;
}

// Writes x_i into a copy of the run's template record (VariableSet::apply): one CTA per run.
__global__ void apply_kernel(const __grid_constant__ VarParams vp, RecordLayout lay,
                             const double* __restrict__ templates, int n_templates,
                             const double* __restrict__ x, double* __restrict__ out, int runs) {
    const int run = blockIdx.x;
    if (run >= runs) return;
    const double* src = templates + static_cast<int64_t>(n_templates == 1 ? 0 : run) * lay.stride;
    double* dst = out + static_cast<int64_t>(run) * lay.stride;
    for (int i = threadIdx.x; i < lay.stride; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) apply_variables(vp, lay, x + static_cast<int64_t>(run) * vp.P, dst);
}

}  // namespace

int launch_apply(const VarParams& vp, const RecordLayout& lay, const double* templates,
                 int n_templates, const double* x, double* out, int runs, cudaStream_t stream) {
    if (runs <= 0) return MKB_OK;
    apply_kernel<<<runs, 128, 0, stream>>>(vp, lay, templates, n_templates, x, out, runs);
    count_launch();
    return cuda_status(cudaGetLastError(), "apply launch");
}

int launch_adjoint_rows(const TraceParams& tp, const VarParams& vp, int64_t rows,
                        const double* records, double* J, bool exact, cudaStream_t stream) {
    AdjointParams ap;
    ap.t = tp;
    ap.v = vp;
    ap.rows = rows;
    const int64_t blocks = static_cast<int64_t>(tp.V) * tp.n_packs;
    if (exact)
        adjoint_rows_kernel<true><<<static_cast<unsigned>(blocks), kAdjThreads, 0, stream>>>(ap, records, J);
    else
        adjoint_rows_kernel<false><<<static_cast<unsigned>(blocks), kAdjThreads, 0, stream>>>(ap, records, J);
    count_launch();
    return cuda_status(cudaGetLastError(), "adjoint rows launch");
}

int launch_projection(const TraceParams& tp, const VarParams& vp, int64_t rows,
                      const uint8_t* status, double* J, bool exact, cudaStream_t stream) {
    AdjointParams ap;
    ap.t = tp;
    ap.v = vp;
    ap.rows = rows;
    const int64_t total = static_cast<int64_t>(tp.V) * tp.n_tuples * vp.P;
    const int threads = 128;
    const int64_t blocks = (total + threads - 1) / threads;
    if (exact)
        projection_kernel<true><<<static_cast<unsigned>(blocks), threads, 0, stream>>>(ap, status, J, total);
    else
        projection_kernel<false><<<static_cast<unsigned>(blocks), threads, 0, stream>>>(ap, status, J, total);
    count_launch();
    return cuda_status(cudaGetLastError(), "projection launch");
}

MKB_DEFINE_ERROR_READER(adjoint_device_error)

}  // namespace mkb

namespace mkb {
// ---- fused adjoint + normal equations ---------------------------------------------------------
// One CTA per run streams the run's rays in chunks of kFusedThreads (one ray per thread):
//   A  forward with checkpoints in shared memory, then the OPL-seed reverse sweep writes the
//      row y_k = [dOPL_k/dx | OPL_k] into shared memory (rays outside the piston: weight 0);
//   B  per tuple segment of the chunk (threads = columns): weighted mean mu_seg, rows centred
//      and scaled in place, x_k = s sqrt(W_k) (y_k - mu_seg), and the segment merged into the
//      tuple's running mean with one extra row s sqrt(W_t W_seg / (W_t + W_seg)) (mu_seg - mu_t)
//      (Chan, Golub, LeVeque): summed over the chunks, sum x x^T is s^2 sum_k W_k (y_k - ybar)
//      (y_k - ybar)^T over the tuple -- exactly [J r]^T [J r] of the piston-projected rows
//      J_k = s sqrt(W_k) (g_k - gbar), r_k = s sqrt(W_k) (OPL_k - piston), without a second
//      pass over the tuple and without J in memory;
//   C  FP64 tensor cores accumulate sum x x^T (mma.sync m8n8k4, 8 x 8 tiles of the upper
//      triangle in registers, owned by the CTA's warps);
//   D  in soft-failure mode, when the chunk has failed rays, the penalty rows
//      [s_p sqrt(W) dpi/dx | p_k] (uncentred) are accumulated the same way.
// Output: gram [runs][P+1][P+1] as the normal-equation kernels write it.
namespace {

constexpr int kFusedThreads = 128;
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr int kExtraRows = 8;
constexpr int kFusedMinBlocks = 3;  // CTAs per SM the register budget is sized for
constexpr int kMaxTileCols = (MKB_MAX_VARIABLES + 1 + 7) / 8;                   // 9
constexpr int kMaxTilePairs = kMaxTileCols * (kMaxTileCols + 1) / 2;             // 45

struct FusedShared {
    uint64_t bar;
    SharedTables tab;
    double w[kFusedThreads];      // sample weight if the ray is in the piston, else 0
    int tuple[kFusedThreads];     // tuple of the ray (-1 past the end)
    double seg_w;                 // weight of the current segment
    double open_w;                // running weight of the open tuple
    int open_tuple;               // tuple whose running mean is kept
    int extra;                    // extra rows pending
    int any_failed;               // chunk has a ray with status != Ok (soft mode)
    int2 tiles[kMaxTilePairs];    // (row tile, column tile) of every upper-triangle pair
};

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// acc += X^T X for X stored column-major, X(k, c) = xt[c * ld + k], k < n (n a multiple of 4;
// the caller pads with zero rows). Warp w owns tile pairs w, w + 4, ...; the 8 x 8 accumulator
// tiles live in shared memory in fragment order (acc[pair][lane][2]), loaded and stored around
// the k loop.
__device__ __forceinline__ void accumulate(const double* xt, int ld, int n, int pairs,
                                           const int2* tiles, double* acc) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    for (int e = warp; e < pairs; e += kFusedWarps) {
        const double* ca = xt + (tiles[e].x * 8 + gid) * ld + tig;
        const double* cb = xt + (tiles[e].y * 8 + gid) * ld + tig;
        double* a = acc + (e * 32 + lane) * 2;
        double d0 = a[0], d1 = a[1];
        for (int k0 = 0; k0 < n; k0 += 4) dmma(d0, d1, ca[k0], cb[k0]);
        a[0] = d0;
        a[1] = d1;
    }
}

template <class N>
__device__ void fused_forward(const TraceParams& p, const double* rec, const RecordLayout& lay,
                              int f, int l, const Sample& smp, bool soft_mode, double* ck,
                              int stride_ck, uint64_t& br_lo, uint64_t& br_hi, int& count,
                              int& image_branch, int& status_out, int& soft_first, double& opl,
                              double& penalty) {
    const int S = p.S, L = p.L;
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
    r.opl = r.py * st;
    SoftT<N> soft{zero, kOk};
    SoftT<N>* sp = soft_mode ? &soft : nullptr;
    auto save = [&](int c) {
        double* q = ck + c * stride_ck;
        q[0] = value_of(r.px);
        q[1 * kFusedThreads] = value_of(r.py);
        q[2 * kFusedThreads] = value_of(r.pz);
        q[3 * kFusedThreads] = value_of(r.dx);
        q[4 * kFusedThreads] = value_of(r.dy);
        q[5 * kFusedThreads] = value_of(r.dz);
    };
    br_lo = br_hi = 0;
    count = 1;
    image_branch = kBranchRegular;
    int status = kOk;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    N n_before = idx[l];
    for (int s = 1; s < S; ++s) {
        const N n_after = idx[s * L + l];
        const N c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        int branch;
        status = step_surface<N>(r, N(thick[s - 1]), c, n_before, n_after, sp, branch);
        if (status != kOk) break;
        count = s + 1;
        if (s < 32) br_lo |= static_cast<uint64_t>(branch) << (2 * s);
        else br_hi |= static_cast<uint64_t>(branch) << (2 * (s - 32));
        if (s % kInterval == 0) save(s / kInterval);
        n_before = n_after;
    }
    if (status == kOk && soft_mode) status = soft.first;
    if (in_piston(status)) {
        if (!(r.dz > zero)) {
            status = kBackward;
        } else {
            int branch;
            const int rst = reference_step<N>(r, N(rec[lay.target + f]), N(thick[S - 1]),
                                              n_before, sp, branch);
            if (!in_piston(rst)) {
                status = rst;
            } else {
                image_branch = branch;
                if (status == kOk) status = rst;
            }
        }
    }
    status_out = status;
    soft_first = soft.first;
    opl = value_of(r.opl);
    penalty = value_of(soft.penalty);
}

// Reverse sweep of one seed writing factor * dPhi/dx into row[col * ld]. One out-of-line copy
// serves both seeds (keeps the kernel's instruction footprint small).
template <class N>
__device__ __noinline__ void fused_backward(const TraceParams& p, const VarParams& v, const double* rec,
                               const RecordLayout& lay, int f, int l, const Sample& smp,
                               const double* ck,
                               int stride_ck, uint64_t br_lo, uint64_t br_hi, int count,
                               int image_branch, bool reached_image, bool soft_mode, N seed_opl,
                               N seed_pen, N factor, double* row, int ld) {
    const int S = p.S, L = p.L;
    const N zero(0.0);
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    RayAdj<N> adj{{zero, zero, zero}, {zero, zero, zero}};
    int next_branch = kBranchRegular;
    const Vec<N> center{zero, N(rec[lay.target + f]), N(thick[S - 1])};
    auto branch_of = [&](int s) {
        return s < 32 ? static_cast<int>((br_lo >> (2 * s)) & 3u)
                      : static_cast<int>((br_hi >> (2 * (s - 32))) & 3u);
    };
    for (int c = (count - 1) / kInterval; c >= 0; --c) {
        const int first = c * kInterval;
        const int n = (count - first) < kInterval ? (count - first) : kInterval;
        Vec<N> sp[kInterval], sd[kInterval];
        if (c == 0) {  // the start ray is recomputed (collimated_ray), not stored
            const N r0 = N(rec[lay.pupil]) * N(smp.rho);
            sp[0] = {r0 * N(smp.sin_phi), r0 * N(smp.cos_phi), zero};
            sd[0] = {zero, N(rec[lay.sin_theta + f]), N(rec[lay.cos_theta + f])};
        } else {
            const double* q = ck + c * stride_ck;
            sp[0] = {N(q[0]), N(q[kFusedThreads]), N(q[2 * kFusedThreads])};
            sd[0] = {N(q[3 * kFusedThreads]), N(q[4 * kFusedThreads]), N(q[5 * kFusedThreads])};
        }
        RayT<N> r{sp[0].x, sp[0].y, sp[0].z, sd[0].x, sd[0].y, sd[0].z, zero};
        SoftT<N> dummy{zero, kOk};
#pragma unroll
        for (int i = 1; i < kInterval; ++i) {
            if (i < n) {
                const int s = first + i;
                const N cs = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
                int branch;
                step_surface<N>(r, N(thick[s - 1]), cs, N(idx[(s - 1) * L + l]),
                                N(idx[s * L + l]), soft_mode ? &dummy : nullptr, branch);
                sp[i] = {r.px, r.py, r.pz};
                sd[i] = {r.dx, r.dy, r.dz};
            }
        }
#pragma unroll
        for (int i = kInterval - 1; i >= 0; --i) {
            if (i < n) {
                const int s = first + i;
                if (s == count - 1) {
                    if (reached_image && count == S) {
                        Vec<N> center_adj{zero, zero, zero};
                        N n_image_adj = zero;
                        reference_step_backward<N>(sp[i], sd[i], center, N(idx[(S - 1) * L + l]),
                                                   image_branch, seed_opl, seed_pen, adj,
                                                   center_adj, n_image_adj);
                        const int col = v.col_thickness[S - 1];
                        if (col >= 0) row[col * ld] = value_of(factor * center_adj.z);
                    }
                } else {
                    const int j = s + 1;
                    const bool sphere = p.type[j] == MKB_SURFACE_SPHERE;
                    const N cj = sphere ? curv[j] : 0.0;
                    StepAdj<N> par{zero, zero, zero, zero};
                    refracting_step_backward<N>(sp[i], sd[i], N(thick[s]), cj, N(idx[s * L + l]),
                                                N(idx[j * L + l]), next_branch, seed_opl,
                                                seed_pen, adj, par);
                    if (sphere && v.col_curvature[j] >= 0)
                        row[v.col_curvature[j] * ld] = value_of(factor * par.curvature);
                    if (v.col_thickness[s] >= 0)
                        row[v.col_thickness[s] * ld] = value_of(factor * par.thickness);
                }
                next_branch = branch_of(s);
            }
        }
    }
}

// Mixed precision: forward in the mixed scheme (FP64 positions, sag root and OPL, FP32
// directions and refraction; checkpoints keep the FP64 position and the FP32 direction), the
// reverse sweep entirely in FP32 on the states rounded to FP32.
struct MixedPrecision {};

__device__ void fused_forward_mixed(const TraceParams& p, const double* rec,
                                    const RecordLayout& lay, int f, int l, const Sample& smp,
                                    bool soft_mode, double* ck, int stride_ck, uint64_t& br_lo,
                                    uint64_t& br_hi, int& count, int& image_branch,
                                    int& status_out, int& soft_first, double& opl,
                                    double& penalty) {
    const int S = p.S, L = p.L;
    const double a = rec[lay.pupil];
    const double st = rec[lay.sin_theta + f];
    const double ct = rec[lay.cos_theta + f];
    const double r0 = a * smp.rho;
    RayMixed r;
    r.px = r0 * smp.sin_phi;
    r.py = r0 * smp.cos_phi;
    r.pz = 0.0;
    r.dx = 0.0f;
    r.dy = static_cast<float>(st);
    r.dz = static_cast<float>(ct);
    r.opl = r.py * st;
    SoftT<double> soft{0.0, kOk};
    SoftT<double>* sp = soft_mode ? &soft : nullptr;
    br_lo = br_hi = 0;
    count = 1;
    image_branch = kBranchRegular;
    int status = kOk;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    double n_before = idx[l];
    for (int s = 1; s < S; ++s) {
        const double n_after = idx[s * L + l];
        const double c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        int branch;
        status = step_surface_mixed(r, thick[s - 1], c, n_before, n_after, sp, branch);
        if (status != kOk) break;
        count = s + 1;
        if (s < 32) br_lo |= static_cast<uint64_t>(branch) << (2 * s);
        else br_hi |= static_cast<uint64_t>(branch) << (2 * (s - 32));
        if (s % kInterval == 0) {
            double* q = ck + (s / kInterval) * stride_ck;
            q[0] = r.px;
            q[1 * kFusedThreads] = r.py;
            q[2 * kFusedThreads] = r.pz;
            q[3 * kFusedThreads] = r.dx;
            q[4 * kFusedThreads] = r.dy;
            q[5 * kFusedThreads] = r.dz;
        }
        n_before = n_after;
    }
    if (status == kOk && soft_mode) status = soft.first;
    if (in_piston(status)) {
        if (!(r.dz > 0.0f)) {
            status = kBackward;
        } else {
            int branch;
            const int rst = reference_step_mixed(r, rec[lay.target + f], thick[S - 1], n_before,
                                                 sp, branch);
            if (!in_piston(rst)) {
                status = rst;
            } else {
                image_branch = branch;
                if (status == kOk) status = rst;
            }
        }
    }
    status_out = status;
    soft_first = soft.first;
    opl = r.opl;
    penalty = soft.penalty;
}

__device__ __noinline__ void fused_backward_mixed(const TraceParams& p, const VarParams& v,
                                                  const double* rec, const RecordLayout& lay,
                                                  int f, int l, const Sample& smp,
                                                  const double* ck, int stride_ck,
                                                  uint64_t br_lo, uint64_t br_hi, int count,
                                                  int image_branch, bool reached_image,
                                                  bool soft_mode, float seed_opl, float seed_pen,
                                                  float factor, double* row, int ld) {
    using F = float;
    const int S = p.S, L = p.L;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    RayAdj<F> adj{{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    int next_branch = kBranchRegular;
    const Vec<F> center{0.f, static_cast<F>(rec[lay.target + f]), static_cast<F>(thick[S - 1])};
    auto branch_of = [&](int s) {
        return s < 32 ? static_cast<int>((br_lo >> (2 * s)) & 3u)
                      : static_cast<int>((br_hi >> (2 * (s - 32))) & 3u);
    };
    for (int c = (count - 1) / kInterval; c >= 0; --c) {
        const int first = c * kInterval;
        const int n = (count - first) < kInterval ? (count - first) : kInterval;
        Vec<F> sp[kInterval], sd[kInterval];
        RayMixed r;
        if (c == 0) {
            const double r0 = rec[lay.pupil] * smp.rho;
            r.px = r0 * smp.sin_phi;
            r.py = r0 * smp.cos_phi;
            r.pz = 0.0;
            r.dx = 0.0f;
            r.dy = static_cast<float>(rec[lay.sin_theta + f]);
            r.dz = static_cast<float>(rec[lay.cos_theta + f]);
        } else {
            const double* q = ck + c * stride_ck;
            r.px = q[0];
            r.py = q[kFusedThreads];
            r.pz = q[2 * kFusedThreads];
            r.dx = static_cast<float>(q[3 * kFusedThreads]);
            r.dy = static_cast<float>(q[4 * kFusedThreads]);
            r.dz = static_cast<float>(q[5 * kFusedThreads]);
        }
        r.opl = 0.0;
        sp[0] = {static_cast<F>(r.px), static_cast<F>(r.py), static_cast<F>(r.pz)};
        sd[0] = {r.dx, r.dy, r.dz};
        SoftT<double> dummy{0.0, kOk};
#pragma unroll
        for (int i = 1; i < kInterval; ++i) {
            if (i < n) {
                const int s = first + i;
                const double cs = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
                int branch;
                step_surface_mixed(r, thick[s - 1], cs, idx[(s - 1) * L + l], idx[s * L + l],
                                   soft_mode ? &dummy : nullptr, branch);
                sp[i] = {static_cast<F>(r.px), static_cast<F>(r.py), static_cast<F>(r.pz)};
                sd[i] = {r.dx, r.dy, r.dz};
            }
        }
#pragma unroll
        for (int i = kInterval - 1; i >= 0; --i) {
            if (i < n) {
                const int s = first + i;
                if (s == count - 1) {
                    if (reached_image && count == S) {
                        Vec<F> center_adj{0.f, 0.f, 0.f};
                        F n_image_adj = 0.f;
                        reference_step_backward<F>(sp[i], sd[i], center,
                                                   static_cast<F>(idx[(S - 1) * L + l]),
                                                   image_branch, seed_opl, seed_pen, adj,
                                                   center_adj, n_image_adj);
                        const int col = v.col_thickness[S - 1];
                        if (col >= 0) row[col * ld] = factor * center_adj.z;
                    }
                } else {
                    const int j = s + 1;
                    const bool sphere = p.type[j] == MKB_SURFACE_SPHERE;
                    const F cj = sphere ? static_cast<F>(curv[j]) : 0.f;
                    StepAdj<F> par{0.f, 0.f, 0.f, 0.f};
                    refracting_step_backward<F>(sp[i], sd[i], static_cast<F>(thick[s]), cj,
                                                static_cast<F>(idx[s * L + l]),
                                                static_cast<F>(idx[j * L + l]), next_branch,
                                                seed_opl, seed_pen, adj, par);
                    if (sphere && v.col_curvature[j] >= 0)
                        row[v.col_curvature[j] * ld] = factor * par.curvature;
                    if (v.col_thickness[s] >= 0) row[v.col_thickness[s] * ld] = factor * par.thickness;
                }
                next_branch = branch_of(s);
            }
        }
    }
}

template <class N>
__global__ void __launch_bounds__(kFusedThreads, kFusedMinBlocks)
adjoint_gram_kernel(const __grid_constant__ AdjointParams ap, const double* __restrict__ records,
                    double* __restrict__ gram) {
    const TraceParams& p = ap.t;
    const VarParams& v = ap.v;
    __shared__ FusedShared sh;
    extern __shared__ __align__(16) double dyn[];
    const int P = v.P;
    const int NP = ((P + 1 + 7) / 8) * 8;
    const int ncols = NP / 8;
    const int pairs = ncols * (ncols + 1) / 2;
    const int nck = (p.S - 1) / kInterval + 1;
    const int stride_ck = 6 * kFusedThreads;
    constexpr int TS = kFusedThreads + 1;              // column stride of Y (odd: no conflicts)
    constexpr int ES = kExtraRows + 1;                 // column stride of E
    double* record = dyn;                              // [stride] (bulk-copy target, 16 B aligned)
    double* Y = record + p.stride;                     // column-major [NP][TS]
    double* E = Y + NP * TS;                           // column-major [NP][ES]
    double* mu_open = E + NP * ES;                     // [NP]
    double* mu_seg = mu_open + NP;                     // [NP]
    double* acc = mu_seg + NP;                         // [pairs][32][2] DMMA accumulators
    double* ckpt = acc + pairs * 64;                   // [nck][6][T], checkpoint 0 unused
    const int tid = threadIdx.x;
    const int run = blockIdx.x;
    const RecordLayout lay = record_layout(p.S, p.L, p.F);
    copy_tables(p, sh.tab);
    if (tid == 0) {
        sh.open_tuple = -1;
        sh.open_w = 0.0;
        sh.extra = 0;
    }
    if (!stage_to_shared(record, records + static_cast<int64_t>(run) * p.stride,
                         static_cast<uint32_t>(p.stride * sizeof(double)), &sh.bar))
        return;
    const bool soft_mode = p.failure == MKB_FAILURE_SOFT;
    for (int e = tid; e < pairs; e += kFusedThreads) {
        int j = 0, rem = e;
        while (rem >= j + 1) {
            rem -= j + 1;
            ++j;
        }
        sh.tiles[e] = make_int2(rem, j);
    }
    for (int i = tid; i < pairs * 64; i += kFusedThreads) acc[i] = 0.0;
    __syncthreads();
    double* my_ck = ckpt + tid;
    for (int base = 0; base < p.rays; base += kFusedThreads) {
        const int q = base + tid;
        double* row = Y + tid;  // this ray's row, column c at row[c * TS]
        for (int c = 0; c < NP; ++c) row[c * TS] = 0.0;
        int f = 0, l = 0, k = 0, tu = -1;
        int status = kMissed, soft_first = kOk, count = 0, image_branch = 0;
        uint64_t br_lo = 0, br_hi = 0;
        double opl = 0.0, penalty = 0.0;
        Sample smp{};
        if (q < p.rays) {
            while (f + 1 < p.F && q >= p.field_offset[f + 1]) ++f;
            const int within = q - p.field_offset[f];
            l = within / p.sample_count[f];
            k = within - l * p.sample_count[f];
            tu = f * p.L + l;
            smp = pupil_sample(p, sh.tab, f, k);
            if constexpr (std::is_same<N, MixedPrecision>::value)
                fused_forward_mixed(p, record, lay, f, l, smp, soft_mode, my_ck, stride_ck, br_lo,
                                    br_hi, count, image_branch, status, soft_first, opl, penalty);
            else
                fused_forward<N>(p, record, lay, f, l, smp, soft_mode, my_ck, stride_ck, br_lo,
                                 br_hi, count, image_branch, status, soft_first, opl, penalty);
            if (in_piston(status)) {
                if constexpr (std::is_same<N, MixedPrecision>::value)
                    fused_backward_mixed(p, v, record, lay, f, l, smp, my_ck, stride_ck, br_lo,
                                         br_hi, count, image_branch, true, soft_mode, 1.0f, 0.0f,
                                         1.0f, row, TS);
                else
                    fused_backward<N>(p, v, record, lay, f, l, smp, my_ck, stride_ck, br_lo,
                                      br_hi, count, image_branch, true, soft_mode, N(1.0),
                                      N(0.0), N(1.0), row, TS);
                row[P * TS] = opl;
            }
        }
        sh.w[tid] = (q < p.rays && in_piston(status)) ? smp.weight : 0.0;
        sh.tuple[tid] = tu;
        if (tid == 0) sh.any_failed = 0;
        __syncthreads();
        if (soft_mode && q < p.rays && status != kOk) sh.any_failed = 1;
        // ---- B: segments (threads = columns) ----
        const int rows_here = p.rays - base < kFusedThreads ? p.rays - base : kFusedThreads;
        int start = 0;
        while (start < rows_here) {
            const int t = sh.tuple[start];
            int end = start + 1;
            while (end < rows_here && sh.tuple[end] == t) ++end;
            if (tid == 0) {
                double w = 0.0;
                for (int r = start; r < end; ++r) w += sh.w[r];
                sh.seg_w = w;
            }
            __syncthreads();
            const double wseg = sh.seg_w;
            const double scale = p.scale[t];
            if (wseg > 0.0) {
                if (tid < NP) {
                    double s = 0.0;
                    double* col = Y + tid * TS;
                    for (int r = start; r < end; ++r) s += sh.w[r] * col[r];
                    const double mean = s / wseg;
                    mu_seg[tid] = mean;
                    for (int r = start; r < end; ++r) {
                        const double x = col[r];
                        col[r] = sh.w[r] > 0.0 ? scale * sqrt(sh.w[r]) * (x - mean) : 0.0;
                    }
                    if (sh.open_tuple == t && sh.open_w > 0.0) {
                        const double wt = sh.open_w;
                        const double fac = scale * sqrt(wt * wseg / (wt + wseg));
                        E[tid * ES + sh.extra] = fac * (mean - mu_open[tid]);
                        mu_open[tid] += (wseg / (wt + wseg)) * (mean - mu_open[tid]);
                    } else {
                        mu_open[tid] = mean;
                    }
                }
                __syncthreads();
                if (tid == 0) {
                    if (sh.open_tuple == t && sh.open_w > 0.0) {
                        sh.extra += 1;
                        sh.open_w += wseg;
                    } else {
                        sh.open_tuple = t;
                        sh.open_w = wseg;
                    }
                }
            } else if (tid < NP) {
                for (int r = start; r < end; ++r) Y[tid * TS + r] = 0.0;
            }
            __syncthreads();
            if (sh.extra == kExtraRows) {  // flush the extra rows
                accumulate(E, ES, kExtraRows, pairs, sh.tiles, acc);
                __syncthreads();
                if (tid == 0) sh.extra = 0;
                __syncthreads();
            }
            start = end;
        }
        // ---- C: accumulate the centred rows and the pending extra rows ----
        for (int r = rows_here + tid; r < ((rows_here + 3) & ~3); r += kFusedThreads)
            for (int c = 0; c < NP; ++c) Y[c * TS + r] = 0.0;
        const int ne = sh.extra;
        for (int r = ne + tid; r < ((ne + 3) & ~3); r += kFusedThreads)
            for (int c = 0; c < NP; ++c) E[c * ES + r] = 0.0;
        __syncthreads();
        accumulate(Y, TS, (rows_here + 3) & ~3, pairs, sh.tiles, acc);
        if (ne > 0) accumulate(E, ES, (ne + 3) & ~3, pairs, sh.tiles, acc);
        __syncthreads();
        if (tid == 0) sh.extra = 0;
        // ---- D: penalty rows ----
        if (sh.any_failed) {
            for (int c = 0; c < NP; ++c) row[c * TS] = 0.0;
            if (q < p.rays && status != kOk) {
                const double factor = p.pscale[tu] * smp.root_weight;
                if (soft_first != kOk) {
                    if constexpr (std::is_same<N, MixedPrecision>::value)
                        fused_backward_mixed(p, v, record, lay, f, l, smp, my_ck, stride_ck,
                                             br_lo, br_hi, count, image_branch, in_piston(status),
                                             soft_mode, 0.0f, 1.0f, static_cast<float>(factor),
                                             row, TS);
                    else
                        fused_backward<N>(p, v, record, lay, f, l, smp, my_ck, stride_ck, br_lo,
                                          br_hi, count, image_branch, in_piston(status),
                                          soft_mode, N(0.0), N(1.0),
                                          N(p.pscale[tu]) * N(smp.root_weight), row, TS);
                }
                const double fp = is_soft(status) ? penalty : penalty + 1.0;
                row[P * TS] = factor * fp;
            }
            __syncthreads();
            accumulate(Y, TS, (rows_here + 3) & ~3, pairs, sh.tiles, acc);
        }
        __syncthreads();
    }
    // ---- write the (P+1) x (P+1) symmetric gram ----
    const int n = P + 1;
    double* G = gram + static_cast<int64_t>(run) * n * n;
    __syncthreads();
    for (int i = tid; i < pairs * 64; i += kFusedThreads) {
        const int e = i / 64, lane = (i / 2) & 31, h = i & 1;
        const int r = sh.tiles[e].x * 8 + (lane >> 2);
        const int c = sh.tiles[e].y * 8 + 2 * (lane & 3) + h;
        if (r < n && c < n) {
            G[static_cast<int64_t>(c) * n + r] = acc[i];
            G[static_cast<int64_t>(r) * n + c] = acc[i];
        }
    }
}

}  // namespace

size_t fused_adjoint_smem(const TraceParams& tp, int P) {
    const int NP = ((P + 1 + 7) / 8) * 8;
    const int nck = (tp.S - 1) / kInterval + 1;
    const int ncols = NP / 8;
    const int pairs = ncols * (ncols + 1) / 2;
    return sizeof(double) * (static_cast<size_t>(tp.stride) +
                             static_cast<size_t>(kFusedThreads + 1) * NP +
                             (kExtraRows + 1) * NP + 2 * NP +
                             static_cast<size_t>(pairs) * 64 +
                             static_cast<size_t>(nck) * 6 * kFusedThreads);
}

int launch_adjoint_gram(const TraceParams& tp, const VarParams& vp, const double* records,
                        double* gram, int precision, cudaStream_t stream) {
    AdjointParams ap;
    ap.t = tp;
    ap.v = vp;
    ap.rows = 0;
    const size_t smem = fused_adjoint_smem(tp, vp.P);
    auto kernel = precision == MKB_PRECISION_FP64    ? adjoint_gram_kernel<Exact64>
                  : precision == MKB_PRECISION_MIXED ? adjoint_gram_kernel<MixedPrecision>
                                                     : adjoint_gram_kernel<double>;
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return cuda_status(err, "fused adjoint: shared memory attribute");
    kernel<<<tp.V, kFusedThreads, smem, stream>>>(ap, records, gram);
    count_launch();
    return cuda_status(cudaGetLastError(), "fused adjoint launch");
}

}  // namespace mkb
