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
