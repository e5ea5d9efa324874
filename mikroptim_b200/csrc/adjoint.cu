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
#include "launch.cuh"
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

// the variant's record is the kernel's dynamic shared memory (16-byte aligned, stride doubles)
struct alignas(16) SharedAdj {
    uint64_t bar;
    SharedTables tab;
    int tuple_start[kMaxPackTuples + 1];
};

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
        GhostData gd;
        const bool plate = ghost_at<true>(p, rec, lay, s, l, gd);
        status = step_surface_xf<N>(r, N(thick[s - 1]), c, n_before, n_before / n_after,
                                    xf_of(rec, lay, s), sp, branch, nullptr,
                                    plate ? &gd : nullptr, n_after);
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
// start[0..2] (when not null) get the adjoint of the start point's x and y and the derivative
// with respect to thickness[0] (the entrance pupil's distance), unscaled, for the aiming fold.
// img_seed (when not null): Phi is g_x x + g_y y of the ray's intersection (x, y) with the
// image plane, thickness[S - 1] behind the last vertex (the transverse ray-error rows), in
// place of the optical path to the reference sphere; seed_opl and seed_pen are then 0.
template <class N>
__device__ void backward_sweep(const TraceParams& p, const VarParams& v, const double* rec,
                               const RecordLayout& lay, int f, int l, const Record<N>& ck,
                               bool reached_image, bool soft_mode, N seed_opl, N seed_pen,
                               N factor, double* col0, int64_t R, int64_t row,
                               double* start = nullptr, const double* img_seed = nullptr) {
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
    // the index of medium s enters the steps onto s and onto s + 1: its adjoint is summed over
    // both (a carry) and written to the glass columns of s with dn/d(n0, nu1, nu2) =
    // (1, w, w^2) at this wavelength (AdjointRowWriter::index, merit/ray_jacobian.hpp:66)
    N n_carry = zero;
    auto index_sink = [&](int s, N value) {
        if (!v.has_glass) return;
        const double w = v.omega[l];
        const N slope[3] = {N(1.0), N(w), N(w) * N(w)};
        for (int c = 0; c < 3; ++c)
            if (v.col_glass[s][c] >= 0) write(v.col_glass[s][c], value * slope[c]);
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
                const N nb = idx[(s - 1) * L + l], na = idx[s * L + l];
                GhostData gd;
                const bool plate = ghost_at<true>(p, rec, lay, s, l, gd);
                step_surface_xf<N>(r, N(thick[s - 1]), cs, nb, nb / na, xf_of(rec, lay, s),
                                   soft_mode ? &dummy : nullptr, branch, nullptr,
                                   plate ? &gd : nullptr, na);
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
                    if (reached_image && count == S && img_seed != nullptr) {
                        // (x, y) = p + s0 (d_x, d_y), s0 = (w - p_z) / d_z (the forward's
                        // transfer_to_image_plane on a copy of the state)
                        const N gx(img_seed[0]), gy(img_seed[1]);
                        const N w = thick[S - 1];
                        const N s0 = (w - sp[i].z) / sd[i].z;
                        const N s0b = gx * sd[i].x + gy * sd[i].y;
                        adj.p = {gx, gy, -s0b / sd[i].z};
                        adj.d = {gx * s0, gy * s0, -(s0b * s0) / sd[i].z};
                        write(v.col_thickness[S - 1], s0b / sd[i].z);
                    } else if (reached_image && count == S) {
                        Vec<N> center_adj{zero, zero, zero};
                        N n_image_adj = zero;
                        reference_step_backward<N>(sp[i], sd[i], center,
                                                   N(idx[(S - 1) * L + l]), ck.image_branch,
                                                   seed_opl, seed_pen, adj, center_adj,
                                                   n_image_adj);
                        write(v.col_thickness[S - 1], center_adj.z);
                        n_carry = n_image_adj;
                    }
                } else {
                    const int j = s + 1;
                    const bool sphere = p.type[j] == MKB_SURFACE_SPHERE;
                    const N cj = sphere ? curv[j] : 0.0;
                    StepAdj<N> par{zero, zero, zero, zero};
                    const double* xf = xf_of(rec, lay, j);
                    const bool moved = xf != nullptr && xf[6] > 0.0;
                    Vec<N> pl = sp[i], dl = sd[i];
                    N tl = thick[s];
                    Transform<N> tr{};
                    if (moved) {
                        tr = transform_at<N>(xf);
                        state_to_surface(tr, pl, dl, tl);
                        tl = zero;
                        adjoint_to_surface(tr, adj);
                    }
                    GhostData gd;
                    if (ghost_at<true>(p, rec, lay, j, l, gd)) {
                        const int g = p.ghost_of[j];
                        const N so[1] = {seed_opl}, sq[1] = {seed_pen};
                        RayAdj<N> a[1] = {adj};
                        StepAdj<N> o[1] = {par};
                        ghost_step_backward_k<N, N, 1>(
                            pl, dl, tl, gd, N(idx[s * L + l]), N(idx[j * L + l]), next_branch,
                            so, sq, a, o,
                            [&](int, int k, N value) { write(v.col_ghost[g][k], value); });
                        adj = a[0];
                        par = o[0];
                    } else {
                        refracting_step_backward<N>(pl, dl, tl, cj, N(idx[s * L + l]),
                                                    N(idx[j * L + l]), next_branch, seed_opl,
                                                    seed_pen, adj, par);
                    }
                    if (moved) {
                        adjoint_from_surface(tr, adj);
                        par.thickness = -adj.p.z;
                    }
                    if (sphere) write(v.col_curvature[j], par.curvature);
                    write(v.col_thickness[s], par.thickness);
                    if (s == 0 && start != nullptr) start[2] = value_of(par.thickness);
                    index_sink(j, par.n_after + n_carry);
                    n_carry = par.n_before;
                }
                next_branch = ck.branch(s);
            }
        }
    }
    index_sink(0, n_carry);
    if (start != nullptr) {
        start[0] = value_of(adj.p.x);
        start[1] = value_of(adj.p.y);
    }
}

// The aiming fold of one row: the entrance pupil's radius a and distance t0 follow the
// variables (aim_record), so every column j gains dPhi/da da/dx_j + dPhi/dt0 dt0/dx_j with
// dPhi/da = rho (sin phi, cos phi) . adj(p0) + seed_opl rho cos phi sin theta (the start point
// a rho (sin phi, cos phi, 0) and its optical path p0 . d0).
__device__ __forceinline__ double aim_start_adjoint(const double* start, const Sample& smp,
                                                    double sin_theta, double seed_opl) {
    return smp.rho * (smp.sin_phi * start[0] + smp.cos_phi * start[1]) +
           seed_opl * smp.rho * smp.cos_phi * sin_theta;
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
    const RecordLayout lay = layout_of(p);
    if (threadIdx.x <= pack.tuples) {
        int start = 0;
        for (int t = 0; t < static_cast<int>(threadIdx.x); ++t)
            start += p.sample_count[(pack.first_tuple + t) / p.L];
        sh.tuple_start[threadIdx.x] = start;
    }
    copy_tables(p, sh.tab);
    extern __shared__ __align__(16) double record[];
    if (!stage_to_shared(record, records + static_cast<int64_t>(v) * p.stride,
                         static_cast<uint32_t>(p.stride * sizeof(double)), &sh.bar))
        return;
    const bool soft_mode = p.failure == MKB_FAILURE_SOFT;
    double* col0 = J + static_cast<int64_t>(v) * ap.v.P * ap.rows;
    // an interior stop: d(a, t0)/dx of the variant's aimed entrance pupil
    __shared__ double aim_da[MKB_MAX_VARIABLES], aim_dt[MKB_MAX_VARIABLES];
    if (lay.stop > 0) {
        for (int k = threadIdx.x; k < ap.v.P; k += kAdjThreads)
            aim_sensitivity(record, lay, ap.v, k, aim_da[k], aim_dt[k]);
        __syncthreads();
    }
    auto aim_fold = [&](const double* start, const Sample& smp, int f, double seed_opl,
                        double factor, int64_t row) {
        const double ga = aim_start_adjoint(start, smp, record[lay.sin_theta + f], seed_opl);
        for (int k = 0; k < ap.v.P; ++k)
            col0[static_cast<int64_t>(k) * ap.rows + row] +=
                factor * (ga * aim_da[k] + start[2] * aim_dt[k]);
    };
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
        const int st = forward_record<N>(p, record, lay, f, l, smp, soft_mode, ck, soft_first);
        const int64_t row = p.field_offset[f] + static_cast<int64_t>(l) * p.sample_count[f] + k;
        const bool reached = in_piston(st);
        double start[3] = {0.0, 0.0, 0.0};
        double* aim = lay.stop > 0 ? start : nullptr;
        if (reached) {
            backward_sweep<N>(p, ap.v, record, lay, f, l, ck, true, soft_mode, N(1.0), N(0.0),
                              N(1.0), col0, ap.rows, row, aim);
            if (aim) aim_fold(start, smp, f, 1.0, 1.0, row);
        }
        if (soft_mode && soft_first != kOk) {
            const N factor = N(p.pscale[tu]) * N(smp.root_weight);
            backward_sweep<N>(p, ap.v, record, lay, f, l, ck, reached, soft_mode, N(0.0),
                              N(1.0), factor, col0, ap.rows, p.rays + row, aim);
            if (aim) aim_fold(start, smp, f, 0.0, value_of(factor), p.rays + row);
        }
        if (reached && p.transverse) {
            // the transverse rows (x errors, then y errors, after the ray and penalty rows):
            // sqrt(w_t W_(f,l)) sqrt(W_k) times the intercept's derivative
            const int64_t base = static_cast<int64_t>(p.rays) * (soft_mode ? 2 : 1);
            const N factor = N(p.tscale[tu]) * N(smp.root_weight);
            for (int axis = 0; axis < 2; ++axis) {
                const double g[2] = {axis == 0 ? 1.0 : 0.0, axis == 1 ? 1.0 : 0.0};
                const int64_t trow = base + axis * p.rays + row;
                backward_sweep<N>(p, ap.v, record, lay, f, l, ck, true, soft_mode, N(0.0),
                                  N(0.0), factor, col0, ap.rows, trow, aim, g);
                if (aim) aim_fold(start, smp, f, 0.0, value_of(factor), trow);
            }
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
// Uneven batches: run i uses the variables rv.table[i] and the row x + i * rv.stride, and its
// record's surface count is copied from its template into rv.vsurf_out.
__global__ void apply_kernel(const __grid_constant__ VarParams vp, RecordLayout lay,
                             const double* __restrict__ templates, int n_templates,
                             const double* __restrict__ x, double* __restrict__ out, int runs,
                             RunVars rv) {
    const int run = blockIdx.x;
    if (run >= runs) return;
    const int t = n_templates == 1 ? 0 : run;
    const double* src = templates + static_cast<int64_t>(t) * lay.stride;
    double* dst = out + static_cast<int64_t>(run) * lay.stride;
    for (int i = threadIdx.x; i < lay.stride; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        const VarParams& v = rv.table != nullptr ? rv.table[run] : vp;
        const int stride = rv.table != nullptr ? rv.stride : vp.P;
        apply_variables(v, lay, x + static_cast<int64_t>(run) * stride, dst);
        if (rv.vsurf_out != nullptr) rv.vsurf_out[run] = rv.tsurf != nullptr ? rv.tsurf[t] : lay.surfaces;
    }
}

}  // namespace

int launch_apply(const VarParams& vp, const RecordLayout& lay, const double* templates,
                 int n_templates, const double* x, double* out, int runs, cudaStream_t stream,
                 RunVars rv) {
    if (runs <= 0) return MKB_OK;
    apply_kernel<<<runs, 128, 0, stream>>>(vp, lay, templates, n_templates, x, out, runs, rv);
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
    const size_t smem = static_cast<size_t>(tp.stride) * sizeof(double);
    auto kernel = exact ? adjoint_rows_kernel<true> : adjoint_rows_kernel<false>;
    const cudaError_t err = cudaFuncSetAttribute(
        kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (err != cudaSuccess) return cuda_status(err, "adjoint rows: shared memory attribute");
    kernel<<<static_cast<unsigned>(blocks), kAdjThreads, smem, stream>>>(ap, records, J);
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
// Persistent CTAs take runs off a work queue; a CTA streams the run's rays in chunks of
// kFusedThreads (one ray per thread):
//   A  forward trace that stores the ray state entering every surface in the CTA's slot of an
//      L2-resident global scratch (thread-minor, coalesced), then ONE reverse sweep over those
//      states carrying two adjoint vectors (seed OPL = 1 and seed penalty = 1) that share the
//      step-local quantities (warps whose rays need one row run the single-seed sweep). The row
//      y_k = [dOPL_k/dx | OPL_k] goes to shared memory (Y, column-major, residual in column
//      P); the scaled penalty row s_p sqrt(W) dpi/dx goes to the scratch slot;
//   B  per tuple segment of the chunk: weighted column means (a warp per column, shuffle sums)
//      and the rows centred and scaled in place by all threads, x_k = s sqrt(W_k) (y_k -
//      mu_seg); the segment is merged into the tuple's running mean with one extra row
//      s sqrt(W_t W_seg / (W_t + W_seg)) (mu_seg - mu_t) (Chan, Golub, LeVeque). Summed over
//      the chunks, sum x x^T is s^2 sum_k W_k (y_k - ybar)(y_k - ybar)^T over the tuple --
//      exactly [J r]^T [J r] of the piston-projected rows J_k = s sqrt(W_k) (g_k - gbar),
//      r_k = s sqrt(W_k) (OPL_k - piston), with no second pass over the tuple and no J in
//      memory;
//   C  FP64 tensor cores accumulate [J r]^T [J r] (mma.sync m8n8k4 on 8 x 8 tiles of the upper
//      triangle, accumulators in shared memory in fragment order);
//   D  in soft-failure mode, when the chunk has failed rays, the penalty rows (uncentred, value
//      s_p sqrt(W) p_k) are loaded from the scratch slot into Y and accumulated the same way.
// Output: gram [runs][P+1][P+1] as the normal-equation kernels write it.
namespace {

constexpr int kFusedThreads = 128;
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr int kExtraRows = 8;
constexpr int kFusedMinBlocks = 3;  // CTAs per SM the register budget is sized for
// Per ray and table surface c the forward pass keeps, in the CTA's scratch slot, the state
// entering the step c -> c + 1 and that step's StepLocal quantities but mu (kSlotDoubles
// values; mu = n / n' per surface and wavelength is in a shared-memory table of the run).
constexpr int kSlotDoubles = 10;
constexpr bool kFusedDual = true;   // one two-seed sweep for rays with both rows
constexpr int kMaxTileCols = MKB_MAX_VARIABLES / 8;                              // 8
constexpr int kMaxTilePairs = kMaxTileCols * (kMaxTileCols + 1) / 2;             // 36
constexpr int kMaxFusedSlots = 148 * 8;  // persistent CTAs at most (SMs x resident CTAs)
constexpr int kSegBatch = 8;             // tuple segments whose means are held at once

// columns of a row: the P derivatives, the residual in column P, zero padding to 8
__host__ __device__ inline int fused_np(int P) { return ((P + 1 + 7) / 8) * 8; }

// tuple (f-major, then l) of ray q of a run
__device__ __forceinline__ int tuple_of(const TraceParams& p, int q) {
    int f = 0;
    while (f + 1 < p.F && q >= p.field_offset[f + 1]) ++f;
    return f * p.L + (q - p.field_offset[f]) / p.sample_count[f];
}

struct FusedShared {
    uint64_t bar;
    SharedTables tab;
    double w[kFusedThreads];      // sample weight if the ray is in the piston, else 0
    int any_pen;                  // chunk has a penalty row (soft mode)
    int run;                      // run taken off the queue
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

// acc += X^T X for the chunk's rows: X(k, c) = Y[c * ld + k] for the derivative columns
// (type YT) and R[k] for the residual column c = P (FP64 in every variant), k < n (n a
// multiple of 4). Fragment columns past P read the zero padding of Y.
template <class YT>
__device__ __forceinline__ void accumulate_rows(const YT* Y, const double* R, int ld, int P, int n,
                                                int pairs, const int2* tiles, double* acc) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    const int last = P >> 3;  // the column tile holding the residual column
    for (int e = warp; e < pairs; e += kFusedWarps) {
        const int col_a = tiles[e].x * 8 + gid, col_b = tiles[e].y * 8 + gid;
        const YT* ya = Y + col_a * ld + tig;
        const YT* yb = Y + col_b * ld + tig;
        double* a = acc + (e * 32 + lane) * 2;
        double d0 = a[0], d1 = a[1];
        if (tiles[e].y != last) {  // warp-uniform: no residual column in the pair
            for (int k0 = 0; k0 < n; k0 += 4)
                dmma(d0, d1, static_cast<double>(ya[k0]), static_cast<double>(yb[k0]));
        } else {  // upper triangle: x <= y, so column tile x holds P only when x == y == last
            const double* r = R + tig;
            const bool ra = col_a == P, rb = col_b == P;
            for (int k0 = 0; k0 < n; k0 += 4) {
                const double fa = ra ? r[k0] : static_cast<double>(ya[k0]);
                const double fb = rb ? r[k0] : static_cast<double>(yb[k0]);
                dmma(d0, d1, fa, fb);
            }
        }
        a[0] = d0;
        a[1] = d1;
    }
}

// Where the reverse sweep writes: the OPL row (seed 0) and the penalty row (seed 1).
template <int K, class YT>
struct RowSinks {
    double factor[K];
    YT* row[K];
    int ld[K];
};

template <class N, class Q, int kFeat>
__device__ void fused_forward(const TraceParams& p, const double* rec, const double* mu_tab,
                              const RecordLayout& lay, int S, int f, int l, const Sample& smp,
                              bool soft_mode, Q* ck,
                              int stride_ck, uint64_t& br_lo, uint64_t& br_hi, int& count,
                              int& image_branch, int& status_out, int& soft_first, double& opl,
                              double& penalty) {
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
    r.opl = r.py * st;
    SoftT<N> soft{zero, kOk};
    SoftT<N>* sp = soft_mode ? &soft : nullptr;
    br_lo = br_hi = 0;
    count = 1;
    image_branch = kBranchRegular;
    int status = kOk;
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    N n_before = idx[l];
    auto keep_state = [&](Q* q) {
        q[0] = Q(value_of(r.px));
        q[1 * kFusedThreads] = Q(value_of(r.py));
        q[2 * kFusedThreads] = Q(value_of(r.pz));
        q[3 * kFusedThreads] = Q(value_of(r.dx));
        q[4 * kFusedThreads] = Q(value_of(r.dy));
        q[5 * kFusedThreads] = Q(value_of(r.dz));
    };
    for (int s = 1; s < S; ++s) {
        const N n_after = idx[s * L + l];
        const N c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        Q* q = ck + (s - 1) * stride_ck;  // slot s - 1: the state entering this step
        keep_state(q);
        int branch;
        StepLocal<N> loc{zero, zero, zero, zero, zero};
        GhostData gd;
        const bool plate = ghost_at<(kFeat & 2) != 0>(p, rec, lay, s, l, gd);
        status = step_surface_xf<N, true>(r, N(thick[s - 1]), c, n_before, N(mu_tab[s * L + l]),
                                          xf_at<(kFeat & 1) != 0>(rec, lay, s), sp, branch, &loc,
                                          plate ? &gd : nullptr, n_after);
        if (status != kOk) break;
        q[6 * kFusedThreads] = Q(value_of(loc.s0));
        q[7 * kFusedThreads] = Q(value_of(loc.s));
        q[8 * kFusedThreads] = Q(value_of(loc.root_d));
        q[9 * kFusedThreads] = Q(value_of(loc.root_k));
        count = s + 1;
        if (s < 32) br_lo |= static_cast<uint64_t>(branch) << (2 * s);
        else br_hi |= static_cast<uint64_t>(branch) << (2 * (s - 32));
        n_before = n_after;
    }
    if (count == S) keep_state(ck + (S - 1) * stride_ck);  // the state entering the image step
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

// fused_forward in MKB_PRECISION_FP32_BULK (coaxial, no ghost plates): the same kept states and
// step quantities (float slots), traced with step_surface_bulk.
template <class Q>
__device__ void fused_forward_bulk(const TraceParams& p, const double* rec, const double* mu_tab,
                                   const RecordLayout& lay, int S, int f, int l,
                                   const Sample& smp, bool soft_mode, Q* ck, int stride_ck,
                                   uint64_t& br_lo, uint64_t& br_hi, int& count,
                                   int& image_branch, int& status_out, int& soft_first,
                                   double& opl, double& penalty) {
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
    auto keep_state = [&](Q* q) {
        q[0] = Q(r.px);
        q[1 * kFusedThreads] = Q(r.py);
        q[2 * kFusedThreads] = Q(r.pz);
        q[3 * kFusedThreads] = Q(r.dx);
        q[4 * kFusedThreads] = Q(r.dy);
        q[5 * kFusedThreads] = Q(r.dz);
    };
    for (int s = 1; s < S; ++s) {
        const double c = p.type[s] == MKB_SURFACE_SPHERE ? curv[s] : 0.0;
        Q* q = ck + (s - 1) * stride_ck;
        keep_state(q);
        int branch;
        StepLocal<float> loc{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        status = step_surface_bulk<true>(r, thick[s - 1], c, n_before,
                                         static_cast<float>(mu_tab[s * L + l]), sp, branch, &loc);
        if (status != kOk) break;
        q[6 * kFusedThreads] = Q(loc.s0);
        q[7 * kFusedThreads] = Q(loc.s);
        q[8 * kFusedThreads] = Q(loc.root_d);
        q[9 * kFusedThreads] = Q(loc.root_k);
        count = s + 1;
        if (s < 32) br_lo |= static_cast<uint64_t>(branch) << (2 * s);
        else br_hi |= static_cast<uint64_t>(branch) << (2 * (s - 32));
        n_before = idx[s * L + l];
    }
    if (count == S) keep_state(ck + (S - 1) * stride_ck);
    if (status == kOk && soft_mode) status = soft.first;
    if (in_piston(status)) {
        if (!(r.dz > 0.0f)) {
            status = kBackward;
        } else {
            int branch;
            const int rst = reference_step_bulk(r, rec[lay.target + f], thick[S - 1], n_before,
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

// Reverse sweep with K adjoint vectors (seed k: OPL seed so[k], penalty seed sp[k]) writing
// factor_k * dPhi_k/dx into sinks.row[k][col * ld_k]. The states and the step-local
// quantities are in N, the adjoint arithmetic in A (N, or float for the mixed precision). One
// out-of-line copy per K keeps the kernel's instruction footprint small.
template <class N, class A, int K, int kFeat, class Q, class YT>
__device__ __noinline__ void fused_backward(const TraceParams& p, const VarParams& v,
                                            const double* rec, const double* mu_tab,
                                            const RecordLayout& lay, int S,
                                            int f, int l, const Sample& smp, const Q* ck,
                                            int stride_ck, uint64_t br_lo, uint64_t br_hi,
                                            int count, int image_branch, bool reached_image,
                                            bool soft_mode, const double (&so)[K],
                                            const double (&spn)[K],
                                            const RowSinks<K, YT>& sinks,
                                            const double* aim_sens) {
    const int L = p.L;
    const N zero(0.0);
    // interior stop (kernel feature 8): the aimed entrance pupil follows the variables
    constexpr bool kAim = (kFeat & 8) != 0;
    A t0_adj[K];
#pragma unroll
    for (int m = 0; m < K; ++m) t0_adj[m] = A(0.0);
    const double* curv = rec + lay.curvature;
    const double* thick = rec + lay.thickness;
    const double* idx = rec + lay.index;
    const A zero_a(0.0);
    A seed_opl[K], seed_pen[K], factor[K];
    RayAdj<A> adj[K];
#pragma unroll
    for (int m = 0; m < K; ++m) {
        seed_opl[m] = A(so[m]);
        seed_pen[m] = A(spn[m]);
        factor[m] = A(sinks.factor[m]);
        adj[m] = {{zero_a, zero_a, zero_a}, {zero_a, zero_a, zero_a}};
    }
    int next_branch = kBranchRegular;
    const Vec<N> center{zero, N(rec[lay.target + f]), N(thick[S - 1])};
    // glass variables (kernel feature 4): the adjoint of the index of each medium, carried from
    // the step onto s + 1 to the step onto s and written with dn/d(n0, nu1, nu2) = (1, w, w^2)
    constexpr bool kGlass = (kFeat & 4) != 0;
    A n_carry[K];
#pragma unroll
    for (int m = 0; m < K; ++m) n_carry[m] = zero_a;
    auto index_sink = [&](int s, const A (&value)[K]) {
        if constexpr (kGlass) {
            const double w = v.omega[l];
            const A slope[3] = {A(1.0), A(w), A(w) * A(w)};
            for (int c = 0; c < 3; ++c) {
                const int col = v.col_glass[s][c];
                if (col < 0) continue;
#pragma unroll
                for (int m = 0; m < K; ++m)
                    sinks.row[m][col * sinks.ld[m]] =
                        YT(value_of(factor[m] * (value[m] * slope[c])));
            }
        }
    };
    auto branch_of = [&](int s) {
        return s < 32 ? static_cast<int>((br_lo >> (2 * s)) & 3u)
                      : static_cast<int>((br_hi >> (2 * (s - 32))) & 3u);
    };
    // slot c: the state entering step c -> c + 1 and the step's local quantities, loaded one
    // step ahead of their use so the load latency hides behind the current step
    struct Slot {
        Vec<N> p, d;
        StepLocal<N> loc;
    };
    auto load = [&](int c, Slot& sl) {
        const Q* q = ck + c * stride_ck;
        sl.p = {N(q[0]), N(q[kFusedThreads]), N(q[2 * kFusedThreads])};
        sl.d = {N(q[3 * kFusedThreads]), N(q[4 * kFusedThreads]), N(q[5 * kFusedThreads])};
        sl.loc = {N(q[6 * kFusedThreads]), N(q[7 * kFusedThreads]), N(q[8 * kFusedThreads]),
                  N(mu_tab[(c + 1) * L + l]), N(q[9 * kFusedThreads])};
    };
    // the steps below the lowest one that writes a column feed no variable (with the aimed
    // pupil, every column takes the start's adjoint: the sweep runs to the start)
    const int floor_c = kAim ? 0 : v.sweep_floor;
    Slot next;
    load(count - 1, next);
    for (int c = count - 1; c >= floor_c; --c) {
        const Slot cur = next;
        if (c > floor_c) load(c - 1, next);
        if (c == count - 1) {
            if (reached_image && count == S) {
                Vec<A> center_adj[K];
                A n_image_adj[K];
#pragma unroll
                for (int m = 0; m < K; ++m) {
                    center_adj[m] = {zero_a, zero_a, zero_a};
                    n_image_adj[m] = zero_a;
                }
                reference_step_backward_k<N, A, K>(cur.p, cur.d, center, N(idx[(S - 1) * L + l]),
                                                   image_branch, seed_opl, seed_pen, adj,
                                                   center_adj, n_image_adj);
                const int col = v.col_thickness[S - 1];
                if (col >= 0) {
#pragma unroll
                    for (int m = 0; m < K; ++m)
                        sinks.row[m][col * sinks.ld[m]] = YT(value_of(factor[m] * center_adj[m].z));
                }
                if constexpr (kGlass) {
#pragma unroll
                    for (int m = 0; m < K; ++m) n_carry[m] = n_image_adj[m];
                }
            }
        } else {
            const int j = c + 1;
            const bool sphere = p.type[j] == MKB_SURFACE_SPHERE;
            const N cj = sphere ? curv[j] : 0.0;
            StepAdj<A> par[K];
#pragma unroll
            for (int m = 0; m < K; ++m) par[m] = {zero_a, zero_a, zero_a, zero_a};
            GhostData gd;
            // feature 16: every plate lies below the sweep floor, so no reverse step is one
            const bool plate =
                ghost_at<(kFeat & 2) != 0 && (kFeat & 16) == 0>(p, rec, lay, j, l, gd);
            // the step in the surface's own frame: a ghost plate (its profile coefficients
            // are variables too) or a refracting sphere / plane
            auto local = [&](Vec<N> pl, Vec<N> dl, N tl) {
                if (plate) {
                    const int g = p.ghost_of[j];
                    ghost_step_backward_k<N, A, K>(
                        pl, dl, tl, gd, N(idx[c * L + l]), N(idx[j * L + l]), next_branch,
                        seed_opl, seed_pen, adj, par, [&](int m, int k, A value) {
                            const int col = v.col_ghost[g][k];
                            if (col >= 0)
                                sinks.row[m][col * sinks.ld[m]] = YT(value_of(factor[m] * value));
                        });
                } else {
                    refracting_step_backward_k<N, A, K>(pl, dl, tl, cj, N(idx[c * L + l]),
                                                        N(idx[j * L + l]), next_branch, seed_opl,
                                                        seed_pen, adj, par, &cur.loc);
                }
            };
            const double* xf = xf_at<(kFeat & 1) != 0>(rec, lay, j);
            if (xf != nullptr && xf[6] > 0.0) {  // decentered / tilted surface
                const Transform<N> tn = transform_at<N>(xf);
                const Transform<A> ta = transform_at<A>(xf);
                Vec<N> pl = cur.p, dl = cur.d;
                state_to_surface(tn, pl, dl, N(thick[c]));
#pragma unroll
                for (int m = 0; m < K; ++m) adjoint_to_surface(ta, adj[m]);
                local(pl, dl, zero);
#pragma unroll
                for (int m = 0; m < K; ++m) {
                    adjoint_from_surface(ta, adj[m]);
                    par[m].thickness = -adj[m].p.z;
                }
            } else {
                local(cur.p, cur.d, N(thick[c]));
            }
            const int cc = sphere ? v.col_curvature[j] : -1;
            const int ct = v.col_thickness[c];
#pragma unroll
            for (int m = 0; m < K; ++m) {
                if (cc >= 0)
                    sinks.row[m][cc * sinks.ld[m]] = YT(value_of(factor[m] * par[m].curvature));
                if (ct >= 0)
                    sinks.row[m][ct * sinks.ld[m]] = YT(value_of(factor[m] * par[m].thickness));
                if (kAim && c == 0) t0_adj[m] = par[m].thickness;
            }
            if constexpr (kGlass) {
                A value[K];
#pragma unroll
                for (int m = 0; m < K; ++m) {
                    value[m] = par[m].n_after + n_carry[m];
                    n_carry[m] = par[m].n_before;
                }
                index_sink(j, value);
            }
        }
        next_branch = branch_of(c);
    }
    index_sink(0, n_carry);
    if constexpr (kAim) {
        // every column gains dPhi/da da/dx_j + dPhi/dt0 dt0/dx_j (aim_start_adjoint)
        const A st = A(rec[lay.sin_theta + f]);
        const A rho = A(smp.rho), sp = A(smp.sin_phi), cp = A(smp.cos_phi);
#pragma unroll
        for (int m = 0; m < K; ++m) {
            const A ga = rho * (sp * adj[m].p.x + cp * adj[m].p.y) + seed_opl[m] * rho * cp * st;
            for (int k = 0; k < v.P; ++k) {
                YT& y = sinks.row[m][k * sinks.ld[m]];
                y = YT(value_of(A(y) + factor[m] * (ga * A(aim_sens[k]) +
                                                    t0_adj[m] * A(aim_sens[MKB_MAX_VARIABLES + k]))));
            }
        }
    }
}

// Mixed precision: the forward trace (OPL, piston, merit, the states the sweep is linearised
// at) in FP64, the reverse sweep in FP32 on those states rounded to FP32 when they are kept
// (an FP32 trace of the rays themselves misses the OPD bar on aberrated systems; the Jacobian
// tolerates single-precision rounding).
struct MixedPrecision {};
// FP32_BULK: as MIXED, with the forward traced by step_surface_bulk (directions and refraction
// in FP32, positions, intersection and optical path in FP64)
struct BulkPrecision {};

// number types per kernel variant: the forward trace (Fwd), the kept states and the
// quantities the reverse sweep recomputes from them (Bwd), the adjoint arithmetic (Adj), the
// type the states are kept in (Keep), and the type of the derivative columns of the rows in
// shared memory and of the penalty rows in the scratch slot (Row; the residual column is FP64)
template <class N> struct FusedTypes {
    using Fwd = N;
    using Bwd = N;
    using Adj = N;
    using Keep = double;
    using Row = double;
};
template <> struct FusedTypes<MixedPrecision> {
    using Fwd = double;
    using Bwd = float;
    using Adj = float;
    using Keep = float;
    using Row = float;
};
template <> struct FusedTypes<BulkPrecision> : FusedTypes<MixedPrecision> {};

template <class N, int K, int kFeat>
__device__ __forceinline__ void run_backward(const TraceParams& p, const VarParams& v,
                                             const double* rec, const double* mu_tab,
                                             const RecordLayout& lay, int S,
                                             int f, int l, const Sample& smp,
                                             const typename FusedTypes<N>::Keep* ck,
                                             int stride_ck, uint64_t br_lo, uint64_t br_hi,
                                             int count, int image_branch, bool reached_image,
                                             bool soft_mode, const double (&so)[K],
                                             const double (&spn)[K],
                                             const RowSinks<K, typename FusedTypes<N>::Row>& sinks,
                                             const double* aim_sens) {
    using T = FusedTypes<N>;
    fused_backward<typename T::Bwd, typename T::Adj, K, kFeat>(p, v, rec, mu_tab, lay, S, f, l, smp, ck, stride_ck,
                                                        br_lo, br_hi, count, image_branch,
                                                        reached_image, soft_mode, so, spn, sinks,
                                                        aim_sens);
}

template <class T>
struct TypeTag {
    using type = T;
};

struct FusedArgs {
    AdjointParams ap;
    const double* records;
    double* gram;
    double* scratch;       // [slots][slot_doubles]: penalty rows and checkpoints per CTA
    int64_t slot_doubles;
    int* queue;            // run counter
    const int* run_mask;   // runs to process (null: all)
    const int* order;      // queue position -> run (null: identity)
    const int* split;      // device: queue positions [0, *split) and [*split, V) are two
                           // launches (runs with <= 31 and with more variables), or null
    int part;              // 0 or 1: which of the two ranges this launch takes; -1: all
    const VarParams* vt;   // per-run variables (null: ap.v for every run)
    int p_max;             // the largest P (sizes the shared memory and the scratch slots)
    int64_t gram_stride;   // doubles per run of `gram`
};

// kWide: the instance for the runs with more than 31 variables in MIXED; their shared memory
// (64 Gram columns) holds three CTAs per SM, so the register budget is that of three CTAs
template <class N, int kFeat, bool kWide = false>
__global__ void __launch_bounds__(kFusedThreads, (std::is_same<N, MixedPrecision>::value ||
                                                  std::is_same<N, BulkPrecision>::value) &&
                                                         !kWide
                                                     ? 4
                                                     : kFusedMinBlocks)
adjoint_gram_kernel(const __grid_constant__ FusedArgs fa) {
    const TraceParams& p = fa.ap.t;
    __shared__ FusedShared sh;
    __shared__ double aim_sens[(kFeat & 8) != 0 ? 2 * MKB_MAX_VARIABLES : 1];
    extern __shared__ __align__(16) double dyn[];
    const int NPM = fused_np(fa.p_max);  // shared-memory and scratch layout: the largest P
    const int pairs_max = (NPM / 8) * (NPM / 8 + 1) / 2;
    const int stride_ck = kSlotDoubles * kFusedThreads;
    // Column strides = 4 (mod 16) doubles, 4 (mod 32) floats: the lanes of a (half-)warp
    // reading a DMMA fragment (8 columns x 4 rows) then hit different banks; lanes that own
    // consecutive rows of one column (the sweep's writes, the centring) stay conflict-free.
    constexpr int TS = kFusedThreads + 4;              // column stride of Y
    constexpr int ES = kExtraRows + 4;                 // column stride of E
    double* record = dyn;                              // [stride] (bulk-copy target, 16 B aligned)
    double* mu_tab = record + ((p.stride + 1) & ~1);   // [S + 1][L]: mu of step s - 1 -> s
    using YT = typename FusedTypes<N>::Row;
    YT* Y = reinterpret_cast<YT*>(mu_tab + (((p.S + 1) * p.L + 1) & ~1));  // [NPM][TS]
    double* R = reinterpret_cast<double*>(Y + NPM * TS);  // [TS] the residual column
    double* E = R + TS;                                // column-major [NPM][ES]
    double* mu_open = E + NPM * ES;                    // [NPM] running mean of the open tuple
    double* seg_mean = mu_open + NPM;                  // [kSegBatch][NPM] segment means
    double* seg_w = seg_mean + kSegBatch * NPM;        // [kSegBatch] segment weights
    double* acc = seg_w + kSegBatch;                   // [pairs][32][2] DMMA accumulators
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const RecordLayout lay = layout_of(p);
    const bool soft_mode = p.failure == MKB_FAILURE_SOFT;
    // this CTA's scratch slot: penalty rows [NPM][T], then per surface [kSlotDoubles][T]
    using Keep = typename FusedTypes<N>::Keep;
    YT* pen_slot =
        reinterpret_cast<YT*>(fa.scratch + static_cast<int64_t>(blockIdx.x) * fa.slot_doubles);
    Keep* ckpt = reinterpret_cast<Keep*>(pen_slot + NPM * kFusedThreads);
    copy_tables(p, sh.tab);
    // upper-triangle tile pairs in column order: the pairs of a smaller P are a prefix
    for (int e = tid; e < pairs_max; e += kFusedThreads) {
        int j = 0, rem = e;
        while (rem >= j + 1) {
            rem -= j + 1;
            ++j;
        }
        sh.tiles[e] = make_int2(rem, j);
    }
    Keep* my_ck = ckpt + tid;
    uint32_t uses = 0;
    for (;;) {
        __syncthreads();  // the previous run's shared state is consumed
        if (tid == 0) sh.run = atomicAdd(fa.queue, 1);
        __syncthreads();
        int lo = 0, hi = p.V;
        if (fa.split != nullptr && fa.part >= 0) {
            const int mid = *fa.split;
            lo = fa.part == 0 ? 0 : mid;
            hi = fa.part == 0 ? mid : p.V;
        }
        if (lo + sh.run >= hi) break;
        const int run = fa.order != nullptr ? fa.order[lo + sh.run] : lo + sh.run;
        if (fa.run_mask != nullptr && fa.run_mask[run] == 0) continue;
        // the run's variables, columns and surfaces
        const VarParams& v = fa.vt != nullptr ? fa.vt[run] : fa.ap.v;
        const int P = v.P;
        const int NP = fused_np(P);
        const int ncols = NP / 8;
        const int pairs = ncols * (ncols + 1) / 2;
        const int S = surfaces_of(p, run);
        for (int i = tid; i < NPM * ES; i += kFusedThreads) E[i] = 0.0;  // padding stays 0
        // the open tuple (kept identically by every thread): its index, weight, extra rows
        int open_tuple = -1, extra = 0;
        double open_w = 0.0;
        for (int i = tid; i < pairs * 64; i += kFusedThreads) acc[i] = 0.0;
        if (!stage_to_shared(record, fa.records + static_cast<int64_t>(run) * p.stride,
                             static_cast<uint32_t>(p.stride * sizeof(double)), &sh.bar, uses++))
            return;
        // mu = n_before / n_after of every step and wavelength, divided as the step divides
        // it (rows 0 and S .. p.S stay 0: no step)
        for (int i = tid; i < (p.S + 1) * p.L; i += kFusedThreads) {
            const int s = i / p.L, l = i - s * p.L;
            using F = typename FusedTypes<N>::Fwd;
            mu_tab[i] = s >= 1 && s < S
                            ? value_of(F(record[lay.index + (s - 1) * p.L + l]) /
                                       F(record[lay.index + s * p.L + l]))
                            : 0.0;
        }
        if constexpr ((kFeat & 8) != 0)  // interior stop: d(a, t0)/dx of the aimed pupil
            for (int k = tid; k < P; k += kFusedThreads)
                aim_sensitivity(record, lay, v, k, aim_sens[k], aim_sens[MKB_MAX_VARIABLES + k]);
        __syncthreads();
        for (int base = 0; base < p.rays; base += kFusedThreads) {
            const int q = base + tid;
            YT* row = Y + tid;  // this ray's row, column c at row[c * TS]
            for (int c = 0; c < NP; ++c) row[c * TS] = YT(0);
            YT* prow = pen_slot + tid;  // this ray's penalty row, column c at prow[c * T]
            int tu = -1, status = kMissed;
            bool has_pen = false;
            double pen_val = 0.0, opl_val = 0.0;
            Sample smp{};
            if (q < p.rays) {
                int f = 0;
                while (f + 1 < p.F && q >= p.field_offset[f + 1]) ++f;
                const int within = q - p.field_offset[f];
                const int l = within / p.sample_count[f];
                const int k = within - l * p.sample_count[f];
                tu = f * p.L + l;
                smp = pupil_sample(p, sh.tab, f, k);
                int soft_first = kOk, count = 0, image_branch = 0;
                uint64_t br_lo = 0, br_hi = 0;
                double opl = 0.0, penalty = 0.0;
                if constexpr (std::is_same<N, BulkPrecision>::value)
                    fused_forward_bulk<Keep>(p, record, mu_tab, lay, S, f, l, smp, soft_mode,
                                             my_ck, stride_ck, br_lo, br_hi, count,
                                             image_branch, status, soft_first, opl, penalty);
                else
                    fused_forward<typename FusedTypes<N>::Fwd, Keep, kFeat>(p, record, mu_tab, lay, S, f, l, smp, soft_mode,
                                                           my_ck, stride_ck, br_lo, br_hi, count,
                                                           image_branch, status, soft_first, opl,
                                                           penalty);
                const bool piston = in_piston(status);
                has_pen = soft_mode && status != kOk;
                const bool pen_sweep = has_pen && soft_first != kOk;
                const double pfac = has_pen ? p.pscale[tu] * smp.root_weight : 0.0;
                if (has_pen) {
                    for (int c = 0; c < NP; ++c) prow[c * kFusedThreads] = YT(0);
                    pen_val = pfac * (is_soft(status) ? penalty : penalty + 1.0);
                }
                if (piston) opl_val = opl;
                // the OPL row into Y, the penalty row into the scratch slot
                if (kFusedDual && __any_sync(__activemask(), piston && pen_sweep)) {
                    if (piston || pen_sweep) {
                        const double so[2] = {piston ? 1.0 : 0.0, 0.0};
                        const double sp[2] = {0.0, pen_sweep ? 1.0 : 0.0};
                        const RowSinks<2, YT> sinks{{1.0, pfac}, {row, prow}, {TS, kFusedThreads}};
                        run_backward<N, 2, kFeat>(p, v, record, mu_tab, lay, S, f, l, smp, my_ck, stride_ck, br_lo,
                                           br_hi, count, image_branch, piston, soft_mode, so, sp,
                                           sinks, aim_sens);
                    }
                } else if (!(piston && pen_sweep)) {
                    if (piston || pen_sweep) {  // one row: its seed and its sink
                        const double so[1] = {piston ? 1.0 : 0.0};
                        const double sp[1] = {pen_sweep ? 1.0 : 0.0};
                        const RowSinks<1, YT> sinks{{piston ? 1.0 : pfac}, {piston ? row : prow},
                                                {piston ? TS : kFusedThreads}};
                        run_backward<N, 1, kFeat>(p, v, record, mu_tab, lay, S, f, l, smp, my_ck, stride_ck,
                                           br_lo, br_hi, count, image_branch, piston, soft_mode,
                                           so, sp, sinks, aim_sens);
                    }
                } else {  // both rows, one sweep each
                    const double so0[1] = {1.0}, sp0[1] = {0.0};
                    const RowSinks<1, YT> s0{{1.0}, {row}, {TS}};
                    run_backward<N, 1, kFeat>(p, v, record, mu_tab, lay, S, f, l, smp, my_ck, stride_ck, br_lo,
                                       br_hi, count, image_branch, true, soft_mode, so0, sp0, s0,
                                       aim_sens);
                    const double so1[1] = {0.0}, sp1[1] = {1.0};
                    const RowSinks<1, YT> s1{{pfac}, {prow}, {kFusedThreads}};
                    run_backward<N, 1, kFeat>(p, v, record, mu_tab, lay, S, f, l, smp, my_ck, stride_ck, br_lo,
                                       br_hi, count, image_branch, true, soft_mode, so1, sp1, s1,
                                       aim_sens);
                }
            }
            R[tid] = opl_val;
            const double wv = (q < p.rays && in_piston(status)) ? smp.weight : 0.0;
            const double swv = sqrt(wv);
            sh.w[tid] = wv;
            if (tid == 0) sh.any_pen = 0;
            __syncthreads();
            if (has_pen) sh.any_pen = 1;
            // ---- B: centre every tuple segment of the chunk ----
            const int rows_here = p.rays - base < kFusedThreads ? p.rays - base : kFusedThreads;
            // Segments are the chunk's pieces of its tuples; rays are ordered by tuple (f-major,
            // then l), so segment k is tuple t0 + k and its rows follow from the plan alone.
            const int t0 = tuple_of(p, base);
            const int nseg = tuple_of(p, base + rows_here - 1) - t0 + 1;
            const int seg = tid < rows_here ? tu - t0 : -1;
            auto seg_rows = [&](int k, int& a, int& n) {
                const int t = t0 + k;
                const int f = t / p.L;
                const int start = p.field_offset[f] + (t - f * p.L) * p.sample_count[f] - base;
                a = start > 0 ? start : 0;
                const int end = start + p.sample_count[f];
                n = (end < rows_here ? end : rows_here) - a;
                if (n < 0) n = 0;
            };
            for (int k0 = 0; k0 < nseg; k0 += kSegBatch) {
                const int kn = nseg - k0 < kSegBatch ? nseg - k0 : kSegBatch;
                // B2: weight and weighted column means of each segment, four lanes per
                // (segment, column) taking rows h, h + 4, ... (h = lane mod 4) and a two-step
                // shuffle sum. The eight columns of a warp and the four row phases then hit
                // 32 different banks (column stride 4 mod 32 floats).
                {
                    const int h = lane & 3;
                    const unsigned quad = 0xFu << (lane & ~3);
                    for (int pr = tid >> 2; pr < kn * (P + 1); pr += kFusedThreads / 4) {
                        const int k = pr / (P + 1), c = pr - k * (P + 1);
                        int a, n;
                        seg_rows(k0 + k, a, n);
                        const YT* col = Y + c * TS + a;
                        const double* rcol = R + a;
                        const double* wr = sh.w + a;
                        double sw_sum = 0.0, sum = 0.0;
                        if (c != P) {
                            for (int r = h; r < n; r += 4) {
                                sw_sum += wr[r];
                                sum += wr[r] * static_cast<double>(col[r]);
                            }
                        } else {
                            for (int r = h; r < n; r += 4) {
                                sw_sum += wr[r];
                                sum += wr[r] * rcol[r];
                            }
                        }
                        sw_sum += __shfl_xor_sync(quad, sw_sum, 1);
                        sum += __shfl_xor_sync(quad, sum, 1);
                        sw_sum += __shfl_xor_sync(quad, sw_sum, 2);
                        sum += __shfl_xor_sync(quad, sum, 2);
                        if (h == 0) {
                            seg_mean[k * NP + c] = sw_sum > 0.0 ? sum / sw_sum : 0.0;
                            if (c == 0) seg_w[k] = sw_sum;
                        }
                    }
                }
                __syncthreads();
                // B3: every row of the batch's segments centred and scaled by its own thread
                if (seg >= k0 && seg < k0 + kn) {
                    const int k = seg - k0;
                    const double f = (seg_w[k] > 0.0 && wv > 0.0) ? p.scale[tu] * swv : 0.0;
                    const double* m = seg_mean + k * NP;
                    for (int c = 0; c < P; ++c) {
                        YT* y = Y + c * TS + tid;
                        *y = f != 0.0 ? YT(f * (static_cast<double>(*y) - m[c])) : YT(0);
                    }
                    R[tid] = f != 0.0 ? f * (R[tid] - m[P]) : 0.0;
                }
                // B4: the segments merged into the open tuple in row order (threads = columns
                // for the vectors; the scalar state is updated identically by every thread)
                for (int k = 0; k < kn; ++k) {
                    const double ws = seg_w[k];
                    if (!(ws > 0.0)) continue;
                    const int t = t0 + k0 + k;
                    const bool open = open_tuple == t && open_w > 0.0;
                    if (tid <= P) {
                        const double mean = seg_mean[k * NP + tid];
                        if (open) {
                            const double fac = p.scale[t] * sqrt(open_w * ws / (open_w + ws));
                            E[tid * ES + extra] = fac * (mean - mu_open[tid]);
                            mu_open[tid] += (ws / (open_w + ws)) * (mean - mu_open[tid]);
                        } else {
                            mu_open[tid] = mean;
                        }
                    }
                    if (open) {
                        extra += 1;
                        open_w += ws;
                    } else {
                        open_tuple = t;
                        open_w = ws;
                    }
                    if (extra == kExtraRows) {  // flush the extra rows
                        __syncthreads();
                        accumulate(E, ES, kExtraRows, pairs, sh.tiles, acc);
                        __syncthreads();
                        extra = 0;
                    }
                }
                // zero padding of the pending extra rows to a multiple of 4 (each column by
                // the thread that writes it)
                if (tid <= P)
                    for (int r = extra; r < ((extra + 3) & ~3); ++r) E[tid * ES + r] = 0.0;
                __syncthreads();
            }
            // ---- C: the centred rows and the pending extra rows ----
            accumulate_rows(Y, R, TS, P, (rows_here + 3) & ~3, pairs, sh.tiles, acc);
            if (extra > 0) accumulate(E, ES, (extra + 3) & ~3, pairs, sh.tiles, acc);
            __syncthreads();
            extra = 0;
            // ---- D: penalty rows ----
            if (sh.any_pen) {
                for (int c = 0; c < NP; ++c) row[c * TS] = has_pen ? prow[c * kFusedThreads] : YT(0);
                R[tid] = pen_val;
                __syncthreads();
                accumulate_rows(Y, R, TS, P, (rows_here + 3) & ~3, pairs, sh.tiles, acc);
                __syncthreads();
            }
        }
        // ---- write the (P+1) x (P+1) symmetric gram ----
        const int n = P + 1;
        double* G = fa.gram + static_cast<int64_t>(run) * fa.gram_stride;
        for (int i = tid; i < pairs * 64; i += kFusedThreads) {
            const int e = i / 64, ln = (i / 2) & 31, h = i & 1;
            const int r = sh.tiles[e].x * 8 + (ln >> 2);
            const int c = sh.tiles[e].y * 8 + 2 * (ln & 3) + h;
            if (r < n && c < n) {
                G[static_cast<int64_t>(c) * n + r] = acc[i];
                G[static_cast<int64_t>(r) * n + c] = acc[i];
            }
        }
    }
}

}  // namespace

size_t fused_adjoint_smem(const TraceParams& tp, int P, size_t row_bytes) {
    const int NP = fused_np(P);
    const int ncols = NP / 8;
    const int pairs = ncols * (ncols + 1) / 2;
    const size_t rows = (static_cast<size_t>(kFusedThreads + 4) * NP * row_bytes + 7) / 8;
    return sizeof(double) * (static_cast<size_t>((tp.stride + 1) & ~1) +
                             static_cast<size_t>(((tp.S + 1) * tp.L + 1) & ~1) + rows +
                             (kFusedThreads + 4) +
                             (kExtraRows + 4) * NP + NP + kSegBatch * (NP + 1) +
                             static_cast<size_t>(pairs) * 64);
}

namespace {
int64_t fused_slot_doubles(int P, int S) {
    return static_cast<int64_t>(fused_np(P) + kSlotDoubles * S) * kFusedThreads;
}
}  // namespace

// Global scratch of the fused kernel: the queue counter, then one slot per persistent CTA with
// its penalty rows and its checkpoints (rewritten for every chunk, so it stays in L2).
size_t fused_scratch_bytes(int runs, int P, int S) {
    const size_t slots = static_cast<size_t>(runs < kMaxFusedSlots ? runs : kMaxFusedSlots);
    return 256 + slots * fused_slot_doubles(P, S) * sizeof(double);
}

int launch_adjoint_gram(const TraceParams& tp, const VarParams& vp, const double* records,
                        double* gram, void* scratch, size_t scratch_bytes, int precision,
                        cudaStream_t stream, const int* run_mask, RunVars rv,
                        const int* order, const int* split, int part, int part_pmax) {
    if (tp.transverse) {
        set_error("fused adjoint: transverse ray-error rows have no fused adjoint (use the "
                  "materialised adjoint Jacobian or FD)");
        return MKB_ERR_UNSUPPORTED;
    }
    if (tp.V <= 0) return MKB_OK;
    const int p_all = rv.table != nullptr ? rv.stride : vp.P;
    const int p_max = part_pmax > 0 ? part_pmax : p_all;  // sizes this launch's shared memory
    if (scratch == nullptr || scratch_bytes < fused_scratch_bytes(tp.V, p_max, tp.S)) {
        set_error("fused adjoint: scratch of %zu bytes needed",
                  fused_scratch_bytes(tp.V, p_max, tp.S));
        return MKB_ERR_WORKSPACE;
    }
    FusedArgs fa;
    fa.ap.t = tp;
    fa.ap.v = vp;
    fa.ap.rows = 0;
    fa.records = records;
    fa.gram = gram;
    fa.queue = static_cast<int*>(scratch);
    fa.scratch = reinterpret_cast<double*>(static_cast<char*>(scratch) + 256);
    fa.slot_doubles = fused_slot_doubles(p_max, tp.S);
    fa.run_mask = run_mask;
    fa.order = order;
    fa.split = split;
    fa.part = part;
    fa.vt = rv.table;
    fa.p_max = p_max;
    fa.gram_stride = static_cast<int64_t>(p_all + 1) * (p_all + 1);
    const bool float_rows =
        precision == MKB_PRECISION_MIXED || precision == MKB_PRECISION_FP32_BULK;
    const size_t smem = fused_adjoint_smem(tp, p_max, float_rows ? sizeof(float) : sizeof(double));
    if (precision == MKB_PRECISION_FP32_BULK && (tp.non_coaxial || tp.G > 0)) {
        set_error("fused adjoint: FP32_BULK is built for coaxial batches without ghost plates");
        return MKB_ERR_UNSUPPORTED;
    }
    // kernel variant per precision and features (1: surface transforms, 2: ghost plates,
    // 4: glass variables of some run)
    const bool glass = vp.has_glass != 0 || rv.any_glass != 0;
    // 8: an interior aperture stop (coaxial, no ghost plates: the batch check refuses others)
    int feat = (tp.non_coaxial ? 1 : 0) | (tp.G > 0 ? 2 : 0) | (glass ? 4 : 0) |
               (tp.stop > 0 ? 8 : 0);
    // 16 (MIXED, FP64_FMA or FP64, coaxial plates): every plate sits at or below every run's
    // sweep floor, so the reverse sweep never reaches one -- the instance without the plate's
    // reverse step (the same arithmetic for every run: the skipped code is never reached)
    if ((precision == MKB_PRECISION_MIXED || precision == MKB_PRECISION_FP64_FMA ||
         precision == MKB_PRECISION_FP64) &&
        feat == 2) {
        int plate_max = 0;
        for (int s = 0; s < tp.S && s < kMaxSurfaces; ++s)
            if (tp.ghost_of[s] >= 0) plate_max = s;
        const int floor_min = rv.table != nullptr ? rv.min_floor : vp.sweep_floor;
        if (floor_min >= plate_max) feat = 18;
    }
    using Fn = void (*)(FusedArgs);
    auto pick = [&](auto tag) -> Fn {
        using N = typename decltype(tag)::type;
        switch (feat) {
        case 0: return adjoint_gram_kernel<N, 0>;
        case 1: return adjoint_gram_kernel<N, 1>;
        case 2: return adjoint_gram_kernel<N, 2>;
        case 3: return adjoint_gram_kernel<N, 3>;
        case 4: return adjoint_gram_kernel<N, 4>;
        case 5: return adjoint_gram_kernel<N, 5>;
        case 6: return adjoint_gram_kernel<N, 6>;
        case 8: return adjoint_gram_kernel<N, 8>;
        case 12: return adjoint_gram_kernel<N, 12>;
        default: return adjoint_gram_kernel<N, 7>;
        }
    };
    // FP32_BULK: coaxial without plates only (features 0, 4, 8, 12)
    auto pick_bulk = [&]() -> Fn {
        switch (feat) {
        case 4: return adjoint_gram_kernel<BulkPrecision, 4>;
        case 8: return adjoint_gram_kernel<BulkPrecision, 8>;
        case 12: return adjoint_gram_kernel<BulkPrecision, 12>;
        default: return adjoint_gram_kernel<BulkPrecision, 0>;
        }
    };
    // MIXED runs with more than 31 variables (three CTAs per SM by shared memory) on the
    // coaxial features: the instance with the three-CTA register budget
    const bool wide = precision == MKB_PRECISION_MIXED && p_max > 31 &&
                      (feat == 0 || feat == 2 || feat == 18);
    const Fn kernel = wide ? (feat == 0   ? adjoint_gram_kernel<MixedPrecision, 0, true>
                              : feat == 2 ? adjoint_gram_kernel<MixedPrecision, 2, true>
                                          : adjoint_gram_kernel<MixedPrecision, 18, true>)
                      : feat == 18 ? (precision == MKB_PRECISION_MIXED
                                          ? adjoint_gram_kernel<MixedPrecision, 18>
                                      : precision == MKB_PRECISION_FP64
                                          ? adjoint_gram_kernel<Exact64, 18>
                                          : adjoint_gram_kernel<double, 18>)
                      : precision == MKB_PRECISION_FP64    ? pick(TypeTag<Exact64>{})
                      : precision == MKB_PRECISION_MIXED ? pick(TypeTag<MixedPrecision>{})
                      : precision == MKB_PRECISION_FP32_BULK ? pick_bulk()
                                                         : pick(TypeTag<double>{});
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return cuda_status(err, "fused adjoint: shared memory attribute");
    int device = 0, sms = 0, per_sm = 0;
    err = cudaGetDevice(&device);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err == cudaSuccess)
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kFusedThreads, smem);
    if (err != cudaSuccess) return cuda_status(err, "fused adjoint: occupancy");
    if (per_sm < 1) {
        set_error("fused adjoint: %zu bytes of shared memory do not fit an SM", smem);
        return MKB_ERR_UNSUPPORTED;
    }
    int grid = sms * per_sm;
    if (grid > kMaxFusedSlots) grid = kMaxFusedSlots;
    if (grid > tp.V) grid = tp.V;
    err = cudaMemsetAsync(fa.queue, 0, sizeof(int), stream);
    if (err != cudaSuccess) return cuda_status(err, "fused adjoint: clear queue");
    kernel<<<grid, kFusedThreads, smem, stream>>>(fa);
    count_launch();
    return cuda_status(cudaGetLastError(), "fused adjoint launch");
}

}  // namespace mkb
