// Jacobian entry points: finite differences (the reference method) and the adjoint sweep.
//
// FD (central scheme, 2P + 1 variants per run; reference: fd_pattern and write_fd_variants,
// src/optim/variant_generator.cpp:177,248; fd_jacobian_from_residuals,
// src/optim/fd_jacobian.cpp:80; fd_difference_kernel, src/cuda/fd_jacobian.cu:65):
//   1. fd_pattern_kernel  one thread per (run, variable): step h, stencil, points, steps
//   2. fd_build_kernel    one CTA per FD variant: template record + x0 + the perturbed entry
//   3. RESIDUALS          the trace kernel over all FD variants of a chunk of runs
//   4. fd_difference_kernel / fd_changes_kernel: columns by fd_derivative, status changes
// Runs are processed in chunks sized by the workspace the caller passes.
//
// Adjoint (reference: DeviceAdjointJacobian::compute, src/cuda/adjoint_jacobian.cu:401):
//   apply x0 -> RESIDUALS (r0, status) -> adjoint rows -> piston projection.
#include "fd.cuh"
#include "launch.cuh"

#include <algorithm>
#include <vector>
#include <type_traits>

namespace mkb {

namespace {

// Run i's variable k is entry i * pstride + k (pstride = P, or the largest P of an uneven batch
// whose run i uses vt[i]).
__global__ void fd_pattern_kernel(const __grid_constant__ VarParams vp, const double* x0, int runs,
                                  FdPattern* pattern, const VarParams* vt, int pstride) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= runs * pstride) return;
    const int run = id / pstride, k = id - run * pstride;
    const VarParams& v = vt != nullptr ? vt[run] : vp;
    if (k >= v.P) return;
    pattern[id] = fd_pattern_of<Exact64>(x0[id], v.lower[k], v.upper[k], v.typical[k]);
}

// One CTA per FD variant j of run i (variant i*n + j, n = 2 pstride + 1): template record, x0
// applied, entry k replaced by x_a (j = 2k + 1) or x_b (j = 2k + 2). active[variant] tells the
// trace which variants to trace (the run is wanted and j < 2 P_i + 1); vsurf[variant] is the
// template's surface count (uneven batches).
__global__ void fd_build_kernel(const __grid_constant__ VarParams vp, RecordLayout lay,
                                const double* __restrict__ templates, int n_templates,
                                const double* __restrict__ x0, const FdPattern* __restrict__ pat,
                                int first_run, int runs, double* __restrict__ out,
                                const int* __restrict__ run_mask, const VarParams* vt,
                                int pstride, const uint8_t* tsurf, int* __restrict__ active,
                                uint8_t* __restrict__ vsurf) {
    const int n = 2 * pstride + 1;
    const int local = blockIdx.x / n;
    const int j = blockIdx.x - local * n;
    const int run = first_run + local;
    const VarParams& v = vt != nullptr ? vt[run] : vp;
    const bool on = (run_mask == nullptr || run_mask[run] != 0) && j < 2 * v.P + 1;
    if (threadIdx.x == 0) active[blockIdx.x] = on ? 1 : 0;
    if (!on) return;
    const int t = n_templates == 1 ? 0 : run;
    if (threadIdx.x == 0 && vsurf != nullptr) vsurf[blockIdx.x] = tsurf != nullptr ? tsurf[t] : lay.surfaces;
    const double* src = templates + static_cast<int64_t>(t) * lay.stride;
    double* dst = out + static_cast<int64_t>(blockIdx.x) * lay.stride;
    for (int i = threadIdx.x; i < lay.stride; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        const double* x = x0 + static_cast<int64_t>(run) * pstride;
        apply_variables(v, lay, x, dst);
        if (j > 0) {
            const int k = (j - 1) / 2;
            const FdPattern& p = pat[static_cast<int64_t>(run) * pstride + k];
            const double y = (j & 1) ? p.xa : p.xb;
            write_variable(v, lay, k, y, dst);
            refresh_glass(v, lay, dst);  // a perturbed Buchdahl coefficient moves the index
            if (lay.stop > 0) aim_record(lay, dst);  // and the entrance pupil follows
        }
    }
}

// J(r, k) = fd_derivative(stencil, r0, r_a, r_b, d_a, d_b) (optim/fd_formula.hpp:40), r0 rows.
template <bool kExact>
__global__ void fd_difference_kernel(const double* __restrict__ res, const FdPattern* __restrict__ pat,
                                     int P, int64_t R, int first_run, int runs,
                                     double* __restrict__ J, double* __restrict__ r0,
                                     const int* __restrict__ run_mask, const VarParams* vt) {
    using N = typename std::conditional<kExact, Exact64, double>::type;
    const int n = 2 * P + 1;
    const int64_t total = static_cast<int64_t>(runs) * (P + 1) * R;
    for (int64_t id = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; id < total;
         id += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t r = id % R;
        const int64_t ck = id / R;
        const int c = static_cast<int>(ck % (P + 1));
        const int local = static_cast<int>(ck / (P + 1));
        const int run = first_run + local;
        if (run_mask != nullptr && run_mask[run] == 0) continue;
        if (vt != nullptr && c < P && c >= vt[run].P) continue;  // past this run's variables
        const double* base = res + static_cast<int64_t>(local) * n * R;
        if (c == P) {
            r0[static_cast<int64_t>(run) * R + r] = base[r];
            continue;
        }
        const FdPattern p = pat[static_cast<int64_t>(run) * P + c];
        J[(static_cast<int64_t>(run) * P + c) * R + r] = fd_derivative_of<N>(
            p.stencil, base[r], base[static_cast<int64_t>(2 * c + 1) * R + r],
            base[static_cast<int64_t>(2 * c + 2) * R + r], p.da, p.db);
    }
}

// Rays whose validity (status Ok) changes between x0 and a perturbed point of column k.
__global__ void fd_changes_kernel(const uint8_t* __restrict__ status, int P, int64_t rays,
                                  int first_run, int64_t* __restrict__ changes,
                                  const VarParams* vt) {
    const int n = 2 * P + 1;
    const int local = blockIdx.x / P;
    const int k = blockIdx.x - local * P;
    if (vt != nullptr && k >= vt[first_run + local].P) {
        if (threadIdx.x == 0) changes[static_cast<int64_t>(first_run + local) * P + k] = 0;
        return;
    }
    const uint8_t* s0 = status + static_cast<int64_t>(local) * n * rays;
    const uint8_t* sa = s0 + static_cast<int64_t>(2 * k + 1) * rays;
    const uint8_t* sb = s0 + static_cast<int64_t>(2 * k + 2) * rays;
    int count = 0;
    for (int64_t r = threadIdx.x; r < rays; r += blockDim.x) {
        const bool ok0 = s0[r] == kOk;
        count += ((sa[r] == kOk) != ok0) || ((sb[r] == kOk) != ok0);
    }
    __shared__ int part[256];
    part[threadIdx.x] = count;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (static_cast<int>(threadIdx.x) < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) changes[static_cast<int64_t>(first_run + local) * P + k] = part[0];
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

struct FdSizes {
    size_t pattern, records, residuals, status, total_fixed, per_run;
};

// Workspace of the FD Jacobian: the step patterns of all runs, then per chunk of runs the FD
// variants' records, residuals, statuses, trace mask and surface counts (each 256-B aligned).
FdSizes fd_sizes(int stride, int P, int64_t R, int64_t rays, int runs) {
    FdSizes z;
    const int n = 2 * P + 1;
    z.pattern = align256(sizeof(FdPattern) * static_cast<size_t>(runs) * P);
    z.per_run = sizeof(double) * static_cast<size_t>(n) * stride +
                sizeof(double) * static_cast<size_t>(n) * R + static_cast<size_t>(n) * rays +
                sizeof(int) * static_cast<size_t>(n) + static_cast<size_t>(n);
    z.total_fixed = z.pattern + 5 * 256;
    return z;
}

int check_templates(const mkb_device_batch* t, int runs) {
    if (t == nullptr || (t->variants != 1 && t->variants != runs)) {
        set_error("templates must hold 1 variant or one per run (%d runs)", runs);
        return MKB_ERR_ARGUMENT;
    }
    return MKB_OK;
}

}  // namespace

MKB_DEFINE_ERROR_READER(jacobian_device_error)

}  // namespace mkb

using namespace mkb;

namespace mkb {

int fd_jacobian(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                const mkb_variables* vars, const double* x0, int runs, double* J, double* r0,
                int64_t* status_changes, void* workspace, size_t workspace_bytes,
                cudaStream_t stream, const int* run_mask, RunVars rv) {
    if (runs < 0) {
        set_error("fd jacobian: runs must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (runs == 0) return MKB_OK;
    int rc = check_templates(templates, runs);
    if (rc != MKB_OK) return rc;
    TraceParams tp;
    mkb_device_batch fdb = *templates;
    fdb.variants = 1;
    rc = make_trace_params(&fdb, plan, pack_rays_default(), &tp);
    if (rc != MKB_OK) return rc;
    if (plan->precision != MKB_PRECISION_FP64 && plan->precision != MKB_PRECISION_FP64_FMA) {
        set_error("fd jacobian: precision %d not available", plan->precision);
        return MKB_ERR_UNSUPPORTED;
    }
    VarParams vp{};
    if (rv.table == nullptr) {
        rc = make_var_params(vars, tp.S, templates->type, &vp, templates->ghost_terms,
                             templates->wavelengths, templates->wavelength_nm,
                             templates->glass);
        if (rc != MKB_OK) return rc;
    }
    if (!x0 || !J || !r0) {
        set_error("fd jacobian: null pointer");
        return MKB_ERR_ARGUMENT;
    }
    const bool exact = plan->precision == MKB_PRECISION_FP64;
    const int P = rv.table != nullptr ? rv.stride : vp.P, n = 2 * P + 1;
    const int64_t R = trace_rows_of(plan, tp.rays);
    const FdSizes z = fd_sizes(tp.stride, P, R, tp.rays, runs);
    if (workspace == nullptr || workspace_bytes < z.total_fixed + z.per_run) {
        set_error("fd jacobian: workspace of at least %zu bytes needed (one run per chunk)",
                  z.total_fixed + z.per_run);
        return MKB_ERR_WORKSPACE;
    }
    const int chunk = static_cast<int>(
        std::min<size_t>((workspace_bytes - z.total_fixed) / z.per_run, static_cast<size_t>(runs)));
    char* ws = static_cast<char*>(workspace);
    FdPattern* pattern = reinterpret_cast<FdPattern*>(ws);
    char* chunk_base = ws + z.pattern;
    double* records = reinterpret_cast<double*>(chunk_base);
    double* res = reinterpret_cast<double*>(
        chunk_base + align256(sizeof(double) * static_cast<size_t>(chunk) * n * tp.stride));
    uint8_t* status = reinterpret_cast<uint8_t*>(
        reinterpret_cast<char*>(res) + align256(sizeof(double) * static_cast<size_t>(chunk) * n * R));
    int* active = reinterpret_cast<int*>(
        reinterpret_cast<char*>(status) + align256(static_cast<size_t>(chunk) * n * tp.rays));
    uint8_t* vsurf = reinterpret_cast<uint8_t*>(
        reinterpret_cast<char*>(active) + align256(sizeof(int) * static_cast<size_t>(chunk) * n));
    const RecordLayout lay = layout_of(tp);
    const bool uneven_surfaces = templates->variant_surfaces != nullptr;

    fd_pattern_kernel<<<(runs * P + 127) / 128, 128, 0, stream>>>(vp, x0, runs, pattern,
                                                                  rv.table, P);
    count_launch();
    rc = cuda_status(cudaGetLastError(), "fd pattern launch");
    for (int first = 0; rc == MKB_OK && first < runs; first += chunk) {
        const int cnt = std::min(chunk, runs - first);
        fd_build_kernel<<<cnt * n, 128, 0, stream>>>(
            vp, lay, templates->records, templates->variants, x0, pattern, first, cnt, records,
            run_mask, rv.table, P, templates->variant_surfaces, active,
            uneven_surfaces ? vsurf : nullptr);
        count_launch();
        rc = cuda_status(cudaGetLastError(), "fd build launch");
        if (rc != MKB_OK) break;
        TraceParams chunk_tp = tp;
        chunk_tp.V = cnt * n;
        chunk_tp.vsurf = uneven_surfaces ? vsurf : nullptr;
        rc = launch_residuals(chunk_tp, records, res, R, nullptr, status, plan->precision, stream,
                              RunMask{active, 1, 0});
        if (rc != MKB_OK) break;
        const int64_t total = static_cast<int64_t>(cnt) * (P + 1) * R;
        const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 64));
        if (exact)
            fd_difference_kernel<true><<<blocks, 256, 0, stream>>>(res, pattern, P, R, first, cnt,
                                                                   J, r0, run_mask, rv.table);
        else
            fd_difference_kernel<false><<<blocks, 256, 0, stream>>>(res, pattern, P, R, first, cnt,
                                                                    J, r0, run_mask, rv.table);
        count_launch();
        rc = cuda_status(cudaGetLastError(), "fd difference launch");
        if (rc != MKB_OK || status_changes == nullptr) continue;
        fd_changes_kernel<<<cnt * P, 256, 0, stream>>>(status, P, tp.rays, first, status_changes,
                                                       rv.table);
        count_launch();
        rc = cuda_status(cudaGetLastError(), "fd status-change launch");
    }
    return rc;
}

}  // namespace mkb

namespace mkb {
namespace {

// The fused adjoint + normal equations of mkb_adjoint_normal_equations_device and, with
// per_run, of mkb_adjoint_normal_equations_runs_device (vars: one set per run).
int adjoint_normal_equations(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, bool per_run, const double* x0,
                             int runs, double* gram, void* workspace, size_t workspace_bytes,
                             cudaStream_t stream) {
    if (runs < 0) {
        set_error("adjoint normal equations: runs must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (runs == 0) return MKB_OK;
    int rc = check_templates(templates, runs);
    if (rc != MKB_OK) return rc;
    if (templates->variant_surfaces != nullptr && templates->variants != runs) {
        set_error("adjoint normal equations: uneven templates need one template per run");
        return MKB_ERR_ARGUMENT;
    }
    TraceParams tp;
    mkb_device_batch b = *templates;
    b.variants = runs;
    rc = make_trace_params(&b, plan, pack_rays_default(), &tp);
    if (rc != MKB_OK) return rc;
    if (plan->precision != MKB_PRECISION_FP64 && plan->precision != MKB_PRECISION_FP64_FMA &&
        plan->precision != MKB_PRECISION_MIXED && plan->precision != MKB_PRECISION_FP32_BULK) {
        set_error("adjoint normal equations: precision %d not available", plan->precision);
        return MKB_ERR_UNSUPPORTED;
    }
    if (vars == nullptr || !x0 || !gram) {
        set_error("adjoint normal equations: null pointer");
        return MKB_ERR_ARGUMENT;
    }
    VarParams vp;
    rc = make_var_params(&vars[0], tp.S, templates->type, &vp, templates->ghost_terms,
                         templates->wavelengths, templates->wavelength_nm,
                         templates->glass);
    if (rc != MKB_OK) return rc;
    std::vector<VarParams> table;
    int pmax = vp.P;
    if (per_run) {
        table.resize(static_cast<size_t>(runs));
        for (int r = 0; r < runs; ++r) {
            rc = make_var_params(&vars[r], tp.S, templates->type, &table[r],
                                 templates->ghost_terms, templates->wavelengths,
                                 templates->wavelength_nm, templates->glass);
            if (rc != MKB_OK) return rc;
            pmax = table[r].P > pmax ? table[r].P : pmax;
        }
    }
    const size_t need = per_run ? mkb_adjoint_normal_equations_runs_workspace_bytes(templates,
                                                                                    vars, runs)
                                : mkb_adjoint_jacobian_workspace_bytes(templates, runs);
    if (workspace == nullptr || workspace_bytes < need) {
        set_error("adjoint normal equations: workspace of %zu bytes needed", need);
        return MKB_ERR_WORKSPACE;
    }
    char* ws = static_cast<char*>(workspace);
    double* records = reinterpret_cast<double*>(ws);
    const size_t rec_bytes = align256(sizeof(double) * static_cast<size_t>(runs) *
                                      templates->record_stride);
    RunVars rv;
    size_t table_bytes = 0;  // per run: the variable table and the run order follow the records
    int* order = nullptr;
    constexpr int kSmallP = 31;  // runs with at most this many variables go first, in a launch
                                 // with a smaller shared-memory footprint
    std::vector<int> host_order;  // [runs] order, then the size of the first group
    if (per_run) {
        table_bytes = align256(sizeof(VarParams) * static_cast<size_t>(runs)) +
                      align256(sizeof(int) * (static_cast<size_t>(runs) + 1));
        VarParams* dtable = reinterpret_cast<VarParams*>(ws + rec_bytes);
        order = reinterpret_cast<int*>(ws + rec_bytes +
                                       align256(sizeof(VarParams) * static_cast<size_t>(runs)));
        for (int r = 0; r < runs; ++r)
            if (table[r].P <= kSmallP) host_order.push_back(r);
        const int small = static_cast<int>(host_order.size());
        for (int r = 0; r < runs; ++r)
            if (table[r].P > kSmallP) host_order.push_back(r);
        host_order.push_back(small);
        rc = cuda_status(cudaMemcpyAsync(dtable, table.data(), sizeof(VarParams) * table.size(),
                                         cudaMemcpyHostToDevice, stream),
                         "adjoint normal equations: upload variables");
        if (rc == MKB_OK)
            rc = cuda_status(cudaMemcpyAsync(order, host_order.data(),
                                             sizeof(int) * host_order.size(),
                                             cudaMemcpyHostToDevice, stream),
                             "adjoint normal equations: upload order");
        if (rc != MKB_OK) return rc;
        rv.table = dtable;
        rv.stride = pmax;
        rv.min_floor = kMaxSurfaces;
        for (const VarParams& t : table) {
            rv.any_glass |= t.has_glass;
            rv.min_floor = t.sweep_floor < rv.min_floor ? t.sweep_floor : rv.min_floor;
        }
    }
    const RecordLayout lay = layout_of(tp);
    rc = launch_apply(vp, lay, templates->records, templates->variants, x0, records, runs, stream,
                      rv);
    if (rc != MKB_OK) return rc;
    void* scratch = ws + rec_bytes + table_bytes;
    const size_t scratch_bytes = workspace_bytes - rec_bytes - table_bytes;
    if (per_run && pmax > kSmallP) {
        rc = launch_adjoint_gram(tp, vp, records, gram, scratch, scratch_bytes, plan->precision,
                                 stream, nullptr, rv, order, order + runs, 0, kSmallP);
        if (rc != MKB_OK) return rc;
        return launch_adjoint_gram(tp, vp, records, gram, scratch, scratch_bytes, plan->precision,
                                   stream, nullptr, rv, order, order + runs, 1, pmax);
    }
    return launch_adjoint_gram(tp, vp, records, gram, scratch, scratch_bytes, plan->precision,
                               stream, nullptr, rv, order);
}

}  // namespace
}  // namespace mkb

extern "C" {

int mkb_fd_pattern_host(const mkb_variables* vars, const double* x, int32_t runs,
                        double* point_plus, double* point_minus, double* step_plus,
                        double* step_minus, int32_t* stencil) {
    if (vars == nullptr || vars->count < 1 || vars->lower == nullptr || vars->upper == nullptr ||
        vars->typical == nullptr || x == nullptr || runs < 0 || point_plus == nullptr ||
        point_minus == nullptr || step_plus == nullptr || step_minus == nullptr ||
        stencil == nullptr) {
        set_error("fd pattern: null argument or no variables");
        return MKB_ERR_ARGUMENT;
    }
    const int P = vars->count;
    for (int64_t i = 0; i < static_cast<int64_t>(runs) * P; ++i) {
        const int k = static_cast<int>(i % P);
        const FdPattern f = fd_pattern_of<double>(x[i], vars->lower[k], vars->upper[k],
                                                  vars->typical[k]);
        point_plus[i] = f.xa;
        point_minus[i] = f.xb;
        step_plus[i] = f.da;
        step_minus[i] = f.db;
        stencil[i] = f.stencil;
    }
    return MKB_OK;
}

int mkb_fd_derivative_host(int32_t stencil, double step_plus, double step_minus, int32_t rows,
                           const double* r0, const double* r_plus, const double* r_minus,
                           double* column) {
    if (rows < 0 || (rows > 0 && (r0 == nullptr || r_plus == nullptr || r_minus == nullptr ||
                                  column == nullptr)) ||
        stencil < kCentral || stencil > kTruncated) {
        set_error("fd derivative: bad arguments");
        return MKB_ERR_ARGUMENT;
    }
    for (int e = 0; e < rows; ++e)
        column[e] = fd_derivative_of<double>(stencil, r0[e], r_plus[e], r_minus[e], step_plus,
                                             step_minus);
    return MKB_OK;
}

size_t mkb_fd_jacobian_workspace_bytes(const mkb_device_batch* templates,
                                       const mkb_residual_plan* plan, int32_t P, int32_t runs,
                                       int32_t runs_per_chunk) {
    TraceParams tp;
    if (templates == nullptr || P < 1 || runs < 1 || runs_per_chunk < 1) return 0;
    mkb_device_batch one = *templates;
    one.variants = 1;
    if (make_trace_params(&one, plan, pack_rays_default(), &tp) != MKB_OK) return 0;
    const int64_t rows = trace_rows_of(plan, tp.rays);
    const FdSizes z = fd_sizes(tp.stride, P, rows, tp.rays, runs);
    return z.total_fixed + z.per_run * static_cast<size_t>(runs_per_chunk < runs ? runs_per_chunk : runs);
}

int mkb_fd_jacobian_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                           const mkb_variables* vars, const double* x0, int32_t runs, double* J,
                           double* r0, int64_t* status_changes, void* workspace,
                           size_t workspace_bytes, void* stream_ptr) {
    return fd_jacobian(templates, plan, vars, x0, runs, J, r0, status_changes, workspace,
                       workspace_bytes, static_cast<cudaStream_t>(stream_ptr), nullptr, {});
}

size_t mkb_adjoint_jacobian_workspace_bytes(const mkb_device_batch* templates, int32_t runs) {
    if (templates == nullptr || runs < 0) return 0;
    return align256(sizeof(double) * static_cast<size_t>(runs) * templates->record_stride) +
           fused_scratch_bytes(runs, MKB_MAX_VARIABLES, templates->surfaces);
}

int mkb_adjoint_jacobian_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                                const mkb_variables* vars, const double* x0, int32_t runs,
                                double* J, double* r0, uint8_t* status, void* workspace,
                                size_t workspace_bytes, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    if (runs < 0) {
        set_error("adjoint jacobian: runs must be >= 0");
        return MKB_ERR_ARGUMENT;
    }
    if (runs == 0) return MKB_OK;
    int rc = check_templates(templates, runs);
    if (rc != MKB_OK) return rc;
    if (templates->variant_surfaces != nullptr) {
        set_error("adjoint jacobian: uneven batches run with the fused adjoint "
                  "(mkb_adjoint_normal_equations_device) or finite differences");
        return MKB_ERR_UNSUPPORTED;
    }
    TraceParams tp;
    mkb_device_batch b = *templates;
    b.variants = runs;
    rc = make_trace_params(&b, plan, pack_rays_default(), &tp);
    if (rc != MKB_OK) return rc;
    if (plan->precision != MKB_PRECISION_FP64 && plan->precision != MKB_PRECISION_FP64_FMA) {
        set_error("adjoint jacobian: precision %d not available", plan->precision);
        return MKB_ERR_UNSUPPORTED;
    }
    VarParams vp;
    rc = make_var_params(vars, tp.S, templates->type, &vp, templates->ghost_terms,
                         templates->wavelengths, templates->wavelength_nm,
                         templates->glass);
    if (rc != MKB_OK) return rc;
    if (!x0 || !J || !r0 || !status) {
        set_error("adjoint jacobian: null pointer");
        return MKB_ERR_ARGUMENT;
    }
    const size_t need = mkb_adjoint_jacobian_workspace_bytes(templates, runs);
    if (workspace == nullptr || workspace_bytes < need) {
        set_error("adjoint jacobian: workspace of %zu bytes needed", need);
        return MKB_ERR_WORKSPACE;
    }
    const bool exact = plan->precision == MKB_PRECISION_FP64;
    const int64_t R = trace_rows_of(plan, tp.rays);
    double* records = static_cast<double*>(workspace);
    const RecordLayout lay = layout_of(tp);
    rc = launch_apply(vp, lay, templates->records, templates->variants, x0, records, runs, stream);
    if (rc != MKB_OK) return rc;
    rc = cuda_status(cudaMemsetAsync(J, 0, sizeof(double) * static_cast<size_t>(runs) * vp.P * R,
                                     stream), "adjoint jacobian: clear J");
    if (rc != MKB_OK) return rc;
    rc = launch_residuals(tp, records, r0, R, nullptr, status, plan->precision, stream);
    if (rc != MKB_OK) return rc;
    rc = launch_adjoint_rows(tp, vp, R, records, J, exact, stream);
    if (rc != MKB_OK) return rc;
    return launch_projection(tp, vp, R, status, J, exact, stream);
}

int mkb_adjoint_normal_equations_runs_device(const mkb_device_batch* templates,
                                             const mkb_residual_plan* plan,
                                             const mkb_variables* vars, const double* x0,
                                             int32_t runs, double* gram, void* workspace,
                                             size_t workspace_bytes, void* stream_ptr);

int mkb_adjoint_normal_equations_device(const mkb_device_batch* templates,
                                        const mkb_residual_plan* plan, const mkb_variables* vars,
                                        const double* x0, int32_t runs, double* gram,
                                        void* workspace, size_t workspace_bytes,
                                        void* stream_ptr) {
    return adjoint_normal_equations(templates, plan, vars, false, x0, runs, gram, workspace,
                                    workspace_bytes, static_cast<cudaStream_t>(stream_ptr));
}

size_t mkb_adjoint_normal_equations_runs_workspace_bytes(const mkb_device_batch* templates,
                                                         const mkb_variables* vars,
                                                         int32_t runs) {
    if (templates == nullptr || vars == nullptr || runs < 0) return 0;
    int pmax = 1;
    for (int r = 0; r < runs; ++r) pmax = vars[r].count > pmax ? vars[r].count : pmax;
    if (pmax > MKB_MAX_VARIABLES) return 0;
    return align256(sizeof(double) * static_cast<size_t>(runs) * templates->record_stride) +
           fused_scratch_bytes(runs, pmax, templates->surfaces) +
           align256(sizeof(VarParams) * static_cast<size_t>(runs)) +
           align256(sizeof(int) * (static_cast<size_t>(runs) + 1));
}

int mkb_adjoint_normal_equations_runs_device(const mkb_device_batch* templates,
                                             const mkb_residual_plan* plan,
                                             const mkb_variables* vars, const double* x0,
                                             int32_t runs, double* gram, void* workspace,
                                             size_t workspace_bytes, void* stream_ptr) {
    return adjoint_normal_equations(templates, plan, vars, true, x0, runs, gram, workspace,
                                    workspace_bytes, static_cast<cudaStream_t>(stream_ptr));
}

}  // extern "C"
