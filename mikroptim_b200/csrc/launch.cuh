// Host-side launchers shared between the library's translation units (each defined once, in
// the file named beside it), and the per-run mask the LM passes to them.
#pragma once

#include "common.cuh"

namespace mkb {

// Which variants a launch works on: variant v is processed when mask[offset + v / div] != 0
// (a null mask processes all). The LM uses it to trace and differentiate only the runs that
// need it in a cycle; the rest of the launch returns at once, so the launch sequence (and a
// CUDA graph of it) stays fixed.
struct RunMask {
    const int* mask = nullptr;
    int div = 1;
    int offset = 0;
};

__device__ __forceinline__ bool run_active(const RunMask& m, int v) {
    return m.mask == nullptr || m.mask[m.offset + v / m.div] != 0;
}

// Per-run variables of an uneven batch: run i uses table[i] (device) and the row x + i * stride
// (stride = the largest P); apply writes each run record's surface count, copied from its
// template's (tsurf, or the table's S when null), into vsurf_out. A null table: every run uses
// the launch's VarParams.
struct RunVars {
    const VarParams* table = nullptr;
    int stride = 0;
    const uint8_t* tsurf = nullptr;
    uint8_t* vsurf_out = nullptr;
    int any_glass = 0;  // some run of the table has glass variables
    int min_floor = 0;  // the smallest sweep floor of the table's runs (0: not known)
};

// trace.cu
// extrema: [V][S][2] per-surface (largest ray height, smallest cos I) of the valid rays, or
// null (TraceSettings::extrema, include/mikroptim/batch/batch_extrema.hpp)
int launch_residuals(const TraceParams& p, const double* records, double* residuals,
                     int64_t stride, double* opd, uint8_t* status, int precision,
                     cudaStream_t stream, RunMask mask = {}, double* extrema = nullptr);
int launch_merit(const TraceParams& p, const double* records, double* merit, int64_t* failed,
                 int64_t* hard, void* workspace, size_t ws_bytes, int precision,
                 cudaStream_t stream, RunMask mask = {}, const double* extra = nullptr,
                 double* extrema = nullptr);
size_t merit_workspace_bytes(int V, int n_tuples);
int pack_rays_default();
// largest pack a caller may ask for (mkb_trace_options.pack_rays is clamped to it)
constexpr int kMaxPackRaysOption = 4096;
// most variants one trace CTA may take (mkb_trace_options.variants_per_cta)
constexpr int kMaxVariantsPerCta = 8;

// adjoint.cu
int launch_apply(const VarParams& vp, const RecordLayout& lay, const double* templates,
                 int n_templates, const double* x, double* out, int runs, cudaStream_t stream,
                 RunVars rv = {});
int launch_adjoint_rows(const TraceParams& tp, const VarParams& vp, int64_t rows,
                        const double* records, double* J, bool exact, cudaStream_t stream);
int launch_projection(const TraceParams& tp, const VarParams& vp, int64_t rows,
                      const uint8_t* status, double* J, bool exact, cudaStream_t stream);
int launch_adjoint_gram(const TraceParams& tp, const VarParams& vp, const double* records,
                        double* gram, void* scratch, size_t scratch_bytes, int precision,
                        cudaStream_t stream, const int* run_mask = nullptr, RunVars rv = {},
                        const int* order = nullptr, const int* split = nullptr, int part = -1,
                        int part_pmax = 0);
size_t fused_scratch_bytes(int runs, int P, int S);

// gram.cu
int launch_gram(const double* J, const double* r, int runs, int P, int64_t R, double* gram,
                bool exact, cudaStream_t stream, const int* run_mask = nullptr, RunVars rv = {});

// jacobian.cu: the FD Jacobian of mkb_fd_jacobian_device for the runs the mask selects
int fd_jacobian(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                const mkb_variables* vars, const double* x0, int runs, double* J, double* r0,
                int64_t* status_changes, void* workspace, size_t workspace_bytes,
                cudaStream_t stream, const int* run_mask, RunVars rv);

// device error words, one per translation unit
int trace_device_error();
int gram_device_error();
int adjoint_device_error();
int jacobian_device_error();
int lm_device_error();
int prefilter_device_error();
int trace_device_error_wait_limit(uint32_t polls);
int gram_device_error_wait_limit(uint32_t polls);
int adjoint_device_error_wait_limit(uint32_t polls);
int jacobian_device_error_wait_limit(uint32_t polls);
int lm_device_error_wait_limit(uint32_t polls);
int prefilter_device_error_wait_limit(uint32_t polls);

}  // namespace mkb
