/*
 * mikroptim_b200.h -- C ABI of the B200 (sm_100a) batched trace-and-optimise path.
 *
 * Plain C: pointers, sizes and status codes, no C++ or torch types. Every entry point
 * returns MKB_OK (0) or a negative mkb_status; mkb_last_error() gives a one-line reason
 * for the calling thread's last failure. Arguments are checked on the host before any
 * device work is queued, as the reference does (it throws std::invalid_argument before a
 * launch; here that is MKB_ERR_ARGUMENT).
 *
 * Device entry points (suffix _device) take device pointers and a CUDA stream passed as
 * `void*` (a cudaStream_t; NULL is the legacy default stream) and only enqueue work: the
 * results are valid once the stream has been synchronised. They allocate nothing; the
 * scratch memory a kernel needs is passed in as `workspace` of at least the size the
 * matching *_workspace_bytes function reports.
 *
 * Layout terms follow the reference (names in parentheses):
 *   V variants, S table surfaces incl. the stop (surface 0), L wavelengths, F fields,
 *   G ghost plates, K ghost terms, P variables, R rows per variant.
 *   Per-variant arrays are variant-major: curvature[v*S+s], index[(v*S+s)*L+l], ...
 *   (include/mikroptim/batch/system_batch_view.hpp:29-95).
 *   Residual rows per variant: tuples (f, l) f-major then l, inside a tuple the pupil
 *   sample k = i*M + j; in soft-failure mode the penalty rows follow the ray rows
 *   (include/mikroptim/batch/batch_residuals.hpp:47-62).
 */
#ifndef MIKROPTIM_B200_H
#define MIKROPTIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- limits of this build ------------------------------------------------------------ */
#define MKB_MAX_SURFACES 64     /* kMaxSurfaces, include/mikroptim/trace/surface_table.hpp:15 */
#define MKB_MAX_RINGS 32        /* the reference caps at 16 (pupil/quadrature.hpp:21) */
#define MKB_MAX_SPOKES 64
#define MKB_MAX_FIELDS 16
#define MKB_MAX_WAVELENGTHS 16
#define MKB_MAX_TUPLES 128      /* F * L */
#define MKB_MAX_VARIABLES 64    /* P */
#define MKB_MAX_GHOST_PLATES 16 /* G (the reference allows one per table surface) */
#define MKB_MAX_GHOST_TERMS 32  /* K, kMaxGhostTerms of trace/surface_table.hpp:20 */

/* ---- status codes --------------------------------------------------------------------- */
typedef enum mkb_status {
    MKB_OK = 0,
    MKB_ERR_ARGUMENT = -1,    /* bad argument; nothing was enqueued */
    MKB_ERR_CUDA = -2,        /* CUDA runtime error (launch or sticky device error) */
    MKB_ERR_WORKSPACE = -3,   /* workspace missing or too small */
    MKB_ERR_TIMEOUT = -4,     /* a bounded device-side wait gave up */
    MKB_ERR_UNSUPPORTED = -5  /* a feature of the input that this build does not trace */
} mkb_status;

/* Values are stable and equal to the reference enums. */
enum { MKB_SURFACE_STOP = 0, MKB_SURFACE_PLANE = 1, MKB_SURFACE_SPHERE = 2,
       MKB_SURFACE_GHOST_PLATE = 3 };                  /* SurfaceKind, surface_table.hpp:25 */
/* An aperture stop inside the system (no counterpart in the reference, whose stop is always
 * table surface 0, docs/adr/0006-blende-erste-flaeche.md): a plane at table surface s_a,
 * 1 <= s_a <= S - 2, at most one per table, whose curvature slot holds the stop's
 * semi-aperture R. Table surface 0 is then the entrance pupil, placed by paraxial ray aiming
 * wherever a record is packed or a variable written: with the y-u trace of the paraxial index
 * (wavelength column 0) from surface 1 to the stop, y_A the stop height of the ray (y = 1,
 * u = 0) and y_B that of the ray (y = 0, u = 1), the pupil radius becomes R / |y_A| and
 * thickness[0] becomes -y_B / y_A (the entrance pupil's distance before surface 1). Every
 * operation separately rounded. Coaxial batches of one table, without ghost plates;
 * thickness[0] is no variable then. */
enum { MKB_SURFACE_APERTURE_STOP = 4 };
enum { MKB_PUPIL_HALF = 0, MKB_PUPIL_FULL = 1, MKB_PUPIL_AXIS = 2 };
                                                       /* PupilMode, pupil/quadrature.hpp:24 */
enum { MKB_FAILURE_SOFT = 0, MKB_FAILURE_HARD = 1 };   /* FailureMode, surface_ops.hpp:74 */
enum { MKB_STATUS_OK = 0, MKB_STATUS_MISSED = 1, MKB_STATUS_TIR = 2, MKB_STATUS_BACKWARD = 3,
       MKB_STATUS_UNSUPPORTED = 4, MKB_STATUS_SOFT_MISSED = 5, MKB_STATUS_SOFT_TIR = 6 };
                                                       /* TraceStatus, surface_ops.hpp:24 */
/* FP64: every operation separately rounded, sums in the reference's order -- bit-identical to
 * the reference CPU build. FP64_FMA: FP64 with a*b+c contracted to FMA and tree sums (faster,
 * equal within the reference's CPU/GPU tolerances). MIXED: the trace (OPL, piston, merit and
 * the ray states) as FP64_FMA, the adjoint reverse sweep in FP32 on those states. */
enum { MKB_PRECISION_FP64 = 0, MKB_PRECISION_MIXED = 1, MKB_PRECISION_FP64_FMA = 2,
       MKB_PRECISION_DF64 = 3, MKB_PRECISION_FP32_BULK = 4 };
/* FP32_BULK (no counterpart in the reference): the trace with its directions and refraction in
 * FP32 (normal, cos I, sqrt k, the refracted direction, renormalised to first order) and in
 * FP64 only what stability needs -- the ray's position and the transfer to the tangent plane,
 * the cancellation-safe sphere intersection s = H / (B + sqrt D), the optical path along the
 * ray, the reference-sphere step and the tuple sums. RESIDUALS, MERIT and the optimiser (the
 * fused adjoint's forward and the LM's trial MERIT; the reverse sweep in FP32 as in MIXED) of
 * coaxial batches without ghost plates; its OPD error against FP64 is stated per workload (tens
 * of nanowaves on singlet-style systems, far more on strongly aberrated ones). */
/* DF64 (RESIDUALS and MERIT only): the reference's reduced-precision trace type
 * (include/mikroptim/math/df64.hpp:108): every per-ray operation in double-float arithmetic
 * (a pair of floats, about 48 bits) on the FP32 pipes, the tuple sums in FP64. */
enum { MKB_VAR_CURVATURE = 0, MKB_VAR_THICKNESS = 1, MKB_VAR_WORKING_DISTANCE = 2,
       MKB_VAR_GHOST_COEFFICIENT = 3, MKB_VAR_GLASS = 4 };
                                                       /* VariableType, model/variables.hpp:18 */

/* ---- batch ------------------------------------------------------------------------------
 * Mirrors SystemBatchView<double> (include/mikroptim/batch/system_batch_view.hpp:108) for a
 * collimated source with the reference sphere through the vertex of the last surface
 * (ReferenceSphereKind::LastSurface) and the ideal image point h_f = field_target. All
 * pointers are host pointers when passed to mkb_pack_batch_host. */
typedef struct mkb_batch_view {
    int32_t variants, surfaces, wavelengths, fields, ghost_plates, ghost_terms;
    double reference_wavelength_nm;
    const uint8_t* type;              /* [S]  surface kind                              */
    const double* wavelength_weight;  /* [L]                                            */
    const double* field_weight;       /* [F]                                            */
    const double* curvature;          /* [V][S]                                         */
    const double* thickness;          /* [V][S]  thickness[S-1] = working distance      */
    const double* index;              /* [V][S][L] medium after surface s               */
    const double* pupil_radius;       /* [V]                                            */
    const double* field_angle;        /* [V][F] radians                                 */
    const double* field_target;       /* [V][F] ideal image height h_f (mm)             */
    /* Non-coaxial batches (BatchTopology::non_coaxial, system_batch.hpp:45): per surface the
     * decenter dx, dy (mm) and the tilts alpha about the local x axis and beta about the local
     * y axis (radians, |.| < pi/2), [V][S][4], rotation R = R_y(beta) R_x(alpha) about the
     * vertex (trace/surface_transform.hpp:8-14). NULL: coaxial. A non-coaxial batch traces
     * Full pupils only. */
    const double* decenter_tilt;
    /* Ghost plates (surfaces of kind MKB_SURFACE_GHOST_PLATE, numbered in table order; K >= 1
     * when G > 0): the Legendre profile coefficients a_1..a_K [V][G][K] (mm), the
     * normalisation radius r_g [G] (mm, shared by the variants as in the reference's
     * SystemBatchHost::ghost_norm_radius(g)) and the plate's glass index [V][G][L]
     * (trace/ghost_plate.hpp:24). NULL when ghost_plates = 0. */
    const double* ghost_coeff;
    const double* ghost_norm_radius;
    const double* ghost_index;
    /* Glass variables: the Buchdahl coefficients (n0, nu1, nu2, nu3) of the medium after every
     * surface [V][S][4] (SystemBatchHost::buchdahl_coeff, system_batch.hpp:147) and the
     * wavelengths [L] in nm; NULL when no variable is a glass. */
    const double* buchdahl_coeff;
    const double* wavelength_nm;
} mkb_batch_view;

/* The device-resident batch: one 16-byte aligned record of `record_stride` doubles per
 * variant (so that a CTA stages its variant with one bulk copy), plus the shared arrays.
 * Record layout (doubles): curvature[S] | thickness[S] | index[S*L] | pupil_radius |
 * sin(field_angle)[F] | cos(field_angle)[F] | field_target[F] | [non-coaxial: per surface
 * dx, dy, cos alpha, sin alpha, cos beta, sin beta, moved, 0] | [ghost plates:
 * coefficients [G][K] | normalisation radius [G] | index [G][L]] | [glass: Buchdahl
 * coefficients [S][4]] | padding. */
typedef struct mkb_device_batch {
    int32_t variants, surfaces, wavelengths, fields;
    int32_t record_stride;            /* doubles per variant, even                      */
    int32_t non_coaxial;              /* 1: the records carry per-surface transforms     */
    const double* records;            /* device [V][record_stride], 16-byte aligned     */
    const uint8_t* type;              /* host [S] (copied into the kernel parameters)   */
    const uint8_t* variant_surfaces;  /* device [V] or NULL: table surfaces each variant
                                         uses (2 .. S; uneven batches, one launch): its
                                         surfaces are 0 .. n-1 of the shared table, its
                                         working distance is thickness[n-1], the entries
                                         past n are ignored. NULL: every variant uses S. */
    int32_t ghost_plates, ghost_terms;  /* G, K: the records carry the plates' data       */
    int32_t glass;                    /* 1: the records carry Buchdahl coefficients [S][4] */
    const double* wavelength_nm;      /* host [L] nm; needed when glass = 1              */
} mkb_device_batch;

/* Doubles per packed variant record for a coaxial batch shape without ghost plates (>= 2,
 * even). */
int32_t mkb_record_stride(int32_t surfaces, int32_t wavelengths, int32_t fields);

/* Doubles per packed variant record for any batch shape. */
int32_t mkb_record_stride_ext(int32_t surfaces, int32_t wavelengths, int32_t fields,
                              int32_t non_coaxial, int32_t ghost_plates, int32_t ghost_terms,
                              int32_t glass);

/* Packs a host SoA view into host records [V][mkb_record_stride_ext(...)] (sin/cos of the
 * field angles and of the tilts are taken here with the host libm, so the start rays and the
 * surface transforms are those of the CPU reference). */
int mkb_pack_batch_host(const mkb_batch_view* view, double* records);

/* The LM variables (VariableSet, include/mikroptim/optim/variable_set.hpp:63): curvature,
 * thickness and working-distance entries of the surface table. The Jacobian and LM entry
 * points write a run point x [P] into a copy of the run's template record on the device
 * (VariableSet::apply, src/optim/variable_set.cpp:237). */
typedef struct mkb_variables {
    int32_t count;                    /* P                                               */
    const int32_t* type;              /* host [P] MKB_VAR_*                              */
    const int32_t* surface;           /* host [P] table surface (batch_surface)          */
    const double* lower;              /* host [P] (-inf allowed)                         */
    const double* upper;              /* host [P] (+inf allowed)                         */
    const double* typical;            /* host [P] > 0                                    */
    /* GhostCoefficient variables (a_k of plate g; their `surface` entry is ignored): host [P]
     * plate g (0 .. G-1, table order) and order k (1 .. K); NULL when there are none. */
    const int32_t* ghost_plate;
    const int32_t* ghost_order;
    /* Glass variables (Buchdahl coordinate of the medium after `surface`; the reference's
     * VariableType::Glass): host [P] component 0 = n0, 1 = nu1, 2 = nu2; NULL when none.
     * Writing one recomputes that medium's index at every wavelength,
     * n = n0 + w (nu1 + w (nu2 + w nu3)), w = the Buchdahl coordinate of the wavelength. */
    const int32_t* glass_component;
} mkb_variables;

/* VariableSet::apply on the device: records_out [runs][record_stride] = the run's template
 * record (templates hold 1 variant or one per run) with the run's point x [runs][P] written
 * into its curvature / thickness / working-distance entries. All pointers except `vars` are
 * device pointers; records_out is 16-byte aligned. */
int mkb_apply_variables_device(const mkb_device_batch* templates, const mkb_variables* vars,
                               const double* x, int32_t runs, double* records_out, void* stream);

/* ---- residual plan -----------------------------------------------------------------------
 * ResidualSettings + ResidualLayout (include/mikroptim/batch/batch_residuals.hpp:24,62)
 * plus the shared weights of the batch. quad_u / quad_w are the Gauss-Legendre radial nodes
 * u_i = rho_i^2 (ascending) and weights W_i (sum 1) for `rings` (pupil/quadrature.hpp:40). */
typedef struct mkb_residual_plan {
    int32_t rings, spokes;
    int32_t failure;                  /* MKB_FAILURE_*                                   */
    int32_t precision;                /* MKB_PRECISION_*                                 */
    double fail_weight;               /* w_fail (ray_residual.hpp:175), >= 0             */
    double reference_wavelength_nm;   /* lambda_ref (residuals in waves at lambda_ref)   */
    int32_t fields, wavelengths;
    const uint8_t* pupil_mode;        /* host [F]                                        */
    const double* field_weight;       /* host [F]                                        */
    const double* wavelength_weight;  /* host [L]                                        */
    const double* quad_u;             /* host [rings]                                    */
    const double* quad_w;             /* host [rings]                                    */
    /* Transverse ray errors as residual rows (>= 0; 0 = none). No counterpart in the
     * reference, whose residual rows are OPD only: after the ray rows and the penalty rows,
     * 2 x rays rows -- the x errors of every ray in the ray-row order, then the y errors --
     * r_x = sqrt(transverse_weight * w_(f,l)) sqrt(W_k) (x_k - 0), r_y likewise with
     * (y_k - h_f), where (x_k, y_k) is the ray's intersection with the image plane
     * (thickness[S-1] behind the last vertex, transfer_to_image_plane,
     * include/mikroptim/trace/trace.hpp:402), w_(f,l) the tuple weight and W_k the pupil
     * weight; 0 for a ray that failed hard. Units: waves^2 per mm^2 (the merit's unit per
     * squared image-plane error). MERIT adds sum_k r_x^2, then sum_k r_y^2 after each tuple's
     * OPD and penalty sums. RESIDUALS, MERIT, the FD Jacobian and the materialised adjoint
     * Jacobian (its sweep seeded at the image-plane intercept); the fused adjoint refuses it. */
    double transverse_weight;
} mkb_residual_plan;

/* Rays per variant (ResidualLayout::rays_per_variant) and trace rows (rays, penalty rows in soft
 * mode, transverse rows with transverse_weight > 0). */
int64_t mkb_rays_per_variant(const mkb_residual_plan* plan);
int64_t mkb_trace_rows(const mkb_residual_plan* plan);

/* ---- forward trace -------------------------------------------------------------------------
 * RESIDUALS: replaces DeviceResiduals::run (src/cuda/residuals.cu:240) behind
 * TraceEngine::run(batch, TraceMode::Residuals, ...) (include/mikroptim/cuda/trace_engine.hpp).
 * residuals [V][stride] (stride >= trace_rows; rows past trace_rows are left untouched),
 * opd [V][rays] (may be NULL), status [V][rays] (may be NULL). */
int mkb_residuals_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                         double* residuals, int64_t stride, double* opd, uint8_t* status,
                         void* stream);

/* MERIT: replaces DeviceMerit::run (src/cuda/merit.cu:339): merit[v] = sum_(f,l) (sum_k r_k^2
 * + sum_k p_k^2), failed[v] / hard_failed[v] ray counts (batch_merit.hpp:32). Scratch: the
 * per-tuple partial sums, mkb_merit_workspace_bytes(V, plan) bytes. */
size_t mkb_merit_workspace_bytes(int32_t variants, const mkb_residual_plan* plan);
int mkb_merit_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                     double* merit, int64_t* failed, int64_t* hard_failed,
                     void* workspace, size_t workspace_bytes, void* stream);

/* Per-run options of the trace (TraceSettings::pack_rays and ::extra_merit,
 * include/mikroptim/cuda/trace_engine.hpp:58).
 *   pack_rays    the largest pack of consecutive tuples one CTA traces, in rays; 0 = 512.
 *                Runtime only: every value gives bit-identical results (a tuple with more rays
 *                gets a pack of its own; values above 4096 are traced as 4096).
 *   extra_merit  MERIT only: device [V] or NULL; extra_merit[v] is added to variant v's merit
 *                after its tuple sums (MeritRunOptions::extra_merit, src/cuda/merit.cu:222).
 *   variants_per_cta  how many variants one CTA traces side by side (0 = 1, at most 8): its
 *                threads, the per-tuple reductions and the barriers are then shared by the
 *                packs of several variants. Runtime only, like pack_rays (bit-identical results
 *                for every value); not with extrema. The trace autotuner picks both.
 *   extrema      device [V][S][2] or NULL: per variant and table surface the largest ray
 *                height sqrt(x^2 + y^2) at the surface and the smallest cos I (d before the
 *                refraction . surface normal) over the rays with status Ok; surface 0 holds
 *                the start point and d_z; neutral 0 and 1 without a valid ray
 *                (SurfaceExtremaResult, include/mikroptim/batch/batch_extrema.hpp, hard
 *                maxima); at a decentered or tilted surface the height and incidence in the
 *                surface's own frame. FP64, FP64_FMA and DF64. */
typedef struct mkb_trace_options {
    int32_t pack_rays;
    int32_t variants_per_cta;
    const double* extra_merit;
    double* extrema;
} mkb_trace_options;

/* mkb_residuals_device / mkb_merit_device with options (NULL = the defaults). */
int mkb_residuals_ex_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                            const mkb_trace_options* options, double* residuals, int64_t stride,
                            double* opd, uint8_t* status, void* stream);
int mkb_merit_ex_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                        const mkb_trace_options* options, double* merit, int64_t* failed,
                        int64_t* hard_failed, void* workspace, size_t workspace_bytes,
                        void* stream);

/* ---- device memory of a TraceEngine run ------------------------------------------------------
 * The tranche plan of TraceEngine::run / run_on_device / max_variants
 * (src/cuda/trace_engine.cu:185-268; usable_bytes and max_variants,
 * include/mikroptim/batch/batch_memory.hpp:119-135), for this library's device layout.
 *
 * usable = free - max(reserve_min_bytes, reserve_fraction * free), at least 0; status
 * MKB_ERR_ARGUMENT when reserve_fraction is outside [0, 1]. */
int mkb_usable_bytes(size_t free_bytes, size_t reserve_min_bytes, double reserve_fraction,
                     size_t* usable);
/* Device bytes a run allocates: `per_variant` for each variant of a tranche (its record, its
 * outputs and scratch) plus `fixed` once (alignment of the buffers). `shape` describes the
 * batch (variants and records are not read). merit_mode 0: RESIDUALS with residual rows of
 * stride trace_rows + extra_residuals, status always, OPD when `opd`; 1: MERIT, with one
 * double per variant more when `extra_merit`. */
int mkb_trace_run_bytes(const mkb_device_batch* shape, const mkb_residual_plan* plan,
                        int32_t merit_mode, int64_t extra_residuals, int32_t opd,
                        int32_t extra_merit, size_t* per_variant, size_t* fixed);
/* The largest tranche for `usable` bytes: a multiple of `granularity` (>= 1) with
 * fixed + tranche * per_variant <= usable and tranche * packs <= 2^31 - 1 CTAs; 0 when not
 * even `granularity` variants fit; negative status on bad arguments. */
int64_t mkb_trace_tranche_variants(size_t usable, const mkb_device_batch* shape,
                                   const mkb_residual_plan* plan,
                                   const mkb_trace_options* options, int32_t merit_mode,
                                   int64_t extra_residuals, int32_t opd, int32_t extra_merit,
                                   int32_t granularity);

/* ---- Jacobians ------------------------------------------------------------------------------
 * Both take `templates` (1 variant for all runs, or one per run), the plan, the variables and
 * the run points x0 [runs][P] (device), and write J [runs][P][R] (column p of run i at
 * J + (i*P + p)*R, R = trace rows) and r0 [runs][R] = residuals at x0 -- the layout of the
 * reference's FdJacobian / AdjointJacobian (include/mikroptim/optim/fd_jacobian.hpp:118). */

/* Finite differences, central scheme with the reference's stencils at bounds: replaces
 * DeviceFdJacobian::compute (src/cuda/fd_jacobian.cu:203, fd_jacobian_cpu in
 * src/optim/fd_jacobian.cpp:182). 2P + 1 traced variants per run; runs are processed in
 * chunks that fit the workspace (mkb_fd_jacobian_workspace_bytes for a chunk size).
 * status_changes [runs][P] (may be NULL): rays whose Ok-status differs between x0 and a
 * perturbed point of the column. */
size_t mkb_fd_jacobian_workspace_bytes(const mkb_device_batch* templates,
                                       const mkb_residual_plan* plan, int32_t P, int32_t runs,
                                       int32_t runs_per_chunk);
int mkb_fd_jacobian_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                           const mkb_variables* vars, const double* x0, int32_t runs, double* J,
                           double* r0, int64_t* status_changes, void* workspace,
                           size_t workspace_bytes, void* stream);

/* Adjoint sweep with checkpoints every 4 surfaces, then the piston projection: replaces
 * DeviceAdjointJacobian::compute (src/cuda/adjoint_jacobian.cu:401) and
 * adjoint_jacobian_cpu (src/optim/adjoint_jacobian.cpp:370). status [runs][rays]. */
size_t mkb_adjoint_jacobian_workspace_bytes(const mkb_device_batch* templates, int32_t runs);
int mkb_adjoint_jacobian_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                                const mkb_variables* vars, const double* x0, int32_t runs,
                                double* J, double* r0, uint8_t* status, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Adjoint Jacobian fused with its normal equations: gram [runs][P+1][P+1] = [J r]^T [J r] of
 * the piston-projected adjoint rows (and the penalty rows), J never written to memory.
 * Replaces DeviceAdjointJacobian::compute + DeviceNormalEquations::compute for the LM. The
 * rows are computed in the plan's precision (FP64: the rows of the exact path; FP64_FMA:
 * contracted), the contraction runs on FP64 tensor cores; the workspace is
 * mkb_adjoint_jacobian_workspace_bytes(templates, runs). */
int mkb_adjoint_normal_equations_device(const mkb_device_batch* templates,
                                        const mkb_residual_plan* plan, const mkb_variables* vars,
                                        const double* x0, int32_t runs, double* gram,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* The same for an uneven batch: `vars` is an array of `runs` variable sets (one per run; the
 * counts may differ), x0 rows are strided by the largest count Pmax and gram [runs] slots by
 * (Pmax + 1)^2 (run i's (P_i + 1)^2 matrix dense at the start of its slot). Templates with
 * variant_surfaces must hold one template per run. */
size_t mkb_adjoint_normal_equations_runs_workspace_bytes(const mkb_device_batch* templates,
                                                         const mkb_variables* vars,
                                                         int32_t runs);
int mkb_adjoint_normal_equations_runs_device(const mkb_device_batch* templates,
                                             const mkb_residual_plan* plan,
                                             const mkb_variables* vars, const double* x0,
                                             int32_t runs, double* gram, void* workspace,
                                             size_t workspace_bytes, void* stream);

/* ---- batched Levenberg-Marquardt ------------------------------------------------------------
 * LmOptions (include/mikroptim/optim/levenberg_marquardt.hpp:85) for one pass (no outer
 * soft-failure penalty rounds), and the per-run state kept in a caller workspace. The device
 * loop replaces the host loop of levenberg_marquardt (src/optim/levenberg_marquardt.cpp:332)
 * with GpuLmBackend (src/cuda/levenberg_marquardt.cpp): mkb_lm_start_device evaluates the
 * merit at x0, each mkb_lm_cycle_device performs one LM cycle for every run (Jacobian and
 * normal equations, damped active-set Cholesky step, trial MERIT, acceptance with Nielsen
 * damping) as a fixed sequence of launches, so cycles can be captured in a CUDA graph.
 * With precision FP64 and gram_exact = 1 every run follows the reference's trajectory bit
 * for bit. Status values are LmStatus (0 running, 1 converged_merit, 2 converged_step,
 * 3 converged_gradient, 5 max_iterations, 6 damping_limit, 7 numerical_error). */
enum { MKB_JACOBIAN_FD = 0, MKB_JACOBIAN_ADJOINT = 1 };
typedef struct mkb_lm_options {
    int32_t max_iterations;           /* 100 */
    int32_t reject_new_failures;      /* 1 */
    double ftol, xtol, gtol;          /* 1e-10 each */
    double initial_damping;           /* 1e-3 */
    double max_damping;               /* 1e16 */
    double diag_floor;                /* 1e-12 */
    int32_t jacobian;                 /* MKB_JACOBIAN_* */
    int32_t gram_exact;               /* 1: FMA-chain normal equations, 0: FP64 DMMA; with
                                         the adjoint, 0 selects the fused adjoint +
                                         normal-equation kernel (no J in memory) */
    int32_t per_run_variables;        /* 0: `vars` is one variable set for all runs. 1: `vars`
                                         points to an array of `runs` sets (uneven batches;
                                         counts may differ), x0 / x rows are then strided by
                                         the largest count; needs gram_exact = 0 */
    /* Paraxial constraints evaluated on the device (ParaxialConstraints as the LM's extra
     * rows, include/mikroptim/optim/paraxial_residuals.hpp:67): `paraxial_count` rows after
     * the trace rows of every run, their Jacobian in every cycle and sum r_e^2 in every merit,
     * with no host phase (a cycle stays one fixed launch sequence). 0 / NULL: none. See
     * mkb_paraxial_constraint and mkb_paraxial_rows_device. */
    int32_t paraxial_count;
    const struct mkb_paraxial_constraint* paraxial;  /* host [paraxial_count] */
    int32_t paraxial_column;          /* wavelength column holding the paraxial index */
    int32_t paraxial_derivative;      /* MKB_PARAXIAL_FD or MKB_PARAXIAL_ADJOINT */
} mkb_lm_options;

/* ---- paraxial constraints on the device -----------------------------------------------------
 * One constraint (ParaxialConstraint, include/mikroptim/optim/paraxial_residuals.hpp:67), its
 * residual r = sqrt(weight) * mode(q + shift) from the y-nu trace at the paraxial index
 * (ynu_trace.hpp; compute_paraxial, src/paraxial/paraxial.cpp:98):
 *   FOCAL_LENGTH      q = f_s (1 - f_s phi), phi = -C (equal only)
 *   PARFOCAL_LENGTH   q = offset + sum_{s >= reference_surface} t_s - L_s
 *   WORKING_DISTANCE  q = t_{S-1} - w_s
 *   PARAXIAL_FOCUS    q = a (A + t_{S-1} C / n'_L) (equal only, target 0)
 *   PETZVAL           q = |kappa_P| - kappa_max, kappa_P = -n'_L P (max only)
 * mode: MKB_MODE_EQUAL q, MIN min(q, 0), MAX max(q, 0); shift moves one-sided limits (0 for
 * equal). The paraxial index of a medium is its index in wavelength column `paraxial_column`
 * of the record (the batch's paraxial_index), or, for a medium with glass variables, the
 * Buchdahl index at the reference wavelength (VariableSet::apply, src/optim/
 * variable_set.cpp:282). A ghost plate is a thin element in the medium n_m of its gap
 * (batch_paraxial, src/batch/system_batch.cpp:965): its power -2 (n_G - n_m) t2 (t2 from its
 * Legendre coefficients, n_G its glass index in the same column) joins the surface's power and
 * that power / (n_m n_G) the Petzval sum; a parfocal reference surface must not be a plate.
 * Coaxial batches. Sine-condition and distortion rows trace real rays and stay host rows. */
enum { MKB_CONSTRAINT_FOCAL_LENGTH = 0, MKB_CONSTRAINT_PARFOCAL_LENGTH = 1,
       MKB_CONSTRAINT_WORKING_DISTANCE = 2, MKB_CONSTRAINT_PARAXIAL_FOCUS = 3,
       MKB_CONSTRAINT_PETZVAL = 4 };          /* ConstraintType, model/constraints.hpp:28 */
enum { MKB_MODE_EQUAL = 0, MKB_MODE_MIN = 1, MKB_MODE_MAX = 2 };  /* ConstraintMode */
/* Jacobian of the constraint rows: central differences with the FD Jacobian's pattern (the
 * reference's extra_rows_cpu, bit for bit), or the analytic adjoint of the y-nu trace (one
 * reverse sweep of the marginal ray per run; exact derivatives). */
enum { MKB_PARAXIAL_FD = 0, MKB_PARAXIAL_ADJOINT = 1 };
#define MKB_MAX_PARAXIAL 16
typedef struct mkb_paraxial_constraint {
    int32_t type, mode;
    double weight, target;
    int32_t reference_surface;        /* PARFOCAL_LENGTH only: table surface */
    int32_t reserved;                 /* 0 */
    double offset;                    /* PARFOCAL_LENGTH only (mm) */
    double shift;                     /* >= 0; 0 for equal */
} mkb_paraxial_constraint;

/* The constraint rows of `runs` runs at x [runs][P] on their templates (1 variant for all runs
 * or one per run): residuals re [runs][E] and Jacobian je [runs][P][E] (column k of run i at
 * (i * P + k) * E). `options` supplies the constraints, the column and the derivative (its
 * other fields must be valid LM options); one variable set for all runs (per_run_variables =
 * 0). Allocates nothing. */
int mkb_paraxial_rows_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const mkb_lm_options* options,
                             const double* x, int32_t runs, double* je, double* re,
                             void* stream);

size_t mkb_lm_workspace_bytes(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                              const mkb_variables* vars, const mkb_lm_options* options,
                              int32_t runs);
int mkb_lm_start_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                        const mkb_variables* vars, const mkb_lm_options* options,
                        const double* x0, int32_t runs, void* workspace, size_t workspace_bytes,
                        void* stream);
int mkb_lm_cycle_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                        const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
                        void* workspace, size_t workspace_bytes, void* stream);

/* Extra residual rows (the reference's LmOptions::jacobian.extra, ExtraResiduals evaluated on
 * the host: paraxial constraints and the like, src/optim/levenberg_marquardt.cpp:659,
 * extra_rows_untraced in src/optim/adjoint_jacobian.cpp:245). A caller with E such rows runs
 * each cycle in phases instead of mkb_lm_cycle_device:
 *   1. mkb_lm_cycle_jacobian_device       trace-row Jacobian and normal equations;
 *      mkb_lm_points_device               want_jacobian [runs] and x [runs][P]: the runs that
 *                                          got normal equations and their points;
 *   2. mkb_lm_extra_rows_device           the caller's rows at those points, J_e [runs][P][E]
 *                                          (column k of run i at (i*P + k)*E) and r_e
 *                                          [runs][E] (device), appended after the trace rows:
 *                                          every entry of [J r]^T [J r] continues its fma chain
 *                                          over e = 0..E-1 (rows of other runs are not read);
 *   3. mkb_lm_cycle_step_device           damped step and trial point;
 *      mkb_lm_points_device               evaluate [runs] and trial [runs][P];
 *   4. mkb_lm_cycle_accept_device         trial MERIT plus extra_merit[run] = sum_e r_e^2 at
 *                                          the trial point (device [runs]; read for the runs to
 *                                          evaluate), then acceptance.
 * Step 4 may itself run in two parts for rows that depend on the trace (the reference's
 * trace_extra, TraceExtraResiduals, which read the per-surface extrema of the same trace):
 *   4a. mkb_lm_cycle_trial_device         trial MERIT (+ extra_merit) and, when `extrema` is
 *                                          given (device [runs][S][2]), the trial points'
 *                                          extrema (mkb_trace_options.extrema);
 *   4b. mkb_lm_cycle_decide_device        acceptance with trace_merit[run] (device [runs]) added
 *                                          to the trial merit after the kernel's sum, as
 *                                          GpuLmBackend::merit does (src/cuda/
 *                                          levenberg_marquardt.cpp:235-240).
 * mkb_lm_start_ex_device is mkb_lm_start_device with the extra merit at x0 (device [runs], in
 * the MERIT kernel) and the trace-dependent merit at x0 (added after it); either may be NULL.
 * The host FD of the extra rows uses mkb_fd_pattern_host / mkb_fd_derivative_host, the
 * pattern and formula of the FD Jacobian. */
int mkb_lm_start_ex_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                           const mkb_variables* vars, const mkb_lm_options* options,
                           const double* x0, const double* extra_merit,
                           const double* trace_merit, int32_t runs, void* workspace,
                           size_t workspace_bytes, void* stream);
int mkb_lm_cycle_trial_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                              const mkb_variables* vars, const mkb_lm_options* options,
                              int32_t runs, void* workspace, size_t workspace_bytes,
                              const double* extra_merit, double* extrema, void* stream);
int mkb_lm_cycle_decide_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                               const mkb_variables* vars, const mkb_lm_options* options,
                               int32_t runs, void* workspace, size_t workspace_bytes,
                               const double* trace_merit, void* stream);
int mkb_lm_cycle_jacobian_device(const mkb_device_batch* templates,
                                 const mkb_residual_plan* plan, const mkb_variables* vars,
                                 const mkb_lm_options* options, int32_t runs, void* workspace,
                                 size_t workspace_bytes, void* stream);
int mkb_lm_extra_rows_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const mkb_lm_options* options,
                             int32_t runs, void* workspace, size_t workspace_bytes,
                             const double* jacobian, const double* residuals, int32_t rows,
                             void* stream);
int mkb_lm_cycle_step_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const mkb_lm_options* options,
                             int32_t runs, void* workspace, size_t workspace_bytes,
                             void* stream);
int mkb_lm_cycle_accept_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                               const mkb_variables* vars, const mkb_lm_options* options,
                               int32_t runs, void* workspace, size_t workspace_bytes,
                               const double* extra_merit, void* stream);
/* Copies want_jacobian [runs], x [runs][P], evaluate [runs] and trial [runs][P] out of the
 * workspace (any may be NULL; host or device pointers). */
int mkb_lm_points_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                         const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
                         const void* workspace, int32_t* want_jacobian, double* x,
                         int32_t* evaluate, double* trial, void* stream);

/* FD pattern of run points on the host (fd_step + fd_pattern, central scheme,
 * src/optim/variant_generator.cpp:177), the same bits as the device FD Jacobian's: for entry
 * i*P + k the perturbed values x_a (point_plus) and x_b (point_minus), the steps
 * d_a = x_a - x and d_b = x_b - x, and the stencil (0 central, 1 one-sided, 2 truncated at a
 * bound). Host arrays [runs][P]. */
int mkb_fd_pattern_host(const mkb_variables* vars, const double* x, int32_t runs,
                        double* point_plus, double* point_minus, double* step_plus,
                        double* step_minus, int32_t* stencil);
/* fd_derivative (optim/fd_formula.hpp:40) of `rows` values on the host: column[e] from r0[e]
 * at x, r_plus[e] at x_a and r_minus[e] at x_b. */
int mkb_fd_derivative_host(int32_t stencil, double step_plus, double step_minus, int32_t rows,
                           const double* r0, const double* r_plus, const double* r_minus,
                           double* column);
/* Copies the run results out of the workspace (any output may be NULL; host or device
 * pointers): x [runs][P], merit, status, iterations, accepted, jacobians, damping mu,
 * history [runs][max_iterations + 1] (NaN-padded), failed / hard-failed rays, and `running`
 * (one int: runs still running after the last cycle). */
int mkb_lm_results_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                          const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
                          const void* workspace, double* x, double* merit, int32_t* status,
                          int32_t* iterations, int32_t* accepted, int32_t* jacobians,
                          double* damping, double* history, int64_t* failed,
                          int64_t* hard_failed, int32_t* running, void* stream);

/* ---- normal equations --------------------------------------------------------------------
 * gram [runs][P+1][P+1] = [J r]^T [J r] for J [runs][P][R] (column p of run i at
 * J + (i*P + p)*R) and r [runs][R]: A = J^T J in the top-left block, g = J^T r in column P.
 * Replaces DeviceNormalEquations::compute (src/cuda/normal_equations.cu:48, gram_kernel).
 * exact != 0: every entry one FMA chain over the rows in ascending order, bit-identical to
 * normal_equations_host (include/mikroptim/optim/normal_equations.hpp:33); exact == 0: FP64
 * tensor cores (mma.sync m8n8k4 f64), deterministic. */
int mkb_normal_equations_device(const double* J, const double* r, int32_t runs, int32_t P,
                                int64_t R, double* gram, int32_t exact, void* stream);

/* MERIT for callers that cannot allocate device memory. No counterpart in the reference.
 * Some callers cannot call cudaMalloc: a host application that gives the library a fixed
 * memory budget and owns the rest of the GPU, or a loop that must never wait on an
 * allocation. This entry point takes the same batch, plan and outputs as mkb_merit_device but
 * no workspace: the per-tuple partial sums go to a 4 MiB array compiled into the library
 * (every GPU that loads the library keeps it until the process exits). Limit: variants x
 * fields x wavelengths <= MKB_NOALLOC_MERIT_MAX_SLOTS per call; larger batches are rejected
 * with MKB_ERR_ARGUMENT before anything is enqueued. The array is shared by all calls, so
 * calls that overlap on the GPU race: run one at a time per device. Every call made outside
 * a stream capture looks up the array's device address in the current context
 * (cudaGetSymbolAddress, no allocation), so switching contexts or resetting the device between
 * calls is safe; a call made while its stream is captured reuses the address the last
 * uncaptured call on that device found, and fails with MKB_ERR_ARGUMENT if there was none. */
#define MKB_NOALLOC_MERIT_MAX_SLOTS 262144
int mkb_merit_noalloc_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                             double* merit, int64_t* failed, int64_t* hard_failed, void* stream);

/* ---- FP32 prefilter of multistart variants ---------------------------------------------------
 * Replaces DevicePrefilter::run / download (include/mikroptim/cuda/prefilter.hpp,
 * src/cuda/prefilter.cu:87,193) behind TraceEngine::prefilter_variants, whose CPU reference is
 * prefilter_stats_cpu (src/batch/batch_prefilter.cpp). Every ray is traced in float with hard
 * failure (prefilter_ray, include/mikroptim/merit/prefilter_ray.hpp) and carries a margin, the
 * distance of its tests (d_z, cos I, cos I', the ghost-plate radicand, the reference sphere's
 * discriminant and denominator) from their failure limits in units of a direction cosine. A
 * ray is certain when its margin exceeds `boundary` (eta). Per variant: merit = sum over the
 * tuples of sum_k r_k^2 over the certainly valid rays (piston over those rays, OPL relative to
 * the tuple's axial optical length), optical_length = the largest |offset| + |OPL - offset| of
 * a certainly valid ray, and the counts of certainly failed, uncertain valid and uncertain
 * failed rays. The arithmetic is the reference's float arithmetic in its order (every
 * operation separately rounded, sums in ascending sample order), so the results equal
 * prefilter_stats_cpu bit for bit. The values only decide which variants are worth an FP64
 * evaluation; they never enter a merit, a Jacobian or the optimiser.
 *
 * field_trig: device [V][F][2] = sinf, cosf of the field angle rounded to float, filled on the
 * host by mkb_prefilter_field_trig_host (the reference takes them with the C library's sinf /
 * cosf). Outputs device [V]. Scratch: mkb_prefilter_workspace_bytes(V, plan) bytes. Status
 * MKB_ERR_ARGUMENT for a boundary that is negative or not finite. */
size_t mkb_prefilter_workspace_bytes(int32_t variants, const mkb_residual_plan* plan);
int mkb_prefilter_field_trig_host(const mkb_batch_view* view, float* field_trig);
int mkb_prefilter_device(const mkb_device_batch* batch, const mkb_residual_plan* plan,
                         const float* field_trig, double boundary, double* merit,
                         double* optical_length, int64_t* failed, int64_t* uncertain_ok,
                         int64_t* uncertain_failed, void* workspace, size_t workspace_bytes,
                         void* stream);

/* Criteria and margins of the prefilter decision (PrefilterCriteria, PrefilterMargins,
 * include/mikroptim/batch/batch_prefilter.hpp:35,52); mkb_prefilter_default_options fills the
 * reference's defaults (0.5, +inf, +inf; 0.15, 32, 0.01). */
typedef struct mkb_prefilter_options {
    double max_failed_fraction;       /* (a) reject when failed > fraction * rays        */
    double max_merit;                 /* (b) reject when the merit exceeds this          */
    double max_merit_factor;          /* (c) reject when the merit exceeds factor * best */
    double boundary;                  /* eta                                             */
    double opl_error_factor;          /* kappa                                           */
    double merit_relative;            /* m, in [0, 1)                                    */
} mkb_prefilter_options;
enum { MKB_PREFILTER_KEEP = 0, MKB_PREFILTER_FAILED_RAYS = 1, MKB_PREFILTER_MERIT_ABSOLUTE = 2,
       MKB_PREFILTER_MERIT_RELATIVE = 4 };   /* PrefilterReason, batch_prefilter.hpp:87 */
void mkb_prefilter_default_options(mkb_prefilter_options* options);

/* The conservative decision from the per-variant results (host arrays; prefilter_decide,
 * src/batch/batch_prefilter.cpp): bounds merit_lower <= F_FP64 <= merit_upper of the FP64 merit
 * and the reason mask per variant (0 = keep), the bound of the best merit that criterion (c)
 * uses and its variant (+inf and -1 when none), and the number kept. extra_merit: [V] or NULL
 * (merit of further rows, added exactly). The plan's failure mode is the FP64 truth's. */
int mkb_prefilter_decide_host(const mkb_residual_plan* plan, const mkb_prefilter_options* options,
                              int32_t variants, const double* merit,
                              const double* optical_length, const int64_t* failed,
                              const int64_t* uncertain_ok, const int64_t* uncertain_failed,
                              const double* extra_merit, double* merit_lower,
                              double* merit_upper, uint8_t* reject, double* reference_merit,
                              int32_t* reference_variant, int32_t* kept);
/* The same rule without margins applied to FP64 merits and failed-ray counts (the truth the
 * prefilter is tested against; prefilter_decide_exact, src/batch/batch_prefilter.cpp). */
int mkb_prefilter_decide_exact_host(const mkb_prefilter_options* options, int32_t variants,
                                    int64_t rays_per_variant, const double* merit,
                                    const int64_t* failed, const double* extra_merit,
                                    uint8_t* reject);

/* ---- EVAL: evaluation on a dense Cartesian pupil grid -----------------------------------------
 * Replaces the kernel EVAL behind TraceEngine::evaluate (src/cuda/eval.cu; CPU reference
 * eval_cpu, src/eval/eval.cpp:307). Every variant, field and wavelength is traced on the grid
 * of cell centres x_i = (2i + 1 - N)/N inside the unit pupil (every failure hard), to the
 * image plane (the spot: image point relative to the ideal image point (0, h_f)) and to the
 * reference sphere about (0, h_f, w): through the paraxial exit pupil (curvature kappa per
 * variant and field, MKB_EVAL_EXIT_PUPIL), through the vertex of the last surface
 * (MKB_EVAL_VERTEX), or of infinite radius (MKB_EVAL_INFINITE). OPD = (OPL - OPL_chief) -
 * piston over the grid weights; four field rays per tuple (chief ray and its neighbours at
 * +-delta for the focus positions): x, y, d_x, d_y, d_z. Failed rays: NaN values, their status.
 * Every operation separately rounded and every sum in ascending grid order: bit-identical to
 * eval_cpu. Outputs are device arrays in the reference's layout: ray (v, f, l, k) at
 * ((v F + f) L + l) n + k, field ray j at ((v F + f) L + l) 4 + j (values x 5). */
enum { MKB_EVAL_EXIT_PUPIL = 0, MKB_EVAL_VERTEX = 1, MKB_EVAL_INFINITE = 2 };
#define MKB_MAX_EVAL_GRID 2048
/* The grid (make_eval_grid): points [n][3] (x, y, weight) in row order; NULL to count only. */
int mkb_eval_grid_host(int32_t size, int32_t half_pupil, double* points, int64_t* count);
/* Reference geometry on the host (eval_reference_geometry): kappa [V][F] and the exit-pupil
 * position [V] (NaN where not used) from the paraxial chief ray at wavelength column
 * `paraxial_column` (the batch's paraxial index). MKB_ERR_ARGUMENT when the image point lies
 * in the exit pupil. */
int mkb_eval_reference_host(const mkb_batch_view* view, int32_t reference,
                            int32_t paraxial_column, double* kappa, double* exit_pupil);
size_t mkb_eval_workspace_bytes(const mkb_device_batch* batch);
/* grid, kappa: device arrays from the two host calls above; half_pupil as for the grid;
 * outputs device [V F L n] (opd, spot_x, spot_y, status) and [V F L 4] x 5 / [V F L 4].
 * precision: MKB_PRECISION_FP64 (the reference's arithmetic) or MKB_PRECISION_FP64_FMA
 * (contracted; the forward of the MIXED mode), for intercept and OPD errors. */
int mkb_eval_device(const mkb_device_batch* batch, int32_t reference, double field_ray_offset,
                    int32_t precision, const double* grid, int64_t n, const double* kappa,
                    double* opd, double* spot_x, double* spot_y, uint8_t* status,
                    double* field_rays, uint8_t* field_status, void* workspace,
                    size_t workspace_bytes, void* stream);

/* ---- PSF and MTF from EVAL OPD maps ------------------------------------------------------
 * Replaces PsfEngine::compute (src/cuda/psf.cu; include/mikroptim/cuda/psf.hpp:44) and the
 * CPU reference psf_cpu (src/eval/psf.cpp:330): per tuple the pupil function
 * P = exp(2 pi i OPD / lambda) of its N x N OPD map (NaN: no transmission) in the corner of an
 * M x M field, the PSF I = |FFT2(P)|^2 / n_full^2 centred at (M/2, M/2) (mirrored along an axis
 * whose sign is -1: a divergent wave), and the MTF cuts |OTF(k, 0)| / OTF(0) (sagittal) and
 * |OTF(0, k)| / OTF(0) (tangential), k = 0 .. N, with OTF = FFT2^-1(I). The transform is this
 * library's own shared-memory FFT (no cuFFT). Outputs are device arrays in the reference's
 * layout: psf [T][M][M] (psf[j M + i] at ((i - M/2) dx, (j - M/2) dy)), mtf [T][2][N + 1]. */
#define MKB_MAX_PSF_FFT 8192
/* PsfPupilParams (include/mikroptim/eval/psf_ops.hpp:48): vacuum wavelength [mm],
 * 1 / n_full^2, +1 (convergent) or -1 (divergent, mirrored) per axis. */
typedef struct mkb_psf_pupil_params {
    double lambda_mm;
    double scale;
    int32_t sign_x, sign_y;
} mkb_psf_pupil_params;
/* The figures of PsfResult (include/mikroptim/eval/psf.hpp:95) that finish_psf and
 * prepare_psf_result fill. */
typedef struct mkb_psf_metrics {
    int64_t transmitted;
    double energy, strehl_fft, strehl_origin, strehl, reference_x, reference_y;
    double peak, peak_x, peak_y;
    double dx, dy, airy_radius;
} mkb_psf_metrics;
/* psf_fft_size (src/eval/psf.cpp:168): the smallest power of two >= max(2N, ceil(padding N));
 * MKB_ERR_ARGUMENT for N outside [1, MKB_MAX_EVAL_GRID], padding < 2 or M > MKB_MAX_PSF_FFT. */
int mkb_psf_fft_size_host(int32_t grid, double padding, int32_t* fft_size);
/* Workspace of mkb_psf_device: twiddles, the N x M row spectra and the projections of every
 * tuple (0 for invalid sizes). */
size_t mkb_psf_workspace_bytes(int32_t tuples, int32_t grid, int32_t fft_size);
/* maps [T][N][N] and params [T] on the device; fft_size a power of two in [2N, 8192]. */
int mkb_psf_device(int32_t tuples, int32_t grid, int32_t fft_size, const double* maps,
                   const mkb_psf_pupil_params* params, double* psf, double* mtf, void* workspace,
                   size_t workspace_bytes, void* stream);
/* OPD maps from EVAL's device outputs without a host round trip (eval_opd_map with piston
 * removal, src/eval/eval.cpp:512): maps [T][N][N] NaN, then the OPD of every ray with status Ok
 * at (row[k], column[k]) of its grid point, also at column N - 1 - column[k] for a half pupil.
 * opd, status [T][samples] as mkb_eval_device writes them; column, row [samples] device. */
int mkb_psf_maps_device(int32_t tuples, int32_t grid, int64_t samples, int32_t half_pupil,
                        const double* opd, const uint8_t* status, const int32_t* column,
                        const int32_t* row, double* maps, void* stream);
/* The NA of the pupil imaging of one tuple from its four EVAL field rays (make_psf_pupil,
 * src/eval/psf.cpp:196): field_rays [4][5], field_status [4], n_image = index of the image
 * space at the tuple's wavelength; numerical_aperture > 0 overrides the field rays. Sets the
 * mirror flags of a divergent wave. MKB_ERR_ARGUMENT when the NA is undetermined. */
int mkb_psf_aperture_host(const double* field_rays, const uint8_t* field_status, double n_image,
                          double field_ray_offset, double numerical_aperture, double* na_x,
                          double* na_y, int32_t* flip_x, int32_t* flip_y);
/* finish_psf and the geometry of prepare_psf_result (src/eval/psf.cpp:262,290) on the host for
 * one tuple: transmitted points, energy, Strehl from the FFT, direct Strehl before and after
 * the least-squares tilt, the tilt's reference point, the peak; host arrays opd_map [N][N] and
 * psf [M][M]. Bit-identical to the reference's finish_psf on the same PSF. */
int mkb_psf_finish_host(int32_t grid, int32_t fft_size, const double* opd_map, int32_t full_count,
                        double wavelength_nm, double na_x, double na_y, int32_t flip_x,
                        int32_t flip_y, const double* psf, mkb_psf_metrics* out);

/* ---- diagnostics ----------------------------------------------------------------------- */
const char* mkb_last_error(void);
const char* mkb_version(void);
/* Reads and clears the device-side error words (synchronising): MKB_OK, or MKB_ERR_TIMEOUT
 * when a bounded wait inside a kernel gave up since the last call. */
int mkb_device_status(void);
/* Polls the first wait on a kernel's bulk copy makes before it gives up, records
 * MKB_ERR_TIMEOUT and leaves the block's outputs unwritten (default MKB_WAIT_POLLS_DEFAULT;
 * 0 makes every such wait give up at once, which lets a test drive the failure path without a
 * fault or a hang). The wait that drains the copy after a give-up keeps the default limit.
 * Synchronising (cudaMemcpyToSymbol per kernel file); set it with no kernel in flight. No
 * counterpart in the reference, whose waits are not bounded. */
#define MKB_WAIT_POLLS_DEFAULT (1u << 24)
int mkb_set_wait_limit(uint32_t polls);
/* Number of kernel launches this library has enqueued in the calling process. */
int64_t mkb_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* MIKROPTIM_B200_H */
