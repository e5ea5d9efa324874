// Paraxial constraints on the device: the checked constraint block the kernels take and the
// launchers (paraxial.cu). Used by the LM cycle (lm.cu) and mkb_paraxial_rows_device.
#pragma once

#include "common.cuh"

namespace mkb {

// The constraints of a launch, checked on the host (check_paraxial_constraints,
// src/optim/paraxial_residuals.cpp:157), passed by value.
struct ParaxialSpec {
    int E;            // rows (0: none)
    int column;       // wavelength column of the paraxial index in the records
    int analytic;     // 1: analytic adjoint Jacobian, 0: central differences
    double omega_ref; // Buchdahl coordinate of the reference wavelength
    int type[MKB_MAX_PARAXIAL], mode[MKB_MAX_PARAXIAL], ref_surface[MKB_MAX_PARAXIAL];
    double root_w[MKB_MAX_PARAXIAL], target[MKB_MAX_PARAXIAL], offset[MKB_MAX_PARAXIAL];
    double shift[MKB_MAX_PARAXIAL];
    // ghost plates: G plates of K profile terms; the plate of a table surface (or -1) and the
    // table surface of a plate
    int G, K;
    int8_t ghost_of[kMaxSurfaces];
    int8_t ghost_surface[kMaxGhostPlates];
};

// buchdahl_index (glass/dispersion.hpp:93): n0 + w (nu1 + w (nu2 + w nu3)), each operation
// separately rounded, as refresh_glass forms it
__device__ __forceinline__ double buchdahl(const double* b, double w) {
    const double inner = __dadd_rn(b[2], __dmul_rn(w, b[3]));
    const double mid = __dadd_rn(b[1], __dmul_rn(w, inner));
    return __dadd_rn(b[0], __dmul_rn(w, mid));
}

// Checks the options' constraints against the batch and fills `sp` (E = 0 without any).
int make_paraxial_spec(const mkb_lm_options* options, const mkb_device_batch* batch,
                       const mkb_residual_plan* plan, ParaxialSpec* sp);

// Rows re [runs][E] and Jacobian je [runs][pstride][E] at x [runs][pstride] for the runs
// mask selects (null: all); the runs' variables are vt[run] (null: vp for every run).
int launch_paraxial_rows(const ParaxialSpec& sp, const VarParams& vp, const VarParams* vt,
                         int pstride, const mkb_device_batch* templates, const double* x,
                         int runs, const int* mask, double* je, double* re,
                         cudaStream_t stream);

// out[run] = sum_e r_e^2 at x[run] for the runs mask selects (others untouched).
int launch_paraxial_merit(const ParaxialSpec& sp, const VarParams& vp, const VarParams* vt,
                          int pstride, const mkb_device_batch* templates, const double* x,
                          int runs, const int* mask, double* out, cudaStream_t stream);

}  // namespace mkb
