/*
 * Test infrastructure (the oracle), not product code.
 *
 * Plain-C restatement of the reference's CPU algorithm for the batched trace-and-optimise
 * path. Built into oracle/liboracle.so; only tests, smoke() and bench.py's CPU legs use it.
 * Every function cites the reference file:line it restates. Inputs are the flat structs of
 * include/mikroptim_b200.h. All functions return 0 on success and -1 on a bad argument.
 */
#ifndef MKO_ORACLE_H
#define MKO_ORACLE_H

#include "mikroptim_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

int64_t mko_port_rays_per_variant(const mkb_residual_plan* plan);

/* Paraxial ray aiming of an interior aperture stop (MKB_SURFACE_APERTURE_STOP; this build's
 * own definition, the reference's stop is always surface 0): per variant the entrance pupil
 * radius R / |y_A| and thickness[0] = -y_B / y_A from the y-u trace of wavelength column 0
 * from surface 1 to the stop. Restated here as the checker of the packed records. */
int mko_port_aim(const mkb_batch_view* view, double* pupil, double* thickness0);

/* residuals_cpu (src/batch/batch_residuals.cpp:272): residuals [V][trace_rows],
 * opd [V][rays], status [V][rays] (opd, status may be NULL). */
int mko_port_residuals(const mkb_batch_view* view, const mkb_residual_plan* plan,
                       double* residuals, double* opd, uint8_t* status, int threads);

/* merit_cpu (src/batch/batch_merit.cpp:61). */
int mko_port_merit(const mkb_batch_view* view, const mkb_residual_plan* plan, double* merit,
                   int64_t* failed, int64_t* hard_failed, int threads);

/* fd_jacobian_cpu, central scheme (src/optim/fd_jacobian.cpp:182): base has 1 variant or
 * one per run; J [runs][P][R], r0 [runs][R], status_changes [runs][P] (may be NULL). */
int mko_port_fd_jacobian(const mkb_batch_view* view, const mkb_residual_plan* plan,
                         const mkb_variables* vars, const double* x0, int runs, double* J,
                         double* r0, int64_t* status_changes, int threads);

/* adjoint_jacobian_cpu (src/optim/adjoint_jacobian.cpp:370), no extra rows. */
int mko_port_adjoint_jacobian(const mkb_batch_view* view, const mkb_residual_plan* plan,
                              const mkb_variables* vars, const double* x0, int runs, double* J,
                              double* r0, uint8_t* status, int threads);

/* normal_equations_host (include/mikroptim/optim/normal_equations.hpp:33). */
int mko_port_normal_equations(const double* J, const double* r, int P, int64_t R, double* A,
                              double* g);

#ifdef __cplusplus
}
#endif

#endif
