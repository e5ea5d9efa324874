// Batched Levenberg-Marquardt on the device.
//
// The control logic of the reference's levenberg_marquardt (src/optim/levenberg_marquardt.cpp:
// 332-589) runs per run on the GPU, with every run's decisions depending only on its own state:
//   lm_update_kernel  one CTA per run: new normal equations -> prepare_step (Marquardt scaling,
//                     projected gradient), the Gauss-Newton model solve (mu = 1e-12) and the
//                     gtol / ftol / xtol tests, then the damped active-set step solve_step(mu)
//                     with the trial point clamp(x + delta)
//   (trial MERIT)     the trace kernels, launched by the entry point
//   lm_accept_kernel  one thread per run: gain ratio, acceptance, Nielsen damping update
// Every operation of prepare_step, cholesky, cholesky_solve and solve_step is a separately
// rounded IEEE operation in the reference's order (sequential where the reference sums
// sequentially), so with bit-identical normal equations and merits the run trajectories equal
// the reference's host loop bit for bit. One cycle is a fixed sequence of launches with
// per-run masks (no host decisions), so a cycle can be captured in a CUDA graph.
#include "launch.cuh"
#include "paraxial.cuh"

#include <algorithm>
#include <vector>
#include <cmath>

namespace mkb {

// LmStatus (include/mikroptim/optim/levenberg_marquardt.hpp:26)
enum : int { kRunning = 0, kConvergedMerit = 1, kConvergedStep = 2, kConvergedGradient = 3,
             kConvergedStall = 4, kMaxIterations = 5, kDampingLimit = 6, kNumericalError = 7 };

struct LmOptionsDev {
    int max_iterations;
    double ftol, xtol, gtol, initial_damping, max_damping, diag_floor;
    int reject_new_failures;
};

// Per-run LM state in the workspace (structure of arrays).
struct LmState {
    double* x;          // [runs][P]
    double* trial;      // [runs][P]
    double* a;          // [runs][P][P]   J^T J (column-major, as the reference)
    double* g;          // [runs][P]
    double* d;          // [runs][P]      Marquardt scaling
    double* merit;      // [runs]
    double* mu;         // [runs]
    double* nu;         // [runs]
    double* predicted;  // [runs]
    double* step_norm;  // [runs]
    double* step_damping;
    double* gradient_norm;
    double* model_decrease;
    double* history;    // [runs][max_iterations + 1]
    int64_t* failed;    // [runs]
    int64_t* hard;      // [runs]
    int* status;        // [runs] LmStatus
    int* iterations;
    int* accepted;
    int* jacobians;
    int* need_jacobian;
    int* rejected;
    int* solved;
    int* in_cycle;      // this cycle took a trial step
    int* evaluate;      // this cycle's trial point is evaluated (mask of the trial MERIT)
    int* want_jacobian; // the next cycle computes this run's Jacobian (mask of the Jacobian)
    int* running;       // [1] runs still running after the last cycle
    const VarParams* vt;  // per-run variables (uneven batches) or null: the launch's VarParams
    int pstride;          // entries per run of x / trial / g / d (the largest P), P*P of a
};

// The next cycle's update reads new normal equations exactly for these runs.
__device__ __forceinline__ int wants_jacobian(const LmState& st, int run, int max_iterations) {
    return st.status[run] == 0 && st.need_jacobian[run] && st.iterations[run] < max_iterations;
}

namespace {

constexpr int kStepThreads = 64;
constexpr int kMaxP = MKB_MAX_VARIABLES;
constexpr double kModelDamping = 1e-12;

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }  // std::max
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }  // std::min

__device__ __forceinline__ Exact64 scale_of(double x, double typical) {
    return Exact64(dmax(fabs(x), typical));
}

__device__ __forceinline__ bool bound_blocks(const VarParams& v, int k, double x, double dir) {
    if (v.lower[k] == v.upper[k]) return true;
    return (x <= v.lower[k] && dir < 0.0) || (x >= v.upper[k] && dir > 0.0);
}

struct StepShared {
    double m[kMaxP * kMaxP];  // damped free block, column-major lower triangle
    double rhs[kMaxP];
    double delta[kMaxP];
    double step[kMaxP];
    double aq[kMaxP];
    int idx[kMaxP];
    int fixed[kMaxP];
    int f;
    int changed;
    int ok;
};

// solve_step (levenberg_marquardt.cpp:149) for one run, by one CTA. a, g, d, x of the run.
// Writes trial, and returns solved / step_norm / predicted through shared memory.
__device__ void solve_step(const VarParams& v, const double* a, const double* g, const double* d,
                           const double* x, double mu, double* trial, StepShared& sh,
                           int& solved, double& step_norm, double& predicted) {
    const int n = v.P;
    const int tid = threadIdx.x;
    for (int k = tid; k < n; k += blockDim.x) sh.fixed[k] = bound_blocks(v, k, x[k], -g[k]) ? 1 : 0;
    __syncthreads();
    solved = 1;
    for (int round = 0; round <= n; ++round) {
        if (tid == 0) {
            int f = 0;
            for (int k = 0; k < n; ++k)
                if (!sh.fixed[k]) sh.idx[f++] = k;
            sh.f = f;
        }
        for (int k = tid; k < n; k += blockDim.x) sh.delta[k] = 0.0;
        __syncthreads();
        const int f = sh.f;
        if (f == 0) break;
        // m = lower triangle of A_FF + mu D_FF, rhs = -g_F
        for (int e = tid; e < f * f; e += blockDim.x) {
            const int j = e / f, i = e - j * f;
            if (i >= j) {
                double val = a[sh.idx[j] * n + sh.idx[i]];
                if (i == j) val = (Exact64(val) + Exact64(mu) * Exact64(d[sh.idx[j]])).v;
                sh.m[j * f + i] = val;
            }
        }
        for (int j = tid; j < f; j += blockDim.x) sh.rhs[j] = -g[sh.idx[j]];
        if (tid == 0) sh.ok = 1;
        __syncthreads();
        // cholesky (levenberg_marquardt.cpp:70): column j, diagonal by one thread, then the
        // rows i > j in parallel; every sum in ascending k
        for (int j = 0; j < f; ++j) {
            if (tid == 0) {
                Exact64 diag = sh.m[j * f + j];
                for (int k = 0; k < j; ++k) diag -= Exact64(sh.m[k * f + j]) * Exact64(sh.m[k * f + j]);
                if (!(diag.v > 0.0) || !isfinite(diag.v)) sh.ok = 0;
                else sh.m[j * f + j] = nsqrt(diag).v;
            }
            __syncthreads();
            if (!sh.ok) break;
            const Exact64 ljj = sh.m[j * f + j];
            for (int i = j + 1 + tid; i < f; i += blockDim.x) {
                Exact64 s = sh.m[j * f + i];
                for (int k = 0; k < j; ++k) s -= Exact64(sh.m[k * f + i]) * Exact64(sh.m[k * f + j]);
                sh.m[j * f + i] = (s / ljj).v;
            }
            __syncthreads();
        }
        if (!sh.ok) {
            solved = 0;
            __syncthreads();
            return;
        }
        // cholesky_solve (levenberg_marquardt.cpp:94): L z = b column-oriented (each b[j]
        // subtracts l[k][j] b[k] for k ascending, as the row loop does), L^T y = z row by row
        for (int i = 0; i < f; ++i) {
            if (tid == 0) sh.rhs[i] = (Exact64(sh.rhs[i]) / Exact64(sh.m[i * f + i])).v;
            __syncthreads();
            const Exact64 bi = sh.rhs[i];
            for (int j = i + 1 + tid; j < f; j += blockDim.x)
                sh.rhs[j] = (Exact64(sh.rhs[j]) - Exact64(sh.m[i * f + j]) * bi).v;
            __syncthreads();
        }
        if (tid == 0) {
            for (int i = f - 1; i >= 0; --i) {
                Exact64 s = sh.rhs[i];
                for (int k = i + 1; k < f; ++k) s -= Exact64(sh.m[i * f + k]) * Exact64(sh.rhs[k]);
                sh.rhs[i] = (s / Exact64(sh.m[i * f + i])).v;
            }
            sh.changed = 0;
        }
        __syncthreads();
        for (int j = tid; j < f; j += blockDim.x) sh.delta[sh.idx[j]] = sh.rhs[j];
        __syncthreads();
        if (tid == 0) {
            int changed = 0;
            for (int j = 0; j < f; ++j) {
                const int k = sh.idx[j];
                if (bound_blocks(v, k, x[k], sh.delta[k])) {
                    sh.fixed[k] = 1;
                    changed = 1;
                }
            }
            sh.changed = changed;
        }
        __syncthreads();
        if (!sh.changed) break;
    }
    // trial point, step norm, predicted decrease -(2 step.g + step.A.step)
    for (int k = tid; k < n; k += blockDim.x) {
        const double t = dmin(dmax((Exact64(x[k]) + Exact64(sh.delta[k])).v, v.lower[k]), v.upper[k]);
        trial[k] = t;
        sh.step[k] = (Exact64(t) - Exact64(x[k])).v;
    }
    __syncthreads();
    for (int q = tid; q < n; q += blockDim.x) {
        Exact64 s = 0.0;
        for (int p = 0; p < n; ++p) s += Exact64(a[q * n + p]) * Exact64(sh.step[p]);
        sh.aq[q] = s.v;
    }
    __syncthreads();
    if (tid == 0) {
        double norm = 0.0;
        for (int k = 0; k < n; ++k)
            norm = dmax(norm, (Exact64(fabs(sh.step[k])) / scale_of(x[k], v.typical[k])).v);
        Exact64 lin = 0.0, quad = 0.0;
        for (int q = 0; q < n; ++q) {
            lin += Exact64(sh.step[q]) * Exact64(g[q]);
            quad += Exact64(sh.step[q]) * Exact64(sh.aq[q]);
        }
        step_norm = norm;
        predicted = (-(Exact64(2.0) * lin + quad)).v;
        sh.ok = 1;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kStepThreads)
lm_update_kernel(const __grid_constant__ VarParams v, LmOptionsDev o, LmState st,
                 const double* __restrict__ gram, int runs) {
    __shared__ StepShared sh;
    __shared__ double s_pred, s_norm;
    __shared__ int s_solved, s_status;
    const int run = blockIdx.x;
    if (run >= runs) return;
    const VarParams& vr = st.vt != nullptr ? st.vt[run] : v;
    const int n = vr.P;
    const int64_t ps = st.pstride;
    const int tid = threadIdx.x;
    double* x = st.x + run * ps;
    double* trial = st.trial + run * ps;
    double* a = st.a + run * ps * ps;
    double* g = st.g + run * ps;
    double* d = st.d + run * ps;
    int status = st.status[run];
    const double merit = st.merit[run];
    // ---- new normal equations ----
    if (status == kRunning && st.need_jacobian[run] && st.iterations[run] < o.max_iterations) {
        const double* G = gram + run * (ps + 1) * (ps + 1);
        __shared__ int s_finite;
        if (tid == 0) s_finite = 1;
        __syncthreads();
        for (int e = tid; e < n * n; e += blockDim.x) {
            const int q = e / n, p = e - q * n;
            const double val = G[q * (n + 1) + p];
            a[e] = val;
            if (!isfinite(val)) s_finite = 0;
        }
        for (int q = tid; q < n; q += blockDim.x) {
            const double val = G[q * (n + 1) + n];
            g[q] = val;
            if (!isfinite(val)) s_finite = 0;
        }
        __syncthreads();
        if (tid == 0) {
            st.need_jacobian[run] = 0;
            st.jacobians[run] += 1;
        }
        if (!s_finite) {
            status = kNumericalError;
        } else {
            // prepare_step (levenberg_marquardt.cpp:122)
            if (tid == 0) {
                double smax = 0.0;
                for (int k = 0; k < n; ++k) {
                    const Exact64 sk = scale_of(x[k], vr.typical[k]);
                    smax = dmax(smax, (Exact64(a[k * n + k]) * sk * sk).v);
                }
                double gmax = 0.0;
                for (int k = 0; k < n; ++k) {
                    const Exact64 sk = scale_of(x[k], vr.typical[k]);
                    const double akk = a[k * n + k];
                    const double floor = smax > 0.0
                                             ? (Exact64(o.diag_floor) * Exact64(smax) / (sk * sk)).v
                                             : (Exact64(1.0) / (sk * sk)).v;
                    d[k] = dmax(akk, floor);
                    if (!bound_blocks(vr, k, x[k], -g[k])) {
                        const double denom = nsqrt(Exact64(akk) * Exact64(merit)).v;
                        if (denom > 0.0) gmax = dmax(gmax, (Exact64(fabs(g[k])) / Exact64(denom)).v);
                    }
                }
                st.gradient_norm[run] = gmax;
            }
            __syncthreads();
            int solved;
            double norm, pred;
            solve_step(vr, a, g, d, x, kModelDamping, trial, sh, solved, norm, pred);
            if (tid == 0) {
                st.model_decrease[run] = solved ? (Exact64(pred) / Exact64(merit)).v : nan("");
                if (st.gradient_norm[run] <= o.gtol) status = kConvergedGradient;
                else if (solved && pred >= 0.0 && pred <= (Exact64(o.ftol) * Exact64(merit)).v)
                    status = kConvergedMerit;
                else if (solved && norm <= o.xtol) status = kConvergedStep;
                s_status = status;
            }
            __syncthreads();
            status = s_status;
        }
    }
    // ---- trial step ----
    int in_cycle = 0, evaluate = 0;
    if (status == kRunning) {
        if (st.iterations[run] >= o.max_iterations) {
            status = kMaxIterations;
        } else {
            in_cycle = 1;
            int solved;
            double norm, pred;
            solve_step(vr, a, g, d, x, st.mu[run], trial, sh, solved, norm, pred);
            if (tid == 0) {
                s_solved = solved;
                s_norm = norm;
                s_pred = pred;
            }
            __syncthreads();
            if (s_solved && st.rejected[run] && s_norm <= o.xtol) status = kConvergedStep;
            else if (s_solved) evaluate = 1;
        }
    }
    if (tid == 0) {
        st.status[run] = status;
        st.in_cycle[run] = in_cycle && status != kConvergedStep;
        st.evaluate[run] = evaluate;
        if (in_cycle) {
            st.solved[run] = s_solved;
            st.step_norm[run] = s_norm;
            st.predicted[run] = s_pred;
            st.step_damping[run] = st.mu[run];
        }
    }
}

// Acceptance (levenberg_marquardt.cpp:518-545) after the trial MERIT.
// post (or null): the caller's merit share added after the kernel's (trace-dependent extra
// rows, src/cuda/levenberg_marquardt.cpp:235-240).
__global__ void lm_accept_kernel(LmOptionsDev o, LmState st, int P, const double* trial_merit,
                                 const int64_t* trial_failed, const int64_t* trial_hard,
                                 int runs, const double* post) {
    const int run = blockIdx.x * blockDim.x + threadIdx.x;
    if (run >= runs) return;
    if (!st.in_cycle[run]) {
        if (st.status[run] == kRunning) atomicAdd(st.running, 1);
        st.want_jacobian[run] = wants_jacobian(st, run, o.max_iterations);
        return;
    }
    st.iterations[run] += 1;
    bool accept = false;
    const int n = st.vt != nullptr ? st.vt[run].P : P;
    const int64_t ps = st.pstride;
    if (st.solved[run]) {
        const double f_new = post != nullptr ? __dadd_rn(trial_merit[run], post[run])
                                             : trial_merit[run];
        const double merit = st.merit[run];
        const double pred = st.predicted[run];
        const double rho = (Exact64(merit) - Exact64(f_new)).v / pred;
        accept = isfinite(f_new) && pred > 0.0 && f_new < merit &&
                 !(o.reject_new_failures && trial_hard[run] > st.hard[run]);
        if (accept) {
            for (int k = 0; k < n; ++k) st.x[run * ps + k] = st.trial[run * ps + k];
            st.merit[run] = f_new;
            st.failed[run] = trial_failed[run];
            st.hard[run] = trial_hard[run];
            const Exact64 t = Exact64(2.0) * Exact64(rho) - Exact64(1.0);
            st.mu[run] = (Exact64(st.mu[run]) *
                          Exact64(dmax(1.0 / 3.0, (Exact64(1.0) - t * t * t).v))).v;
            st.nu[run] = 2.0;
            st.need_jacobian[run] = 1;
            st.rejected[run] = 0;
            st.accepted[run] += 1;
            if (f_new == 0.0) st.status[run] = kConvergedMerit;
        }
    }
    if (!accept) {
        st.mu[run] = (Exact64(st.mu[run]) * Exact64(st.nu[run])).v;
        st.nu[run] = (Exact64(st.nu[run]) * Exact64(2.0)).v;
        st.rejected[run] = 1;
        if (st.mu[run] > o.max_damping) st.status[run] = kDampingLimit;
    }
    st.history[static_cast<int64_t>(run) * (o.max_iterations + 1) + st.iterations[run]] =
        st.merit[run];
    if (st.status[run] == kRunning) atomicAdd(st.running, 1);
    st.want_jacobian[run] = wants_jacobian(st, run, o.max_iterations);
}

// Start: merit at x0 (already evaluated into merit/failed/hard), status, damping.
__global__ void lm_init_kernel(LmOptionsDev o, LmState st, int P, const double* x0, int runs,
                               const double* post) {
    const int run = blockIdx.x * blockDim.x + threadIdx.x;
    if (run >= runs) return;
    if (post != nullptr) st.merit[run] = __dadd_rn(st.merit[run], post[run]);
    const int64_t ps = st.pstride;  // x0 rows have the same stride (P, or the largest P)
    for (int k = 0; k < ps; ++k) {
        const double xv = x0[run * ps + k];
        st.x[run * ps + k] = xv;
        st.trial[run * ps + k] = xv;
    }
    const double m = st.merit[run];
    int status = kRunning;
    if (!isfinite(m)) status = kNumericalError;
    else if (m == 0.0) status = kConvergedMerit;
    st.status[run] = status;
    st.mu[run] = o.initial_damping;
    st.nu[run] = 2.0;
    st.need_jacobian[run] = 1;
    st.rejected[run] = 0;
    st.iterations[run] = st.accepted[run] = st.jacobians[run] = 0;
    st.gradient_norm[run] = 0.0;
    st.model_decrease[run] = nan("");
    st.history[static_cast<int64_t>(run) * (o.max_iterations + 1)] = m;
    for (int h = 1; h <= o.max_iterations; ++h)
        st.history[static_cast<int64_t>(run) * (o.max_iterations + 1) + h] = nan("");
    if (status == kRunning) atomicAdd(st.running, 1);
    st.want_jacobian[run] = wants_jacobian(st, run, o.max_iterations);
}

// Rows of the caller's own (the reference's extra residuals, appended after the trace rows):
// every entry of [J r]^T [J r] of the runs that got normal equations in this cycle continues
// its chain over the extra rows e = 0 .. E-1, acc = fma(u_e, v_e, acc), as the reference's
// normal_equations_host does over all rows in ascending order. je [runs][pstride][E] (column
// k of run i at (i * pstride + k) * E), re [runs][E].
__global__ void gram_extend_kernel(const VarParams v, LmState st, double* __restrict__ gram,
                                   const double* __restrict__ je, const double* __restrict__ re,
                                   int E, int runs) {
    const int run = blockIdx.x;
    if (run >= runs || !st.want_jacobian[run]) return;
    const int n = st.vt != nullptr ? st.vt[run].P : v.P;
    const int64_t ps = st.pstride;
    double* G = gram + run * (ps + 1) * (ps + 1);
    const double* col = je + run * ps * E;
    const double* r = re + static_cast<int64_t>(run) * E;
    for (int e = threadIdx.x; e < (n + 1) * (n + 1); e += blockDim.x) {
        const int q = e / (n + 1), p = e - q * (n + 1);
        const double* u = q < n ? col + static_cast<int64_t>(q) * E : r;
        const double* w = p < n ? col + static_cast<int64_t>(p) * E : r;
        double acc = G[e];
        for (int k = 0; k < E; ++k) acc = fma(u[k], w[k], acc);
        G[e] = acc;
    }
}

}  // namespace

int launch_lm_init(const LmOptionsDev& o, const LmState& st, int P, const double* x0, int runs,
                   cudaStream_t stream, const double* post = nullptr) {
    lm_init_kernel<<<(runs + 127) / 128, 128, 0, stream>>>(o, st, P, x0, runs, post);
    count_launch();
    return cuda_status(cudaGetLastError(), "lm init launch");
}

int launch_lm_update(const VarParams& v, const LmOptionsDev& o, const LmState& st,
                     const double* gram, int runs, cudaStream_t stream) {
    lm_update_kernel<<<runs, kStepThreads, 0, stream>>>(v, o, st, gram, runs);
    count_launch();
    return cuda_status(cudaGetLastError(), "lm update launch");
}

int launch_lm_accept(const LmOptionsDev& o, const LmState& st, int P, const double* trial_merit,
                     const int64_t* trial_failed, const int64_t* trial_hard, int runs,
                     cudaStream_t stream, const double* post = nullptr) {
    lm_accept_kernel<<<(runs + 127) / 128, 128, 0, stream>>>(o, st, P, trial_merit, trial_failed,
                                                             trial_hard, runs, post);
    count_launch();
    return cuda_status(cudaGetLastError(), "lm accept launch");
}

MKB_DEFINE_ERROR_READER(lm_device_error)

int launch_gram_extend(const VarParams& v, const LmState& st, double* gram, const double* je,
                       const double* re, int E, int runs, cudaStream_t stream) {
    if (runs <= 0 || E <= 0) return MKB_OK;
    gram_extend_kernel<<<runs, 256, 0, stream>>>(v, st, gram, je, re, E, runs);
    count_launch();
    return cuda_status(cudaGetLastError(), "lm extra rows launch");
}

}  // namespace mkb

// ---- entry points ------------------------------------------------------------------------------
namespace mkb {

namespace {

size_t al(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

struct LmLayout {
    size_t total;
    LmState st;
    double* gram;
    double* J;
    double* r0;
    uint8_t* status;
    double* records;
    void* merit_ws;
    size_t merit_ws_bytes;
    double* trial_merit;
    int64_t* trial_failed;
    int64_t* trial_hard;
    void* fd_ws;
    size_t fd_ws_bytes;
    void* fused_ws;
    size_t fused_ws_bytes;
    VarParams* vt;      // per-run variables (uneven batches), else null
    uint8_t* vsurf;     // surface count of each run's record (uneven surfaces), else null
    int* order;         // processing order (uneven batches), else null
    int* split;         // [1] runs of the first group of `order`
    double* px_je;      // device paraxial rows: Jacobian [runs][pmax][E], rows [runs][E],
    double* px_re;      // and sum r_e^2 at the points of the merit [runs]
    double* px_merit;
};

constexpr int kFdChunkRuns = 64;

struct LmSetup {
    TraceParams tp;
    VarParams vp;       // the variables (uniform) or those of run 0 (per run)
    LmOptionsDev o;
    bool fd, exact, gram_exact, fused;
    bool per_run;       // per-run variables
    bool any_glass;     // some run has glass variables
    int min_floor;      // the smallest sweep floor of the runs' variable sets
    int pmax;           // P, or the largest P of the runs
    int precision;
    int64_t R;
    ParaxialSpec px;    // paraxial constraints evaluated on the device (px.E = 0: none)
};

// Carves the workspace (base may be null to only size it).
LmLayout lm_layout(char* base, const LmSetup& s, int runs, const mkb_device_batch* templates,
                   const mkb_residual_plan* plan) {
    LmLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off += al(bytes);
        return p;
    };
    const TraceParams& tp = s.tp;
    const size_t P = static_cast<size_t>(s.pmax);
    const int max_it = s.o.max_iterations;
    const size_t r = static_cast<size_t>(runs);
    const int64_t R = s.R;
    L.st.x = reinterpret_cast<double*>(take(8 * r * P));
    L.st.trial = reinterpret_cast<double*>(take(8 * r * P));
    L.st.a = reinterpret_cast<double*>(take(8 * r * P * P));
    L.st.g = reinterpret_cast<double*>(take(8 * r * P));
    L.st.d = reinterpret_cast<double*>(take(8 * r * P));
    L.st.merit = reinterpret_cast<double*>(take(8 * r));
    L.st.mu = reinterpret_cast<double*>(take(8 * r));
    L.st.nu = reinterpret_cast<double*>(take(8 * r));
    L.st.predicted = reinterpret_cast<double*>(take(8 * r));
    L.st.step_norm = reinterpret_cast<double*>(take(8 * r));
    L.st.step_damping = reinterpret_cast<double*>(take(8 * r));
    L.st.gradient_norm = reinterpret_cast<double*>(take(8 * r));
    L.st.model_decrease = reinterpret_cast<double*>(take(8 * r));
    L.st.history = reinterpret_cast<double*>(take(8 * r * (max_it + 1)));
    L.st.failed = reinterpret_cast<int64_t*>(take(8 * r));
    L.st.hard = reinterpret_cast<int64_t*>(take(8 * r));
    L.st.status = reinterpret_cast<int*>(take(4 * r));
    L.st.iterations = reinterpret_cast<int*>(take(4 * r));
    L.st.accepted = reinterpret_cast<int*>(take(4 * r));
    L.st.jacobians = reinterpret_cast<int*>(take(4 * r));
    L.st.need_jacobian = reinterpret_cast<int*>(take(4 * r));
    L.st.rejected = reinterpret_cast<int*>(take(4 * r));
    L.st.solved = reinterpret_cast<int*>(take(4 * r));
    L.st.in_cycle = reinterpret_cast<int*>(take(4 * r));
    L.st.evaluate = reinterpret_cast<int*>(take(4 * r));
    L.st.want_jacobian = reinterpret_cast<int*>(take(4 * r));
    L.st.running = reinterpret_cast<int*>(take(4));
    L.vt = s.per_run ? reinterpret_cast<VarParams*>(take(sizeof(VarParams) * r)) : nullptr;
    L.st.vt = L.vt;
    L.st.pstride = s.pmax;
    const bool uneven = templates->variant_surfaces != nullptr;
    L.vsurf = uneven ? reinterpret_cast<uint8_t*>(take(r)) : nullptr;
    L.order = uneven || s.per_run ? reinterpret_cast<int*>(take(4 * r)) : nullptr;
    L.split = uneven || s.per_run ? reinterpret_cast<int*>(take(4)) : nullptr;
    L.gram = reinterpret_cast<double*>(take(8 * r * (P + 1) * (P + 1)));
    const size_t jr = s.fused ? 0 : r;  // the fused adjoint keeps J out of memory
    L.J = reinterpret_cast<double*>(take(8 * jr * P * R));
    L.r0 = reinterpret_cast<double*>(take(8 * jr * R));
    L.status = reinterpret_cast<uint8_t*>(take(jr * tp.rays));
    L.records = reinterpret_cast<double*>(take(8 * r * tp.stride));
    L.merit_ws_bytes = merit_workspace_bytes(runs, tp.n_tuples);
    L.merit_ws = take(L.merit_ws_bytes);
    L.trial_merit = reinterpret_cast<double*>(take(8 * r));
    L.trial_failed = reinterpret_cast<int64_t*>(take(8 * r));
    L.trial_hard = reinterpret_cast<int64_t*>(take(8 * r));
    L.fused_ws_bytes = s.fused ? fused_scratch_bytes(runs, s.pmax, tp.S) : 0;
    L.fused_ws = take(L.fused_ws_bytes);
    L.fd_ws_bytes = 0;
    if (s.fd) {
        mkb_device_batch t = *templates;
        L.fd_ws_bytes = mkb_fd_jacobian_workspace_bytes(&t, plan, s.pmax, runs,
                                                        runs < kFdChunkRuns ? runs : kFdChunkRuns);
        L.fd_ws = take(L.fd_ws_bytes);
    }
    const size_t E = static_cast<size_t>(s.px.E);
    L.px_je = reinterpret_cast<double*>(take(8 * r * P * E));
    L.px_re = reinterpret_cast<double*>(take(8 * r * E));
    L.px_merit = E > 0 ? reinterpret_cast<double*>(take(8 * r)) : nullptr;
    L.total = off;
    return L;
}

// table != null (start): every run's variables are validated and built into it.
int lm_setup(const mkb_device_batch* templates, const mkb_residual_plan* plan,
             const mkb_variables* vars, const mkb_lm_options* options, int runs, LmSetup& s,
             std::vector<VarParams>* table = nullptr) {
    if (templates == nullptr || options == nullptr || runs < 1 || vars == nullptr) {
        set_error("lm: null templates/options/variables or runs < 1");
        return MKB_ERR_ARGUMENT;
    }
    if (templates->variants != 1 && templates->variants != runs) {
        set_error("lm: templates must hold 1 variant or one per run");
        return MKB_ERR_ARGUMENT;
    }
    mkb_device_batch b = *templates;
    b.variants = runs;
    int rc = make_trace_params(&b, plan, pack_rays_default(), &s.tp);
    if (rc != MKB_OK) return rc;
    if (plan->precision != MKB_PRECISION_FP64 && plan->precision != MKB_PRECISION_FP64_FMA &&
        plan->precision != MKB_PRECISION_MIXED && plan->precision != MKB_PRECISION_FP32_BULK) {
        set_error("lm: precision %d not available", plan->precision);
        return MKB_ERR_UNSUPPORTED;
    }
    const mkb_lm_options& o = *options;
    s.per_run = o.per_run_variables != 0;
    rc = make_var_params(&vars[0], s.tp.S, templates->type, &s.vp, templates->ghost_terms,
                         templates->wavelengths, templates->wavelength_nm,
                         templates->glass);
    if (rc != MKB_OK) return rc;
    s.pmax = s.vp.P;
    s.any_glass = s.vp.has_glass != 0;
    s.min_floor = s.vp.sweep_floor;
    if (s.per_run) {
        if (table != nullptr) table->resize(static_cast<size_t>(runs));
        for (int r = 0; r < runs; ++r) {
            if (vars[r].count > s.pmax) s.pmax = vars[r].count;
            if (vars[r].count >= 1 && vars[r].type != nullptr && vars[r].surface != nullptr) {
                const int fl = sweep_floor_of(&vars[r], s.tp.S, templates->type);
                if (fl < s.min_floor) s.min_floor = fl;
            }
            for (int k = 0; k < vars[r].count; ++k)
                if (vars[r].type[k] == MKB_VAR_GLASS) s.any_glass = true;
            if (table != nullptr) {
                rc = make_var_params(&vars[r], s.tp.S, templates->type, &(*table)[r],
                                     templates->ghost_terms, templates->wavelengths,
                                     templates->wavelength_nm, templates->glass);
                if (rc != MKB_OK) return rc;
            }
        }
        if (s.pmax > MKB_MAX_VARIABLES) {
            set_error("lm: a run has more than %d variables", MKB_MAX_VARIABLES);
            return MKB_ERR_ARGUMENT;
        }
    }
    auto ok = [](double v) { return std::isfinite(v) && v >= 0.0; };
    if (o.max_iterations < 0 || !ok(o.ftol) || !ok(o.xtol) || !ok(o.gtol) || !ok(o.diag_floor) ||
        !(o.initial_damping > 0.0) || !std::isfinite(o.initial_damping) ||
        !(o.max_damping > o.initial_damping)) {
        set_error("lm: invalid options (check_options, levenberg_marquardt.cpp:226)");
        return MKB_ERR_ARGUMENT;
    }
    if (o.jacobian != MKB_JACOBIAN_FD && o.jacobian != MKB_JACOBIAN_ADJOINT) {
        set_error("lm: unknown jacobian method %d", o.jacobian);
        return MKB_ERR_ARGUMENT;
    }
    s.o = {o.max_iterations, o.ftol, o.xtol, o.gtol, o.initial_damping, o.max_damping,
           o.diag_floor, o.reject_new_failures};
    s.fd = o.jacobian == MKB_JACOBIAN_FD;
    s.exact = plan->precision == MKB_PRECISION_FP64;
    s.precision = plan->precision;
    s.gram_exact = o.gram_exact != 0;
    s.fused = !s.fd && !s.gram_exact;
    if ((plan->precision == MKB_PRECISION_MIXED || plan->precision == MKB_PRECISION_FP32_BULK) &&
        !s.fused) {
        set_error("lm: mixed precision runs with the fused adjoint (jacobian = adjoint, "
                  "gram_exact = 0)");
        return MKB_ERR_UNSUPPORTED;
    }
    if (!s.fd && !s.fused && (s.per_run || templates->variant_surfaces != nullptr)) {
        set_error("lm: uneven batches run with the fused adjoint (gram_exact = 0) or FD");
        return MKB_ERR_UNSUPPORTED;
    }
    s.R = trace_rows_of(plan, s.tp.rays);
    if (s.tp.transverse && s.fused) {
        set_error("lm: transverse ray-error rows have no fused adjoint; use the materialised "
                  "adjoint (gram_exact = 1) or the FD Jacobian");
        return MKB_ERR_UNSUPPORTED;
    }
    return make_paraxial_spec(options, templates, plan, &s.px);
}

// The LM's own records are one per run: their surface counts and processing order are the
// workspace's.
TraceParams run_params(const LmSetup& s, const LmLayout& L) {
    TraceParams tp = s.tp;
    tp.vsurf = L.vsurf;
    tp.order = L.order;
    return tp;
}

RunVars run_vars(const LmSetup& s, const LmLayout& L, const mkb_device_batch* templates) {
    RunVars rv;
    rv.table = L.vt;
    rv.stride = s.pmax;
    rv.tsurf = templates->variant_surfaces;
    rv.vsurf_out = L.vsurf;
    rv.any_glass = s.any_glass ? 1 : 0;
    rv.min_floor = s.min_floor;
    return rv;
}

// merit at the run points `x` (applied to the templates) into merit/failed/hard
int lm_merit_at(const LmSetup& s, const LmLayout& L, const mkb_device_batch* templates,
                const double* x, int runs, double* merit, int64_t* failed, int64_t* hard,
                cudaStream_t stream, const int* run_mask = nullptr,
                const double* extra_merit = nullptr, double* extrema = nullptr) {
    const RecordLayout lay = layout_of(s.tp);
    int rc = launch_apply(s.vp, lay, templates->records, templates->variants, x, L.records, runs,
                          stream, run_vars(s, L, templates));
    if (rc != MKB_OK) return rc;
    return launch_merit(run_params(s, L), L.records, merit, failed, hard, L.merit_ws,
                        L.merit_ws_bytes, s.precision, stream, RunMask{run_mask, 1, 0},
                        extra_merit, extrema);
}

// Processing order of the runs: those with at most kSmallP variables first (their fused
// adjoint launch needs less shared memory per CTA, so more CTAs fit an SM), each group by
// surface count, largest first. *split = size of the first group. Counting sort in one CTA;
// the order inside a bucket is not fixed, and only the scheduling depends on it.
constexpr int kSmallP = 31;
constexpr int kBuckets = 2 * (MKB_MAX_SURFACES + 1);

__global__ void order_kernel(const uint8_t* __restrict__ vsurf, const VarParams* vt, int P,
                             int runs, int S, int* __restrict__ order, int* __restrict__ split) {
    __shared__ int start[kBuckets];
    for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) start[i] = 0;
    __syncthreads();
    auto key = [&](int r) {
        int n = vsurf != nullptr ? vsurf[r] : S;
        n = n < 2 ? 2 : (n > S ? S : n);
        const int big = (vt != nullptr ? vt[r].P : P) > kSmallP ? 1 : 0;
        return big * (MKB_MAX_SURFACES + 1) + (MKB_MAX_SURFACES - n);
    };
    for (int r = threadIdx.x; r < runs; r += blockDim.x) atomicAdd(&start[key(r)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int at = 0;
        for (int k = 0; k < kBuckets; ++k) {
            if (k == MKB_MAX_SURFACES + 1) *split = at;
            const int c = start[k];
            start[k] = at;
            at += c;
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < runs; r += blockDim.x) order[atomicAdd(&start[key(r)], 1)] = r;
}

// Everything a phase of a cycle needs, checked once.
struct LmCall {
    LmSetup s;
    LmLayout L;
};

int lm_call(const mkb_device_batch* templates, const mkb_residual_plan* plan,
            const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
            void* workspace, size_t workspace_bytes, LmCall& c,
            std::vector<VarParams>* table = nullptr) {
    int rc = lm_setup(templates, plan, vars, options, runs, c.s, table);
    if (rc != MKB_OK) return rc;
    c.L = lm_layout(static_cast<char*>(workspace), c.s, runs, templates, plan);
    if (workspace == nullptr || workspace_bytes < c.L.total) {
        set_error("lm: workspace of %zu bytes needed", c.L.total);
        return MKB_ERR_WORKSPACE;
    }
    return MKB_OK;
}

// 1. Jacobian and normal equations at x for the runs whose update will read them
int phase_jacobian(const LmCall& c, const mkb_device_batch* templates,
                   const mkb_residual_plan* plan, const mkb_variables* vars, int32_t runs,
                   cudaStream_t stream) {
    const LmSetup& s = c.s;
    const LmLayout& L = c.L;
    const TraceParams tp = run_params(s, L);
    const RunVars rv = run_vars(s, L, templates);
    const int* want = L.st.want_jacobian;
    int rc;
    if (s.fd) {
        rc = fd_jacobian(templates, plan, vars, L.st.x, runs, L.J, L.r0, nullptr, L.fd_ws,
                         L.fd_ws_bytes, stream, want, rv);
    } else if (s.fused) {
        const RecordLayout lay = layout_of(s.tp);
        rc = launch_apply(s.vp, lay, templates->records, templates->variants, L.st.x, L.records,
                          runs, stream, rv);
        if (rc == MKB_OK && L.order != nullptr && s.pmax > kSmallP) {
            // two launches: the runs with few variables with a smaller shared-memory footprint
            rc = launch_adjoint_gram(tp, s.vp, L.records, L.gram, L.fused_ws, L.fused_ws_bytes,
                                     s.precision, stream, want, rv, L.order, L.split, 0,
                                     kSmallP);
            if (rc == MKB_OK)
                rc = launch_adjoint_gram(tp, s.vp, L.records, L.gram, L.fused_ws,
                                         L.fused_ws_bytes, s.precision, stream, want, rv, L.order,
                                         L.split, 1, s.pmax);
        } else if (rc == MKB_OK) {
            rc = launch_adjoint_gram(tp, s.vp, L.records, L.gram, L.fused_ws, L.fused_ws_bytes,
                                     s.precision, stream, want, rv, L.order);
        }
    } else {
        const RecordLayout lay = layout_of(s.tp);
        rc = launch_apply(s.vp, lay, templates->records, templates->variants, L.st.x, L.records,
                          runs, stream);
        if (rc == MKB_OK)
            rc = cuda_status(cudaMemsetAsync(L.J, 0, sizeof(double) * size_t(runs) * s.vp.P * s.R,
                                             stream), "lm: clear J");
        if (rc == MKB_OK)
            rc = launch_residuals(s.tp, L.records, L.r0, s.R, nullptr, L.status, s.precision,
                                  stream, RunMask{want, 1, 0});
        if (rc == MKB_OK)
            rc = launch_adjoint_rows(s.tp, s.vp, s.R, L.records, L.J, s.exact, stream);
        if (rc == MKB_OK)
            rc = launch_projection(s.tp, s.vp, s.R, L.status, L.J, s.exact, stream);
    }
    if (rc != MKB_OK) return rc;
    if (!s.fused) rc = launch_gram(L.J, L.r0, runs, s.vp.P, s.R, L.gram, s.gram_exact, stream,
                                   want, rv);
    if (rc != MKB_OK || s.px.E == 0) return rc;
    // paraxial constraint rows at x, appended after the trace rows of every entry's chain
    rc = launch_paraxial_rows(s.px, s.vp, L.vt, s.pmax, templates, L.st.x, runs, want, L.px_je,
                              L.px_re, stream);
    if (rc != MKB_OK) return rc;
    return launch_gram_extend(s.vp, L.st, L.gram, L.px_je, L.px_re, s.px.E, runs, stream);
}

// 3. trial MERIT (+ the caller's extra merit; extrema of the trial points when asked)
int phase_trial(const LmCall& c, const mkb_device_batch* templates, int32_t runs,
                const double* extra_merit, double* extrema, cudaStream_t stream) {
    if (c.s.px.E > 0) {  // the paraxial rows' sum of squares at the trial points
        if (extra_merit != nullptr) {
            set_error("lm: device paraxial constraints and host extra rows cannot be combined");
            return MKB_ERR_UNSUPPORTED;
        }
        const int rc = launch_paraxial_merit(c.s.px, c.s.vp, c.L.vt, c.s.pmax, templates,
                                             c.L.st.trial, runs, c.L.st.evaluate,
                                             c.L.px_merit, stream);
        if (rc != MKB_OK) return rc;
        extra_merit = c.L.px_merit;
    }
    return lm_merit_at(c.s, c.L, templates, c.L.st.trial, runs, c.L.trial_merit,
                       c.L.trial_failed, c.L.trial_hard, stream, c.L.st.evaluate, extra_merit,
                       extrema);
}

// 4. acceptance (post: a merit share added after the trial MERIT's, or null)
int phase_decide(const LmCall& c, int32_t runs, const double* post, cudaStream_t stream) {
    int rc = cuda_status(cudaMemsetAsync(c.L.st.running, 0, sizeof(int), stream),
                         "lm: clear count");
    if (rc != MKB_OK) return rc;
    return launch_lm_accept(c.s.o, c.L.st, c.s.vp.P, c.L.trial_merit, c.L.trial_failed,
                            c.L.trial_hard, runs, stream, post);
}

int phase_accept(const LmCall& c, const mkb_device_batch* templates, int32_t runs,
                 const double* extra_merit, cudaStream_t stream) {
    int rc = phase_trial(c, templates, runs, extra_merit, nullptr, stream);
    if (rc != MKB_OK) return rc;
    return phase_decide(c, runs, nullptr, stream);
}

}  // namespace
}  // namespace mkb

using namespace mkb;

extern "C" {

size_t mkb_lm_workspace_bytes(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                              const mkb_variables* vars, const mkb_lm_options* options,
                              int32_t runs) {
    LmSetup s;
    if (lm_setup(templates, plan, vars, options, runs, s) != MKB_OK) return 0;
    return lm_layout(nullptr, s, runs, templates, plan).total;
}

int mkb_lm_start_ex_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                           const mkb_variables* vars, const mkb_lm_options* options,
                           const double* x0, const double* extra_merit,
                           const double* trace_merit, int32_t runs, void* workspace,
                           size_t workspace_bytes, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    LmCall c;
    std::vector<VarParams> table;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c, &table);
    if (rc != MKB_OK) return rc;
    const LmSetup& s = c.s;
    const LmLayout& L = c.L;
    if (x0 == nullptr) {
        set_error("lm: x0 is null");
        return MKB_ERR_ARGUMENT;
    }
    if (L.vt != nullptr) {  // pageable source: the copy has consumed it when the call returns
        rc = cuda_status(cudaMemcpyAsync(L.vt, table.data(), sizeof(VarParams) * table.size(),
                                         cudaMemcpyHostToDevice, stream),
                         "lm: upload variables");
        if (rc != MKB_OK) return rc;
    }
    if (L.order != nullptr) {  // surface counts of the runs' records, then their order
        const RecordLayout lay = layout_of(s.tp);
        rc = launch_apply(s.vp, lay, templates->records, templates->variants, x0, L.records, runs,
                          stream, run_vars(s, L, templates));
        if (rc != MKB_OK) return rc;
        order_kernel<<<1, 1024, 0, stream>>>(L.vsurf, L.vt, s.vp.P, runs, s.tp.S, L.order,
                                             L.split);
        count_launch();
        rc = cuda_status(cudaGetLastError(), "lm order launch");
        if (rc != MKB_OK) return rc;
    }
    if (s.px.E > 0) {
        if (extra_merit != nullptr) {
            set_error("lm: device paraxial constraints and host extra rows cannot be combined");
            return MKB_ERR_UNSUPPORTED;
        }
        rc = launch_paraxial_merit(s.px, s.vp, L.vt, s.pmax, templates, x0, runs, nullptr,
                                   L.px_merit, stream);
        if (rc != MKB_OK) return rc;
        extra_merit = L.px_merit;
    }
    rc = lm_merit_at(s, L, templates, x0, runs, L.st.merit, L.st.failed, L.st.hard, stream,
                     nullptr, extra_merit);
    if (rc != MKB_OK) return rc;
    rc = cuda_status(cudaMemsetAsync(L.st.running, 0, sizeof(int), stream), "lm: clear count");
    if (rc != MKB_OK) return rc;
    return launch_lm_init(s.o, L.st, s.pmax, x0, runs, stream, trace_merit);
}

int mkb_lm_start_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                        const mkb_variables* vars, const mkb_lm_options* options,
                        const double* x0, int32_t runs, void* workspace, size_t workspace_bytes,
                        void* stream_ptr) {
    return mkb_lm_start_ex_device(templates, plan, vars, options, x0, nullptr, nullptr, runs,
                                  workspace, workspace_bytes, stream_ptr);
}

int mkb_lm_cycle_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                        const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
                        void* workspace, size_t workspace_bytes, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    rc = phase_jacobian(c, templates, plan, vars, runs, stream);
    if (rc != MKB_OK) return rc;
    rc = launch_lm_update(c.s.vp, c.s.o, c.L.st, c.L.gram, runs, stream);  // 2. step
    if (rc != MKB_OK) return rc;
    return phase_accept(c, templates, runs, nullptr, stream);
}

int mkb_paraxial_rows_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const mkb_lm_options* options,
                             const double* x, int32_t runs, double* je, double* re,
                             void* stream_ptr) {
    LmSetup s;
    int rc = lm_setup(templates, plan, vars, options, runs, s);
    if (rc != MKB_OK) return rc;
    if (s.per_run) {
        set_error("paraxial rows: one variable set for all runs (the LM takes per-run sets)");
        return MKB_ERR_UNSUPPORTED;
    }
    if (s.px.E == 0) return MKB_OK;
    if (x == nullptr || je == nullptr || re == nullptr) {
        set_error("paraxial rows: null x, je or re");
        return MKB_ERR_ARGUMENT;
    }
    return launch_paraxial_rows(s.px, s.vp, nullptr, s.pmax, templates, x, runs, nullptr, je, re,
                                static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_cycle_jacobian_device(const mkb_device_batch* templates,
                                 const mkb_residual_plan* plan, const mkb_variables* vars,
                                 const mkb_lm_options* options, int32_t runs, void* workspace,
                                 size_t workspace_bytes, void* stream_ptr) {
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    return phase_jacobian(c, templates, plan, vars, runs, static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_extra_rows_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const mkb_lm_options* options,
                             int32_t runs, void* workspace, size_t workspace_bytes,
                             const double* jacobian, const double* residuals, int32_t rows,
                             void* stream_ptr) {
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    if (rows < 0 || (rows > 0 && (jacobian == nullptr || residuals == nullptr))) {
        set_error("lm extra rows: %d rows, jacobian and residuals needed", rows);
        return MKB_ERR_ARGUMENT;
    }
    return launch_gram_extend(c.s.vp, c.L.st, c.L.gram, jacobian, residuals, rows, runs,
                              static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_cycle_step_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                             const mkb_variables* vars, const mkb_lm_options* options,
                             int32_t runs, void* workspace, size_t workspace_bytes,
                             void* stream_ptr) {
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    return launch_lm_update(c.s.vp, c.s.o, c.L.st, c.L.gram, runs,
                            static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_cycle_accept_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                               const mkb_variables* vars, const mkb_lm_options* options,
                               int32_t runs, void* workspace, size_t workspace_bytes,
                               const double* extra_merit, void* stream_ptr) {
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    return phase_accept(c, templates, runs, extra_merit, static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_cycle_trial_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                              const mkb_variables* vars, const mkb_lm_options* options,
                              int32_t runs, void* workspace, size_t workspace_bytes,
                              const double* extra_merit, double* extrema, void* stream_ptr) {
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    return phase_trial(c, templates, runs, extra_merit, extrema,
                       static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_cycle_decide_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                               const mkb_variables* vars, const mkb_lm_options* options,
                               int32_t runs, void* workspace, size_t workspace_bytes,
                               const double* trace_merit, void* stream_ptr) {
    LmCall c;
    int rc = lm_call(templates, plan, vars, options, runs, workspace, workspace_bytes, c);
    if (rc != MKB_OK) return rc;
    return phase_decide(c, runs, trace_merit, static_cast<cudaStream_t>(stream_ptr));
}

int mkb_lm_points_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                         const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
                         const void* workspace, int32_t* want_jacobian, double* x,
                         int32_t* evaluate, double* trial, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    LmSetup s;
    int rc = lm_setup(templates, plan, vars, options, runs, s);
    if (rc != MKB_OK) return rc;
    const LmLayout L = lm_layout(static_cast<char*>(const_cast<void*>(workspace)), s, runs,
                                 templates, plan);
    const size_t r = static_cast<size_t>(runs);
    struct Copy {
        void* dst;
        const void* src;
        size_t bytes;
    } copies[] = {
        {want_jacobian, L.st.want_jacobian, 4 * r},
        {x, L.st.x, 8 * r * s.pmax},
        {evaluate, L.st.evaluate, 4 * r},
        {trial, L.st.trial, 8 * r * s.pmax},
    };
    for (const Copy& cp : copies) {
        if (cp.dst == nullptr) continue;
        rc = cuda_status(cudaMemcpyAsync(cp.dst, cp.src, cp.bytes, cudaMemcpyDefault, stream),
                         "lm points copy");
        if (rc != MKB_OK) return rc;
    }
    return MKB_OK;
}

int mkb_lm_results_device(const mkb_device_batch* templates, const mkb_residual_plan* plan,
                          const mkb_variables* vars, const mkb_lm_options* options, int32_t runs,
                          const void* workspace, double* x, double* merit, int32_t* status,
                          int32_t* iterations, int32_t* accepted, int32_t* jacobians,
                          double* damping, double* history, int64_t* failed,
                          int64_t* hard_failed, int32_t* running, void* stream_ptr) {
    const cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    LmSetup s;
    int rc = lm_setup(templates, plan, vars, options, runs, s);
    if (rc != MKB_OK) return rc;
    const LmLayout L = lm_layout(static_cast<char*>(const_cast<void*>(workspace)), s, runs,
                                 templates, plan);
    const size_t r = static_cast<size_t>(runs);
    struct Copy {
        void* dst;
        const void* src;
        size_t bytes;
    } copies[] = {
        {x, L.st.x, 8 * r * s.pmax},
        {merit, L.st.merit, 8 * r},
        {status, L.st.status, 4 * r},
        {iterations, L.st.iterations, 4 * r},
        {accepted, L.st.accepted, 4 * r},
        {jacobians, L.st.jacobians, 4 * r},
        {damping, L.st.mu, 8 * r},
        {history, L.st.history, 8 * r * (s.o.max_iterations + 1)},
        {failed, L.st.failed, 8 * r},
        {hard_failed, L.st.hard, 8 * r},
        {running, L.st.running, 4},
    };
    for (const Copy& c : copies) {
        if (c.dst == nullptr) continue;
        rc = cuda_status(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDefault, stream),
                         "lm results copy");
        if (rc != MKB_OK) return rc;
    }
    return MKB_OK;
}

}  // extern "C"
