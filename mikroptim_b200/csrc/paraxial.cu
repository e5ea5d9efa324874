// Paraxial constraints (focal length, parfocal length, working distance, paraxial focus,
// Petzval curvature) as extra rows of the LM on the device, for sm_100a.
//
// Every residual comes from the y-nu trace of the marginal ray at the paraxial index of each
// medium (paraxial_trace / petzval_sum, include/mikroptim/paraxial/ynu_trace.hpp:56,84;
// compute_paraxial, src/paraxial/paraxial.cpp:98; paraxial_deviation / paraxial_residual,
// src/optim/paraxial_residuals.cpp:254,338), in Exact64 in the reference's order of operations.
// The rows' Jacobian is either
//   * MKB_PARAXIAL_FD: central differences with the FD Jacobian's pattern at every variable,
//     the 2P + 1 points of a run traced by the threads of its CTA (extra_rows_untraced,
//     src/optim/adjoint_jacobian.cpp:270), bit for bit the reference's extra rows; or
//   * MKB_PARAXIAL_ADJOINT: the analytic derivatives, from one reverse sweep of the marginal
//     ray per run (seeds dA and dC) and the closed-form derivatives of the Petzval sum.
// Ghost plates enter as thin elements in the medium of their gap (batch_paraxial,
// src/batch/system_batch.cpp:965): power phi_G = -2 (n_G - n_m) t2 added to the surface's power
// and phi_G / (n_m n_G) added to the Petzval sum, t2 from the plate's Legendre coefficients.
// Kernels: paraxial_rows_kernel (rows and Jacobian of the runs a mask selects) and
// paraxial_merit_kernel (sum r_e^2 at the points a mask selects, added to the MERIT).
#include "fd.cuh"
#include "launch.cuh"
#include "paraxial.cuh"

#include <cmath>
#include <cstring>

namespace mkb {

namespace {

constexpr int kRowThreads = 128;

// The y-nu quantities a residual reads, from the arrays of one point.
struct Paraxial {
    double A, C, power, kappa;
};

// The ghost plates of one point: the template's plate data with the run's GhostCoefficient
// variables at x applied; variable `pk` (or -1) takes the value `pv` instead of x[pk].
struct Plates {
    const ParaxialSpec* sp;
    const VarParams* v;
    const double* tmpl;
    const double* x;
    RecordLayout lay;
    int L, pk;
    double pv;

    __device__ double coefficient(int g, int j) const {
        const int col = v->col_ghost[g][j];
        if (col < 0) return tmpl[lay.ghost_coeff + g * sp->K + j];
        return col == pk ? pv : x[col];
    }
    // ghost_profile_t2 (include/mikroptim/trace/ghost_plate.hpp:95)
    __device__ double t2(int g) const {
        double sum = 0.0;
        for (int k = 1; k <= sp->K; ++k) {
            const double term = __dmul_rn(coefficient(g, k - 1), static_cast<double>(k * (k + 1)));
            sum = __dadd_rn(sum, (k & 1) ? term : -term);
        }
        const double r = tmpl[lay.ghost_radius + g];
        return __ddiv_rn(sum, __dmul_rn(r, r));
    }
    __device__ double glass(int g) const { return tmpl[lay.ghost_index + g * L + sp->column]; }
    // ghost_plate_power / ghost_plate_petzval (ghost_plate.hpp:107,114) of surface s in the
    // medium n_m; 0 and 0 on a surface without a plate
    __device__ void at(int s, double n_m, double& power, double& petzval) const {
        power = petzval = 0.0;
        const int g = sp->ghost_of[s];
        if (g < 0) return;
        const double n_g = glass(g);
        power = __dmul_rn(__dmul_rn(-2.0, __dsub_rn(n_g, n_m)), t2(g));
        petzval = __ddiv_rn(power, __dmul_rn(n_m, n_g));
    }
};

__device__ inline Paraxial ynu(const double* c, const double* t, const double* n, int S,
                               const Plates& pl) {
    using N = Exact64;
    N y(1.0), u(0.0), nb(1.0);
    for (int s = 0; s < S; ++s) {
        if (s > 0) y = y + N(t[s - 1]) * u;
        N phi = N(c[s]) * (N(n[s]) - nb);
        double pw, pz;
        pl.at(s, n[s], pw, pz);
        phi = phi + N(pw);  // the plates' extra power (0 elsewhere), added as the reference adds
        u = (nb * u - y * phi) / N(n[s]);
        nb = n[s];
    }
    N p(0.0);
    nb = N(1.0);
    for (int s = 0; s < S; ++s) {
        p = p + (N(c[s]) * (N(n[s]) - nb)) / (nb * N(n[s]));
        double pw, pz;
        pl.at(s, n[s], pw, pz);
        p = p + N(pz);
        nb = n[s];
    }
    Paraxial out;
    out.A = y.v;
    out.C = (N(n[S - 1]) * u).v;
    out.power = out.C == 0.0 ? 0.0 : -out.C;
    out.kappa = (-N(n[S - 1]) * p).v;
    return out;
}

// deviation q of constraint e with its shift (paraxial_deviation, paraxial_residual)
__device__ inline double deviation(const ParaxialSpec& sp, int e, const Paraxial& px,
                                   const double* t, const double* n, int S, double a) {
    using N = Exact64;
    double q = 0.0;
    switch (sp.type[e]) {
    case MKB_CONSTRAINT_FOCAL_LENGTH:
        q = (N(sp.target[e]) * (N(1.0) - N(sp.target[e]) * N(px.power))).v;
        break;
    case MKB_CONSTRAINT_WORKING_DISTANCE:
        q = (N(t[S - 1]) - N(sp.target[e])).v;
        break;
    case MKB_CONSTRAINT_PARFOCAL_LENGTH: {
        N length(sp.offset[e]);
        for (int s = sp.ref_surface[e]; s < S; ++s) length += N(t[s]);
        q = (length - N(sp.target[e])).v;
        break;
    }
    case MKB_CONSTRAINT_PARAXIAL_FOCUS:
        q = (N(a) * (N(px.A) + N(t[S - 1]) * N(px.C) / N(n[S - 1]))).v;
        break;
    default:  // MKB_CONSTRAINT_PETZVAL
        q = (N(fabs(px.kappa)) - N(sp.target[e])).v;
        break;
    }
    if (sp.shift[e] != 0.0) {
        if (sp.mode[e] == MKB_MODE_MAX) q = __dadd_rn(q, sp.shift[e]);
        else if (sp.mode[e] == MKB_MODE_MIN) q = __dsub_rn(q, sp.shift[e]);
    }
    return q;
}

// apply_mode: equal q, min std::min(q, 0), max std::max(q, 0)
__device__ inline double mode_of(int mode, double q) {
    if (mode == MKB_MODE_MIN) return (0.0 < q) ? 0.0 : q;
    if (mode == MKB_MODE_MAX) return (q < 0.0) ? 0.0 : q;
    return q;
}

__device__ inline void residuals_at(const ParaxialSpec& sp, const double* c, const double* t,
                                    const double* n, int S, const Plates& pl, double a,
                                    double* r) {
    const Paraxial px = ynu(c, t, n, S, pl);
    for (int e = 0; e < sp.E; ++e)
        r[e] = __dmul_rn(sp.root_w[e], mode_of(sp.mode[e], deviation(sp, e, px, t, n, S, a)));
}

// The arrays of run `run` at the point x (its template with every variable applied, the
// paraxial index of a glass medium refreshed from its Buchdahl coefficients at the reference
// wavelength): c, t, n [S], Buchdahl coefficients bu [S][4] of the glass media; returns S.
__device__ inline int build_point(const ParaxialSpec& sp, const VarParams& v,
                                  const RecordLayout& lay, const double* tmpl, int S, int L,
                                  const double* x, double* c, double* t, double* n, double* bu) {
    for (int s = 0; s < S; ++s) {
        c[s] = tmpl[lay.curvature + s];
        t[s] = tmpl[lay.thickness + s];
        n[s] = tmpl[lay.index + s * L + sp.column];
        if (lay.glass >= 0)
            for (int j = 0; j < 4; ++j) bu[4 * s + j] = tmpl[lay.glass + s * 4 + j];
    }
    for (int k = 0; k < v.P; ++k) {
        const int s = v.surface[k];
        if (v.type[k] == MKB_VAR_CURVATURE) c[s] = x[k];
        else if (v.type[k] == MKB_VAR_GLASS) bu[4 * s + v.glass_component[k]] = x[k];
        else if (v.type[k] != MKB_VAR_GHOST_COEFFICIENT) t[s] = x[k];
    }
    if (v.has_glass)
        for (int s = 0; s < S; ++s)
            if (v.col_glass[s][0] >= 0 || v.col_glass[s][1] >= 0 || v.col_glass[s][2] >= 0)
                n[s] = buchdahl(bu + 4 * s, sp.omega_ref);
    return S;
}

// One CTA per run (mask[run] != 0, or every run without a mask): rows re[run][E] and columns
// je[run][k][E] at x[run].
__global__ void __launch_bounds__(kRowThreads)
paraxial_rows_kernel(const __grid_constant__ ParaxialSpec sp, const __grid_constant__ VarParams vp,
                     const VarParams* vt, int pstride, RecordLayout lay, int L,
                     const double* __restrict__ templates, int n_templates, int stride,
                     const uint8_t* __restrict__ tsurf, int S_table, const double* __restrict__ x,
                     const int* __restrict__ mask, double* __restrict__ je,
                     double* __restrict__ re) {
    const int run = blockIdx.x;
    if (mask != nullptr && mask[run] == 0) return;
    const VarParams& v = vt != nullptr ? vt[run] : vp;
    const int tmpl_i = n_templates == 1 ? 0 : run;
    const double* tmpl = templates + static_cast<int64_t>(tmpl_i) * stride;
    int S = tsurf != nullptr ? tsurf[tmpl_i] : S_table;
    S = S < 2 ? 2 : (S > S_table ? S_table : S);
    const double* xr = x + static_cast<int64_t>(run) * pstride;
    __shared__ double c0[kMaxSurfaces], t0[kMaxSurfaces], n0[kMaxSurfaces];
    __shared__ double bu0[4 * kMaxSurfaces];
    __shared__ double rs[(2 * MKB_MAX_VARIABLES + 1) * MKB_MAX_PARAXIAL];
    __shared__ FdPattern pat[MKB_MAX_VARIABLES];
    if (threadIdx.x == 0) build_point(sp, v, lay, tmpl, S, L, xr, c0, t0, n0, bu0);
    for (int k = threadIdx.x; k < v.P; k += kRowThreads)
        pat[k] = fd_pattern_of<Exact64>(xr[k], v.lower[k], v.upper[k], v.typical[k]);
    __syncthreads();
    const double a = tmpl[lay.pupil];
    const int E = sp.E;
    double* rrow = re + static_cast<int64_t>(run) * E;
    double* jcol = je + static_cast<int64_t>(run) * pstride * E;
    if (!sp.analytic) {
        // point j: x (j = 0), x with x_k = x_a (j = 2k + 1) or x_b (j = 2k + 2)
        for (int j = threadIdx.x; j < 2 * v.P + 1; j += kRowThreads) {
            double c[kMaxSurfaces], t[kMaxSurfaces], n[kMaxSurfaces];
            for (int s = 0; s < S; ++s) {
                c[s] = c0[s];
                t[s] = t0[s];
                n[s] = n0[s];
            }
            Plates pl{&sp, &v, tmpl, xr, lay, L, -1, 0.0};
            if (j > 0) {
                const int k = (j - 1) / 2;
                const double val = (j & 1) ? pat[k].xa : pat[k].xb;
                const int s = v.surface[k];
                if (v.type[k] == MKB_VAR_CURVATURE) {
                    c[s] = val;
                } else if (v.type[k] == MKB_VAR_GLASS) {
                    double b[4] = {bu0[4 * s], bu0[4 * s + 1], bu0[4 * s + 2], bu0[4 * s + 3]};
                    b[v.glass_component[k]] = val;
                    n[s] = buchdahl(b, sp.omega_ref);
                } else if (v.type[k] == MKB_VAR_GHOST_COEFFICIENT) {
                    pl.pk = k;
                    pl.pv = val;
                } else {
                    t[s] = val;
                }
            }
            residuals_at(sp, c, t, n, S, pl, a, rs + j * E);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < v.P * E; i += kRowThreads) {
            const int k = i / E, e = i - k * E;
            jcol[k * E + e] = fd_derivative_of<Exact64>(pat[k].stencil, rs[e],
                                                        rs[(2 * k + 1) * E + e],
                                                        rs[(2 * k + 2) * E + e], pat[k].da,
                                                        pat[k].db);
        }
        for (int e = threadIdx.x; e < E; e += kRowThreads) rrow[e] = rs[e];
        return;
    }
    // ---- analytic: thread 0 per run (S <= 64 steps, a handful of rows) ------------------
    if (threadIdx.x != 0) return;
    const Plates pl{&sp, &v, tmpl, xr, lay, L, -1, 0.0};
    double y[kMaxSurfaces], u[kMaxSurfaces];  // marginal height at s, angle after s
    double pw[kMaxSurfaces];                  // the plates' extra power (0 elsewhere)
    {
        double yy = 1.0, uu = 0.0, nb = 1.0;
        for (int s = 0; s < S; ++s) {
            double pz;
            pl.at(s, n0[s], pw[s], pz);
            if (s > 0) yy = yy + t0[s - 1] * uu;
            const double phi = c0[s] * (n0[s] - nb) + pw[s];
            uu = (nb * uu - yy * phi) / n0[s];
            y[s] = yy;
            u[s] = uu;
            nb = n0[s];
        }
    }
    const Paraxial px = ynu(c0, t0, n0, S, pl);
    // gradients of A = y_{S-1} and C = n_{S-1} u_{S-1} with respect to c_s, t_s, n_s by one
    // reverse sweep carrying both seeds; gradient of the Petzval sum in closed form
    double gA_c[kMaxSurfaces], gA_t[kMaxSurfaces], gA_n[kMaxSurfaces], gA_p[kMaxSurfaces];
    double gC_c[kMaxSurfaces], gC_t[kMaxSurfaces], gC_n[kMaxSurfaces], gC_p[kMaxSurfaces];
    for (int s = 0; s < S; ++s)
        gA_c[s] = gA_t[s] = gA_n[s] = gA_p[s] = gC_c[s] = gC_t[s] = gC_n[s] = gC_p[s] = 0.0;
    {
        double ay[2] = {1.0, 0.0};           // adjoint of y_s (seed A, seed C)
        double au[2] = {0.0, n0[S - 1]};     // adjoint of u_s
        gC_n[S - 1] += u[S - 1];
        for (int s = S - 1; s >= 0; --s) {
            const double nb = s > 0 ? n0[s - 1] : 1.0;
            const double u_in = s > 0 ? u[s - 1] : 0.0;
            const double phi = c0[s] * (n0[s] - nb) + pw[s];
            double* gc[2] = {gA_c, gC_c};
            double* gt[2] = {gA_t, gC_t};
            double* gn[2] = {gA_n, gC_n};
            double* gp[2] = {gA_p, gC_p};
            for (int q = 0; q < 2; ++q) {
                // u_s = (nb u_in - y_s phi) / n_s
                const double w = au[q] / n0[s];
                double a_uin = w * nb;
                ay[q] += -w * phi;
                const double a_phi = -w * y[s];
                gn[q][s] += -w * u[s];  // d/dn_s of 1/n_s
                double a_nb = w * u_in;
                // phi = c_s (n_s - nb) + the plate's power
                gp[q][s] += a_phi;
                gc[q][s] += a_phi * (n0[s] - nb);
                gn[q][s] += a_phi * c0[s];
                a_nb += -a_phi * c0[s];
                if (s > 0) {
                    gn[q][s - 1] += a_nb;
                    // y_s = y_{s-1} + t_{s-1} u_{s-1}
                    gt[q][s - 1] += ay[q] * u[s - 1];
                    a_uin += ay[q] * t0[s - 1];
                }
                au[q] = a_uin;  // adjoint of u_{s-1}
                // ay[q] stays: adjoint of y_{s-1} (dy_s/dy_{s-1} = 1)
            }
        }
    }
    // dP/dc_s = 1/nb - 1/n_s; dP/dn_s = c_s / n_s^2 - c_{s+1} / n_s^2; a plate on surface s
    // adds through its medium n_m = n_s: d(phi_G)/dn_m = 2 t2 and
    // d(phi_G / (n_m n_G))/dn_m = 2 t2 / (n_m n_G) - phi_G / (n_m^2 n_G)
    double gP_c[kMaxSurfaces], gP_n[kMaxSurfaces];
    {
        double nb = 1.0;
        for (int s = 0; s < S; ++s) {
            gP_c[s] = 1.0 / nb - 1.0 / n0[s];
            gP_n[s] = c0[s] / (n0[s] * n0[s]) - (s + 1 < S ? c0[s + 1] / (n0[s] * n0[s]) : 0.0);
            const int g = sp.ghost_of[s];
            if (g >= 0) {
                const double ng = pl.glass(g), dpw = 2.0 * pl.t2(g);
                gA_n[s] += gA_p[s] * dpw;
                gC_n[s] += gC_p[s] * dpw;
                gP_n[s] += dpw / (n0[s] * ng) - pw[s] / (n0[s] * n0[s] * ng);
            }
            nb = n0[s];
        }
    }
    const double nL = n0[S - 1], tL = t0[S - 1];
    const double petz = px.kappa / -nL;  // P
    for (int e = 0; e < E; ++e) {
        const double q = deviation(sp, e, px, t0, n0, S, a);
        rrow[e] = __dmul_rn(sp.root_w[e], mode_of(sp.mode[e], q));
        const int md = sp.mode[e];
        const bool active = md == MKB_MODE_EQUAL || (md == MKB_MODE_MIN && !(0.0 < q)) ||
                            (md == MKB_MODE_MAX && !(q < 0.0));
        for (int k = 0; k < v.P; ++k) {
            const int s = v.surface[k];
            // dq/d(theta) for the parameter of variable k: c_s, t_s, or n_s (glass, times the
            // Buchdahl slope of its component at the reference wavelength)
            int kind = 0;  // 0 curvature, 1 thickness, 2 index, 3 none
            double slope = 1.0;
            if (v.type[k] == MKB_VAR_CURVATURE) kind = 0;
            else if (v.type[k] == MKB_VAR_GLASS) {
                kind = 2;
                const int comp = v.glass_component[k];
                slope = comp == 0 ? 1.0 : comp == 1 ? sp.omega_ref : sp.omega_ref * sp.omega_ref;
            } else if (v.type[k] == MKB_VAR_GHOST_COEFFICIENT) kind = 3;
            else kind = 1;
            double dA = 0.0, dC = 0.0, dP = 0.0, dt_last = 0.0, dn_last = 0.0, dt_sum = 0.0;
            if (kind == 0) {
                dA = gA_c[s];
                dC = gC_c[s];
                dP = gP_c[s];
            } else if (kind == 1) {
                dA = gA_t[s];
                dC = gC_t[s];
                dt_last = s == S - 1 ? 1.0 : 0.0;
                dt_sum = 1.0;
            } else if (kind == 2) {
                dA = gA_n[s] * slope;
                dC = gC_n[s] * slope;
                dP = gP_n[s] * slope;
                dn_last = s == S - 1 ? slope : 0.0;
            } else {
                // coefficient a_o of plate g: dt2/da_o = (-1)^{o+1} o (o + 1) / r^2
                const int g = v.ghost_plate[k], o = v.ghost_order[k];
                const int sg = sp.ghost_surface[g];
                if (sg < S) {
                    const double r = tmpl[lay.ghost_radius + g], ng = pl.glass(g);
                    const double dt2 = ((o & 1) ? 1.0 : -1.0) * o * (o + 1) / (r * r);
                    const double dpw = -2.0 * (ng - n0[sg]) * dt2;
                    dA = gA_p[sg] * dpw;
                    dC = gC_p[sg] * dpw;
                    dP = dpw / (n0[sg] * ng);
                }
            }
            double dq = 0.0;
            switch (sp.type[e]) {
            case MKB_CONSTRAINT_FOCAL_LENGTH:  // q = f (1 - f phi), phi = -C
                dq = sp.target[e] * sp.target[e] * dC;
                break;
            case MKB_CONSTRAINT_WORKING_DISTANCE:
                dq = dt_last;
                break;
            case MKB_CONSTRAINT_PARFOCAL_LENGTH:
                dq = (kind == 1 && s >= sp.ref_surface[e]) ? dt_sum : 0.0;
                break;
            case MKB_CONSTRAINT_PARAXIAL_FOCUS:  // q = a (A + t_L C / n_L)
                dq = a * (dA + (tL * dC + px.C * dt_last) / nL - tL * px.C * dn_last / (nL * nL));
                break;
            default: {  // |kappa| - max, kappa = -n_L P
                const double dk = -(petz * dn_last + nL * dP);
                dq = px.kappa >= 0.0 ? dk : -dk;
                break;
            }
            }
            jcol[k * E + e] = active ? sp.root_w[e] * dq : 0.0;
        }
    }
}

// sum_e r_e^2 (in ascending e) at the points x[run] of the runs mask selects; 0 elsewhere is
// left untouched.
__global__ void paraxial_merit_kernel(const __grid_constant__ ParaxialSpec sp,
                                      const __grid_constant__ VarParams vp, const VarParams* vt,
                                      int pstride, RecordLayout lay, int L,
                                      const double* __restrict__ templates, int n_templates,
                                      int stride, const uint8_t* __restrict__ tsurf, int S_table,
                                      const double* __restrict__ x, int runs,
                                      const int* __restrict__ mask, double* __restrict__ out) {
    const int run = blockIdx.x * blockDim.x + threadIdx.x;
    if (run >= runs || (mask != nullptr && mask[run] == 0)) return;
    const VarParams& v = vt != nullptr ? vt[run] : vp;
    const int tmpl_i = n_templates == 1 ? 0 : run;
    const double* tmpl = templates + static_cast<int64_t>(tmpl_i) * stride;
    int S = tsurf != nullptr ? tsurf[tmpl_i] : S_table;
    S = S < 2 ? 2 : (S > S_table ? S_table : S);
    double c[kMaxSurfaces], t[kMaxSurfaces], n[kMaxSurfaces], bu[4 * kMaxSurfaces];
    const double* xr = x + static_cast<int64_t>(run) * pstride;
    build_point(sp, v, lay, tmpl, S, L, xr, c, t, n, bu);
    double r[MKB_MAX_PARAXIAL];
    residuals_at(sp, c, t, n, S, Plates{&sp, &v, tmpl, xr, lay, L, -1, 0.0}, tmpl[lay.pupil], r);
    double sum = 0.0;
    for (int e = 0; e < sp.E; ++e) sum = __dadd_rn(sum, __dmul_rn(r[e], r[e]));
    out[run] = sum;
}

}  // namespace

int make_paraxial_spec(const mkb_lm_options* o, const mkb_device_batch* b,
                       const mkb_residual_plan* plan, ParaxialSpec* sp) {
    std::memset(sp, 0, sizeof(*sp));
    if (o == nullptr || o->paraxial_count == 0) return MKB_OK;
    const int E = o->paraxial_count;
    if (E < 0 || E > MKB_MAX_PARAXIAL || o->paraxial == nullptr) {
        set_error("paraxial constraints: count must be in [0, %d] with an array",
                  MKB_MAX_PARAXIAL);
        return MKB_ERR_ARGUMENT;
    }
    if (b->non_coaxial) {
        set_error("paraxial constraints on the device: coaxial batches");
        return MKB_ERR_UNSUPPORTED;
    }
    if (b->ghost_plates < 0 || b->ghost_plates > kMaxGhostPlates || b->ghost_terms < 0 ||
        b->ghost_terms > kMaxGhostTerms || b->surfaces > kMaxSurfaces) {
        set_error("paraxial constraints: ghost plates (G=%d, K=%d) or %d surfaces out of range",
                  b->ghost_plates, b->ghost_terms, b->surfaces);
        return MKB_ERR_ARGUMENT;
    }
    if (o->paraxial_column < 0 || o->paraxial_column >= b->wavelengths) {
        set_error("paraxial constraints: column %d outside [0, %d)", o->paraxial_column,
                  b->wavelengths);
        return MKB_ERR_ARGUMENT;
    }
    if (o->paraxial_derivative != MKB_PARAXIAL_FD && o->paraxial_derivative != MKB_PARAXIAL_ADJOINT) {
        set_error("paraxial constraints: unknown derivative %d", o->paraxial_derivative);
        return MKB_ERR_ARGUMENT;
    }
    sp->E = E;
    sp->column = o->paraxial_column;
    // the plates in table order (the surface table's ghost_of)
    sp->G = b->ghost_plates;
    sp->K = b->ghost_terms;
    for (int s = 0; s < kMaxSurfaces; ++s) sp->ghost_of[s] = -1;
    for (int g = 0; g < kMaxGhostPlates; ++g) sp->ghost_surface[g] = kMaxSurfaces;
    for (int s = 1, g = 0; s < b->surfaces; ++s)
        if (b->type[s] == MKB_SURFACE_GHOST_PLATE && g < sp->G) {
            sp->ghost_of[s] = static_cast<int8_t>(g);
            sp->ghost_surface[g++] = static_cast<int8_t>(s);
        }
    sp->analytic = o->paraxial_derivative == MKB_PARAXIAL_ADJOINT ? 1 : 0;
    // the Buchdahl coordinate of the reference wavelength (buchdahl_omega,
    // glass/dispersion.hpp:87), as make_var_params forms it for the batch's wavelengths
    const double dl = plan->reference_wavelength_nm / 1000.0 - 0.546074;
    const double den = 1.0 + 2.5 * dl;
    sp->omega_ref = den > 0.0 ? dl / den : 0.0;
    // check_paraxial_constraints (src/optim/paraxial_residuals.cpp:157)
    for (int e = 0; e < E; ++e) {
        const mkb_paraxial_constraint& c = o->paraxial[e];
        auto fail = [&](const char* what) {
            set_error("paraxial constraint %d: %s", e, what);
            return MKB_ERR_ARGUMENT;
        };
        if (c.type < MKB_CONSTRAINT_FOCAL_LENGTH || c.type > MKB_CONSTRAINT_PETZVAL)
            return fail("unknown type");
        if (c.mode < MKB_MODE_EQUAL || c.mode > MKB_MODE_MAX) return fail("unknown mode");
        if (!(std::isfinite(c.weight) && c.weight >= 0.0)) return fail("weight must be >= 0");
        if (!std::isfinite(c.target)) return fail("target must be finite");
        if (!(std::isfinite(c.shift) && c.shift >= 0.0)) return fail("shift must be >= 0");
        if (c.mode == MKB_MODE_EQUAL && c.shift != 0.0) return fail("an equation has no shift");
        if (c.type == MKB_CONSTRAINT_FOCAL_LENGTH && (c.target == 0.0 || c.mode != MKB_MODE_EQUAL))
            return fail("focal length: an equation with a target != 0");
        if (c.type == MKB_CONSTRAINT_PARAXIAL_FOCUS && c.mode != MKB_MODE_EQUAL)
            return fail("paraxial focus: an equation");
        if (c.type == MKB_CONSTRAINT_PETZVAL && (c.mode != MKB_MODE_MAX || c.target < 0.0))
            return fail("Petzval: an upper limit >= 0");
        if (c.type == MKB_CONSTRAINT_PARFOCAL_LENGTH &&
            (c.reference_surface < 0 || c.reference_surface >= b->surfaces ||
             !std::isfinite(c.offset)))
            return fail("parfocal length: reference surface outside the table");
        if (c.type == MKB_CONSTRAINT_PARFOCAL_LENGTH &&
            b->type[c.reference_surface] == MKB_SURFACE_GHOST_PLATE)
            return fail("parfocal length: the reference surface is a ghost plate");
        sp->type[e] = c.type;
        sp->mode[e] = c.mode;
        sp->root_w[e] = std::sqrt(c.weight);
        sp->target[e] = c.target;
        sp->offset[e] = c.offset;
        sp->shift[e] = c.shift;
        sp->ref_surface[e] = c.reference_surface;
    }
    return MKB_OK;
}

int launch_paraxial_rows(const ParaxialSpec& sp, const VarParams& vp, const VarParams* vt,
                         int pstride, const mkb_device_batch* templates, const double* x,
                         int runs, const int* mask, double* je, double* re,
                         cudaStream_t stream) {
    const RecordLayout lay = record_layout(templates->surfaces, templates->wavelengths,
                                           templates->fields, templates->non_coaxial,
                                           templates->ghost_plates, templates->ghost_terms,
                                           templates->glass ? 1 : 0);
    paraxial_rows_kernel<<<runs, kRowThreads, 0, stream>>>(
        sp, vp, vt, pstride, lay, templates->wavelengths, templates->records,
        templates->variants, templates->record_stride, templates->variant_surfaces,
        templates->surfaces, x, mask, je, re);
    count_launch();
    return cuda_status(cudaGetLastError(), "paraxial rows launch");
}

int launch_paraxial_merit(const ParaxialSpec& sp, const VarParams& vp, const VarParams* vt,
                          int pstride, const mkb_device_batch* templates, const double* x,
                          int runs, const int* mask, double* out, cudaStream_t stream) {
    const RecordLayout lay = record_layout(templates->surfaces, templates->wavelengths,
                                           templates->fields, templates->non_coaxial,
                                           templates->ghost_plates, templates->ghost_terms,
                                           templates->glass ? 1 : 0);
    paraxial_merit_kernel<<<(runs + 63) / 64, 64, 0, stream>>>(
        sp, vp, vt, pstride, lay, templates->wavelengths, templates->records,
        templates->variants, templates->record_stride, templates->variant_surfaces,
        templates->surfaces, x, runs, mask, out);
    count_launch();
    return cuda_status(cudaGetLastError(), "paraxial merit launch");
}

}  // namespace mkb
