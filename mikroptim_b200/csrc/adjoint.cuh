// Reverse-mode derivative of the surface chain, templated on the number type N (Exact64 for
// the bit-identical path, double for the contracted one). Formulas and order of operations
// follow the reference's reverse sweep:
//   refracting_step_backward   trace/adjoint_backward.hpp:118
//   reference_step_backward    trace/adjoint_backward.hpp:376
//   transfer_backward          trace/adjoint_backward.hpp:91
// Each function takes the state (p, d) that entered the step, the adjoint of the state that
// left it, and returns the adjoint of the entering state plus the adjoints of the step's
// parameters (thickness of the transfer, curvature, indices before and after).
#pragma once

#include "common.cuh"

namespace mkb {

template <class N>
struct Vec {
    N x, y, z;
};

template <class N>
__device__ __forceinline__ Vec<N> vadd(Vec<N> a, Vec<N> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class N>
__device__ __forceinline__ Vec<N> vsub(Vec<N> a, Vec<N> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class N>
__device__ __forceinline__ Vec<N> vscale(N s, Vec<N> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class N>
__device__ __forceinline__ N vdot(Vec<N> a, Vec<N> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class N>
__device__ __forceinline__ N vnorm(Vec<N> a) { return nsqrt(vdot(a, a)); }

template <class N>
struct RayAdj {
    Vec<N> p, d;
};

template <class N>
struct StepAdj {
    N thickness, curvature, n_before, n_after;
};

// Conversion of a forward quantity (type N) to the adjoint arithmetic (type A): the identity
// when N == A, a rounding to float when the reverse sweep runs in FP32 on FP64 states.
template <class A, class N>
__device__ __forceinline__ A cv(N x) { return A(value_of(x)); }
template <class A, class N>
__device__ __forceinline__ Vec<A> cv(Vec<N> v) { return {cv<A>(v.x), cv<A>(v.y), cv<A>(v.z)}; }

// Decentered and tilted surfaces (backward_ray, trace/adjoint_backward.hpp:539-569): the step
// is differentiated in the surface's tilted frame, with the entering state
// R^T (p - t e_z - D), R^T d and a transfer by 0; the adjoints of the leaving state are turned
// in with R^T and those of the entering state back with R, and t-bar = -p-bar_z.
template <class N>
__device__ __forceinline__ void state_to_surface(const Transform<N>& t, Vec<N>& p, Vec<N>& d,
                                                 N thickness) {
    N x = p.x - t.dx, y = p.y - t.dy, z = p.z - thickness;
    rotate_to(t, x, y, z);
    p = {x, y, z};
    rotate_to(t, d.x, d.y, d.z);
}

template <class A>
__device__ __forceinline__ void adjoint_to_surface(const Transform<A>& t, RayAdj<A>& a) {
    rotate_to(t, a.p.x, a.p.y, a.p.z);
    rotate_to(t, a.d.x, a.d.y, a.d.z);
}

template <class A>
__device__ __forceinline__ void adjoint_from_surface(const Transform<A>& t, RayAdj<A>& a) {
    rotate_from(t, a.p.x, a.p.y, a.p.z);
    rotate_from(t, a.d.x, a.d.y, a.d.z);
}

// A divisor of the adjoint arithmetic. FP32 (the mixed sweep): the SFU reciprocal, taken once
// per step and shared by the K seeds, and a multiply -- a few ulp of single precision, inside
// that sweep's rounding budget. FP64: the rounded division in the reference's order, so the
// FP64 sweeps stay bit-identical.
__device__ __forceinline__ float sfu_reciprocal(float x) { return __fdividef(1.0f, x); }

template <class A>
struct Divisor {
    A d;
    __device__ __forceinline__ explicit Divisor(A x) : d(x) {}
    __device__ __forceinline__ A div(A a) const { return a / d; }
};
template <>
struct Divisor<float> {
    float r;
    __device__ __forceinline__ explicit Divisor(float x) : r(sfu_reciprocal(x)) {}
    __device__ __forceinline__ float div(float a) const { return a * r; }
};

// K adjoint vectors through one step (K seeds of the same ray: the OPL and the penalty). The
// step-local forward quantities are recomputed in N, the adjoint arithmetic runs in A (N for
// the FP64 paths; float on FP64 states for the mixed path). The forward recompute and the
// seed-independent reverse quantities are shared; every adjoint vector goes through the
// reference's statements in the reference's order, so for N == A and K = 1 (and for each k)
// the result equals the single-seed sweep bit for bit.
// `known` (optional): the step's StepLocal quantities kept by the forward pass, used instead
// of recomputing the divisions and square roots (the values are the same).
template <class N, class A, int K>
__device__ __forceinline__ void refracting_step_backward_k(Vec<N> p, Vec<N> d, N t, N c,
                                                           N n_before, N n_after, int branch,
                                                           const A (&seed_opl)[K],
                                                           const A (&seed_pen)[K],
                                                           RayAdj<A> (&adj)[K],
                                                           StepAdj<A> (&out)[K],
                                                           const StepLocal<N>* known = nullptr) {
    const N one(1.0), two(2.0);
    // forward recompute of the step's local quantities
    const N z = p.z - t;
    const N s0 = known ? known->s0 : -z / d.z;
    const N x = p.x + s0 * d.x;
    const N y = p.y + s0 * d.y;
    const N rr = x * x + y * y;
    const N H = c * rr;
    const N xd = x * d.x + y * d.y;
    const N B = d.z - c * xd;
    const N D = B * B - c * H;
    const bool missed = (branch & kBranchSoftMissed) != 0;
    const bool tir = (branch & kBranchSoftTir) != 0;
    N root_d(0.0), s;
    if (known) {
        root_d = known->root_d;
        s = known->s;
    } else if (missed) {
        s = B / c;
    } else {
        root_d = nsqrt(D);
        s = H / (B + root_d);
    }
    const Vec<N> q{x + s * d.x, y + s * d.y, s * d.z};
    const Vec<N> n_raw{-c * q.x, -c * q.y, one - c * q.z};
    N inv_norm = one;
    Vec<N> Nv = n_raw;
    if (missed) {
        inv_norm = one / vnorm(n_raw);
        Nv = vscale(inv_norm, n_raw);
    }
    const N mu = known ? known->mu : n_before / n_after;
    const N cos_i = vdot(d, Nv);
    const N sin2 = one - cos_i * cos_i;
    const N k = one - mu * mu * sin2;
    // seed-independent reverse quantities
    Vec<N> d1{N(0.0), N(0.0), N(0.0)};
    N inv_tau(0.0), root_k(0.0), a(0.0), inv(0.0);
    if (tir) {
        const Vec<N> tau = vsub(d, vscale(cos_i, Nv));
        inv_tau = one / vnorm(tau);
        d1 = vscale(inv_tau, tau);
    } else {
        root_k = known ? known->root_k : nsqrt(k);
        a = root_k - mu * cos_i;
    }
    if (!missed) inv = Divisor<N>(two * root_d).div(one);
    // the same quantities in the adjoint arithmetic
    const A zero_a(0.0), two_a(2.0);
    const Vec<A> ad = cv<A>(d), aNv = cv<A>(Nv), aq = cv<A>(q), ad1 = cv<A>(d1);
    const A ac = cv<A>(c), amu = cv<A>(mu), acos = cv<A>(cos_i), asin2 = cv<A>(sin2);
    const A ainv_tau = cv<A>(inv_tau), aroot_k = cv<A>(root_k), aa = cv<A>(a);
    const A ainv_norm = cv<A>(inv_norm), ainv = cv<A>(inv), as = cv<A>(s), as0 = cv<A>(s0);
    const A ann = cv<A>(n_after), anb = cv<A>(n_before), aB = cv<A>(B), aH = cv<A>(H);
    const A arr = cv<A>(rr), ax = cv<A>(x), ay = cv<A>(y), axd = cv<A>(xd);
    const Divisor<A> by_2root_k(two_a * aroot_k), by_n_after(ann), by_c(ac), by_dz(ad.z);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const Vec<A> qb_out = adj[m].p;
        const Vec<A> d1b = adj[m].d;
        RayAdj<A> in{{zero_a, zero_a, zero_a}, {zero_a, zero_a, zero_a}};
        Vec<A> nb{zero_a, zero_a, zero_a};
        A cosb = zero_a, kb = zero_a, mub = zero_a;
        if (tir) {
            const Vec<A> taub = vscale(ainv_tau, vsub(d1b, vscale(vdot(ad1, d1b), ad1)));
            in.d = vadd(in.d, taub);
            cosb += -vdot(taub, aNv);
            nb = vadd(nb, vscale(-acos, taub));
            kb += -seed_pen[m];
        } else {
            in.d = vadd(in.d, vscale(amu, d1b));
            nb = vadd(nb, vscale(aa, d1b));
            const A ab = vdot(d1b, aNv);
            mub += vdot(d1b, ad);
            kb += by_2root_k.div(ab);
            mub += -ab * acos;
            cosb += -ab * amu;
        }
        mub += -kb * two_a * amu * asin2;
        cosb += kb * two_a * amu * amu * acos;
        in.d = vadd(in.d, vscale(cosb, aNv));
        nb = vadd(nb, vscale(cosb, ad));
        out[m].n_before += by_n_after.div(mub);
        out[m].n_after += by_n_after.div(-mub * amu);
        Vec<A> nrb = nb;
        if (missed) nrb = vscale(ainv_norm, vsub(nb, vscale(vdot(aNv, nb), aNv)));
        const Vec<A> qb = vadd(qb_out, vscale(-ac, nrb));
        A cb = -vdot(aq, nrb);
        A xb = qb.x, yb = qb.y;
        A sb = vdot(qb, ad);
        in.d = vadd(in.d, vscale(as, qb));
        sb += seed_opl[m] * anb;
        A s0b = seed_opl[m] * anb;
        out[m].n_before += seed_opl[m] * (as0 + as);
        A hb = zero_a, bb = zero_a;
        if (missed) {
            bb += by_c.div(sb);
            cb += by_c.div(-sb * as);
            const A db = -seed_pen[m];
            bb += db * two_a * aB;
            cb += -db * aH;
            hb += -db * ac;
        } else {
            hb += sb * ainv;
            bb += -sb * as * two_a * ainv;
            cb += sb * as * as * ainv;
        }
        cb += hb * arr;
        xb += hb * two_a * ac * ax;
        yb += hb * two_a * ac * ay;
        in.d.z += bb;
        cb += -bb * axd;
        xb += -bb * ac * ad.x;
        yb += -bb * ac * ad.y;
        in.d.x += -bb * ac * ax;
        in.d.y += -bb * ac * ay;
        // transfer: s0 = (t - p_z) / d_z
        in.p.x += xb;
        in.p.y += yb;
        s0b += xb * ad.x + yb * ad.y;
        in.d.x += xb * as0;
        in.d.y += yb * as0;
        const A qq = by_dz.div(s0b);
        out[m].thickness += qq;
        in.p.z += -qq;
        in.d.z += -qq * as0;
        out[m].curvature += cb;
        adj[m] = in;
    }
}

// K adjoint vectors through a ghost-plate step (ghost_step_backward,
// trace/adjoint_backward.hpp:253): the forward quantities recomputed in N, the adjoint
// arithmetic in A, every statement in the reference's order. The profile's second derivative
// comes from P''_{k+1} = P''_{k-1} + (2k + 1) P'_k. coeff(m, k, value) receives the adjoint of
// a_{k+1} for seed m (k = 0 .. K-1); out[m].curvature is left alone.
template <class N, class A, int K, class CoeffSink>
__device__ __forceinline__ void ghost_step_backward_k(Vec<N> p, Vec<N> d, N t, const GhostData& g,
                                                      N n_before, N n_after, int branch,
                                                      const A (&seed_opl)[K],
                                                      const A (&seed_pen)[K],
                                                      RayAdj<A> (&adj)[K], StepAdj<A> (&out)[K],
                                                      CoeffSink&& coeff) {
    const N one(1.0), two(2.0);
    // ---- forward ----
    const N z = p.z - t;
    const N s0 = -z / d.z;
    const N x = p.x + s0 * d.x;
    const N y = p.y + s0 * d.y;
    const N radius = g.radius;
    const N inv_r2 = Divisor<N>(radius * radius).div(one);
    const N u = (x * x + y * y) * inv_r2;
    const N xi = two * u - one;
    N prof_t(0.0), sum_dp(0.0), sum_ddp(0.0);
    {
        N p_prev = one, p_cur = xi, dp_prev(0.0), dp_cur = one, ddp_prev(0.0), ddp_cur(0.0);
        for (int k = 1; k <= g.K; ++k) {
            const N a = g.coeff[k - 1];
            prof_t += a * p_cur;
            sum_dp += a * dp_cur;
            sum_ddp += a * ddp_cur;
            const N p_next =
                legendre_div<N>(N(double(2 * k + 1)) * xi * p_cur - N(double(k)) * p_prev, k);
            const N dp_next = dp_prev + N(double(2 * k + 1)) * p_cur;
            const N ddp_next = ddp_prev + N(double(2 * k + 1)) * dp_cur;
            p_prev = p_cur;
            p_cur = p_next;
            dp_prev = dp_cur;
            dp_cur = dp_next;
            ddp_prev = ddp_cur;
            ddp_cur = ddp_next;
        }
    }
    const N dt_du = two * sum_dp;
    const N d2t_du2 = N(4.0) * sum_ddp;
    const N dn = N(g.n_glass) - n_before;
    const N radial = dn * dt_du * two * inv_r2;
    N dx, dy;
    if constexpr (kMulByReciprocal<N>) {  // as ghost_step forms them
        const N inv_after = one / n_after;
        dx = (n_before * d.x + radial * x) * inv_after;
        dy = (n_before * d.y + radial * y) * inv_after;
    } else {
        dx = (n_before * d.x + radial * x) / n_after;
        dy = (n_before * d.y + radial * y) / n_after;
    }
    const N radicand = one - dx * dx - dy * dy;
    const bool tir = (branch & kBranchSoftTir) != 0;
    N inv_m(0.0), ex(0.0), ey(0.0), root(0.0);
    if (tir) {
        inv_m = one / nsqrt(dx * dx + dy * dy);
        ex = dx * inv_m;
        ey = dy * inv_m;
    } else {
        root = nsqrt(radicand);
    }
    // ---- reverse, in A ----
    const A zero_a(0.0), two_a(2.0);
    const A adx = cv<A>(dx), ady = cv<A>(dy), ax = cv<A>(x), ay = cv<A>(y);
    const A ainv_m = cv<A>(inv_m), aex = cv<A>(ex), aey = cv<A>(ey), aroot = cv<A>(root);
    const A anb = cv<A>(n_before), ana = cv<A>(n_after), ad_x = cv<A>(d.x), ad_y = cv<A>(d.y);
    const A aradial = cv<A>(radial), as0 = cv<A>(s0), adn = cv<A>(dn), aprof = cv<A>(prof_t);
    const A adtdu = cv<A>(dt_du), ad2t = cv<A>(d2t_du2), ainv_r2 = cv<A>(inv_r2);
    const A axi = cv<A>(xi), ad_z = cv<A>(d.z);
    // the seed-independent divisors (FP32: one SFU reciprocal each, shared by the K seeds)
    const Divisor<A> by_2root(two_a * aroot), by_after(ana), by_dz(ad_z);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const Vec<A> qb = adj[m].p;
        const Vec<A> d1b = adj[m].d;
        RayAdj<A> in{{zero_a, zero_a, zero_a}, {zero_a, zero_a, zero_a}};
        A dxb, dyb, radb;
        if (tir) {
            const A proj = aex * d1b.x + aey * d1b.y;
            dxb = (d1b.x - proj * aex) * ainv_m;
            dyb = (d1b.y - proj * aey) * ainv_m;
            radb = -seed_pen[m];
        } else {
            dxb = d1b.x;
            dyb = d1b.y;
            radb = by_2root.div(d1b.z);
        }
        dxb += -two_a * adx * radb;
        dyb += -two_a * ady * radb;
        in.d.x += by_after.div(dxb * anb);
        in.d.y += by_after.div(dyb * anb);
        out[m].n_before += by_after.div(dxb * ad_x + dyb * ad_y);
        out[m].n_after += by_after.div(-(dxb * adx + dyb * ady));
        const A gxb = by_after.div(dxb);
        const A gyb = by_after.div(dyb);
        const A radialb = gxb * ax + gyb * ay;
        A xb = qb.x + gxb * aradial;
        A yb = qb.y + gyb * aradial;
        A s0b = seed_opl[m] * anb;
        out[m].n_before += seed_opl[m] * as0;
        const A phaseb = seed_opl[m];
        const A dnb = phaseb * aprof + radialb * adtdu * two_a * ainv_r2;
        const A tb = phaseb * adn;
        const A dtdub = radialb * adn * two_a * ainv_r2;
        out[m].n_before += -dnb;
        const A ub = tb * adtdu + dtdub * ad2t;
        {
            A p_prev(1.0), p_cur = axi, dp_prev(0.0), dp_cur(1.0);
            for (int k = 1; k <= g.K; ++k) {
                coeff(m, k - 1, tb * p_cur + dtdub * two_a * dp_cur);
                const A p_next =
                    legendre_div<A>(A(double(2 * k + 1)) * axi * p_cur - A(double(k)) * p_prev, k);
                const A dp_next = dp_prev + A(double(2 * k + 1)) * p_cur;
                p_prev = p_cur;
                p_cur = p_next;
                dp_prev = dp_cur;
                dp_cur = dp_next;
            }
        }
        xb += ub * two_a * ax * ainv_r2;
        yb += ub * two_a * ay * ainv_r2;
        // transfer: s0 = (t - p_z) / d_z (transfer_backward, adjoint_backward.hpp:91)
        in.p.x += xb;
        in.p.y += yb;
        s0b += xb * ad_x + yb * ad_y;
        in.d.x += xb * as0;
        in.d.y += yb * as0;
        const A qq = by_dz.div(s0b);
        out[m].thickness += qq;
        in.p.z += -qq;
        in.d.z += -qq * as0;
        adj[m] = in;
    }
}

template <class N>
__device__ __forceinline__ void refracting_step_backward(Vec<N> p, Vec<N> d, N t, N c, N n_before,
                                                         N n_after, int branch, N seed_opl,
                                                         N seed_pen, RayAdj<N>& adj,
                                                         StepAdj<N>& out) {
    const N so[1] = {seed_opl}, sp[1] = {seed_pen};
    RayAdj<N> a[1] = {adj};
    StepAdj<N> o[1] = {out};
    refracting_step_backward_k<N, N, 1>(p, d, t, c, n_before, n_after, branch, so, sp, a, o);
    adj = a[0];
    out = o[0];
}

// Step onto the reference sphere through the last vertex about M = (0, h, w), K seeds
// (forward quantities in N, adjoint arithmetic in A, as above).
template <class N, class A, int K>
__device__ __forceinline__ void reference_step_backward_k(Vec<N> p, Vec<N> d, Vec<N> center,
                                                          N n_image, int branch,
                                                          const A (&seed_opl)[K],
                                                          const A (&seed_pen)[K],
                                                          RayAdj<A> (&adj)[K],
                                                          Vec<A> (&center_adj)[K],
                                                          A (&n_image_adj)[K]) {
    const N zero(0.0), one(1.0), two(2.0);
    const Vec<N> q = vsub(p, center);
    const N b = -vdot(q, d);
    const N g = vdot(p, vsub(p, vscale(two, center)));
    const N disc = b * b - g;
    const bool missed = (branch & kBranchSoftMissed) != 0;
    const N sigma = center.z >= zero ? one : N(-1.0);
    N s, root = zero;
    if (missed) {
        s = b;
    } else {
        root = nsqrt(disc);
        s = g / (b + sigma * root);
    }
    const N radius_sq = missed ? vdot(center, center) : zero;
    const A zero_a(0.0), two_a(2.0), m2_a(-2.0);
    const Vec<A> ad = cv<A>(d), aq = cv<A>(q), ap = cv<A>(p), acenter = cv<A>(center);
    const A as = cv<A>(s), ab = cv<A>(b), adisc = cv<A>(disc), asigma = cv<A>(sigma);
    const A aroot = cv<A>(root), arsq = cv<A>(radius_sq), an = cv<A>(n_image);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const A sb = seed_opl[m] * an;
        n_image_adj[m] += seed_opl[m] * as;
        A bb, gb;
        if (missed) {
            bb = sb;
            gb = zero_a;
            const A discb = -seed_pen[m] / arsq;
            bb += discb * two_a * ab;
            gb += -discb;
            center_adj[m] = vadd(center_adj[m],
                                 vscale(seed_pen[m] * two_a * adisc / (arsq * arsq), acenter));
        } else {
            gb = sb * asigma / (two_a * aroot);
            bb = -sb * asigma * as / aroot;
        }
        RayAdj<A> in{{zero_a, zero_a, zero_a}, {zero_a, zero_a, zero_a}};
        in.p = vadd(in.p, vscale(-bb, ad));
        in.d = vadd(in.d, vscale(-bb, aq));
        center_adj[m] = vadd(center_adj[m], vscale(bb, ad));
        in.p = vadd(in.p, vscale(two_a * gb, vsub(ap, acenter)));
        center_adj[m] = vadd(center_adj[m], vscale(m2_a * gb, ap));
        adj[m] = in;
    }
}

template <class N>
__device__ __forceinline__ void reference_step_backward(Vec<N> p, Vec<N> d, Vec<N> center,
                                                        N n_image, int branch, N seed_opl,
                                                        N seed_pen, RayAdj<N>& adj,
                                                        Vec<N>& center_adj, N& n_image_adj) {
    const N so[1] = {seed_opl}, sp[1] = {seed_pen};
    RayAdj<N> a[1] = {adj};
    Vec<N> ca[1] = {center_adj};
    N na[1] = {n_image_adj};
    reference_step_backward_k<N, N, 1>(p, d, center, n_image, branch, so, sp, a, ca, na);
    adj = a[0];
    center_adj = ca[0];
    n_image_adj = na[0];
}

}  // namespace mkb
