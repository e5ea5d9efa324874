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

// K adjoint vectors through one step (K seeds of the same ray: the OPL and the penalty). The
// forward recompute and the seed-independent reverse quantities are shared; every adjoint
// vector goes through the reference's statements in the reference's order, so for K = 1 (and
// for each k) the result equals the single-seed sweep bit for bit.
template <class N, int K>
__device__ __forceinline__ void refracting_step_backward_k(Vec<N> p, Vec<N> d, N t, N c,
                                                           N n_before, N n_after, int branch,
                                                           const N (&seed_opl)[K],
                                                           const N (&seed_pen)[K],
                                                           RayAdj<N> (&adj)[K],
                                                           StepAdj<N> (&out)[K]) {
    const N zero(0.0), one(1.0), two(2.0);
    // forward recompute of the step's local quantities
    const N z = p.z - t;
    const N s0 = -z / d.z;
    const N x = p.x + s0 * d.x;
    const N y = p.y + s0 * d.y;
    const N rr = x * x + y * y;
    const N H = c * rr;
    const N xd = x * d.x + y * d.y;
    const N B = d.z - c * xd;
    const N D = B * B - c * H;
    const bool missed = (branch & kBranchSoftMissed) != 0;
    const bool tir = (branch & kBranchSoftTir) != 0;
    N root_d = zero, s;
    if (missed) {
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
    const N mu = n_before / n_after;
    const N cos_i = vdot(d, Nv);
    const N sin2 = one - cos_i * cos_i;
    const N k = one - mu * mu * sin2;
    // seed-independent reverse quantities
    Vec<N> d1{zero, zero, zero};
    N inv_tau = zero, root_k = zero, a = zero, inv = zero;
    if (tir) {
        const Vec<N> tau = vsub(d, vscale(cos_i, Nv));
        inv_tau = one / vnorm(tau);
        d1 = vscale(inv_tau, tau);
    } else {
        root_k = nsqrt(k);
        a = root_k - mu * cos_i;
    }
    if (!missed) inv = one / (two * root_d);
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const Vec<N> qb_out = adj[m].p;
        const Vec<N> d1b = adj[m].d;
        RayAdj<N> in{{zero, zero, zero}, {zero, zero, zero}};
        Vec<N> nb{zero, zero, zero};
        N cosb = zero, kb = zero, mub = zero;
        if (tir) {
            const Vec<N> taub = vscale(inv_tau, vsub(d1b, vscale(vdot(d1, d1b), d1)));
            in.d = vadd(in.d, taub);
            cosb += -vdot(taub, Nv);
            nb = vadd(nb, vscale(-cos_i, taub));
            kb += -seed_pen[m];
        } else {
            in.d = vadd(in.d, vscale(mu, d1b));
            nb = vadd(nb, vscale(a, d1b));
            const N ab = vdot(d1b, Nv);
            mub += vdot(d1b, d);
            kb += ab / (two * root_k);
            mub += -ab * cos_i;
            cosb += -ab * mu;
        }
        mub += -kb * two * mu * sin2;
        cosb += kb * two * mu * mu * cos_i;
        in.d = vadd(in.d, vscale(cosb, Nv));
        nb = vadd(nb, vscale(cosb, d));
        out[m].n_before += mub / n_after;
        out[m].n_after += -mub * mu / n_after;
        Vec<N> nrb = nb;
        if (missed) nrb = vscale(inv_norm, vsub(nb, vscale(vdot(Nv, nb), Nv)));
        const Vec<N> qb = vadd(qb_out, vscale(-c, nrb));
        N cb = -vdot(q, nrb);
        N xb = qb.x, yb = qb.y;
        N sb = vdot(qb, d);
        in.d = vadd(in.d, vscale(s, qb));
        sb += seed_opl[m] * n_before;
        N s0b = seed_opl[m] * n_before;
        out[m].n_before += seed_opl[m] * (s0 + s);
        N hb = zero, bb = zero;
        if (missed) {
            bb += sb / c;
            cb += -sb * s / c;
            const N db = -seed_pen[m];
            bb += db * two * B;
            cb += -db * H;
            hb += -db * c;
        } else {
            hb += sb * inv;
            bb += -sb * s * two * inv;
            cb += sb * s * s * inv;
        }
        cb += hb * rr;
        xb += hb * two * c * x;
        yb += hb * two * c * y;
        in.d.z += bb;
        cb += -bb * xd;
        xb += -bb * c * d.x;
        yb += -bb * c * d.y;
        in.d.x += -bb * c * x;
        in.d.y += -bb * c * y;
        // transfer: s0 = (t - p_z) / d_z
        in.p.x += xb;
        in.p.y += yb;
        s0b += xb * d.x + yb * d.y;
        in.d.x += xb * s0;
        in.d.y += yb * s0;
        const N qq = s0b / d.z;
        out[m].thickness += qq;
        in.p.z += -qq;
        in.d.z += -qq * s0;
        out[m].curvature += cb;
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
    refracting_step_backward_k<N, 1>(p, d, t, c, n_before, n_after, branch, so, sp, a, o);
    adj = a[0];
    out = o[0];
}

// Step onto the reference sphere through the last vertex about M = (0, h, w), K seeds.
template <class N, int K>
__device__ __forceinline__ void reference_step_backward_k(Vec<N> p, Vec<N> d, Vec<N> center,
                                                          N n_image, int branch,
                                                          const N (&seed_opl)[K],
                                                          const N (&seed_pen)[K],
                                                          RayAdj<N> (&adj)[K],
                                                          Vec<N> (&center_adj)[K],
                                                          N (&n_image_adj)[K]) {
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
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const N sb = seed_opl[m] * n_image;
        n_image_adj[m] += seed_opl[m] * s;
        N bb, gb;
        if (missed) {
            bb = sb;
            gb = zero;
            const N discb = -seed_pen[m] / radius_sq;
            bb += discb * two * b;
            gb += -discb;
            center_adj[m] = vadd(center_adj[m],
                                 vscale(seed_pen[m] * two * disc / (radius_sq * radius_sq),
                                        center));
        } else {
            gb = sb * sigma / (two * root);
            bb = -sb * sigma * s / root;
        }
        RayAdj<N> in{{zero, zero, zero}, {zero, zero, zero}};
        in.p = vadd(in.p, vscale(-bb, d));
        in.d = vadd(in.d, vscale(-bb, q));
        center_adj[m] = vadd(center_adj[m], vscale(bb, d));
        in.p = vadd(in.p, vscale(two * gb, vsub(p, center)));
        center_adj[m] = vadd(center_adj[m], vscale(N(-2.0) * gb, p));
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
    reference_step_backward_k<N, 1>(p, d, center, n_image, branch, so, sp, a, ca, na);
    adj = a[0];
    center_adj = ca[0];
    n_image_adj = na[0];
}

}  // namespace mkb
