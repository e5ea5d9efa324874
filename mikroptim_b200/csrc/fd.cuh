// Finite-difference pattern and derivative shared by the FD Jacobian (jacobian.cu) and the
// device paraxial constraint rows (paraxial.cu): the reference's fd_step / fd_pattern
// (src/optim/variant_generator.cpp:177) and fd_derivative (include/mikroptim/optim/
// fd_formula.hpp:40), every operation separately rounded so that host and device agree bit for
// bit with the reference CPU build.
#pragma once

#include "common.cuh"

namespace mkb {

enum : int { kCentral = 0, kOneSided = 1, kTruncated = 2 };  // FdStencil, optim/fd_formula.hpp:16

struct FdPattern {
    double xa, xb, da, db;
    int stencil;
    int pad;
};

__host__ __device__ inline double raw(double a) { return a; }
__host__ __device__ inline double raw(Exact64 a) { return a.v; }

// fd_step + fd_pattern (central) of one variable (src/optim/variant_generator.cpp:177), every
// operation separately rounded: Exact64 on the device, plain double on the host (x86-64 without
// contraction), so both give the same bits.
template <class N>
__host__ __device__ inline FdPattern fd_pattern_of(double x0, double lower, double upper,
                                                   double typical) {
    const N x = x0;
    const N lo = lower, up = upper;
    const double ax = fabs(x0);
    const N h = N(6.0554544523933395e-06) * N(ax < typical ? typical : ax);
    const N plus = x + h, minus = x - h;
    FdPattern out;
    out.stencil = kCentral;
    out.pad = 0;
    N a, b;
    if (raw(plus) <= raw(up) && raw(minus) >= raw(lo)) {
        a = plus;
        b = minus;
    } else {
        const bool towards_upper = raw(up - x) >= raw(x - lo);
        const N two_h = N(2.0) * h;
        const N far = towards_upper ? x + two_h : x - two_h;
        if (towards_upper ? raw(far) <= raw(up) : raw(far) >= raw(lo)) {
            out.stencil = kOneSided;
            a = towards_upper ? plus : minus;
            b = far;
        } else {
            out.stencil = kTruncated;
            a = raw(plus) <= raw(up) ? plus : up;
            b = raw(minus) >= raw(lo) ? minus : lo;
        }
    }
    out.xa = raw(a);
    out.xb = raw(b);
    out.da = raw(a - x);
    out.db = raw(b - x);
    return out;
}

// fd_derivative (optim/fd_formula.hpp:40)
template <class N>
__host__ __device__ inline double fd_derivative_of(int stencil, double r0, double ra, double rb,
                                                   double da_, double db_) {
    const N v0 = r0, va = ra, vb = rb, da = da_, db = db_;
    N d;
    if (stencil == kOneSided) {
        const N ga = va - v0;
        const N gb = vb - v0;
        d = (db * db * ga - da * da * gb) / (da * db * (db - da));
    } else {
        d = (va - vb) / (da - db);
    }
    return raw(d);
}

}  // namespace mkb
