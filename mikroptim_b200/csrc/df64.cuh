// Double-float ("df64") arithmetic: a value is the unevaluated sum hi + lo of two floats with
// |lo| <= ulp(hi) / 2, about 48 significant bits on the FP32 pipes. The reference's reduced-
// precision trace type (include/mikroptim/math/df64.hpp:108); restated here from the published
// error-free transformations and double-word algorithms:
//   TwoSum (Knuth), FastTwoSum (Dekker 1971), TwoProd with an FMA;
//   double-word + double-word (Joldes, Muller, Popescu 2017, "AccurateDWPlusDW", Algorithm 6),
//   double-word x double-word (Algorithm 12 with an FMA), division and square root by one
//   Newton correction of the float quotient / root.
// Every float operation is a separately rounded IEEE operation (the __f*_rn intrinsics), so the
// compiler cannot contract or reorder the error-free transformations.
#pragma once

#include <cuda_runtime.h>

namespace mkb {

struct Df64 {
    float hi, lo;
    Df64() = default;
    __host__ __device__ constexpr Df64(float h, float l) : hi(h), lo(l) {}
    __device__ Df64(double x) {
        hi = __double2float_rn(x);
        lo = __double2float_rn(x - static_cast<double>(hi));
    }
};

__device__ __forceinline__ Df64 df_two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float err = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return Df64(s, err);
}
__device__ __forceinline__ Df64 df_fast_two_sum(float a, float b) {  // |a| >= |b|
    const float s = __fadd_rn(a, b);
    return Df64(s, __fsub_rn(b, __fsub_rn(s, a)));
}
__device__ __forceinline__ Df64 df_two_prod(float a, float b) {
    const float p = __fmul_rn(a, b);
    return Df64(p, __fmaf_rn(a, b, -p));
}

__device__ __forceinline__ Df64 operator+(Df64 x, Df64 y) {
    const Df64 s = df_two_sum(x.hi, y.hi);
    const Df64 t = df_two_sum(x.lo, y.lo);
    const float c = __fadd_rn(s.lo, t.hi);
    const Df64 v = df_fast_two_sum(s.hi, c);
    const float w = __fadd_rn(t.lo, v.lo);
    return df_fast_two_sum(v.hi, w);
}
__device__ __forceinline__ Df64 operator-(Df64 x) { return Df64(-x.hi, -x.lo); }
__device__ __forceinline__ Df64 operator-(Df64 x, Df64 y) { return x + (-y); }
__device__ __forceinline__ Df64 operator*(Df64 x, Df64 y) {
    const Df64 c = df_two_prod(x.hi, y.hi);
    const float tl0 = __fmul_rn(x.lo, y.lo);
    const float tl1 = __fmaf_rn(x.hi, y.lo, tl0);
    const float cl2 = __fmaf_rn(x.lo, y.hi, tl1);
    const float cl3 = __fadd_rn(c.lo, cl2);
    return df_fast_two_sum(c.hi, cl3);
}
__device__ __forceinline__ Df64 operator/(Df64 x, Df64 y) {
    const float q1 = __fdiv_rn(x.hi, y.hi);
    const Df64 r = x - y * Df64(q1, 0.0f);  // remainder in double-word
    const float q2 = __fdiv_rn(r.hi, y.hi);
    return df_fast_two_sum(q1, q2);
}
__device__ __forceinline__ Df64& operator+=(Df64& a, Df64 b) { return a = a + b; }
__device__ __forceinline__ Df64& operator-=(Df64& a, Df64 b) { return a = a - b; }
__device__ __forceinline__ bool operator<(Df64 a, Df64 b) {
    return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}
__device__ __forceinline__ bool operator>(Df64 a, Df64 b) { return b < a; }
__device__ __forceinline__ bool operator>=(Df64 a, Df64 b) { return !(a < b) && a.hi == a.hi &&
                                                                   b.hi == b.hi; }
__device__ __forceinline__ Df64 nsqrt(Df64 a) {
    if (!(a.hi > 0.0f)) return Df64(__fsqrt_rn(a.hi), 0.0f);  // 0, or NaN below 0
    const float s = __fsqrt_rn(a.hi);
    const Df64 r = a - df_two_prod(s, s);
    const float c = __fdiv_rn(r.hi, __fmul_rn(2.0f, s));
    return df_fast_two_sum(s, c);
}
__device__ __forceinline__ double value_of(Df64 a) {
    return static_cast<double>(a.hi) + static_cast<double>(a.lo);
}

}  // namespace mkb
