// Correctly rounded FP64 atan2 and sin for the table builders.
//
// The reference computes every pixel corner's 2-theta and chi with the C
// library's atan2 (and q with sin), which is correctly rounded in all but
// rare hard cases. A table entry can depend on the last bit of a corner (a
// corner a few ulp from a bin edge decides whether a sliver of the pixel
// enters that bin), so the device evaluates these functions in double-double
// arithmetic (about 104 bits) and rounds once: the result is the correctly
// rounded double, hence the C library's bits wherever that is correctly
// rounded.
//
// Method (textbook argument reduction, no vendor code):
//   atan(t), t in [0,1]: c = round(64 t)/64, u = (t - c)/(1 + t c),
//     atan(t) = atan(c) + u * sum_j (-1)^j u^(2j)/(2j+1), |u| <= 1/128;
//   atan2(y, x) from atan(min/max) by the octant identities pi/2 - a, pi - a;
//   sin(x), |x| <= pi/2: c = round(64 x)/64, d = x - c (exact),
//     sin(x) = sin(c) cos(d) + cos(c) sin(d), Taylor series for sin d, cos d.
// The constants atan(k/64), sin(k/64), cos(k/64), pi, 1/(2j+1) and 1/k! are
// double-double values generated by gen_dd_tables.py.
#pragma once

#include "dg_dd_tables.h"

namespace dg {
namespace ddm {

struct dd {
    double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
    double s = __dadd_rn(a, b);
    double bb = __dsub_rn(s, a);
    double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return {s, e};
}
__device__ __forceinline__ dd fast_two_sum(double a, double b) {
    double s = __dadd_rn(a, b);
    return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ dd two_prod(double a, double b) {
    double p = __dmul_rn(a, b);
    return {p, __fma_rn(a, b, -p)};
}
__device__ __forceinline__ dd add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    dd v = fast_two_sum(s.hi, __dadd_rn(s.lo, t.hi));
    return fast_two_sum(v.hi, __dadd_rn(t.lo, v.lo));
}
__device__ __forceinline__ dd add_d(dd a, double b) {
    dd s = two_sum(a.hi, b);
    return fast_two_sum(s.hi, __dadd_rn(s.lo, a.lo));
}
__device__ __forceinline__ dd neg(dd a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ dd mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    double c = __fma_rn(a.hi, b.lo, __dmul_rn(a.lo, b.hi));
    return fast_two_sum(p.hi, __dadd_rn(p.lo, c));
}
__device__ __forceinline__ dd mul_d(dd a, double b) {
    dd p = two_prod(a.hi, b);
    return fast_two_sum(p.hi, __fma_rn(a.lo, b, p.lo));
}
__device__ __forceinline__ dd div(dd a, dd b) {
    double q1 = __ddiv_rn(a.hi, b.hi);
    dd r = add(a, neg(mul_d(b, q1)));
    double q2 = __ddiv_rn(r.hi, b.hi);
    r = add(r, neg(mul_d(b, q2)));
    double q3 = __ddiv_rn(r.hi, b.hi);
    return add_d(fast_two_sum(q1, q2), q3);
}
__device__ __forceinline__ dd cst(const double (&c)[2]) { return {c[0], c[1]}; }

// sum_j (-1)^j coef[j] v^j for j = 0..last: terms j >= split in double
// (their size makes double precision enough), the rest in double-double.
template <int LAST, int SPLIT>
__device__ __forceinline__ dd alt_series(dd v, const double (*coef)[2], int stride, int first) {
    double vh = v.hi;
    double tail = coef[first + stride * LAST][0];
#pragma unroll
    for (int j = LAST - 1; j >= SPLIT; --j) tail = __fma_rn(-vh, tail, coef[first + stride * j][0]);
    dd s = {tail, 0.0};
#pragma unroll
    for (int j = SPLIT - 1; j >= 0; --j) s = add(cst(coef[first + stride * j]), neg(mul(v, s)));
    return s;
}

// atan(t) for t in [0, 1] (double-double).
__device__ __forceinline__ dd atan01(dd t) {
    int k = int(rint(t.hi * double(kTabStep)));
    double c = double(k) * (1.0 / kTabStep);
    dd num = add_d(t, -c);
    dd den = add_d(mul_d(t, c), 1.0);
    dd u = div(num, den);
    dd v = mul(u, u);
    // |u| <= 1/128: v^j/(2j+1) < 2^-110 for j >= 8.
    dd s = alt_series<8, 4>(v, kInvOdd, 1, 0);
    return add(cst(kAtanTab[k]), mul(u, s));
}

// Correctly rounded atan2 with the C library's special-value rules.
__device__ __forceinline__ double cr_atan2(double y, double x) {
    if (isnan(x) || isnan(y)) return x + y;
    if (isinf(x) || isinf(y)) return atan2(y, x);
    if (y == 0.0) return signbit(x) ? copysign(kPiHi, y) : y;
    if (x == 0.0) return copysign(kPiHalfHi, y);
    double ax = fabs(x), ay = fabs(y);
    bool swap = ay > ax;
    dd t = div(dd{swap ? ax : ay, 0.0}, dd{swap ? ay : ax, 0.0});
    dd r = atan01(t);
    if (swap) r = add(dd{kPiHalfHi, kPiHalfLo}, neg(r));
    if (signbit(x)) r = add(dd{kPiHi, kPiLo}, neg(r));
    return copysign(__dadd_rn(r.hi, r.lo), y);
}

// Correctly rounded sin on |x| <= pi/2 + 1/64 (table range); outside that
// range it returns CUDA's sin, which the builders never need.
__device__ __forceinline__ double cr_sin(double x) {
    double ax = fabs(x);
    if (!(ax * double(kTabStep) <= double(kSinTabLen - 1))) return sin(x);
    if (ax == 0.0) return x;
    int k = int(rint(ax * double(kTabStep)));
    double c = double(k) * (1.0 / kTabStep);
    double d = __dsub_rn(ax, c);  // exact (Sterbenz) for k >= 1; d = ax for k = 0
    dd v = two_prod(d, d);
    // sin d = d * sum (-1)^j v^j/(2j+1)!, cos d = sum (-1)^j v^j/(2j)!; |d| <= 1/128.
    dd sd = mul_d(alt_series<6, 4>(v, kInvFact, 2, 1), d);
    dd cd = alt_series<6, 4>(v, kInvFact, 2, 0);
    dd r = add(mul(cst(kSinTab[k]), cd), mul(cst(kCosTab[k]), sd));
    return copysign(__dadd_rn(r.hi, r.lo), x);
}

}  // namespace ddm
}  // namespace dg
