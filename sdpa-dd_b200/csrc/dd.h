// Double-double (dd) arithmetic for host and device.
//
// A dd value is an unevaluated sum hi + lo of two IEEE doubles with
// |lo| <= ulp(hi)/2.  The operations below are the error-free
// transformations of Knuth (TwoSum), Dekker (FastTwoSum, exact products)
// and the "sloppy" double-double formulas of Hida, Li and Bailey
// (QD library, 2.3.x), written so that every intermediate double rounds
// exactly as in that library's default x86-64 build (no fused
// multiply-add anywhere except for the exact product error, which equals
// Dekker's split product bit for bit in the normal range).
//
// The reference solver uses three distinct rounding shapes for addition
// (dd_real::operator+, operator+= and operator-/-=) and two for
// multiplication (operator* and operator*=); the names below keep them apart
// so that each call site can use the shape the reference uses there
// (QD dd_inline.h: operator+ sloppy_add, operator+=, operator-, operator*,
// operator*=, sloppy_div; dd_real.cpp: sqrt).
//
// Device code uses the explicitly rounded intrinsics (__dadd_rn, __dmul_rn,
// __fma_rn, __ddiv_rn, __dsqrt_rn), so nothing here depends on the
// compiler's contraction settings.  Host code must be compiled with
// -ffp-contract=off.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define DD_HD __host__ __device__ __forceinline__
#else
#define DD_HD inline
#endif

struct __attribute__((aligned(16))) dd_t {
    double hi, lo;
};

namespace ddm {

// ------------------------------------------------------------ IEEE primitives
DD_HD double add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
DD_HD double sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
DD_HD double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
DD_HD double div(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
DD_HD double sqrt_(double a) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(a);
#else
    return ::sqrt(a);
#endif
}
// exact a*b - p for p = fl(a*b)
DD_HD double prod_err(double a, double b, double p) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, -p);
#else
    return ::fma(a, b, -p);
#endif
}

// --------------------------------------------------- error-free transforms
// s + e == a + b exactly, s = fl(a + b)          (Knuth)
DD_HD double two_sum(double a, double b, double &e) {
    double s = add(a, b);
    double v = sub(s, a);
    e = add(sub(a, sub(s, v)), sub(b, v));
    return s;
}
// s + e == a - b exactly, s = fl(a - b)
DD_HD double two_diff(double a, double b, double &e) {
    double s = sub(a, b);
    double v = sub(s, a);
    e = sub(sub(a, sub(s, v)), add(b, v));
    return s;
}
// s + e == a + b exactly when |a| >= |b|          (Dekker)
DD_HD double fast_two_sum(double a, double b, double &e) {
    double s = add(a, b);
    e = sub(b, sub(s, a));
    return s;
}
// p + e == a * b exactly
DD_HD double two_prod(double a, double b, double &e) {
    double p = mul(a, b);
    e = prod_err(a, b, p);
    return p;
}

} // namespace ddm

DD_HD dd_t dd_make(double hi, double lo) {
    dd_t r;
    r.hi = hi;
    r.lo = lo;
    return r;
}
DD_HD dd_t dd_from(double a) { return dd_make(a, 0.0); }
DD_HD dd_t dd_zero() { return dd_make(0.0, 0.0); }
DD_HD dd_t dd_neg(dd_t a) { return dd_make(-a.hi, -a.lo); }
DD_HD dd_t dd_abs(dd_t a) { return a.hi < 0.0 ? dd_neg(a) : a; }

// a + b, the shape of dd_real operator+ (lo parts summed first)
DD_HD dd_t dd_add(dd_t a, dd_t b) {
    using namespace ddm;
    double e, s = two_sum(a.hi, b.hi, e);
    e = add(e, add(a.lo, b.lo));
    s = fast_two_sum(s, e, e);
    return dd_make(s, e);
}
// x += a, the shape of dd_real::operator+= (lo parts added one by one)
DD_HD dd_t dd_acc(dd_t x, dd_t a) {
    using namespace ddm;
    double e, s = two_sum(x.hi, a.hi, e);
    e = add(e, x.lo);
    e = add(e, a.lo);
    s = fast_two_sum(s, e, e);
    return dd_make(s, e);
}
// a - b, the shape of dd_real operator- and operator-= (identical to
// dd_acc(a, -b) bit for bit)
DD_HD dd_t dd_sub(dd_t a, dd_t b) {
    using namespace ddm;
    double e, s = two_diff(a.hi, b.hi, e);
    e = add(e, a.lo);
    e = sub(e, b.lo);
    s = fast_two_sum(s, e, e);
    return dd_make(s, e);
}
// a * b, the shape of dd_real operator* (commutative bit for bit)
DD_HD dd_t dd_mul(dd_t a, dd_t b) {
    using namespace ddm;
    double e, p = two_prod(a.hi, b.hi, e);
    e = add(e, add(mul(a.hi, b.lo), mul(a.lo, b.hi)));
    p = fast_two_sum(p, e, e);
    return dd_make(p, e);
}
// x *= a, the shape of dd_real::operator*=
DD_HD dd_t dd_muleq(dd_t x, dd_t a) {
    using namespace ddm;
    double e, p = two_prod(x.hi, a.hi, e);
    e = add(e, mul(a.lo, x.hi));
    e = add(e, mul(a.hi, x.lo));
    p = fast_two_sum(p, e, e);
    return dd_make(p, e);
}
// a * b for a double b (dd_real * double)
DD_HD dd_t dd_mul_d(dd_t a, double b) {
    using namespace ddm;
    double e, p = two_prod(a.hi, b, e);
    e = add(e, mul(a.lo, b));
    p = fast_two_sum(p, e, e);
    return dd_make(p, e);
}
// a + b for a double b (dd_real + double)
DD_HD dd_t dd_add_d(dd_t a, double b) {
    using namespace ddm;
    double e, s = two_sum(a.hi, b, e);
    e = add(e, a.lo);
    s = fast_two_sum(s, e, e);
    return dd_make(s, e);
}
// a - b for a double b (dd_real - double)
DD_HD dd_t dd_sub_d(dd_t a, double b) {
    using namespace ddm;
    double e, s = two_diff(a.hi, b, e);
    e = add(e, a.lo);
    s = fast_two_sum(s, e, e);
    return dd_make(s, e);
}
// a - b for a double a (double - dd_real)
DD_HD dd_t d_sub_dd(double a, dd_t b) {
    using namespace ddm;
    double e, s = two_diff(a, b.hi, e);
    e = sub(e, b.lo);
    s = fast_two_sum(s, e, e);
    return dd_make(s, e);
}
// exact sum of two doubles (dd_real::add(double, double))
DD_HD dd_t dd_add_dd_exact(double a, double b) {
    double e, s = ddm::two_sum(a, b, e);
    return dd_make(s, e);
}
// a / b, the "sloppy" division of the QD library
DD_HD dd_t dd_div(dd_t a, dd_t b) {
    using namespace ddm;
    double q1 = div(a.hi, b.hi);
    dd_t r = dd_mul_d(b, q1);
    double s2, s1 = two_diff(a.hi, r.hi, s2);
    s2 = sub(s2, r.lo);
    s2 = add(s2, a.lo);
    double q2 = div(add(s1, s2), b.hi);
    double e, q = fast_two_sum(q1, q2, e);
    return dd_make(q, e);
}
// a / b for a double b (dd_real / double)
DD_HD dd_t dd_div_d(dd_t a, double b) {
    using namespace ddm;
    double q1 = div(a.hi, b);
    double p2, p1 = two_prod(q1, b, p2);
    double e, s = two_diff(a.hi, p1, e);
    e = add(e, a.lo);
    e = sub(e, p2);
    double q2 = div(add(s, e), b);
    double r2, r1 = fast_two_sum(q1, q2, r2);
    return dd_make(r1, r2);
}
// square of a double as an exact dd (dd_real::sqr(double))
DD_HD dd_t dd_sqr_d(double a) {
    double e, p = ddm::two_prod(a, a, e);
    return dd_make(p, e);
}
// sqr(a) (QD's dd squaring)
DD_HD dd_t dd_sqr(dd_t a) {
    using namespace ddm;
    double p2, p1 = two_prod(a.hi, a.hi, p2);
    p2 = add(p2, mul(mul(2.0, a.hi), a.lo));
    p2 = add(p2, mul(a.lo, a.lo));
    double s2, s1 = fast_two_sum(p1, p2, s2);
    return dd_make(s1, s2);
}
// sqrt(a) by Karp's trick: with x ~ 1/sqrt(a.hi),
// sqrt(a) ~ a*x + (a - (a*x)^2) * x / 2.  Negative input gives NaN.
DD_HD dd_t dd_sqrt(dd_t a) {
    using namespace ddm;
    if (a.hi == 0.0) return dd_zero();
    if (a.hi < 0.0) {
        double nan = 0.0 / 0.0;
        return dd_make(nan, nan);
    }
    double x = div(1.0, sqrt_(a.hi));
    double ax = mul(a.hi, x);
    dd_t d = dd_sub(a, dd_sqr_d(ax));
    return dd_add_dd_exact(ax, mul(d.hi, mul(x, 0.5)));
}

// 10^p as QD's npwr(10, p) forms it (src/dd_real.cpp): for |p| > 1 the
// binary powers of 10 (QD's sqr) multiplied in ("*=" shape) where p has a
// bit, for |p| == 1 ten itself; for p < 0 one division of 1 by the power.
DD_HD dd_t dd_pow10(int p) {
    if (p == 0) return dd_from(1.0);
    const dd_t ten = dd_from(10.0);
    unsigned bits = (unsigned)(p < 0 ? -p : p);
    dd_t power = ten;
    if (bits > 1) {
        dd_t acc = dd_from(1.0), base = ten;
        for (; bits != 0; bits >>= 1) {
            if (bits & 1u) acc = dd_muleq(acc, base);
            if (bits > 1) base = dd_sqr(base);
        }
        power = acc;
    }
    return p < 0 ? dd_div(dd_from(1.0), power) : power;
}

// ----------------------------------------------------------- comparisons
DD_HD bool dd_lt(dd_t a, dd_t b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
DD_HD bool dd_gt(dd_t a, dd_t b) { return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo); }
DD_HD bool dd_le(dd_t a, dd_t b) { return a.hi < b.hi || (a.hi == b.hi && a.lo <= b.lo); }
DD_HD bool dd_ge(dd_t a, dd_t b) { return a.hi > b.hi || (a.hi == b.hi && a.lo >= b.lo); }
DD_HD bool dd_eq(dd_t a, dd_t b) { return a.hi == b.hi && a.lo == b.lo; }
DD_HD bool dd_lt_d(dd_t a, double b) { return a.hi < b || (a.hi == b && a.lo < 0.0); }
DD_HD bool dd_gt_d(dd_t a, double b) { return a.hi > b || (a.hi == b && a.lo > 0.0); }
DD_HD bool dd_le_d(dd_t a, double b) { return a.hi < b || (a.hi == b && a.lo <= 0.0); }
DD_HD bool dd_ge_d(dd_t a, double b) { return a.hi > b || (a.hi == b && a.lo >= 0.0); }
DD_HD bool dd_is_zero(dd_t a) { return a.hi == 0.0 && a.lo == 0.0; }
DD_HD bool dd_isnan(dd_t a) { return a.hi != a.hi || a.lo != a.lo; }
DD_HD dd_t dd_max(dd_t a, dd_t b) { return dd_gt(a, b) ? a : b; }
DD_HD dd_t dd_min(dd_t a, dd_t b) { return dd_lt(a, b) ? a : b; }

// c - a*b with the product rounded first: the reference's accumulation
// step "c -= a*b" / "c = c - a*b" (operator- of an operator* product).
DD_HD dd_t dd_fms(dd_t c, dd_t a, dd_t b) { return dd_sub(c, dd_mul(a, b)); }
// c += a*b: the reference's "c += a*b" (operator+= of an operator* product).
DD_HD dd_t dd_fma(dd_t c, dd_t a, dd_t b) { return dd_acc(c, dd_mul(a, b)); }
