// Correctly rounded binary32 exp and log for host and device.
//
// The reference physiology (src/physiology.cuh, src/lp_cell.cuh,
// src/prinz_cell.cuh of mixic/neural-selection) calls expf/logf. glibc's
// expf/logf and CUDA's expf/logf round differently in a small fraction of
// arguments, so the reference's CPU and GPU runs diverge
// (docs/GYM_PERFORMANCE.md:57). This engine instead evaluates both functions
// correctly rounded (round to nearest, ties to even): the result is the one
// binary32 value nearest to the exact mathematical exp(x) / log(x). That value
// is unique, so the host oracle, the CUDA kernels and a C compiler folding
// expf(constant) all agree bit for bit.
//
// Method (Tang, "Table-driven implementation of the exponential function in
// IEEE floating-point arithmetic", ACM TOMS 15(2), 1989, evaluated in binary64
// with a rounding test in the style of Ziv's strategy):
//   fast path  exp: x = k ln2/128 + r, exp(x) = 2^(k>>7) * T[k&127] * e^r,
//                   e^r by a degree-5 Taylor polynomial, |r| <= ln2/256.
//              log: x = m 2^e, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
//                   s = (m-1)/(m+1), odd series to s^23.
//   The binary64 fast result has relative error below 2^-50. If it lies
//   within 2^-48 (relative) of a binary32 rounding midpoint the result is
//   recomputed in double-double arithmetic (Dekker/Knuth error-free
//   transforms, relative error below 2^-95) and rounded with the sign of the
//   low word breaking an exact-midpoint tie.
//
// Only IEEE binary64 +, -, *, / and fused multiply-add are used, all
// correctly rounded on both x86-64 (SSE2/FMA) and sm_100a, so results do not
// depend on the compiler as long as floating-point contraction is disabled
// (-ffp-contract=off on the host, --fmad=false on the device). Exhaustive
// agreement with an independent long-double/binary128 implementation over all
// 2^32 inputs is checked by the oracle's exhaustive test.
#pragma once

#include <stdint.h>
#include "ns_crmath_consts.h"

#if defined(__CUDACC__)
#define NSX_HD __host__ __device__ __forceinline__
#define NSX_COLD static __host__ __device__ __noinline__
#else
#define NSX_HD static inline
#define NSX_COLD static
#include <string.h>
#include <math.h>
#endif

namespace nsx {

NSX_HD uint64_t dbits(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u; memcpy(&u, &d, 8); return u;
#endif
}
NSX_HD double bitsd(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d; memcpy(&d, &u, 8); return d;
#endif
}
NSX_HD uint32_t fbits(float f) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)__float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
NSX_HD float bitsf(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}
NSX_HD double dfma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

// Round-to-nearest-even integer value (exact IEEE rint on both sides).
NSX_HD double round_shift(double t) {
    return rint(t);
}
NSX_HD float f32_inf() { return bitsf(0x7f800000u); }

// ---- double-double arithmetic (value = hi + lo, |lo| <= ulp(hi)/2) -------
struct dd { double hi, lo; };

NSX_HD dd two_sum(double a, double b) {
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
NSX_HD dd fast_two_sum(double a, double b) {  // requires |a| >= |b|
    double s = a + b;
    return {s, b - (s - a)};
}
NSX_HD dd two_prod(double a, double b) {
    double p = a * b;
    return {p, dfma(a, b, -p)};
}
NSX_HD dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
NSX_HD dd dd_mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return fast_two_sum(p.hi, p.lo);
}
NSX_HD dd dd_div_d(double a, double b) {  // a / b for doubles, as dd
    double q1 = a / b;
    double r = dfma(-q1, b, a);           // exact remainder
    double q2 = r / b;
    return fast_two_sum(q1, q2);
}

// Round hi + lo (|lo| <= ulp(hi)/2) to binary32, nearest-even. RN(hi)
// differs from RN(hi + lo) only when hi is exactly a binary32 midpoint
// (midpoints are binary64 numbers), and then the sign of lo decides.
NSX_HD float round_dd_to_float(double hi, double lo) {
    float f = (float)hi;
    double fd = (double)f;
    if (fd == hi) return f;
    uint32_t fb = fbits(f);
    bool toward_pos = hi > fd;        // the other neighbour lies above f
    uint32_t gb;
    if ((fb & 0x7fffffffu) == 0u) {
        gb = toward_pos ? 0x00000001u : 0x80000001u;
    } else {
        bool f_neg = (fb >> 31) != 0;
        gb = (toward_pos != f_neg) ? fb + 1u : fb - 1u;
    }
    float g = bitsf(gb);
    double fdv = fd;
    if ((fb & 0x7fffffffu) == 0x7f800000u) fdv = (fb >> 31) ? -0x1p128 : 0x1p128;
    double mid = 0.5 * (fdv + (double)g);
    if (hi != mid) return f;
    if (lo == 0.0) return f;          // exact tie: RN already chose even
    bool true_above = lo > 0.0;
    bool g_above = (double)g > hi;
    return (g_above == true_above) ? g : f;
}

// Is the binary64 value y (a normal binary32-range result) within
// `margin` binary64 ulps of a binary32 rounding midpoint?
NSX_HD bool near_midpoint(double y, uint64_t margin) {
    uint64_t low = dbits(y) & ((1ull << 29) - 1ull);
    uint64_t mid = 1ull << 28;
    uint64_t d = low > mid ? low - mid : mid - low;
    return d <= margin;
}

// Constant tables: one copy in host memory, one in device global memory.
static const double kInvFactDD_h[2 * NSX_INV_FACT_COUNT] = {NSX_INV_FACT_DD};
static const double kInvOddDD_h[2 * NSX_INV_ODD_COUNT] = {NSX_INV_ODD_DD};
static const double kExp2Tab_h[128] = {NSX_EXP2_128_TABLE};
static const float kExp2F_h[256] = {NSX_EXP2F_128_TABLE};
#if defined(__CUDACC__)
static __device__ const float kExp2F_d[256] = {NSX_EXP2F_128_TABLE};
static __device__ const double kInvFactDD_d[2 * NSX_INV_FACT_COUNT] = {NSX_INV_FACT_DD};
static __device__ const double kInvOddDD_d[2 * NSX_INV_ODD_COUNT] = {NSX_INV_ODD_DD};
static __device__ const double kExp2Tab_d[128] = {NSX_EXP2_128_TABLE};
#endif
NSX_HD const double *inv_fact_dd() {
#if defined(__CUDA_ARCH__)
    return kInvFactDD_d;
#else
    return kInvFactDD_h;
#endif
}
NSX_HD const double *inv_odd_dd() {
#if defined(__CUDA_ARCH__)
    return kInvOddDD_d;
#else
    return kInvOddDD_h;
#endif
}
NSX_HD const float *exp2f_table() {
#if defined(__CUDA_ARCH__)
    return kExp2F_d;
#else
    return kExp2F_h;
#endif
}
NSX_HD const double *exp2_table() {
#if defined(__CUDA_ARCH__)
    return kExp2Tab_d;
#else
    return kExp2Tab_h;
#endif
}

// exp(x) for -104 < x < 88.8 in double-double, rounded to binary32.
NSX_COLD float expf_slow(float x) {
    double xd = (double)x;
    double md = round_shift(xd * NSX_INV_LN2);
    // r = x - m ln2 with ln2 = A + B + C; m*A and m*B are exact.
    double rh = xd - md * NSX_LN2_A;          // exact (cancellation)
    dd r = two_sum(rh, -(md * NSX_LN2_B));
    r.lo -= md * NSX_LN2_C;
    r = fast_two_sum(r.hi, r.lo);
    // Horner: p = sum_{n=0}^{24} r^n / n!
    const double *c = inv_fact_dd();
    dd p = {c[2 * (NSX_INV_FACT_COUNT - 1)], c[2 * (NSX_INV_FACT_COUNT - 1) + 1]};
    for (int n = NSX_INV_FACT_COUNT - 2; n >= 0; --n) {
        p = dd_mul(p, r);
        p = dd_add(p, dd{c[2 * n], c[2 * n + 1]});
    }
    int m = (int)md;
    // 2^m as two factors so that the intermediate stays normal.
    int m1 = m / 2, m2 = m - m1;
    double s1 = bitsd((uint64_t)(int64_t)(m1 + 1023) << 52);
    double s2 = bitsd((uint64_t)(int64_t)(m2 + 1023) << 52);
    double hi = p.hi * s1 * s2, lo = p.lo * s1 * s2;  // exact scalings
    return round_dd_to_float(hi, lo);
}

// Correctly rounded exp for binary32 using table `tab` (NSX_EXP2_128_TABLE).
NSX_HD float expf_cr_tab(float x, const double *tab) {
    if (x != x) return x + x;
    if (x > 88.8f) return f32_inf();
    if (x < -104.0f) return 0.0f;
    double xd = (double)x;
    double kd = round_shift(xd * NSX_INV_LN2_128);
    double r = dfma(-kd, NSX_LN2_128_HI, xd);
    r = dfma(-kd, NSX_LN2_128_LO, r);
    // q = 1 + r/2 + r^2/6 + r^3/24 + r^4/120, e^r = 1 + r q
    double q = dfma(r, 1.0 / 120.0, 1.0 / 24.0);
    q = dfma(r, q, 1.0 / 6.0);
    q = dfma(r, q, 0.5);
    q = dfma(r, q, 1.0);
    double rq = r * q;
    int64_t k = (int64_t)kd;
    int j = (int)(k & 127);
    int64_t m = k >> 7;                       // floor(k / 128)
    double t = tab[j];
    double y = dfma(t, rq, t);
    y *= bitsd((uint64_t)(m + 1023) << 52);   // exact power of two, -151 < m < 129
    if (y < 0x1p-126 || near_midpoint(y, 32)) return expf_slow(x);
    return (float)y;
}

NSX_HD float sfma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

// Binary64 path, out of line on the device (used for the rare arguments the
// binary32 fast path below cannot decide).
NSX_COLD float expf_cr_wide(float x) { return expf_cr_tab(x, exp2_table()); }

// Correctly rounded exp, binary32 fast path. `tabf` is NSX_EXP2F_128_TABLE
// (2^(j/128) as binary32 hi/lo pairs). Float-float evaluation on the FP32
// pipes: x = k ln2/128 + r (Cody-Waite with a 10-bit first constant, so the
// first product is exact, and an error-free product for the second),
// exp(x) = 2^(k>>7) (T_hi + T_lo)(1 + r + q(r)); relative error below 2^-41.
// The result is returned only if it is at least 2^-38 (relative) away from a
// rounding midpoint; otherwise, and outside [-86, 88.5] (results near the
// normal range limits, NaN, infinities), the binary64 path decides.
NSX_HD float expf_cr_ff(float x, const float *tabf) {
    if (!(x >= -86.0f && x <= 88.5f)) return expf_cr_wide(x);
    const float shifter = 0x1.8p23f;
    const float t = sfma(x, NSX_F_INV_LN2_128, shifter);
    const int ki = (int)fbits(t) - 0x4B400000;
    const float kf = t - shifter;
    const float r1 = sfma(-kf, NSX_F_LN2_128_A, x);      // exact
    const float p = kf * NSX_F_LN2_128_B;
    const float pe = sfma(kf, NSX_F_LN2_128_B, -p);       // exact error of p
    const float rh = r1 - p;                              // two-sum(r1, -p)
    const float bb = rh - r1;
    const float re = (r1 - (rh - bb)) + (-p - bb);
    const float rl = (re - pe) - kf * NSX_F_LN2_128_C;
    float h = sfma(rh, 1.0f / 120.0f, 1.0f / 24.0f);
    h = sfma(rh, h, 1.0f / 6.0f);
    h = sfma(rh, h, 0.5f);
    const float q = (rh * rh) * h;                        // e^r - 1 - r, |q| < 2^-17
    const float sm = sfma(rh, rl, rl) + q;                // rl (1 + rh) + q
    const int j = ki & 127;
    const float th = tabf[2 * j], tl = tabf[2 * j + 1];
    const float ph = th * rh;
    const float pl = sfma(th, rh, -ph);
    const float low = sfma(th, sm, sfma(tl, rh, tl)) + pl;
    const float sh = th + ph;                             // fast two-sum, |th| > |ph|
    const float sl = ph - (sh - th);
    const float c = sl + low;
    const float y = sh + c;
    const float d = (sh - y) + c;                         // residual below ulp(y)/2
    const uint32_t yb = fbits(y);
    const float half = bitsf((yb & 0x7f800000u) - (24u << 23));   // ulp(y)/2
    const float gap = half - fabsf(d);
    if ((yb & 0x007fffffu) == 0u || gap <= half * 0x1p-14f) return expf_cr_wide(x);
    return bitsf((uint32_t)((int)yb + (ki >> 7) * (1 << 23)));
}

// Correctly rounded exp using the built-in table of the calling side.
NSX_HD float expf_cr(float x) { return expf_cr_ff(x, exp2f_table()); }

// log(x) for finite x > 0, x != 1, in double-double, rounded to binary32.
NSX_COLD float logf_slow(double md, int e) {
    // s = (m-1)/(m+1); m-1 and m+1 are exact.
    dd s = dd_div_d(md - 1.0, md + 1.0);
    dd z = dd_mul(s, s);
    const double *c = inv_odd_dd();
    dd p = {c[2 * (NSX_INV_ODD_COUNT - 1)], c[2 * (NSX_INV_ODD_COUNT - 1) + 1]};
    for (int n = NSX_INV_ODD_COUNT - 2; n >= 0; --n) {
        p = dd_mul(p, z);
        p = dd_add(p, dd{c[2 * n], c[2 * n + 1]});
    }
    dd lm = dd_mul(s, p);
    lm.hi *= 2.0; lm.lo *= 2.0;
    double ed = (double)e;
    dd el = two_sum(ed * NSX_LN2_A, ed * NSX_LN2_B);   // both exact products
    el.lo += ed * NSX_LN2_C;
    dd res = dd_add(el, lm);
    return round_dd_to_float(res.hi, res.lo);
}

// Correctly rounded log for binary32.
NSX_HD float logf_cr(float x) {
    uint32_t u = fbits(x);
    if (x != x) return x + x;
    if (u == 0x7f800000u) return x;                       // +inf
    if ((u & 0x7fffffffu) == 0u) return -f32_inf();
    if (u >> 31) return (x - x) / (x - x);                // negative: NaN
    if (x == 1.0f) return 0.0f;
    int e;
    double md;
    if (u < 0x00800000u) {                                // subnormal
        double xd = (double)x * 0x1p24;
        uint64_t b = dbits(xd);
        e = (int)((b >> 52) & 0x7ff) - 1023 - 24;
        md = bitsd((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    } else {
        e = (int)(u >> 23) - 127;
        md = (double)bitsf((u & 0x007fffffu) | 0x3f800000u);
    }
    if (md > NSX_SQRT2) { md *= 0.5; e += 1; }
    double s = (md - 1.0) / (md + 1.0);
    double z = s * s;
    // atanh(s)/s = sum z^n/(2n+1), n = 0..11
    double p = 1.0 / 23.0;
    p = dfma(p, z, 1.0 / 21.0);
    p = dfma(p, z, 1.0 / 19.0);
    p = dfma(p, z, 1.0 / 17.0);
    p = dfma(p, z, 1.0 / 15.0);
    p = dfma(p, z, 1.0 / 13.0);
    p = dfma(p, z, 1.0 / 11.0);
    p = dfma(p, z, 1.0 / 9.0);
    p = dfma(p, z, 1.0 / 7.0);
    p = dfma(p, z, 1.0 / 5.0);
    p = dfma(p, z, 1.0 / 3.0);
    double lm = 2.0 * dfma(s * z, p, s);
    double ed = (double)e;
    double y = dfma(ed, NSX_LN2_LOG_HI, dfma(ed, NSX_LN2_LOG_LO, lm));
    double ay = y < 0 ? -y : y;
    if (ay < 0x1p-126 || near_midpoint(ay, 32)) return logf_slow(md, e);
    return (float)y;
}

}  // namespace nsx
