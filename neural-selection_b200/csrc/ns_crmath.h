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
// expf_cr_fast is the binary32 part alone: its result stands when `ok`.
NSX_HD float expf_cr_fast(float x, const float *tabf, bool &ok) {
    // Branch-free, so that independent exponentials can be interleaved: an
    // argument outside [-86, 88.5] is replaced by 0 for the arithmetic (the
    // table index stays in range) and reported through `ok`.
    const bool in = x >= -86.0f && x <= 88.5f;
    const float xs = in ? x : 0.0f;
    const float shifter = 0x1.8p23f;
    const float t = sfma(xs, NSX_F_INV_LN2_128, shifter);
    const int ki = (int)fbits(t) - 0x4B400000;
    const float kf = t - shifter;
    const float r1 = sfma(-kf, NSX_F_LN2_128_A, xs);     // exact
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
    ok = in && (yb & 0x007fffffu) != 0u && gap > half * 0x1p-14f;
    return bitsf((uint32_t)((int)yb + (ki >> 7) * (1 << 23)));
}

NSX_HD float expf_cr_ff(float x, const float *tabf) {
    bool ok;
    const float y = expf_cr_fast(x, tabf, ok);
    return ok ? y : expf_cr_wide(x);
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

// ---- sin, cos, hypot ----------------------------------------------------------
// The reference world's body and sense kernels (src/main.cu:619-657,
// 1146-1249) call cosf, sinf and hypotf. They are evaluated here correctly
// rounded as well, with the same fast-path / double-double strategy:
//   reduction  |x| = (4j + q) pi/2 + r, |r| <= pi/4, by Payne and Hanek's
//              method ("Radian reduction for trigonometric functions",
//              SIGNUM Newsletter 18(1), 1983): the 24-bit significand times a
//              192-bit window of 2/pi in integer arithmetic, keeping at least
//              159 fraction bits, so r carries a relative error below 2^-100;
//   fast path  Taylor polynomials of sin and cos to degree 17/18 in binary64
//              (relative error below 2^-50), accepted unless within 2^-47 of a
//              binary32 rounding midpoint;
//   slow path  the Taylor series to degree 24 in double-double.
// hypot: x^2 and y^2 are exact in binary64; sqrt(x^2 + y^2) in binary64 is
// within 2^-52 (relative); near a midpoint the midpoint m is compared with the
// exact sum of squares (m^2 has at most 50 significant bits).
static const uint32_t k2OverPi_h[NSX_2OPI_COUNT] = {NSX_2OPI_WORDS};
#if defined(__CUDACC__)
static __device__ const uint32_t k2OverPi_d[NSX_2OPI_COUNT] = {NSX_2OPI_WORDS};
#endif
NSX_HD const uint32_t *two_over_pi() {
#if defined(__CUDA_ARCH__)
    return k2OverPi_d;
#else
    return k2OverPi_h;
#endif
}

NSX_HD int clz32(uint32_t v) {   // v != 0
#if defined(__CUDA_ARCH__)
    return __clz((int)v);
#else
    return __builtin_clz(v);
#endif
}

// Bits [lo, lo + 64) of the 256-bit little-endian value L (zero below bit 0).
NSX_HD uint64_t window64(const uint32_t *L, int lo) {
    int shift = 0;
    if (lo < 0) {
        if (lo <= -64) return 0;
        shift = -lo;
        lo = 0;
    }
    const int w = lo >> 5, s = lo & 31;
    const uint64_t a = (uint64_t)L[w] | ((uint64_t)(w + 1 < 8 ? L[w + 1] : 0u) << 32);
    const uint64_t c = w + 2 < 8 ? L[w + 2] : 0u;
    const uint64_t v = s ? (a >> s) | (c << (64 - s)) : a;
    return v << shift;
}

// |x| (binary32 bits u, finite, above pi/4) = (4j + q) pi/2 + r.
NSX_COLD dd reduce_pio2(uint32_t u, int *quadrant) {
    const uint32_t *W = two_over_pi();
    const uint64_t m = (u & 0x7fffffu) | 0x800000u;
    const int E = (int)(u >> 23) - 150;                 // |x| = m 2^E
    const int i0 = E >= 2 ? (E - 2) >> 5 : 0;           // earlier words add multiples of 4
    uint64_t p[6];
    for (int k = 0; k < 6; ++k) p[k] = m * W[i0 + k];
    uint32_t L[8];                                      // S = sum_k p[k] 2^(32 (5 - k))
    uint64_t acc = 0;
    for (int j = 0; j < 7; ++j) {
        if (j <= 5) acc += p[5 - j] & 0xffffffffu;
        if (j >= 1) acc += p[6 - j] >> 32;
        L[j] = (uint32_t)acc;
        acc >>= 32;
    }
    L[7] = (uint32_t)acc;
    const int sh = 32 * (i0 + 6) - E;                   // fraction bits of S, 159..216
    int q = (int)((L[sh >> 5] >> (sh & 31)) & 1u);
    q |= (int)((L[(sh + 1) >> 5] >> ((sh + 1) & 31)) & 1u) << 1;
    for (int j = 0; j < 8; ++j) {                       // keep the fraction F = S mod 2^sh
        const int lo = 32 * j;
        if (lo >= sh) L[j] = 0;
        else if (lo + 32 > sh) L[j] &= (1u << (sh - lo)) - 1u;
    }
    const bool neg = (L[(sh - 1) >> 5] >> ((sh - 1) & 31)) & 1u;   // F >= 1/2: r = (F - 1) pi/2
    if (neg) {
        q = (q + 1) & 3;
        uint64_t c = 1;                                 // 2^sh - F
        for (int j = 0; j < 8; ++j) {
            c += (uint64_t)(uint32_t)~L[j];
            L[j] = (uint32_t)c;
            c >>= 32;
        }
        for (int j = 0; j < 8; ++j) {
            const int lo = 32 * j;
            if (lo >= sh) L[j] = 0;
            else if (lo + 32 > sh) L[j] &= (1u << (sh - lo)) - 1u;
        }
    }
    *quadrant = q;
    int top = -1;
    for (int j = 7; j >= 0 && top < 0; --j)
        if (L[j]) top = 32 * j + 31 - clz32(L[j]);
    if (top < 0) return dd{0.0, 0.0};
    const uint64_t mask53 = (1ull << 53) - 1ull;
    const double a = (double)(window64(L, top - 52) & mask53);
    const double b = (double)(window64(L, top - 105) & mask53);
    const double fa = a * bitsd((uint64_t)(int64_t)(1023 + top - 52 - sh) << 52);
    const double fb = b * bitsd((uint64_t)(int64_t)(1023 + top - 105 - sh) << 52);
    dd r = dd_mul(fast_two_sum(fa, fb), dd{NSX_PIO2_HI, NSX_PIO2_LO});
    if (neg) { r.hi = -r.hi; r.lo = -r.lo; }
    return r;
}

// sin(r) (odd = 1) or cos(r) (odd = 0) for |r| <= pi/4 in double-double.
NSX_COLD float sincos_slow(dd r, bool odd, bool negate) {
    const double *c = inv_fact_dd();
    const dd z = dd_mul(r, r);
    int n = odd ? NSX_INV_FACT_COUNT - 2 : NSX_INV_FACT_COUNT - 1;   // 23 or 24
    dd p = {c[2 * n], c[2 * n + 1]};
    if ((n / 2) & 1) { p.hi = -p.hi; p.lo = -p.lo; }
    for (n -= 2; n >= 0; n -= 2) {
        dd t = {c[2 * n], c[2 * n + 1]};
        if ((n / 2) & 1) { t.hi = -t.hi; t.lo = -t.lo; }
        p = dd_add(dd_mul(p, z), t);
    }
    if (odd) p = dd_mul(p, r);
    if (negate) { p.hi = -p.hi; p.lo = -p.lo; }
    return round_dd_to_float(p.hi, p.lo);
}

// Correctly rounded sin (odd = 1) or cos (odd = 0) of binary32 x.
NSX_HD float sincosf_cr(float x, bool want_sin) {
    const uint32_t u = fbits(x) & 0x7fffffffu;
    if (u >= 0x7f800000u) return (x - x) / (x - x);     // NaN, +-inf: NaN
    if (u == 0u) return want_sin ? x : 1.0f;
    const bool xneg = fbits(x) >> 31;
    int q = 0;
    dd r;
    if (u <= 0x3f490fdau) r = dd{(double)bitsf(u), 0.0};  // |x| < pi/4
    else r = reduce_pio2(u, &q);
    const bool odd = want_sin ? (q & 1) == 0 : (q & 1) != 0;
    bool negate = want_sin ? (q >= 2) != xneg : (q == 1 || q == 2);
    const double rh = r.hi, rl = r.lo, z = rh * rh;
    double y;
    if (odd) {
        double s = dfma(z, 1.0 / 355687428096000.0, -1.0 / 1307674368000.0);
        s = dfma(z, s, 1.0 / 6227020800.0);
        s = dfma(z, s, -1.0 / 39916800.0);
        s = dfma(z, s, 1.0 / 362880.0);
        s = dfma(z, s, -1.0 / 5040.0);
        s = dfma(z, s, 1.0 / 120.0);
        s = dfma(z, s, -1.0 / 6.0);
        y = rh + dfma(rh * z, s, rl);                   // sin(rh + rl) ~ sin rh + rl
    } else {
        double s = dfma(z, 1.0 / 6402373705728000.0, -1.0 / 20922789888000.0);
        s = dfma(z, s, 1.0 / 87178291200.0);
        s = dfma(z, s, -1.0 / 479001600.0);
        s = dfma(z, s, 1.0 / 3628800.0);
        s = dfma(z, s, -1.0 / 40320.0);
        s = dfma(z, s, 1.0 / 720.0);
        s = dfma(z, s, -1.0 / 24.0);
        s = dfma(z, s, 0.5);
        y = 1.0 - dfma(z, s, rh * rl);                  // cos(rh + rl) ~ cos rh - rh rl
    }
    const double ay = y < 0 ? -y : y;
    if (ay < 0x1p-126 || near_midpoint(ay, 64)) return sincos_slow(r, odd, negate);
    return negate ? -(float)y : (float)y;
}
NSX_HD float sinf_cr(float x) { return sincosf_cr(x, true); }
NSX_HD float cosf_cr(float x) { return sincosf_cr(x, false); }

// Correctly rounded hypot of binary32 x, y (C99 special cases: an infinite
// argument gives +inf even with a NaN, otherwise NaN propagates).
NSX_HD float hypotf_cr(float x, float y) {
    const uint32_t ux = fbits(x) & 0x7fffffffu, uy = fbits(y) & 0x7fffffffu;
    if (ux == 0x7f800000u || uy == 0x7f800000u) return f32_inf();
    if (ux > 0x7f800000u || uy > 0x7f800000u) return x + y;
    const double a = (double)x * (double)x, b = (double)y * (double)y;   // exact
    const double h = sqrt(a + b);
    if (h >= 0x1p-126 && !near_midpoint(h, 16)) return (float)h;
    if (h == 0.0) return 0.0f;
    // The binary32 neighbours f, g around h and their midpoint (exact in
    // binary64; +inf stands for 2^128 as round-to-nearest treats it).
    const float f = (float)h;
    const double fd = fbits(f) == 0x7f800000u ? 0x1p128 : (double)f;
    if (fd == h) return f;
    const float g = bitsf(fd < h ? fbits(f) + 1u : fbits(f) - 1u);
    const double gd = fbits(g) == 0x7f800000u ? 0x1p128 : (double)g;
    const double mid = 0.5 * (fd + gd);
    const dd s = two_sum(a, b);                         // x^2 + y^2 exactly
    const double d = mid * mid - s.hi;                  // exact: mid^2 has <= 50 bits, close to s.hi
    const float below = fd < gd ? f : g, above = fd < gd ? g : f;
    if (d > s.lo) return below;
    if (d < s.lo) return above;
    return (fbits(f) & 1u) ? g : f;                     // exact midpoint: even
}

}  // namespace nsx
