/* ORACLE — test infrastructure only. Not linked into, or called by, the
 * product library.
 *
 * Correctly rounded binary32 exp and log for the oracle, written independently
 * of the product's binary64 implementation so the two can check each other.
 *
 * Method: evaluate with glibc's binary64 exp/log (relative error < 2^-51);
 * if the result +-2^-48 rounds to one binary32 value, that value is correctly
 * rounded. Otherwise evaluate in x87 80-bit long double (glibc expl/logl, error
 * < 2^-62 relative). If the long-double result brackets a unique binary32 value within
 * a 2^-58 relative margin, that value is the correctly rounded result. Otherwise
 * re-evaluate in IEEE binary128 (libquadmath expq/logq, error < 2^-110) with a
 * 2^-100 margin. A remaining ambiguity aborts (none exists for binary32 inputs;
 * the exhaustive test would report it).
 *
 * The reference calls expf/logf in src/physiology.cuh:215,227,266,271,309,
 * 369,371,411,419,429,431,434,514-515,537-538,576-577,581-582, src/lp_cell.cuh
 * and src/prinz_cell.cuh; the oracle binds all of those to or_cr_expf /
 * or_cr_logf in its default build.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <quadmath.h>

static float bracket_ld(long double y, long double margin, int *ok) {
    float lo = (float)(y * (1.0L - margin));
    float hi = (float)(y * (1.0L + margin));
    *ok = memcmp(&lo, &hi, sizeof lo) == 0;
    return lo;
}

static float bracket_d(double y, double margin, int *ok) {
    float lo = (float)(y * (1.0 - margin));
    float hi = (float)(y * (1.0 + margin));
    *ok = memcmp(&lo, &hi, sizeof lo) == 0;
    return lo;
}

static float bracket_q(__float128 y, __float128 margin, int *ok) {
    float lo = (float)(y * (1 - margin));
    float hi = (float)(y * (1 + margin));
    *ok = memcmp(&lo, &hi, sizeof lo) == 0;
    return lo;
}

float or_cr_expf(float x) {
    if (isnan(x)) return x + x;
    if (isinf(x)) return x > 0 ? x : 0.0f;
    int ok;
    /* glibc's binary64 exp: relative error < 2^-51; bracket at 2^-48. */
    float r = bracket_d(exp((double)x), 0x1p-48, &ok);
    if (ok) return r;
    long double y = expl((long double)x);
    r = bracket_ld(y, 0x1p-58L, &ok);
    if (ok) return r;
    __float128 q = expq((__float128)x);
    r = bracket_q(q, 0x1p-100Q, &ok);
    if (ok) return r;
    abort();
}

float or_cr_logf(float x) {
    if (isnan(x)) return x + x;
    if (x < 0) return (x - x) / (x - x);
    if (x == 0) return -INFINITY;
    if (isinf(x)) return x;
    if (x == 1.0f) return 0.0f;
    int ok;
    float r = bracket_d(log((double)x), 0x1p-48, &ok);
    if (ok) return r;
    long double y = logl((long double)x);
    r = bracket_ld(y, 0x1p-58L, &ok);
    if (ok) return r;
    __float128 q = logq((__float128)x);
    r = bracket_q(q, 0x1p-100Q, &ok);
    if (ok) return r;
    abort();
}

/* sin, cos, hypot for the reference world's body and sense kernels
 * (src/main.cu:619-657, 1146-1249), bracketed the same way: glibc binary64
 * (error below 1 ulp of binary64), then x87 long double, then binary128. */
float or_cr_sinf(float x) {
    if (isnan(x) || isinf(x)) return (x - x) / (x - x);
    if (x == 0) return x;
    int ok;
    float r = bracket_d(sin((double)x), 0x1p-48, &ok);
    if (ok) return r;
    r = bracket_ld(sinl((long double)x), 0x1p-58L, &ok);
    if (ok) return r;
    r = bracket_q(sinq((__float128)x), 0x1p-100Q, &ok);
    if (ok) return r;
    abort();
}

float or_cr_cosf(float x) {
    if (isnan(x) || isinf(x)) return (x - x) / (x - x);
    int ok;
    float r = bracket_d(cos((double)x), 0x1p-48, &ok);
    if (ok) return r;
    r = bracket_ld(cosl((long double)x), 0x1p-58L, &ok);
    if (ok) return r;
    r = bracket_q(cosq((__float128)x), 0x1p-100Q, &ok);
    if (ok) return r;
    abort();
}

float or_cr_hypotf(float x, float y) {
    if (isinf(x) || isinf(y)) return INFINITY;
    if (isnan(x) || isnan(y)) return x + y;
    if (x == 0 && y == 0) return 0.0f;
    int ok;
    float r = bracket_d(hypot((double)x, (double)y), 0x1p-48, &ok);
    if (ok) return r;
    r = bracket_ld(hypotl((long double)x, (long double)y), 0x1p-58L, &ok);
    if (ok) return r;
    /* x^2 and y^2 are exact in binary128; an exact midpoint (possible for
     * sums of squares) is settled by comparing squares exactly. */
    __float128 xq = x, yq = y, q = sqrtq(xq * xq + yq * yq);
    r = bracket_q(q, 0x1p-100Q, &ok);
    if (ok) return r;
    float lo = (float)(q * (1 - 0x1p-100Q)), hi = (float)(q * (1 + 0x1p-100Q));
    __float128 mid = ((__float128)lo + (__float128)hi) / 2, s = xq * xq + yq * yq;
    if (mid * mid < s) return hi;
    if (mid * mid > s) return lo;
    uint32_t lb; memcpy(&lb, &lo, 4);
    return (lb & 1u) ? hi : lo;
}
