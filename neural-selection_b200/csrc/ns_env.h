// Device-resident pole-on-cart environment for the serving loop, with the
// Gym adapter's observation encoding and action decoding, host and device.
//
// Every function here is written so that the host build (x86-64 SSE2 double,
// -ffp-contract=off) and the device build (--fmad=false) perform the same
// IEEE-754 operations in the same order, so episodes give bit-identical
// results on either side: exp, tanh, sin and cos are this file's own
// polynomial evaluations (Taylor series after Cody-Waite reduction), not the
// platform math library, whose last-place rounding differs between glibc and
// CUDA.
//
// Dynamics: the classic cart-pole of Barto, Sutton & Anderson (1983) in the
// form Gymnasium's CartPole uses (gravity 9.8, cart 1.0 kg, pole 0.1 kg, half
// length 0.5 m, force 10 N, explicit Euler with tau = 0.02 s, failure at
// |x| > 2.4 m or |theta| > 12 degrees).
// Encoding: gym_adapter/adapter.py:153-169 (opponent code of tanh((x - c)/s)
// of the float32 observation, two channels per dimension).
// Decoding: gym_adapter/gpu.py:66-83 and adapter.py:171-176 (smoothed spike
// counts activity = activity*(1-s) + s*spikes; the larger of two wins; a tie
// is a coin flip, drawn here from Philox4x32-10 instead of NumPy's PCG64).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define NSE_HD __host__ __device__ __forceinline__
#else
#define NSE_HD inline
#endif

namespace nse {

// ---- Philox4x32-10 (Salmon et al., SC'11) -----------------------------------
struct U4 { uint32_t x, y, z, w; };
NSE_HD uint32_t mulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }
NSE_HD U4 philox(U4 c, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint32_t h0 = mulhi32(0xD2511F53u, c.x), l0 = 0xD2511F53u * c.x;
        const uint32_t h1 = mulhi32(0xCD9E8D57u, c.z), l1 = 0xCD9E8D57u * c.z;
        c = U4{h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0};
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return c;
}
// Uniform [0, 1) from the top 24 bits (exact in double).
NSE_HD double unit24(uint32_t w) { return (double)(w >> 8) * (1.0 / 16777216.0); }

constexpr uint32_t kKeyInit = 0xCA27901Eu;   // stream of initial states (counter: reset index)
constexpr uint32_t kKeyTie = 0x7E1B0C11u;    // stream of tie-breaking coin flips (counter: step)

// ---- deterministic binary64 elementary functions ----------------------------
constexpr double kLn2Hi = 0x1.62e42ff000000p-1;     // ln 2 to 32 bits: k*kLn2Hi exact for |k| < 2^21
constexpr double kLn2Lo = -0x1.718432a1b0e26p-35;   // ln 2 - kLn2Hi
constexpr double kInvLn2 = 1.4426950408889634;
constexpr double kPio2Hi = 0x1.921fb54400000p+0;    // pi/2 to 33 bits
constexpr double kPio2Lo = 0x1.0b4611a626331p-34;   // pi/2 - kPio2Hi
constexpr double kTwoOverPi = 0.6366197723675814;

NSE_HD double round_half_even(double x) {
    // x in (-2^51, 2^51): adding and subtracting 1.5*2^52 rounds to an integer
    // in round-to-nearest-even.
    const double big = 6755399441055744.0;
    return (x + big) - big;
}

NSE_HD double scale2(double v, int k) {
    // v * 2^k for a result in the normal range, k in [-1022, 1023].
    union { double d; uint64_t u; } s;
    s.u = (uint64_t)(k + 1023) << 52;
    return v * s.d;
}

// e^x for |x| <= 700: x = k ln 2 + r, |r| <= ln2/2, Taylor series of degree 13.
NSE_HD double det_exp(double x) {
    if (x > 700.0) x = 700.0;
    if (x < -700.0) x = -700.0;
    const double k = round_half_even(x * kInvLn2);
    const double r = (x - k * kLn2Hi) - k * kLn2Lo;
    double p = 1.6059043836821613e-10;          // 1/13!
    p = p * r + 2.08767569878681e-09;           // 1/12!
    p = p * r + 2.505210838544172e-08;
    p = p * r + 2.755731922398589e-07;
    p = p * r + 2.7557319223985893e-06;
    p = p * r + 2.48015873015873e-05;
    p = p * r + 0.0001984126984126984;
    p = p * r + 0.001388888888888889;
    p = p * r + 0.008333333333333333;
    p = p * r + 0.041666666666666664;
    p = p * r + 0.16666666666666666;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return scale2(p, (int)k);
}

NSE_HD double det_tanh(double z) {
    const double a = z < 0 ? -z : z;
    double t;
    if (a > 20.0) t = 1.0;
    else if (a < 1.0 / 268435456.0) t = a;      // 2^-28
    else t = 1.0 - 2.0 / (det_exp(2.0 * a) + 1.0);
    return z < 0 ? -t : t;
}

// sin and cos of r, |r| <= pi/4 (+ margin): Taylor series to degree 17 / 18.
NSE_HD double sin_poly(double r) {
    const double q = r * r;
    double p = 2.8114572543455206e-15;          // 1/17!
    p = p * q - 7.647163731819816e-13;          // 1/15!
    p = p * q + 1.6059043836821613e-10;
    p = p * q - 2.505210838544172e-08;
    p = p * q + 2.7557319223985893e-06;
    p = p * q - 0.0001984126984126984;
    p = p * q + 0.008333333333333333;
    p = p * q - 0.16666666666666666;
    return r + r * q * p;
}
NSE_HD double cos_poly(double r) {
    const double q = r * r;
    double p = 1.5619206968586225e-16;          // 1/18!
    p = p * q - 4.779477332387385e-14;          // 1/16!
    p = p * q + 1.1470745597729725e-11;
    p = p * q - 2.08767569878681e-09;
    p = p * q + 2.755731922398589e-07;
    p = p * q - 2.48015873015873e-05;
    p = p * q + 0.001388888888888889;
    p = p * q - 0.041666666666666664;
    p = p * q + 0.5;
    return 1.0 - q * p;
}
// sin and cos of x, |x| < 1e6: x = k pi/2 + r.
NSE_HD void det_sincos(double x, double *s, double *c) {
    const double k = round_half_even(x * kTwoOverPi);
    const double r = (x - k * kPio2Hi) - k * kPio2Lo;
    const double sr = sin_poly(r), cr = cos_poly(r);
    switch (((long long)k) & 3) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
    }
}

// ---- cart-pole ------------------------------------------------------------------
struct Cart { double x, xd, th, thd; };

constexpr double kThetaLimit = 0.20943951023931953;   // 12 * 2 * pi / 360
constexpr double kXLimit = 2.4;

NSE_HD Cart cart_initial(uint32_t seed, uint32_t reset_index) {
    const U4 w = philox(U4{reset_index, 0u, 0u, 0u}, seed, kKeyInit);
    return Cart{-0.05 + 0.1 * unit24(w.x), -0.05 + 0.1 * unit24(w.y), -0.05 + 0.1 * unit24(w.z),
                -0.05 + 0.1 * unit24(w.w)};
}

// One Euler step of 20 ms; returns true when the pole has fallen or the cart left the track.
NSE_HD bool cart_step(Cart &s, int action) {
    const double force = action ? 10.0 : -10.0;
    double sn, cs;
    det_sincos(s.th, &sn, &cs);
    const double temp = (force + 0.05 * s.thd * s.thd * sn) / 1.1;
    const double thacc = (9.8 * sn - cs * temp) / (0.5 * (4.0 / 3.0 - 0.1 * cs * cs / 1.1));
    const double xacc = temp - 0.05 * thacc * cs / 1.1;
    s.x = s.x + 0.02 * s.xd;
    s.xd = s.xd + 0.02 * xacc;
    s.th = s.th + 0.02 * s.thd;
    s.thd = s.thd + 0.02 * thacc;
    return s.x < -kXLimit || s.x > kXLimit || s.th < -kThetaLimit || s.th > kThetaLimit;
}

// Opponent code of the float32 observation into 8 channels. Scales are the
// bounds of the observation box (float32 4.8 m and 24 degrees); unbounded
// velocities use scale 1; every centre is 0.
NSE_HD void cart_encode(const Cart &s, float *out) {
    const double kScale[4] = {4.800000190734863, 1.0, 0.41887903213500977, 1.0};
    const double obs[4] = {(double)(float)s.x, (double)(float)s.xd, (double)(float)s.th, (double)(float)s.thd};
    for (int i = 0; i < 4; ++i) {
        const double sg = det_tanh(obs[i] / kScale[i]);
        out[2 * i] = (float)((1.0 + sg) / 2.0);
        out[2 * i + 1] = (float)((1.0 - sg) / 2.0);
    }
}

// Smoothed motor activity and the chosen action (0 or 1). keep and smoothing
// are the float32 values of 1 - s and s (NumPy casts both Python floats to
// float32 before the array arithmetic).
NSE_HD int decode_action(float &a0, float &a1, float spikes0, float spikes1, float keep, float smoothing,
                         uint32_t seed, uint32_t step) {
    a0 = a0 * keep; a1 = a1 * keep;
    a0 = a0 + smoothing * spikes0; a1 = a1 + smoothing * spikes1;
    if (a0 > a1) return 0;
    if (a1 > a0) return 1;
    return (int)(philox(U4{step, 0u, 0u, 0u}, seed, kKeyTie).x & 1u);
}

// FNV-1a accumulation of one step's action and motor counts (episode trace).
NSE_HD uint32_t trace_step(uint32_t h, int action, float spikes0, float spikes1) {
    const uint32_t v[3] = {(uint32_t)action, (uint32_t)spikes0, (uint32_t)spikes1};
    for (int i = 0; i < 3; ++i)
        for (int b = 0; b < 4; ++b) { h ^= (v[i] >> (8 * b)) & 0xffu; h *= 16777619u; }
    return h;
}

}  // namespace nse
