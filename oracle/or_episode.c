/* ORACLE — test infrastructure only (see ns_oracle.h).
 *
 * One genome-evaluation episode on the CPU: the brain stepped by or_step
 * (ns_step semantics, 16 ticks per environment step) and the pole-on-cart
 * environment of the serving loop, with the Gym adapter's observation encoding
 * (gym_adapter/adapter.py:153-169) and smoothed two-action decoding
 * (gym_adapter/gpu.py:66-83, adapter.py:171-176).
 *
 * The environment's arithmetic is a definition shared with the library: its
 * exp/tanh/sin/cos are fixed polynomial evaluations in binary64 (Taylor
 * series after Cody-Waite reduction by ln 2 and pi/2) and the cart-pole step is
 * the Barto-Sutton-Anderson model as Gymnasium writes it, so that the CPU and
 * the GPU produce the same bits. Built with -ffp-contract=off.
 */
#include "ns_oracle.h"

#include <string.h>

/* ---- Philox4x32-10 -------------------------------------------------------- */
typedef struct { uint32_t v[4]; } ep_u4;
static ep_u4 ep_philox(uint32_t c0, uint32_t k0, uint32_t k1) {
    uint32_t x = c0, y = 0, z = 0, w = 0;
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * x, p1 = (uint64_t)0xCD9E8D57u * z;
        const uint32_t nx = (uint32_t)(p1 >> 32) ^ y ^ k0, ny = (uint32_t)p1;
        const uint32_t nz = (uint32_t)(p0 >> 32) ^ w ^ k1, nw = (uint32_t)p0;
        x = nx; y = ny; z = nz; w = nw;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    ep_u4 o = {{x, y, z, w}};
    return o;
}
static double ep_unit24(uint32_t w) { return (double)(w >> 8) * (1.0 / 16777216.0); }
#define EP_KEY_INIT 0xCA27901Eu
#define EP_KEY_TIE 0x7E1B0C11u

/* ---- binary64 polynomial elementary functions ---------------------------- */
static double ep_round(double x) { const double big = 6755399441055744.0; return (x + big) - big; }
static double ep_scale2(double v, int k) {
    union { double d; uint64_t u; } s;
    s.u = (uint64_t)(k + 1023) << 52;
    return v * s.d;
}
static double ep_exp(double x) {
    static const double c[14] = {1.0, 1.0, 0.5, 0.16666666666666666, 0.041666666666666664, 0.008333333333333333,
                                 0.001388888888888889, 0.0001984126984126984, 2.48015873015873e-05,
                                 2.7557319223985893e-06, 2.755731922398589e-07, 2.505210838544172e-08,
                                 2.08767569878681e-09, 1.6059043836821613e-10};
    if (x > 700.0) x = 700.0;
    if (x < -700.0) x = -700.0;
    const double k = ep_round(x * 1.4426950408889634);
    const double r = (x - k * 0x1.62e42ff000000p-1) - k * -0x1.718432a1b0e26p-35;
    double p = c[13];
    for (int i = 12; i >= 0; --i) p = p * r + c[i];
    return ep_scale2(p, (int)k);
}
static double ep_tanh(double z) {
    const double a = z < 0 ? -z : z;
    double t;
    if (a > 20.0) t = 1.0;
    else if (a < 1.0 / 268435456.0) t = a;
    else t = 1.0 - 2.0 / (ep_exp(2.0 * a) + 1.0);
    return z < 0 ? -t : t;
}
static void ep_sincos(double x, double *s, double *c) {
    /* odd / even Taylor coefficients 1/n! with alternating signs */
    static const double sc[8] = {-0.16666666666666666, 0.008333333333333333, -0.0001984126984126984,
                                 2.7557319223985893e-06, -2.505210838544172e-08, 1.6059043836821613e-10,
                                 -7.647163731819816e-13, 2.8114572543455206e-15};
    static const double cc[9] = {0.5, -0.041666666666666664, 0.001388888888888889, -2.48015873015873e-05,
                                 2.755731922398589e-07, -2.08767569878681e-09, 1.1470745597729725e-11,
                                 -4.779477332387385e-14, 1.5619206968586225e-16};
    const double k = ep_round(x * 0.6366197723675814);
    const double r = (x - k * 0x1.921fb54400000p+0) - k * 0x1.0b4611a626331p-34;
    const double q = r * r;
    double ps = sc[7];
    for (int i = 6; i >= 0; --i) ps = ps * q + sc[i];
    double pc = cc[8];
    for (int i = 7; i >= 0; --i) pc = pc * q + cc[i];
    const double sr = r + r * q * ps, cr = 1.0 - q * pc;
    switch (((long long)k) & 3) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
    }
}

/* ---- cart-pole ------------------------------------------------------------------ */
typedef struct { double x, xd, th, thd; } ep_cart;
static ep_cart ep_initial(uint32_t seed, uint32_t reset_index) {
    const ep_u4 w = ep_philox(reset_index, seed, EP_KEY_INIT);
    ep_cart c = {-0.05 + 0.1 * ep_unit24(w.v[0]), -0.05 + 0.1 * ep_unit24(w.v[1]), -0.05 + 0.1 * ep_unit24(w.v[2]),
                 -0.05 + 0.1 * ep_unit24(w.v[3])};
    return c;
}
static int ep_step(ep_cart *s, int action) {
    const double force = action ? 10.0 : -10.0;
    double sn, cs;
    ep_sincos(s->th, &sn, &cs);
    const double temp = (force + 0.05 * s->thd * s->thd * sn) / 1.1;
    const double thacc = (9.8 * sn - cs * temp) / (0.5 * (4.0 / 3.0 - 0.1 * cs * cs / 1.1));
    const double xacc = temp - 0.05 * thacc * cs / 1.1;
    s->x = s->x + 0.02 * s->xd;
    s->xd = s->xd + 0.02 * xacc;
    s->th = s->th + 0.02 * s->thd;
    s->thd = s->thd + 0.02 * thacc;
    return s->x < -2.4 || s->x > 2.4 || s->th < -0.20943951023931953 || s->th > 0.20943951023931953;
}
static void ep_encode(const ep_cart *s, float *out) {
    static const double scale[4] = {4.800000190734863, 1.0, 0.41887903213500977, 1.0};
    const double obs[4] = {(double)(float)s->x, (double)(float)s->xd, (double)(float)s->th, (double)(float)s->thd};
    for (int i = 0; i < 4; ++i) {
        const double sg = ep_tanh(obs[i] / scale[i]);
        out[2 * i] = (float)((1.0 + sg) / 2.0);
        out[2 * i + 1] = (float)((1.0 - sg) / 2.0);
    }
}
static uint32_t ep_trace(uint32_t h, int action, float s0, float s1) {
    const uint32_t v[3] = {(uint32_t)action, (uint32_t)s0, (uint32_t)s1};
    for (int i = 0; i < 3; ++i)
        for (int b = 0; b < 4; ++b) { h ^= (v[i] >> (8 * b)) & 0xffu; h *= 16777619u; }
    return h;
}

double or_env_exp(double x) { return ep_exp(x); }
double or_env_tanh(double x) { return ep_tanh(x); }
void or_env_sincos(double x, double *s, double *c) { ep_sincos(x, s, c); }

int or_episode(or_brain *b, uint32_t seed, int steps, int ticks, float gain, double smoothing, int32_t *out) {
    if (or_count(b) < 1 || steps < 1) return -1;
    float input[8], motor[2];
    const float keep = (float)(1.0 - smoothing), sm = (float)smoothing;
    float a0 = 0.0f, a1 = 0.0f;
    int reward = 0, failures = 0, done = 0, status = 0;
    uint32_t trace = 2166136261u;
    or_reset(b, seed);
    ep_cart c = ep_initial(seed, 0u);
    ep_encode(&c, input);
    for (; done < steps; ++done) {
        if (or_step(b, input, ticks, gain, motor, NULL, 0) != 0) { status = -1; break; }
        a0 = a0 * keep; a1 = a1 * keep;
        a0 = a0 + sm * motor[0]; a1 = a1 + sm * motor[1];
        int action;
        if (a0 > a1) action = 0;
        else if (a1 > a0) action = 1;
        else action = (int)(ep_philox((uint32_t)done, seed, EP_KEY_TIE).v[0] & 1u);
        trace = ep_trace(trace, action, motor[0], motor[1]);
        if (ep_step(&c, action)) {
            ++failures;
            c = ep_initial(seed, (uint32_t)failures);
        } else {
            ++reward;
        }
        if (done + 1 < steps) ep_encode(&c, input);
    }
    out[0] = done; out[1] = reward; out[2] = failures; out[3] = (int32_t)trace; out[4] = status;
    return 0;
}

/* A fixed environment sequence for comparing host builds: 500 steps of the
 * action pattern (t / 7) & 1 from seed 12345 with resets on failure, an FNV
 * hash of every encoded observation, and 64 decoded actions of synthetic
 * motor counts. out = {bits of x, bits of theta_dot, hash, action code}. */
void or_env_sequence(uint64_t *out) {
    ep_cart cart = ep_initial(12345u, 0u);
    float enc[8];
    uint32_t h = 2166136261u;
    for (int t = 0; t < 500; ++t) {
        const int a = (t / 7) & 1;
        if (ep_step(&cart, a)) cart = ep_initial(12345u, (uint32_t)t + 1);
        ep_encode(&cart, enc);
        for (int i = 0; i < 8; ++i) { uint32_t u; memcpy(&u, &enc[i], 4); h = (h ^ u) * 16777619u; }
    }
    float a0 = 0, a1 = 0;
    uint32_t acts = 0;
    for (int t = 0; t < 64; ++t) {
        const float s0 = (float)(t % 3), s1 = (float)(t % 2);
        a0 = a0 * 0.6f; a1 = a1 * 0.6f;
        a0 = a0 + 0.4f * s0; a1 = a1 + 0.4f * s1;
        int action;
        if (a0 > a1) action = 0;
        else if (a1 > a0) action = 1;
        else action = (int)(ep_philox((uint32_t)t, 7u, EP_KEY_TIE).v[0] & 1u);
        acts = acts * 3u + (uint32_t)action;
    }
    memcpy(&out[0], &cart.x, 8);
    memcpy(&out[1], &cart.thd, 8);
    out[2] = h;
    out[3] = acts;
}
