// Device physiology of the neural tick (CUDA, sm_100a).
//
// The arithmetic restates the reference model (mixic/neural-selection
// src/physiology.cuh:206-586, src/lp_cell.cuh:28-113,
// src/prinz_cell.cuh:45-121) operation for operation: every binary32 add,
// multiply and divide happens in the reference's order with IEEE rounding
// (built with --fmad=false; divisions and square roots are IEEE), and every
// exponential/logarithm is correctly rounded (ns_crmath.h). Constant-argument
// and gene-constant exponentials are precomputed on the host with the same
// correctly rounded function. Together this makes the engine's results
// bit-identical to the CPU oracle.
#pragma once
#include <stdint.h>
#include "ns_crmath.h"
#include "ns_layout.h"

namespace nsb {

// Correctly rounded constant exponentials, identical for every engine (set by
// the host once per device).
static __constant__ PhysConst c_K;

struct NeuronRegs {
    float v, w, adp, inh, depol, rec_ns;
    uint32_t rng;
    float d0, d1, d2, d3;
    int total;
    uint32_t spike;
};

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }

__device__ __forceinline__ uint32_t xorshift32(uint32_t x) {
    x ^= x << 13; x ^= x >> 17; x ^= x << 5; return x;
}

__device__ __forceinline__ float crexp(float x, const float *tab) { return nsx::expf_cr_ff(x, tab); }

// The reference's uniform draws are u = (x >> 8) * 2^-24 for a 32-bit
// xorshift state x (physiology.cuh:211-213, 384-391), tested as u < p. Both
// u and p * 2^24 are exact binary32 values, so u < p holds exactly when the
// 24-bit integer x >> 8 is below ceil(p * 2^24); a NaN or non-positive p
// never passes. The integer test needs no int-to-float conversion per draw.
__device__ __forceinline__ uint32_t draw_threshold(float p) {
    const float t = p * 16777216.0f;
    if (!(t > 0.0f)) return 0u;
    if (t >= 16777216.0f) return 16777216u;
    return (uint32_t)ceilf(t);
}

// physiology.cuh:226-230: thin-branch input/output curve (type 0 only).
// When gs - 4 rounds to exactly -4 (|gs| below half an ulp of 4, about
// 2.4e-7: a branch decaying after its last input), the exponent -(gs - 4)/0.4
// is exactly 10, the same binary32 value as in the offset 5/(1 + exp(10)), so
// regen equals the offset bit for bit and the exponential is skipped.
__device__ __forceinline__ float branch_gain(float gs, float offset, const float *tab) {
    const float t = gs - 4.0f;
    const float regen = t == -4.0f ? offset : 5.0f / (1.0f + crexp(-t / 0.4f, tab));
    return fminf(11.0f, gs + regen - offset);
}

// physiology.cuh:206-219: receptor events (type 5 with a receptor channel).
__device__ __forceinline__ float receptor_drive(const float *g, uint32_t flags, NeuronRegs &s,
                                                float level) {
    if (!(flags & NF_GENE_SENS) || !(g[G_RECEVENT] > 0)) return 0.0f;
    float rate = clampf(g[G_RECBASE] + g[G_RECGAIN] * level, 0.0f, 1000.0f);
    s.rng = xorshift32(s.rng);
    s.rec_ns *= g[G_RECDECAY];
    if ((s.rng >> 8) < draw_threshold(rate * (1.0f / 1000.0f))) s.rec_ns += g[G_RECEVENT];
    return s.rec_ns * (0.0f - s.v);
}

// physiology.cuh:290-374, AdEx path (types 0, 1, 4, 5), four 0.25 ms substeps.
// exc0..3/inh_in: this tick's summed synaptic input.
__device__ __forceinline__ void adex_tick(const float *g, uint32_t type, uint32_t flags, NeuronRegs &s,
                                          float cur, float e0, float e1, float e2, float e3, float inh_in,
                                          const float *tab) {
    s.d0 += e0; s.d1 += e1; s.d2 += e2; s.d3 += e3;
    float sub = fmaxf(0.0f, fminf(s.v, -50.0f) - g[G_EL]);
    s.depol += 0.1f * (sub - s.depol);
    s.inh += inh_in;
    s.spike = 0;
    const float h = 0.25f;
    const float clamp_leak = 0.0f, clamp_rev = -68.0f;
#pragma unroll 1
    for (int step = 0; step < 4; ++step) {
        float v = s.v;
        s.w += h * (g[G_A] * (v - g[G_EL]) - s.w) / g[G_TAUW];
        float expo = clampf((v - g[G_VT]) / g[G_SLOPE], -20.0f, 10.0f);
        float soma;
        if (type == 0) {
            // branch_gain(0) is exactly +0 (its two exponentials are the same
            // value) and soma >= +0, so a branch with no conductance adds
            // nothing and is skipped; warps sorted by branch usage skip it
            // together.
            soma = 0.0f;
            if (s.d0 != 0.0f) soma += branch_gain(s.d0, c_K.dend_offset, tab);
            if (s.d1 != 0.0f) soma += branch_gain(s.d1, c_K.dend_offset, tab);
            if (s.d2 != 0.0f) soma += branch_gain(s.d2, c_K.dend_offset, tab);
            if (s.d3 != 0.0f) soma += branch_gain(s.d3, c_K.dend_offset, tab);
        } else {
            soma = 0.0f + s.d0;
            soma += s.d1; soma += s.d2; soma += s.d3;
        }
        float dv = g[G_GL] * (g[G_EL] - v) + g[G_GLSLOPE] * crexp(expo, tab) + soma * (0.0f - v) +
                   s.inh * (-75.0f - v) + cur + s.adp - s.w - clamp_leak * (v - clamp_rev);
        s.v = v + h * dv / g[G_CAP];
        if (s.v >= 0.0f) {
            s.spike = 1; ++s.total;
            s.v = g[G_VR]; s.w += g[G_B]; s.adp += g[G_ADPB];
        }
        if (flags & NF_ADP) s.adp *= g[G_ADPDECAY];
        s.d0 *= c_K.exc_sub; s.d1 *= c_K.exc_sub; s.d2 *= c_K.exc_sub; s.d3 *= c_K.exc_sub;
        s.inh *= c_K.inh_sub;
    }
}

// ---- LFS cell (physiology.cuh:258-287); x = {v, thr, act[3], open[3]} -------------
static __device__ __noinline__ void lfs_tick(const float *g, NeuronRegs &s, float *x, float cur, float exc, float inh) {
    const float wt[3] = {250.0f, 10.0f, 4.0f}, op[3] = {10.0f, 40.0f, 750.0f}, cl[3] = {50.0f, 750.0f, 2000.0f};
    x[1] = g[G_VT] + (x[1] - g[G_VT]) * c_K.lfs_thr;
    float under = 0;
    for (int j = 0; j < 3; ++j) {
        x[5 + j] += x[2 + j] / op[j] - x[5 + j] / cl[j];
        x[2 + j] *= c_K.lfs_open[j];
        under += wt[j] * x[5 + j];
    }
    const float v = x[0];
    const float i = g[G_GL] * (g[G_EL] - v) + exc * (10.0f - v) + inh * (-60.0f - v) + under * (-80.0f - v) + cur;
    x[0] = v + i / g[G_CAP];
    s.spike = x[0] >= x[1] ? 1u : 0u;
    if (s.spike) {
        x[1] = 200.0f;
        for (int j = 0; j < 3; ++j) x[2 + j] += 1.0f;
        ++s.total;
    }
    s.v = x[0];
}

// ---- LP cell (lp_cell.cuh:28-113) --------------------------------------------------
// The reference's sigmoid gates are 1 / (1 + exp((v - mid) / slope)) and its
// rate ratios num / den, or a limit when |den| < 1e-5; lp_rates and
// lp_rates_warp evaluate them in place, in batches.

// N independent quotients a[i] / b[i] (IEEE division). The compiled division
// was measured against straight-line alternatives on B200 (a binary64
// Newton-Raphson quotient rounded once; a binary32 Markstein quotient proved by
// its exact remainder): both gave the same bits and both were slower, since
// every reciprocal goes through the special-function unit and the proof adds
// a dozen dependent operations per quotient.
template <int N> __device__ __forceinline__ void fdiv_n(const float (&a)[N], const float (&b)[N], float (&q)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) q[i] = a[i] / b[i];
}

// N independent quotients on a warp: lane i < N divides a[i] by b[i] (the
// operands are the same in every lane) and shuffles give every lane all N,
// so the IEEE divisions run at once instead of one after another. All 32
// lanes call it together.
template <int N>
__device__ __forceinline__ void fdiv_warp(const float (&a)[N], const float (&b)[N], float (&q)[N], int lane) {
    float n = a[0], d = b[0];
#pragma unroll
    for (int i = 1; i < N; ++i) {
        n = lane == i ? a[i] : n;
        d = lane == i ? b[i] : d;
    }
    const float r = n / d;
#pragma unroll
    for (int i = 0; i < N; ++i) q[i] = __shfl_sync(0xffffffffu, r, i);
}

// Exponentials in the LP and Prinz models. A batch whose binary64 fallback
// (expf_cr_wide, an out-of-line call) sits inside the integration loop was
// measured 2.7 times slower per exponential on B200 than the same binary32
// fast paths alone, although the fallback almost never runs: the call's
// register contract weighs on the whole loop. So the models' hot loops use
// the fast paths alone (exp_n<false>), which report in `ok` whether every
// result stands; an integration step with any undecided exponential (about
// one argument in 8,000) is recomputed from its saved state by an out-of-line
// copy of the same step that uses crexp_n (exp_n<true>). The results are the
// correctly rounded ones either way.
//
// Correctly rounded exponentials of N independent arguments: every binary32
// fast path first, with no branch between them, so that they interleave;
// then the binary64 path for any argument that needs it (rare).
template <int N> __device__ __forceinline__ void crexp_n(const float (&x)[N], float (&y)[N], const float *tab) {
    bool ok[N];
    bool all = true;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        y[i] = nsx::expf_cr_fast(x[i], tab, ok[i]);
        all = all && ok[i];
    }
    if (!all) {
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (!ok[i]) y[i] = nsx::expf_cr_wide(x[i]);
    }
}
// SAFE: crexp_n. Otherwise the binary32 fast paths alone; `ok` is cleared when
// any of them is undecided (its result then must not be used).
template <bool SAFE, int N>
__device__ __forceinline__ void exp_n(const float (&x)[N], float (&y)[N], const float *tab, bool &ok) {
    if (SAFE) {
        crexp_n(x, y, tab);
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            bool oi;
            y[i] = nsx::expf_cr_fast(x[i], tab, oi);
            ok = ok && oi;
        }
    }
}
template <bool SAFE> __device__ __forceinline__ float exp1(float x, const float *tab, bool &ok) {
    if (SAFE) return crexp(x, tab);
    bool oi;
    const float y = nsx::expf_cr_fast(x, tab, oi);
    ok = ok && oi;
    return y;
}

// lp_rates with its 21 exponentials computed as one batch (crexp_n) and its
// 40 quotients as three (fdiv_n: the exponents' arguments; the sigmoids and
// ratios; the three that use those). Every argument, sigmoid and assembly is
// the reference's operation in its order; x / 4 and x / 8 are written as the
// products by 0.25 and 0.125, which round the same exact value.
template <bool SAFE>
__device__ __forceinline__ void lp_rates(const float (&x)[16], float i_na, const float (&sc)[4], float (&d)[16],
                                         const float *tab, bool &ok) {
    const float va = x[0], vs = x[15], cai = x[13];
    float N1[17], D1[17], Q1[17];
    N1[0] = vs;                          D1[0] = 11.4866f;
    N1[1] = vs - 55.0f;                  D1[1] = -15.0f;
    N1[2] = va;                          D1[2] = 5.0f;
    N1[3] = va;                          D1[3] = 18.0f;
    N1[4] = va;                          D1[4] = 40.0f;
    N1[5] = vs - 15.0f;                  D1[5] = -9.8f;
    N1[6] = vs - -40.0f;                 D1[6] = 3.2f;
    N1[7] = vs - -15.0f;                 D1[7] = -10.0f;
    N1[8] = vs - 29.1336f;               D1[8] = -4.43083f;
    N1[9] = vs - -.6f * cai;             D1[9] = -23.0f;
    N1[10] = vs - (-16.0f - .6f * cai);  D1[10] = -5.0f;
    N1[11] = vs - -12.0f;                D1[11] = -26.0f;
    N1[12] = vs - -62.0f;                D1[12] = 6.0f;
    N1[13] = vs - -40.0f;                D1[13] = -12.0f;
    N1[14] = vs - -110.0f;               D1[14] = -21.6f;
    N1[15] = va - -26.9916223f;          D1[15] = -5.957441281f;
    N1[16] = va - -60.57875745f;         D1[16] = -13.25674673f;
    fdiv_n(N1, D1, Q1);
    float A[21], E[21];
    A[0] = Q1[0];
    A[1] = Q1[1];
    A[2] = -13.0f - va * 0.25f;          // va / 4
    A[3] = Q1[2] + 5.0f;
    A[4] = -2.66666666667f - Q1[3];
    A[5] = -5.0f - Q1[2];
    A[6] = -10.0f - Q1[2];
    A[7] = -1.375f - Q1[4];
    A[8] = Q1[5];
    A[9] = Q1[6];
    A[10] = Q1[7];
    A[11] = Q1[8];
    A[12] = Q1[9];
    A[13] = Q1[10];
    A[14] = Q1[11];
    A[15] = Q1[12];
    A[16] = Q1[13];
    A[17] = (vs - -70.0f) * 0.125f;      // (vs + 70) / 8
    A[18] = Q1[14];
    A[19] = Q1[15];
    A[20] = Q1[16];
    exp_n<SAFE>(A, E, tab, ok);
    const float na = x[1] * x[1] * x[1] * x[2] * 7.15f * (va - 50.0f);
    const float kd = x[8] * x[8] * x[8] * x[8] * 1.43f * (va + 72.0f);
    const float km = .2613041227f * x[14] * (va + 80.0f);
    const float aleak = sc[3] * .001004288227f * (va + 50.0f);
    const float cpl = .004017089073f * (vs - va);
    const float ev = E[0];
    // the sigmoids 1 / (1 + E[i]) of i = 1, 8..20 (Q2[0], Q2[i - 7]), the GHK
    // quotient, the rate ratios, the calcium-dependent quotient and d[0]
    float N2[21], D2[21], Q2[21];
    N2[0] = 1.0f;                                D2[0] = 1.0f + E[1];
#pragma unroll
    for (int i = 8; i <= 20; ++i) { N2[i - 7] = 1.0f; D2[i - 7] = 1.0f + E[i]; }
    N2[14] = vs * (x[13] * ev - 15123.5f);       D2[14] = ev - 1.0f;
    N2[15] = -16.64f - .32f * va;                D2[15] = E[2] - 1.0f;
    N2[16] = .28f * va + 7.0f;                   D2[16] = E[3] - 1.0f;
    N2[17] = 4.0f;                               D2[17] = E[5] + 1.0f;
    N2[18] = -1.6f - .032f * va;                 D2[18] = E[6] - 1.0f;
    N2[19] = .7f;                                D2[19] = .6f + cai;
    N2[20] = -na - kd - km - aleak + cpl;        D2[20] = .1148312178f;
    fdiv_n(N2, D2, Q2);
    auto sig = [&](int i) { return i == 1 ? Q2[0] : Q2[i - 7]; };
    d[0] = Q2[20];
    const float ghk = fabsf(vs) < .001f ? 11.4866f * (x[13] - 15123.5f) : Q2[14];
    const float ca = sc[0] * (x[3] * x[4] * .1247796343f + x[5] * .07142141077f) * .00155982f * ghk * .9f;
    const float kca = sc[1] * x[6] * x[7] * 1.663612026f * (vs + 72.0f) * .9f;
    const float amix = sig(1);
    const float ka = x[9] * x[9] * x[9] * .8008791415f * (vs + 72.0f) * (amix * x[10] + (1.0f - amix) * x[11]) * .9f;
    const float ih = sc[2] * x[12] * .0126874385f * (vs + 20.0f) * .9f;
    const float sleak = sc[3] * .0006901584324f * (vs + 50.0f);
    float N3[3], D3[3], Q3[3];
    N3[0] = -ca - kca - ka - ih - sleak - cpl + (i_na - 2.0f) * .01222505828f;   D3[0] = .0543909161f;
    N3[1] = sig(12) * sig(13) * cai;                                              D3[1] = 2.5f + cai;
    N3[2] = (sig(17) - x[12]) * .00033f;                                          D3[2] = sig(18);
    fdiv_n(N3, D3, Q3);
    d[15] = Q3[0];
    float a = fabsf(D2[15]) < 1e-5f ? 1.28f : Q2[15];
    float b = fabsf(D2[16]) < 1e-5f ? 1.4f : Q2[16];
    d[1] = a * (1.0f - x[1]) - b * x[1];
    a = .128f * E[4];
    b = Q2[17];
    d[2] = a * (1.0f - x[2]) - b * x[2];
    a = fabsf(D2[18]) < 1e-5f ? .16f : Q2[18];
    b = .5f * E[7];
    d[8] = a * (1.0f - x[8]) - b * x[8];
    d[3] = (sig(8) - x[3]) * .045f;
    d[4] = (sig(9) - x[4]) * .02f * sig(10);
    d[5] = (sig(11) - x[5]) * .0608644f;
    const float kinf = Q3[1];
    d[6] = (kinf - x[6]) * .6f;
    d[7] = (Q2[19] - x[7]) * .035f;
    d[9] = (sig(14) - x[9]) * .14f;
    const float ainf = sig(15);
    d[10] = (ainf - x[10]) * .05f;
    d[11] = (ainf - x[11]) * .0036f * sig(16);
    d[12] = Q3[2];
    d[13] = -.05049639866f * ca - .01729930764f * (cai - .02f);
    d[14] = (sig(19) - x[14]) * .0001386796618f * sig(20);
}
// One classical RK4 step of 0.05 ms from x into xn: lp_rates at x, x + dt/2 k1,
// x + dt/2 k2 and x + dt k3, as one loop over a single copy of lp_rates. The
// stage sum k1 + 2 k2 + 2 k3 + k4 accumulates left to right, the order of the
// reference's expression, so every rounding is the same.
template <bool SAFE>
__device__ __forceinline__ void lp_rk4(const float (&x)[16], float (&xn)[16], float i_na, const float (&sc)[4],
                                       const float *tab, bool &ok) {
    const float dt = .05f;
    float y[16], k[16], acc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) y[j] = x[j];
#pragma unroll 1
    for (int st = 0; st < 4; ++st) {
        lp_rates<SAFE>(y, i_na, sc, k, tab, ok);
        if (st == 0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = k[j];
        } else if (st < 3) {
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = acc[j] + 2 * k[j];
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = acc[j] + k[j];
        }
        const float c = st < 2 ? .5f * dt : dt;
#pragma unroll
        for (int j = 0; j < 16; ++j) y[j] = x[j] + c * k[j];
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) xn[j] = x[j] + dt * acc[j] / 6.0f;
}

// The RK4 step with every exponential decided (crexp_n), on the state xs in
// memory: the rare recomputation of a step whose fast paths left one undecided.
static __device__ __noinline__ void lp_rk4_safe(float *xs, float i_na, const float *scs, const float *tab) {
    float x[16], xn[16], sc[4];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 4; ++j) sc[j] = scs[j];
    bool ok = true;
    lp_rk4<true>(x, xn, i_na, sc, tab, ok);
#pragma unroll
    for (int j = 0; j < 16; ++j) xs[j] = xn[j];
}

// lp_integrate on the state xs (16 floats in memory): 20 RK4 steps with the
// state and the four scales in registers.
static __device__ __noinline__ void lp_integrate(float *xs, float i_na, const float *scs, const float *tab) {
    float x[16], sc[4];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 4; ++j) sc[j] = scs[j];
#pragma unroll 1
    for (int step = 0; step < 20; ++step) {
        float xn[16];
        bool ok = true;
        lp_rk4<false>(x, xn, i_na, sc, tab, ok);
        if (!ok) {
#pragma unroll
            for (int j = 0; j < 16; ++j) xs[j] = x[j];
            lp_rk4_safe(xs, i_na, scs, tab);
#pragma unroll
            for (int j = 0; j < 16; ++j) xn[j] = xs[j];
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = xn[j];
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) xs[j] = x[j];
}

// ---- Prinz pacemaker (prinz_cell.cuh:45-121); u = {v, ca, m[7], h[4]} -------------
// The reference's gates pz_gate(v, a, b) = 1 / (1 + exp((v + a) / b)) and its
// two-exponential time constants 1 / (exp((v + a) / b) + exp((v + c) / d))
// are evaluated in place by pz_substep and pz_substep_warp, in batches.
// pz_substep with its exponentials computed as two batches (crexp_n: the
// voltage's gates and time constants, then the relaxations that use them) and
// its quotients as three (fdiv_n: the exponents' arguments and the calcium
// quotients; the gates and time constants; the relaxation rates, the voltage's
// target and the calcium current). Every operation is the reference's, in its
// order; (v + 65) / -16 is written as the product by -0.0625, which rounds the
// same exact value.
template <bool SAFE>
__device__ __forceinline__ void pz_substep(float (&u)[13], const float (&g)[9], float ext, float clamp_ns,
                                           float clamp_rev, const float *tab, bool &ok) {
    const float dt = .025f;
    float *m = u + 2, *h = u + 9;
    const float v = u[0], ca = fmaxf(u[1], 0.000001f);
    // level 1: pz_gate(v, a, b) = 1 / (1 + exp((v + a) / b)) and the raw exponentials
    const float ga[18] = {25.5f, 27.1f, 33, 27.2f, 28.3f, 12.3f, 75,          // mi
                          120, 68.1f, 32.9f, 46, 28.3f,                       // mt 0 1 3 4 5
                          48.9f, 32.1f, 60, 56.9f,                            // hi
                          55, 38.9f};                                         // ht 1 3
    const float gb[18] = {-5.29f, -7.2f, -8.1f, -8.7f, -12.6f, -11.8f, 5.5f,
                          -25, -20.5f, -15.2f, -22.7f, -19.2f,
                          5.18f, 5.5f, 6.2f, 4.9f,
                          -16.9f, -26.5f};
    float N1[25], D1[25], Q1[25];
#pragma unroll
    for (int i = 0; i < 18; ++i) { N1[i] = v + ga[i]; D1[i] = gb[i]; }
    N1[18] = v + 27;       D1[18] = 10;          // mt 2
    N1[19] = v + 70;       D1[19] = -13;
    N1[20] = v + 62.9f;    D1[20] = -10;         // ht 0
    N1[21] = v + 34.9f;    D1[21] = 3.6f;
    N1[22] = v + 55;       D1[22] = 9;           // ht 2
    N1[23] = 3000.0f;      D1[23] = ca;          // calcium reversal
    N1[24] = ca;           D1[24] = ca + 3;      // calcium factor of mi[4]
    fdiv_n(N1, D1, Q1);
    float A[26], E[26];
#pragma unroll
    for (int i = 0; i < 20; ++i) A[i] = Q1[i];
    A[20] = -14.59f - .086f * v;     // mt 6
    A[21] = -1.87f + .0701f * v;
    A[22] = Q1[20];
    A[23] = Q1[21];
    A[24] = Q1[22];
    A[25] = (v + 65) * -0.0625f;     // (v + 65) / -16
    exp_n<SAFE>(A, E, tab, ok);
    float N2[23], D2[23], Q2[23];
#pragma unroll
    for (int i = 0; i < 18; ++i) { N2[i] = 1.0f; D2[i] = 1.0f + E[i]; }
    N2[18] = 1.0f;         D2[18] = E[18] + E[19];
    N2[19] = 2.0f;         D2[19] = E[20] + E[21];
    N2[20] = 1.34f;        D2[20] = 1 + E[22];
    N2[21] = 1;            D2[21] = 1 + E[23];
    N2[22] = 1.0f;         D2[22] = E[24] + E[25];
    fdiv_n(N2, D2, Q2);
    auto gate = [&](int i) { return Q2[i]; };
    const float eca = (8.31451e3f * 283.0f / (2.0f * 96485.3415f)) * nsx::logf_cr(Q1[23]);
    const float c[8] = {g[0] * m[0] * m[0] * m[0] * h[0], g[1] * m[1] * m[1] * m[1] * h[1],
                        g[2] * m[2] * m[2] * m[2] * h[2], g[3] * m[3] * m[3] * m[3] * h[3],
                        g[4] * m[4] * m[4] * m[4] * m[4], g[5] * m[5] * m[5] * m[5] * m[5],
                        g[6] * m[6], g[7]};
    const float rev[8] = {50, eca, eca, -80, -80, -80, -20, -50};
    float gt = clamp_ns, ws = ext + clamp_ns * clamp_rev;
#pragma unroll
    for (int i = 0; i < 8; ++i) { gt += c[i]; ws += c[i] * rev[i]; }
    const float mi[7] = {gate(0), gate(1), gate(2), gate(3), Q1[24] * gate(4), gate(5), gate(6)};
    const float mt[7] = {2.64f - 2.52f * gate(7), 43.4f - 42.6f * gate(8), 2.8f + 14 * Q2[18],
                         23.2f - 20.8f * gate(9), 180.6f - 150.2f * gate(10), 14.4f - 12.8f * gate(11), Q2[19]};
    const float hi[4] = {gate(12), gate(13), gate(14), gate(15)};
    const float ht[4] = {Q2[20] * (1.5f + Q2[21]), 210 - 179.6f * gate(16), 120 + 300 * Q2[22],
                         77.2f - 58.4f * gate(17)};
    // level 2: the voltage's relaxation and the gates'
    float N3[15], D3[15], Q3[15];
    N3[0] = -dt * gt;      D3[0] = 628.3f;
#pragma unroll
    for (int i = 0; i < 7; ++i) { N3[1 + i] = -dt; D3[1 + i] = mt[i]; }
#pragma unroll
    for (int i = 0; i < 4; ++i) { N3[8 + i] = -dt; D3[8 + i] = ht[i]; }
    N3[12] = dt * ws;                     D3[12] = 628.3f;
    N3[13] = ws;                          D3[13] = gt;
    N3[14] = (c[1] + c[2]) * (v - eca);   D3[14] = 1000000.0f;
    fdiv_n(N3, D3, Q3);
    float B[12], F[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) B[i] = Q3[i];
    exp_n<SAFE>(B, F, tab, ok);
    if (fabsf(gt) < .000001f) u[0] = v + Q3[12];
    else { const float tg = Q3[13]; u[0] = tg + (v - tg) * F[0]; }
    const float ica = Q3[14];
    const float cat = .05f - 14961.0f * ica;
    u[1] = fmaxf(.000001f, cat + (ca - cat) * c_K.prinz_ca);
#pragma unroll
    for (int i = 0; i < 7; ++i) m[i] = mi[i] + (m[i] - mi[i]) * F[1 + i];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = hi[i] + (h[i] - hi[i]) * F[8 + i];
}

// The substep with every exponential decided (crexp_n), on the state xs in
// memory: the rare recomputation of a substep whose fast paths left one
// undecided.
static __device__ __noinline__ void pz_substep_safe(float *xs, const float *gs, float ext, float clamp_ns,
                                                    float clamp_rev, const float *tab) {
    float u[13], g[9];
#pragma unroll
    for (int j = 0; j < 13; ++j) u[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 9; ++j) g[j] = gs[j];
    bool ok = true;
    pz_substep<true>(u, g, ext, clamp_ns, clamp_rev, tab, ok);
#pragma unroll
    for (int j = 0; j < 13; ++j) xs[j] = u[j];
}

// The Prinz cell's 40 substeps of one tick on xs (13 state floats in memory),
// with the state and conductances in registers; returns whether the voltage
// crossed 0 mV upwards in any substep.
static __device__ __noinline__ bool prinz_tick(float *xs, const float *gs, float ext, float clamp_ns, float clamp_rev,
                                               const float *tab) {
    float u[13], g[9];
#pragma unroll
    for (int j = 0; j < 13; ++j) u[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 9; ++j) g[j] = gs[j];
    bool spiked = false;
#pragma unroll 1
    for (int i = 0; i < 40; ++i) {
        const float before = u[0];
        float uo[13];
#pragma unroll
        for (int j = 0; j < 13; ++j) uo[j] = u[j];
        bool ok = true;
        pz_substep<false>(u, g, ext, clamp_ns, clamp_rev, tab, ok);
        if (!ok) {
#pragma unroll
            for (int j = 0; j < 13; ++j) xs[j] = uo[j];
            pz_substep_safe(xs, gs, ext, clamp_ns, clamp_rev, tab);
#pragma unroll
            for (int j = 0; j < 13; ++j) u[j] = xs[j];
        }
        spiked |= before < 0 && u[0] >= 0;
    }
#pragma unroll
    for (int j = 0; j < 13; ++j) xs[j] = u[j];
    return spiked;
}

// Heavy cell types (2 LP, 3 Prinz, 6 LFS) on their extended state x (16 floats).
static __device__ __noinline__ NeuronRegs heavy_tick(const float *g, uint32_t type, const float *xg, float *x, NeuronRegs s,
                                        float cur, float e0, float e1, float e2, float e3, float inh_in,
                                        const float *tab) {
    const float clamp_leak = 0.0f, clamp_rev = -68.0f;
    s.d0 += e0; s.d1 += e1; s.d2 += e2; s.d3 += e3;
    float sub = fmaxf(0.0f, fminf(s.v, -50.0f) - g[G_EL]);
    s.depol += 0.1f * (sub - s.depol);
    s.inh += inh_in;
    s.spike = 0;
    float exc = 0;
    exc += s.d0; exc += s.d1; exc += s.d2; exc += s.d3;
    if (type == 6) {
        lfs_tick(g, s, x, cur, exc, s.inh);
    } else if (type == 2) {
        float axon_before = x[0];
        float ext = cur + exc * (0.0f - s.v) + s.inh * (-75.0f - s.v) - clamp_leak * (s.v - clamp_rev);
        lp_integrate(x, ext / 1000.0f, xg, tab);
        s.v = x[15] - 9.342518882f;
        s.spike = (axon_before < 0 && x[0] >= 0) ? 1u : 0u;
        s.total += (int)s.spike;
    } else {
        const float ext = cur + exc * (0.0f - s.v) + s.inh * (-75.0f - s.v);
        const bool spiked = prinz_tick(x, xg, ext, xg[8] + clamp_leak, clamp_rev, tab);
        s.spike = spiked ? 1u : 0u;
        s.total += (int)s.spike;
        s.v = x[0];
    }
    s.d0 *= c_K.exc_ms; s.d1 *= c_K.exc_ms; s.d2 *= c_K.exc_ms; s.d3 *= c_K.exc_ms;
    s.inh *= c_K.inh_ms;
    return s;
}

// ---- LP and Prinz cells on a whole warp ------------------------------------------
// The same arithmetic as lp_integrate and pz_substep, spread over the 32
// lanes of a warp. Each exponential (and the one logarithm) of a derivative
// evaluation is computed by a lane of its own from the same operands in the
// same order, and each state component is then assembled by one lane exactly
// as the one-thread code assembles it, so the results are identical bit for
// bit. The exponentials' operands are formed by code that is the same for
// every lane, from per-lane constants (forms below), so the 20-odd
// exponentials of an evaluation run at once instead of one after another.
// All 32 lanes call these functions together (converged); w is the warp's
// kHeavyWarpScratch floats of shared memory.
constexpr int kHeavyWarpScratch = 48;

// Operand forms of a lane's exponential: x is the lane's voltage, m, k, c its
// constants. LP: A (x - m) / k; B c - x / k; C x / k + c; D x / k.
// Prinz: G (x + m) / k; P c - k * x; Q c + k * x.
enum : int { F_A = 0, F_B, F_C, F_D, F_G, F_P, F_Q };
struct LaneTerm {
    int form;
    float m, k, c;
    int sig;       // 1: 1 / (1 + e) (the model's sigmoid gates)
    int use_va;    // LP: the axon voltage instead of the soma's
};

// The lane's exponential term of an LP derivative evaluation (lp_rates).
__device__ __forceinline__ LaneTerm lp_term(int lane) {
    switch (lane) {
    case 0: return {F_D, 0.0f, 11.4866f, 0.0f, 0, 0};
    case 1: return {F_A, 55.0f, -15.0f, 0.0f, 1, 0};
    case 2: return {F_B, 0.0f, 4.0f, -13.0f, 0, 1};
    case 3: return {F_C, 0.0f, 5.0f, 5.0f, 0, 1};
    case 4: return {F_B, 0.0f, 18.0f, -2.66666666667f, 0, 1};
    case 5: return {F_B, 0.0f, 5.0f, -5.0f, 0, 1};
    case 6: return {F_B, 0.0f, 5.0f, -10.0f, 0, 1};
    case 7: return {F_B, 0.0f, 40.0f, -1.375f, 0, 1};
    case 8: return {F_A, 15.0f, -9.8f, 0.0f, 1, 0};
    case 9: return {F_A, -40.0f, 3.2f, 0.0f, 1, 0};
    case 10: return {F_A, -15.0f, -10.0f, 0.0f, 1, 0};
    case 11: return {F_A, 29.1336f, -4.43083f, 0.0f, 1, 0};
    case 12: return {F_A, 0.0f, -23.0f, 0.0f, 1, 0};     // mid -.6 * cai
    case 13: return {F_A, 0.0f, -5.0f, 0.0f, 1, 0};      // mid -16 - .6 * cai
    case 14: return {F_A, -12.0f, -26.0f, 0.0f, 1, 0};
    case 15: return {F_A, -62.0f, 6.0f, 0.0f, 1, 0};
    case 16: return {F_A, -40.0f, -12.0f, 0.0f, 1, 0};
    case 17: return {F_A, -70.0f, 8.0f, 0.0f, 1, 0};
    case 18: return {F_A, -110.0f, -21.6f, 0.0f, 1, 0};
    case 19: return {F_A, -26.9916223f, -5.957441281f, 0.0f, 1, 1};
    case 20: return {F_A, -60.57875745f, -13.25674673f, 0.0f, 1, 1};
    default: return {F_B, 0.0f, 1e30f, -1.0f, 0, 0};     // idle lanes: exp(-1), unused
    }
}

// lp_rates on a warp: lane i < 21 forms the i-th exponential of lp_rates and,
// for the gates, its sigmoid 1 / (1 + e), each exactly as lp_rates forms it;
// shuffles give every lane all 21 values, and every lane then assembles all
// 16 derivatives with lp_rates' operations (the same values in every lane,
// so the assembly runs converged, with no divergence and no shared memory),
// nine of its ten quotients spread over the lanes in one round (fdiv_warp).
template <bool SAFE>
__device__ __forceinline__ void lp_rates_warp(const float (&x)[16], float i_na, const float (&sc)[4], float (&d)[16],
                                              int lane, const LaneTerm &q, const float *tab, bool &ok) {
    const float va = x[0], vs = x[15], cai = x[13];
    float t;
    {
        const float xs = q.use_va ? va : vs;
        const float m = lane == 12 ? -.6f * cai : lane == 13 ? -16.0f - .6f * cai : q.m;
        const float r = (q.form == F_A ? xs - m : xs) / q.k;
        const float arg = q.form == F_B ? q.c - r : q.form == F_C ? r + q.c : r;
        const float e = exp1<SAFE>(arg, tab, ok);
        t = q.sig ? 1.0f / (1.0f + e) : e;
    }
    // T[i] = E[i] for i = 0, 2..7 and sig(i) for i = 1, 8..20 (lp_rates' names)
    float T[21];
#pragma unroll
    for (int i = 0; i < 21; ++i) T[i] = __shfl_sync(0xffffffffu, t, i);
    const float na = x[1] * x[1] * x[1] * x[2] * 7.15f * (va - 50.0f);
    const float kd = x[8] * x[8] * x[8] * x[8] * 1.43f * (va + 72.0f);
    const float km = .2613041227f * x[14] * (va + 80.0f);
    const float aleak = sc[3] * .001004288227f * (va + 50.0f);
    const float cpl = .004017089073f * (vs - va);
    const float ev = T[0];
    // every quotient but d[15]'s (which needs the first) in one round
    float N2[9], D2[9], Q2[9];
    N2[0] = vs * (x[13] * ev - 15123.5f);       D2[0] = ev - 1.0f;
    N2[1] = -16.64f - .32f * va;                D2[1] = T[2] - 1.0f;
    N2[2] = .28f * va + 7.0f;                   D2[2] = T[3] - 1.0f;
    N2[3] = 4.0f;                               D2[3] = T[5] + 1.0f;
    N2[4] = -1.6f - .032f * va;                 D2[4] = T[6] - 1.0f;
    N2[5] = .7f;                                D2[5] = .6f + cai;
    N2[6] = -na - kd - km - aleak + cpl;        D2[6] = .1148312178f;
    N2[7] = T[12] * T[13] * cai;                D2[7] = 2.5f + cai;
    N2[8] = (T[17] - x[12]) * .00033f;          D2[8] = T[18];
    fdiv_warp(N2, D2, Q2, lane);
    d[0] = Q2[6];
    const float ghk = fabsf(vs) < .001f ? 11.4866f * (x[13] - 15123.5f) : Q2[0];
    const float ca = sc[0] * (x[3] * x[4] * .1247796343f + x[5] * .07142141077f) * .00155982f * ghk * .9f;
    const float kca = sc[1] * x[6] * x[7] * 1.663612026f * (vs + 72.0f) * .9f;
    const float amix = T[1];
    const float ka = x[9] * x[9] * x[9] * .8008791415f * (vs + 72.0f) * (amix * x[10] + (1.0f - amix) * x[11]) * .9f;
    const float ih = sc[2] * x[12] * .0126874385f * (vs + 20.0f) * .9f;
    const float sleak = sc[3] * .0006901584324f * (vs + 50.0f);
    d[15] = (-ca - kca - ka - ih - sleak - cpl + (i_na - 2.0f) * .01222505828f) / .0543909161f;
    float a = fabsf(D2[1]) < 1e-5f ? 1.28f : Q2[1];
    float b = fabsf(D2[2]) < 1e-5f ? 1.4f : Q2[2];
    d[1] = a * (1.0f - x[1]) - b * x[1];
    a = .128f * T[4];
    b = Q2[3];
    d[2] = a * (1.0f - x[2]) - b * x[2];
    a = fabsf(D2[4]) < 1e-5f ? .16f : Q2[4];
    b = .5f * T[7];
    d[8] = a * (1.0f - x[8]) - b * x[8];
    d[3] = (T[8] - x[3]) * .045f;
    d[4] = (T[9] - x[4]) * .02f * T[10];
    d[5] = (T[11] - x[5]) * .0608644f;
    d[6] = (Q2[7] - x[6]) * .6f;
    d[7] = (Q2[5] - x[7]) * .035f;
    d[9] = (T[14] - x[9]) * .14f;
    d[10] = (T[15] - x[10]) * .05f;
    d[11] = (T[15] - x[11]) * .0036f * T[16];
    d[12] = Q2[8];
    d[13] = -.05049639866f * ca - .01729930764f * (cai - .02f);
    d[14] = (T[19] - x[14]) * .0001386796618f * T[20];
}

// lp_rk4 on the whole warp (lp_rates_warp); every lane computes xn.
template <bool SAFE>
__device__ __forceinline__ void lp_rk4_warp(const float (&x)[16], float (&xn)[16], float i_na, const float (&sc)[4],
                                            int lane, const LaneTerm &q, const float *tab, bool &ok) {
    const float dt = .05f;
    float y[16], k[16], acc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) y[j] = x[j];
#pragma unroll 1
    for (int st = 0; st < 4; ++st) {
        lp_rates_warp<SAFE>(y, i_na, sc, k, lane, q, tab, ok);
        if (st == 0) {
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = k[j];
        } else if (st < 3) {
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = acc[j] + 2 * k[j];
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = acc[j] + k[j];
        }
        const float c = st < 2 ? .5f * dt : dt;
#pragma unroll
        for (int j = 0; j < 16; ++j) y[j] = x[j] + c * k[j];
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) xn[j] = x[j] + dt * acc[j] / 6.0f;
}

// The warp's RK4 step with every exponential decided, on xs in memory (lane 0
// writes the result); all 32 lanes call it together.
static __device__ __noinline__ void lp_rk4_warp_safe(float *xs, float i_na, const float *scs, int lane,
                                                     const float *tab) {
    const LaneTerm q = lp_term(lane);
    float x[16], xn[16], sc[4];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 4; ++j) sc[j] = scs[j];
    bool ok = true;
    lp_rk4_warp<true>(x, xn, i_na, sc, lane, q, tab, ok);
    __syncwarp();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < 16; ++j) xs[j] = xn[j];
    }
    __syncwarp();
}

// lp_integrate on the whole warp: every lane holds the state and the scales
// in registers and runs lp_integrate's 20 RK4 steps (a step with an undecided
// exponential in any lane is recomputed by lp_rk4_warp_safe); lane 0 writes
// the state back. All 32 lanes call it together. The scratch argument `w` is
// unused (kept for the callers' interface).
static __device__ __noinline__ void lp_integrate_warp(float *xs, float i_na, const float *scs, float *w, int lane,
                                                      const float *tab) {
    (void)w;
    const LaneTerm q = lp_term(lane);
    float x[16], sc[4];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 4; ++j) sc[j] = scs[j];
#pragma unroll 1
    for (int step = 0; step < 20; ++step) {
        float xn[16];
        bool ok = true;
        lp_rk4_warp<false>(x, xn, i_na, sc, lane, q, tab, ok);
        if (__any_sync(0xffffffffu, !ok)) {
            __syncwarp();
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) xs[j] = x[j];
            }
            __syncwarp();
            lp_rk4_warp_safe(xs, i_na, scs, lane, tab);
#pragma unroll
            for (int j = 0; j < 16; ++j) xn[j] = xs[j];
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = xn[j];
    }
    __syncwarp();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < 16; ++j) xs[j] = x[j];
    }
    __syncwarp();
}

// The lane's term of a Prinz substep, level 1 (pz_substep's A, E and the
// quotients on them): lanes 0-17 the gates pz_gate (1 / (1 + e) of
// (v + a) / b), 18, 19 and 24, 25 the raw exponentials of the two-exponential
// time constants, 20 and 21 those of mt[6] (c - k v, c + k v), 22 and 23 the
// factors 1.34 / (1 + e) and 1 / (1 + e) of ht[0]; lane 26 takes the
// logarithm of 3000 / ca and lane 27 the quotient ca / (ca + 3).
struct PzTerm {
    int form;       // F_G: (v + a) / b; F_P: c - k v; F_Q: c + k v
    float a, b;     // F_G: a, b; F_P, F_Q: c, k
    float num;      // the numerator over 1 + e; 0: the raw exponential
};
__device__ __forceinline__ PzTerm pz_term(int lane) {
    switch (lane) {
    case 0: return {F_G, 25.5f, -5.29f, 1.0f};
    case 1: return {F_G, 27.1f, -7.2f, 1.0f};
    case 2: return {F_G, 33.0f, -8.1f, 1.0f};
    case 3: return {F_G, 27.2f, -8.7f, 1.0f};
    case 4: return {F_G, 28.3f, -12.6f, 1.0f};
    case 5: return {F_G, 12.3f, -11.8f, 1.0f};
    case 6: return {F_G, 75.0f, 5.5f, 1.0f};
    case 7: return {F_G, 120.0f, -25.0f, 1.0f};
    case 8: return {F_G, 68.1f, -20.5f, 1.0f};
    case 9: return {F_G, 32.9f, -15.2f, 1.0f};
    case 10: return {F_G, 46.0f, -22.7f, 1.0f};
    case 11: return {F_G, 28.3f, -19.2f, 1.0f};
    case 12: return {F_G, 48.9f, 5.18f, 1.0f};
    case 13: return {F_G, 32.1f, 5.5f, 1.0f};
    case 14: return {F_G, 60.0f, 6.2f, 1.0f};
    case 15: return {F_G, 56.9f, 4.9f, 1.0f};
    case 16: return {F_G, 55.0f, -16.9f, 1.0f};
    case 17: return {F_G, 38.9f, -26.5f, 1.0f};
    case 18: return {F_G, 27.0f, 10.0f, 0.0f};
    case 19: return {F_G, 70.0f, -13.0f, 0.0f};
    case 20: return {F_P, -14.59f, .086f, 0.0f};
    case 21: return {F_Q, -1.87f, .0701f, 0.0f};
    case 22: return {F_G, 62.9f, -10.0f, 1.34f};
    case 23: return {F_G, 34.9f, 3.6f, 1.0f};
    case 24: return {F_G, 55.0f, 9.0f, 0.0f};
    case 25: return {F_G, 65.0f, -16.0f, 0.0f};
    default: return {F_P, -1.0f, 0.0f, 0.0f};    // lanes 26-31: exp(-1), unused
    }
}

// One pz_substep on the whole warp: every lane holds u (v, ca, m[7], h[4]) and
// g in registers. Level 1: lane i forms pz_substep's i-th exponential and the
// quotient on it (PzTerm), lanes 26 and 27 the calcium terms; shuffles give
// every lane all 28. Every lane then assembles the gates, time constants and
// currents with pz_substep's operations; level 2: lane i < 12 forms the i-th
// relaxation exponential, lanes 12-14 the voltage target and the calcium
// current; shuffles again, and every lane updates u the same way.
template <bool SAFE>
__device__ __forceinline__ void pz_substep_warp(float (&u)[13], const float (&g)[9], float ext, float clamp_ns,
                                                float clamp_rev, int lane, const PzTerm &q, const float *tab,
                                                bool &ok) {
    const float dt = .025f;
    float *m = u + 2, *h = u + 9;
    const float v = u[0], ca = fmaxf(u[1], 0.000001f);
    float t;
    {
        const float n = lane == 26 ? 3000.0f : lane == 27 ? ca : v + q.a;
        const float dd = lane == 26 ? ca : lane == 27 ? ca + 3 : q.form == F_G ? q.b : 1.0f;
        const float r = n / dd;
        const float arg = lane >= 26 ? -1.0f : q.form == F_G ? r : q.form == F_P ? q.a - q.b * v : q.a + q.b * v;
        const float e = exp1<SAFE>(arg, tab, ok);
        const float s = q.num / (1 + e);
        t = lane == 27 ? r : q.num != 0.0f ? s : e;
        if (lane == 26) t = nsx::logf_cr(r);
    }
    float T[28];
#pragma unroll
    for (int i = 0; i < 28; ++i) T[i] = __shfl_sync(0xffffffffu, t, i);
    float N1[3], D1[3], Q1[3];
    N1[0] = 1.0f;  D1[0] = T[18] + T[19];
    N1[1] = 2.0f;  D1[1] = T[20] + T[21];
    N1[2] = 1.0f;  D1[2] = T[24] + T[25];
    fdiv_warp(N1, D1, Q1, lane);
    const float eca = (8.31451e3f * 283.0f / (2.0f * 96485.3415f)) * T[26];
    const float c[8] = {g[0] * m[0] * m[0] * m[0] * h[0], g[1] * m[1] * m[1] * m[1] * h[1],
                        g[2] * m[2] * m[2] * m[2] * h[2], g[3] * m[3] * m[3] * m[3] * h[3],
                        g[4] * m[4] * m[4] * m[4] * m[4], g[5] * m[5] * m[5] * m[5] * m[5],
                        g[6] * m[6], g[7]};
    const float rev[8] = {50, eca, eca, -80, -80, -80, -20, -50};
    float gt = clamp_ns, ws = ext + clamp_ns * clamp_rev;
#pragma unroll
    for (int i = 0; i < 8; ++i) { gt += c[i]; ws += c[i] * rev[i]; }
    const float mi[7] = {T[0], T[1], T[2], T[3], T[27] * T[4], T[5], T[6]};
    const float mt[7] = {2.64f - 2.52f * T[7], 43.4f - 42.6f * T[8], 2.8f + 14 * Q1[0],
                         23.2f - 20.8f * T[9], 180.6f - 150.2f * T[10], 14.4f - 12.8f * T[11], Q1[1]};
    const float hi[4] = {T[12], T[13], T[14], T[15]};
    const float ht[4] = {T[22] * (1.5f + T[23]), 210 - 179.6f * T[16], 120 + 300 * Q1[2], 77.2f - 58.4f * T[17]};
    // level 2: lane 0 the voltage's relaxation, 1-7 and 8-11 the gates',
    // 12-14 the voltage target's two forms and the calcium current
    float f;
    {
        float n = -dt, dd = 628.3f;
        if (lane == 0) n = -dt * gt;
        else if (lane == 12) n = dt * ws;
        else if (lane == 13) { n = ws; dd = gt; }
        else if (lane == 14) { n = (c[1] + c[2]) * (v - eca); dd = 1000000.0f; }
#pragma unroll
        for (int i = 0; i < 7; ++i) dd = lane == 1 + i ? mt[i] : dd;
#pragma unroll
        for (int i = 0; i < 4; ++i) dd = lane == 8 + i ? ht[i] : dd;
        const float r = n / dd;
        const float e = exp1<SAFE>(lane < 12 ? r : -1.0f, tab, ok);
        f = lane < 12 ? e : r;
    }
    float F[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) F[i] = __shfl_sync(0xffffffffu, f, i);
    if (fabsf(gt) < .000001f) u[0] = v + F[12];
    else { const float tg = F[13]; u[0] = tg + (v - tg) * F[0]; }
    const float ica = F[14];
    const float cat = .05f - 14961.0f * ica;
    u[1] = fmaxf(.000001f, cat + (ca - cat) * c_K.prinz_ca);
#pragma unroll
    for (int i = 0; i < 7; ++i) m[i] = mi[i] + (m[i] - mi[i]) * F[1 + i];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = hi[i] + (h[i] - hi[i]) * F[8 + i];
}

// The warp's substep with every exponential decided, on xs in memory (lane 0
// writes the result); all 32 lanes call it together.
static __device__ __noinline__ void pz_substep_warp_safe(float *xs, const float *xg, float ext, float clamp_ns,
                                                         float clamp_rev, int lane, const float *tab) {
    const PzTerm q = pz_term(lane);
    float u[13], g[9];
#pragma unroll
    for (int j = 0; j < 13; ++j) u[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 9; ++j) g[j] = xg[j];
    bool ok = true;
    pz_substep_warp<true>(u, g, ext, clamp_ns, clamp_rev, lane, q, tab, ok);
    __syncwarp();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < 13; ++j) xs[j] = u[j];
    }
    __syncwarp();
}

// The Prinz cell's 40 substeps of one tick on x (13 state floats) on the whole
// warp (a substep with an undecided exponential in any lane is recomputed by
// pz_substep_warp_safe); lane 0 writes the state back. Returns whether the
// voltage crossed 0 mV upwards in any substep (all lanes). The scratch
// argument `w` is unused (kept for the callers' interface).
static __device__ __noinline__ bool prinz_tick_warp(float *x, const float *xg, float ext, float clamp_ns,
                                                    float clamp_rev, float *w, int lane, const float *tab) {
    (void)w;
    const PzTerm q = pz_term(lane);
    float u[13], g[9];
#pragma unroll
    for (int j = 0; j < 13; ++j) u[j] = x[j];
#pragma unroll
    for (int j = 0; j < 9; ++j) g[j] = xg[j];
    bool spiked = false;
#pragma unroll 1
    for (int i = 0; i < 40; ++i) {
        const float before = u[0];
        float uo[13];
#pragma unroll
        for (int j = 0; j < 13; ++j) uo[j] = u[j];
        bool ok = true;
        pz_substep_warp<false>(u, g, ext, clamp_ns, clamp_rev, lane, q, tab, ok);
        if (__any_sync(0xffffffffu, !ok)) {
            __syncwarp();
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < 13; ++j) x[j] = uo[j];
            }
            __syncwarp();
            pz_substep_warp_safe(x, xg, ext, clamp_ns, clamp_rev, lane, tab);
#pragma unroll
            for (int j = 0; j < 13; ++j) u[j] = x[j];
        }
        spiked |= before < 0 && u[0] >= 0;
    }
    __syncwarp();
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < 13; ++j) x[j] = u[j];
    }
    __syncwarp();
    return spiked;
}

// A heavy unit steps its pooled LP and Prinz cells on whole warps, one after
// another per warp (lp_integrate_warp, prinz_tick_warp), when the pool holds at
// most this many cells per warp on average; with more, each cell runs on its
// own lane at once (lp_integrate, prinz_tick). Measured on B200, one cell-tick
// costs about 142 k (LP) and 97 k (Prinz) cycles on a warp and about 435 k on
// a lane, and a warp whose lanes hold both kinds runs the two one after the
// other; on whole warps the pool also spreads evenly. The Gym batches measured
// were fastest on whole warps up to about eight cells per warp.
#ifndef NSB_WARP_CELLS_MAX
#define NSB_WARP_CELLS_MAX 8
#endif
constexpr int kWarpCellsMax = NSB_WARP_CELLS_MAX;

// The cell model of one LP (type 2) or Prinz (type 3) cell on its own lane,
// between heavy_pre and heavy_post: returns the LP axon voltage before the
// tick (type 2) and sets `spiked` (type 3).
__device__ __forceinline__ float heavy_model_lane(uint32_t type, float *x, const float *xg, float ext, bool &spiked,
                                                  const float *tab) {
    if (type == 2) {
        const float ab = x[0];
        lp_integrate(x, ext / 1000.0f, xg, tab);
        return ab;
    }
    spiked = prinz_tick(x, xg, ext, xg[8] + 0.0f, -68.0f, tab);
    return 0.0f;
}

// heavy_tick in three parts for the warp form: heavy_pre and heavy_post run
// on the cell's own lane, the cell model in between on the whole warp.
// heavy_pre returns the external current the cell model receives (the LP
// cell's is divided by 1000 there, as in heavy_tick).
__device__ __forceinline__ float heavy_pre(const float *g, uint32_t type, NeuronRegs &s, float cur, float e0,
                                           float e1, float e2, float e3, float inh_in) {
    const float clamp_leak = 0.0f, clamp_rev = -68.0f;
    s.d0 += e0; s.d1 += e1; s.d2 += e2; s.d3 += e3;
    float sub = fmaxf(0.0f, fminf(s.v, -50.0f) - g[G_EL]);
    s.depol += 0.1f * (sub - s.depol);
    s.inh += inh_in;
    s.spike = 0;
    float exc = 0;
    exc += s.d0; exc += s.d1; exc += s.d2; exc += s.d3;
    if (type == 2) return cur + exc * (0.0f - s.v) + s.inh * (-75.0f - s.v) - clamp_leak * (s.v - clamp_rev);
    return cur + exc * (0.0f - s.v) + s.inh * (-75.0f - s.v);
}
__device__ __forceinline__ void heavy_post(uint32_t type, NeuronRegs &s, const float *x, float axon_before,
                                           bool spiked) {
    if (type == 2) {
        s.v = x[15] - 9.342518882f;
        s.spike = (axon_before < 0 && x[0] >= 0) ? 1u : 0u;
    } else {
        s.spike = spiked ? 1u : 0u;
        s.v = x[0];
    }
    s.total += (int)s.spike;
    s.d0 *= c_K.exc_ms; s.d1 *= c_K.exc_ms; s.d2 *= c_K.exc_ms; s.d3 *= c_K.exc_ms;
    s.inh *= c_K.inh_ms;
}

// ---- homeostasis (physiology.cuh:243-253) ----------------------------------------
__device__ __forceinline__ float homeostasis(uint32_t type, float log_ampa, float elapsed, float hz) {
    if (type != 0) return log_ampa;
    float ratio = clampf(hz / 0.4f, 0.0f, 2.65f);
    float change = ratio < 1.0f ? c_K.log_up * (1.0f - ratio) : c_K.log_down * ((ratio - 1.0f) / 1.65f);
    return clampf(log_ampa + change * (elapsed / 172800000.0f), -3.0f, 3.0f);
}

// ---- synapse -----------------------------------------------------------------------
// Release (physiology.cuh:425-454) on a synapse state record in registers.
// L: type of the last-arrival tick (int in the batch pools, int64_t in the
// world simulator's SynapseState records).
template <class L> struct SynReleaseT {
    float w, ru, slow;
    uint64_t ready;
    uint32_t rng;
    L last;
};
using SynRelease = SynReleaseT<int>;
template <class L>
__device__ __forceinline__ float release(const float *y, SynReleaseT<L> &s, int64_t tick, const float *tab) {
    float p_rec = 0;
    if (s.last > -1000000) {
        float dt = (float)(tick - (int64_t)s.last) * 1.0f;
        p_rec = 1.0f - crexp(-dt / y[Y_TREC], tab);
        if (y[Y_TFAC] > 0) s.ru *= crexp(-dt / y[Y_TFAC], tab);
        if (y[Y_SLOWREC] > 0) s.slow = 1.0f - (1.0f - s.slow) * crexp(-dt / y[Y_SLOWREC], tab);
    }
    s.ru = y[Y_TFAC] > 0 ? s.ru + y[Y_U] * (1.0f - s.ru) : y[Y_U];
    const int n = (int)(__float_as_uint(y[Y_INFO]) & 0xffu);
    int released = 0;
    uint32_t rng = s.rng;
    uint64_t ready = s.ready;
    const uint32_t t_rec = draw_threshold(p_rec), t_ru = draw_threshold(s.ru);
    for (int site = 0; site < n; ++site) {
        uint64_t bit = 1ull << site;
        if (!(ready & bit)) {
            rng = xorshift32(rng);
            if ((rng >> 8) < t_rec) ready |= bit;
        }
        if (ready & bit) {
            rng = xorshift32(rng);
            if ((rng >> 8) < t_ru) { ready &= ~bit; ++released; }
        }
    }
    s.rng = rng; s.ready = ready;
    s.last = (L)tick;
    float out = s.w * (float)released / (float)n * s.slow;
    if (y[Y_SLOWREC] > 0) s.slow *= 1.0f - y[Y_SLOWDEPL];
    return out;
}

// Plasticity state in registers.
struct SynPlast {
    float w, pre_tr, post_tr, eltp, eltd, da_age, spine, st_age, pre_age, post_age;
};

__device__ __forceinline__ float da_window(float age, const float *tab) {
    if (age < 0 || age > 20000.0f) return 0;
    float x = age / 2000.0f;
    return x * x * x * x * crexp(4.0f * (1.0f - x), tab);
}
__device__ __forceinline__ float spine_window(float age, const float *tab) {
    if (age < 0 || age > 5000.0f) return 0;
    float x = age / 1000.0f;
    return x * x * x * crexp(3.0f * (1.0f - x), tab);
}

// One plasticity tick (physiology.cuh:459-555) for a plastic synapse
// (plasticity != 0 and excitatory pair), all channels available.
__device__ __forceinline__ void plasticity_tick(uint32_t prof, uint32_t receptors, float w0, SynPlast &s,
                                                bool arrived, bool post, float depol, uint32_t mod,
                                                const float *tab) {
    if (prof == 6) {
        // Triplet STDP (Pfister & Gerstner 2006, minimal all-to-all model:
        // tau+ 16.8, tau- 33.7, tau_y 114 ms, A3+ 6.5e-3, A2- 7.1e-3) written
        // into an eligibility trace (tau 200 ms) that a dopamine event turns
        // into a weight change. pre_tr = r1, post_tr = o1, eltd = o2, eltp = e.
        s.pre_tr *= c_K.tp; s.post_tr *= c_K.tm; s.eltd *= c_K.ty; s.eltp *= c_K.te;
        s.pre_age += 1.0f; s.post_age += 1.0f;
        if (arrived) { s.eltp -= 0.0071f * s.post_tr; s.pre_tr += 1.0f; s.pre_age = 0; }
        if (post) { s.eltp += 0.0065f * s.pre_tr * s.eltd; s.post_tr += 1.0f; s.eltd += 1.0f; s.post_age = 0; }
        if ((mod & 4u) && (receptors & 4u)) s.w += w0 * s.eltp;
        s.w = clampf(s.w, 0.0f, 2.0f * w0);
        return;
    }
    if (prof == 5) {
        if (s.st_age >= 0) { s.st_age += 1.0f; if (s.st_age > 5000.0f) s.st_age = -1; }
        s.pre_age += 1.0f;
        if (arrived) s.pre_age = 0;
        if (post && s.pre_age <= 15.0f && s.st_age < 0) s.st_age = 0;
        if ((mod & 4u) && (receptors & 4u)) s.spine = clampf(s.spine + 0.025f * spine_window(s.st_age, tab), 1.0f, 2.0f);
        return;
    }
    if (prof == 4) {
        if (s.da_age >= 0) { s.da_age += 1.0f; if (s.da_age > 20000.0f) s.da_age = -1; }
        s.pre_age += 1.0f;
        if (arrived) s.pre_age = 0;
        if (post && s.pre_age <= 15.0f && (s.da_age < 0 || s.da_age > 30.0f)) {
            s.da_age = 0;
            s.w -= 0.005383f * w0;
        }
        if ((mod & 4u) && (receptors & 4u)) {
            s.w += 0.00453f * da_window(s.da_age, tab) * w0;
            s.da_age = -1;
        }
        s.w = clampf(s.w, 0.0f, 2.0f * w0);
        return;
    }
    if (prof == 3) {
        s.eltp *= c_K.ne; s.eltd *= c_K.sht;
        s.pre_age += 1.0f; s.post_age += 1.0f;
        if (arrived) { if (s.post_age <= 15.0f) s.eltd += 1.0f; s.pre_age = 0; }
        if (post) { if (s.pre_age <= 15.0f) s.eltp += 1.0f; s.post_age = 0; }
        if ((mod & 1u) && (receptors & 1u)) { s.w += 0.0048f * s.eltp * w0; s.eltp = 0; }
        if ((mod & 2u) && (receptors & 2u)) { s.w -= 0.0075f * s.eltd * w0; s.eltd = 0; }
        s.w = clampf(s.w, 0.0f, 2.0f * w0);
        return;
    }
    s.pre_tr *= c_K.ltp; s.post_tr *= c_K.ltd;
    s.pre_age += 1.0f; s.post_age += 1.0f;
    if (arrived) {
        if (s.post_age <= (prof == 2 ? 50.0f : 20.0f)) s.w *= 1.0f - 0.004f * s.post_tr;
        s.pre_tr += 1.0f;
        s.pre_age = 0;
    }
    if (post) {
        if (s.pre_age <= 20.0f && (prof == 1 || depol >= 2.3f)) s.w += 0.016f * s.pre_tr * (2.0f * w0 - s.w);
        s.post_tr += 1.0f;
        s.post_age = 0;
    }
    s.w = clampf(s.w, 0.0f, 2.0f * w0);
}

// k consecutive ticks with no arrival, no postsynaptic spike and no relevant
// modulator event: exactly k applications of plasticity_tick's quiet branch
// (each field evolves independently; the weight bound is idempotent).
__device__ __forceinline__ void plasticity_quiet(uint32_t prof, float w0, SynPlast &s, int k) {
    if (k <= 0) return;
    if (prof == 6) {
        for (int i = 0; i < k; ++i) {
            s.pre_tr *= c_K.tp; s.post_tr *= c_K.tm; s.eltd *= c_K.ty; s.eltp *= c_K.te;
            s.pre_age += 1.0f; s.post_age += 1.0f;
        }
        s.w = clampf(s.w, 0.0f, 2.0f * w0);
        return;
    }
    if (prof == 5) {
        for (int i = 0; i < k; ++i) {
            if (s.st_age >= 0) { s.st_age += 1.0f; if (s.st_age > 5000.0f) s.st_age = -1; }
            s.pre_age += 1.0f;
        }
        return;
    }
    if (prof == 4) {
        for (int i = 0; i < k; ++i) {
            if (s.da_age >= 0) { s.da_age += 1.0f; if (s.da_age > 20000.0f) s.da_age = -1; }
            s.pre_age += 1.0f;
        }
        s.w = clampf(s.w, 0.0f, 2.0f * w0);
        return;
    }
    if (prof == 3) {
        for (int i = 0; i < k; ++i) { s.eltp *= c_K.ne; s.eltd *= c_K.sht; s.pre_age += 1.0f; s.post_age += 1.0f; }
        s.w = clampf(s.w, 0.0f, 2.0f * w0);
        return;
    }
    for (int i = 0; i < k; ++i) { s.pre_tr *= c_K.ltp; s.post_tr *= c_K.ltd; s.pre_age += 1.0f; s.post_age += 1.0f; }
    s.w = clampf(s.w, 0.0f, 2.0f * w0);
}

// Does a modulator bit set at the postsynaptic neuron affect this profile?
__device__ __forceinline__ bool mod_relevant(uint32_t prof, uint32_t receptors, uint32_t mod) {
    if (prof == 3) return (mod & receptors & 3u) != 0;
    if (prof == 4 || prof == 5 || prof == 6) return (mod & receptors & 4u) != 0;
    return false;
}

}  // namespace nsb
