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
__device__ __forceinline__ float lp_sig(float v, float mid, float slope, const float *tab) {
    return 1.0f / (1.0f + crexp((v - mid) / slope, tab));
}
__device__ __forceinline__ float lp_ratio(float num, float den, float lim) { return fabsf(den) < 1e-5f ? lim : num / den; }
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

// lp_rates with its 21 exponentials computed as one batch (crexp_n): the
// arguments, the sigmoids 1 / (1 + e) and the derivative assembly are the
// operations of the reference, in its order.
__device__ __forceinline__ void lp_rates(const float (&x)[16], float i_na, const float (&sc)[4], float (&d)[16],
                                         const float *tab) {
    const float va = x[0], vs = x[15], cai = x[13];
    float A[21], E[21];
    A[0] = vs / 11.4866f;
    A[1] = (vs - 55.0f) / -15.0f;
    A[2] = -13.0f - va / 4.0f;
    A[3] = va / 5.0f + 5.0f;
    A[4] = -2.66666666667f - va / 18.0f;
    A[5] = -5.0f - va / 5.0f;
    A[6] = -10.0f - va / 5.0f;
    A[7] = -1.375f - va / 40.0f;
    A[8] = (vs - 15.0f) / -9.8f;
    A[9] = (vs - -40.0f) / 3.2f;
    A[10] = (vs - -15.0f) / -10.0f;
    A[11] = (vs - 29.1336f) / -4.43083f;
    A[12] = (vs - -.6f * cai) / -23.0f;
    A[13] = (vs - (-16.0f - .6f * cai)) / -5.0f;
    A[14] = (vs - -12.0f) / -26.0f;
    A[15] = (vs - -62.0f) / 6.0f;
    A[16] = (vs - -40.0f) / -12.0f;
    A[17] = (vs - -70.0f) / 8.0f;
    A[18] = (vs - -110.0f) / -21.6f;
    A[19] = (va - -26.9916223f) / -5.957441281f;
    A[20] = (va - -60.57875745f) / -13.25674673f;
    crexp_n(A, E, tab);
    auto sig = [&](int i) { return 1.0f / (1.0f + E[i]); };
    const float na = x[1] * x[1] * x[1] * x[2] * 7.15f * (va - 50.0f);
    const float kd = x[8] * x[8] * x[8] * x[8] * 1.43f * (va + 72.0f);
    const float km = .2613041227f * x[14] * (va + 80.0f);
    const float aleak = sc[3] * .001004288227f * (va + 50.0f);
    const float cpl = .004017089073f * (vs - va);
    d[0] = (-na - kd - km - aleak + cpl) / .1148312178f;
    const float ev = E[0];
    const float ghk = fabsf(vs) < .001f ? 11.4866f * (x[13] - 15123.5f) : vs * (x[13] * ev - 15123.5f) / (ev - 1.0f);
    const float ca = sc[0] * (x[3] * x[4] * .1247796343f + x[5] * .07142141077f) * .00155982f * ghk * .9f;
    const float kca = sc[1] * x[6] * x[7] * 1.663612026f * (vs + 72.0f) * .9f;
    const float amix = sig(1);
    const float ka = x[9] * x[9] * x[9] * .8008791415f * (vs + 72.0f) * (amix * x[10] + (1.0f - amix) * x[11]) * .9f;
    const float ih = sc[2] * x[12] * .0126874385f * (vs + 20.0f) * .9f;
    const float sleak = sc[3] * .0006901584324f * (vs + 50.0f);
    d[15] = (-ca - kca - ka - ih - sleak - cpl + (i_na - 2.0f) * .01222505828f) / .0543909161f;
    float a = lp_ratio(-16.64f - .32f * va, E[2] - 1.0f, 1.28f);
    float b = lp_ratio(.28f * va + 7.0f, E[3] - 1.0f, 1.4f);
    d[1] = a * (1.0f - x[1]) - b * x[1];
    a = .128f * E[4];
    b = 4.0f / (E[5] + 1.0f);
    d[2] = a * (1.0f - x[2]) - b * x[2];
    a = lp_ratio(-1.6f - .032f * va, E[6] - 1.0f, .16f);
    b = .5f * E[7];
    d[8] = a * (1.0f - x[8]) - b * x[8];
    d[3] = (sig(8) - x[3]) * .045f;
    d[4] = (sig(9) - x[4]) * .02f * sig(10);
    d[5] = (sig(11) - x[5]) * .0608644f;
    const float kinf = sig(12) * sig(13) * cai / (2.5f + cai);
    d[6] = (kinf - x[6]) * .6f;
    d[7] = (.7f / (.6f + cai) - x[7]) * .035f;
    d[9] = (sig(14) - x[9]) * .14f;
    const float ainf = sig(15);
    d[10] = (ainf - x[10]) * .05f;
    d[11] = (ainf - x[11]) * .0036f * sig(16);
    d[12] = (sig(17) - x[12]) * .00033f / sig(18);
    d[13] = -.05049639866f * ca - .01729930764f * (cai - .02f);
    d[14] = (sig(19) - x[14]) * .0001386796618f * sig(20);
}
// lp_integrate on the state xs (16 floats in memory): 20 classical RK4 steps
// of 0.05 ms with the state, the four scales and the stage sums in registers.
// The four stages run as one loop over a single copy of lp_rates. The stage
// sum k1 + 2 k2 + 2 k3 + k4 accumulates left to right, the order of the
// reference's expression, so every rounding is the same.
static __device__ __noinline__ void lp_integrate(float *xs, float i_na, const float *scs, const float *tab) {
    const float dt = .05f;
    float x[16], y[16], k[16], acc[16], sc[4];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = xs[j];
#pragma unroll
    for (int j = 0; j < 4; ++j) sc[j] = scs[j];
#pragma unroll 1
    for (int step = 0; step < 20; ++step) {
#pragma unroll
        for (int j = 0; j < 16; ++j) y[j] = x[j];
#pragma unroll 1
        for (int st = 0; st < 4; ++st) {
            lp_rates(y, i_na, sc, k, tab);
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
        for (int j = 0; j < 16; ++j) x[j] += dt * acc[j] / 6.0f;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) xs[j] = x[j];
}

// ---- Prinz pacemaker (prinz_cell.cuh:45-121); u = {v, ca, m[7], h[4]} -------------
__device__ __forceinline__ float pz_gate(float v, float a, float b, const float *tab) {
    return 1.0f / (1.0f + crexp((v + a) / b, tab));
}
__device__ __forceinline__ float pz_gate2(float v, float a, float b, float c, float d, const float *tab) {
    return 1.0f / (crexp((v + a) / b, tab) + crexp((v + c) / d, tab));
}
// pz_substep with its exponentials computed as two batches (crexp_n): the
// voltage's gates and time constants, then the relaxations that use them.
__device__ __forceinline__ void pz_substep(float (&u)[13], const float (&g)[9], float ext, float clamp_ns,
                                           float clamp_rev, const float *tab) {
    const float dt = .025f;
    float *m = u + 2, *h = u + 9;
    const float v = u[0], ca = fmaxf(u[1], 0.000001f);
    // level 1: pz_gate(v, a, b) = 1 / (1 + exp((v + a) / b)) and the raw exponentials
    float A[26], E[26];
    const float ga[20] = {25.5f, 27.1f, 33, 27.2f, 28.3f, 12.3f, 75,          // mi
                          120, 68.1f, 32.9f, 46, 28.3f,                       // mt 0 1 3 4 5
                          48.9f, 32.1f, 60, 56.9f,                            // hi
                          55, 38.9f,                                          // ht 1 3
                          0, 0};
    const float gb[20] = {-5.29f, -7.2f, -8.1f, -8.7f, -12.6f, -11.8f, 5.5f,
                          -25, -20.5f, -15.2f, -22.7f, -19.2f,
                          5.18f, 5.5f, 6.2f, 4.9f,
                          -16.9f, -26.5f,
                          1, 1};
#pragma unroll
    for (int i = 0; i < 18; ++i) A[i] = (v + ga[i]) / gb[i];
    A[18] = (v + 27) / 10;           // mt 2
    A[19] = (v + 70) / -13;
    A[20] = -14.59f - .086f * v;     // mt 6
    A[21] = -1.87f + .0701f * v;
    A[22] = (v + 62.9f) / -10;       // ht 0
    A[23] = (v + 34.9f) / 3.6f;
    A[24] = (v + 55) / 9;            // ht 2
    A[25] = (v + 65) / -16;
    crexp_n(A, E, tab);
    auto gate = [&](int i) { return 1.0f / (1.0f + E[i]); };
    const float eca = (8.31451e3f * 283.0f / (2.0f * 96485.3415f)) * nsx::logf_cr(3000.0f / ca);
    const float c[8] = {g[0] * m[0] * m[0] * m[0] * h[0], g[1] * m[1] * m[1] * m[1] * h[1],
                        g[2] * m[2] * m[2] * m[2] * h[2], g[3] * m[3] * m[3] * m[3] * h[3],
                        g[4] * m[4] * m[4] * m[4] * m[4], g[5] * m[5] * m[5] * m[5] * m[5],
                        g[6] * m[6], g[7]};
    const float rev[8] = {50, eca, eca, -80, -80, -80, -20, -50};
    float gt = clamp_ns, ws = ext + clamp_ns * clamp_rev;
#pragma unroll
    for (int i = 0; i < 8; ++i) { gt += c[i]; ws += c[i] * rev[i]; }
    const float mi[7] = {gate(0), gate(1), gate(2), gate(3), (ca / (ca + 3)) * gate(4), gate(5), gate(6)};
    const float mt[7] = {2.64f - 2.52f * gate(7), 43.4f - 42.6f * gate(8), 2.8f + 14 * (1.0f / (E[18] + E[19])),
                         23.2f - 20.8f * gate(9), 180.6f - 150.2f * gate(10), 14.4f - 12.8f * gate(11),
                         2.0f / (E[20] + E[21])};
    const float hi[4] = {gate(12), gate(13), gate(14), gate(15)};
    const float ht[4] = {(1.34f / (1 + E[22])) * (1.5f + 1 / (1 + E[23])), 210 - 179.6f * gate(16),
                         120 + 300 * (1.0f / (E[24] + E[25])), 77.2f - 58.4f * gate(17)};
    // level 2: the voltage's relaxation and the gates'
    float B[12], F[12];
    B[0] = -dt * gt / 628.3f;
#pragma unroll
    for (int i = 0; i < 7; ++i) B[1 + i] = -dt / mt[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) B[8 + i] = -dt / ht[i];
    crexp_n(B, F, tab);
    if (fabsf(gt) < .000001f) u[0] = v + dt * ws / 628.3f;
    else { const float tg = ws / gt; u[0] = tg + (v - tg) * F[0]; }
    const float ica = (c[1] + c[2]) * (v - eca) / 1000000.0f;
    const float cat = .05f - 14961.0f * ica;
    u[1] = fmaxf(.000001f, cat + (ca - cat) * c_K.prinz_ca);
#pragma unroll
    for (int i = 0; i < 7; ++i) m[i] = mi[i] + (m[i] - mi[i]) * F[1 + i];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = hi[i] + (h[i] - hi[i]) * F[8 + i];
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
        pz_substep(u, g, ext, clamp_ns, clamp_rev, tab);
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

// lp_rates on the state y (16 floats) for lanes 0..15: returns d[lane].
__device__ __forceinline__ float lp_rate_warp(const float *y, float i_na, const float *sc, float *T, int lane,
                                              const LaneTerm &q, const float *tab) {
    const float va = y[0], vs = y[15], cai = y[13];
    {   // every lane: one exponential, formed the same way in every lane
        const float x = q.use_va ? va : vs;
        const float m = lane == 12 ? -.6f * cai : lane == 13 ? -16.0f - .6f * cai : q.m;
        const float r = (q.form == F_A ? x - m : x) / q.k;
        const float arg = q.form == F_B ? q.c - r : q.form == F_C ? r + q.c : r;
        const float e = crexp(arg, tab);
        T[lane] = q.sig ? 1.0f / (1.0f + e) : e;
    }
    __syncwarp();
    const float *x = y;
    float d = 0.0f;
    if (lane == 0) {
        const float na = x[1] * x[1] * x[1] * x[2] * 7.15f * (va - 50.0f);
        const float kd = x[8] * x[8] * x[8] * x[8] * 1.43f * (va + 72.0f);
        const float km = .2613041227f * x[14] * (va + 80.0f);
        const float aleak = sc[3] * .001004288227f * (va + 50.0f);
        const float cpl = .004017089073f * (vs - va);
        d = (-na - kd - km - aleak + cpl) / .1148312178f;
    } else if (lane == 13 || lane == 15) {
        const float ev = T[0];
        const float ghk = fabsf(vs) < .001f ? 11.4866f * (x[13] - 15123.5f) : vs * (x[13] * ev - 15123.5f) / (ev - 1.0f);
        const float ca = sc[0] * (x[3] * x[4] * .1247796343f + x[5] * .07142141077f) * .00155982f * ghk * .9f;
        if (lane == 13) {
            d = -.05049639866f * ca - .01729930764f * (cai - .02f);
        } else {
            const float cpl = .004017089073f * (vs - va);
            const float kca = sc[1] * x[6] * x[7] * 1.663612026f * (vs + 72.0f) * .9f;
            const float amix = T[1];
            const float ka = x[9] * x[9] * x[9] * .8008791415f * (vs + 72.0f) * (amix * x[10] + (1.0f - amix) * x[11]) * .9f;
            const float ih = sc[2] * x[12] * .0126874385f * (vs + 20.0f) * .9f;
            const float sleak = sc[3] * .0006901584324f * (vs + 50.0f);
            d = (-ca - kca - ka - ih - sleak - cpl + (i_na - 2.0f) * .01222505828f) / .0543909161f;
        }
    } else if (lane == 1 || lane == 2 || lane == 8) {
        float a, b;
        if (lane == 1) {
            a = lp_ratio(-16.64f - .32f * va, T[2] - 1.0f, 1.28f);
            b = lp_ratio(.28f * va + 7.0f, T[3] - 1.0f, 1.4f);
        } else if (lane == 2) {
            a = .128f * T[4];
            b = 4.0f / (T[5] + 1.0f);
        } else {
            a = lp_ratio(-1.6f - .032f * va, T[6] - 1.0f, .16f);
            b = .5f * T[7];
        }
        d = a * (1.0f - x[lane]) - b * x[lane];
    } else if (lane < 16) {
        // gating variables: ((A - x) * k) [* or / B]
        const int ia = lane == 3 ? 8 : lane == 4 ? 9 : lane == 5 ? 11 : lane == 9 ? 14 : lane == 10 ? 15
                       : lane == 11 ? 15 : lane == 12 ? 17 : 19;
        const float A = lane == 6 ? T[12] * T[13] * cai / (2.5f + cai) : lane == 7 ? .7f / (.6f + cai) : T[ia];
        const float k = lane == 3 ? .045f : lane == 4 ? .02f : lane == 5 ? .0608644f : lane == 6 ? .6f
                        : lane == 7 ? .035f : lane == 9 ? .14f : lane == 10 ? .05f : lane == 11 ? .0036f
                        : lane == 12 ? .00033f : .0001386796618f;
        d = (A - x[lane]) * k;
        if (lane == 4 || lane == 11 || lane == 14) d = d * T[lane == 4 ? 10 : lane == 11 ? 16 : 20];
        else if (lane == 12) d = d / T[18];
    }
    __syncwarp();
    return d;
}

// lp_integrate on x (16 floats, any memory the warp can read and write).
static __device__ __noinline__ void lp_integrate_warp(float *x, float i_na, const float *sc, float *w, int lane,
                                                      const float *tab) {
    const float dt = .05f;
    float *y = w, *T = w + 16;
    const LaneTerm q = lp_term(lane);
    float xj = lane < 16 ? x[lane] : 0.0f;
    if (lane < 16) y[lane] = xj;
    __syncwarp();
    for (int step = 0; step < 20; ++step) {
        const float k1 = lp_rate_warp(y, i_na, sc, T, lane, q, tab);
        if (lane < 16) y[lane] = xj + .5f * dt * k1;
        __syncwarp();
        const float k2 = lp_rate_warp(y, i_na, sc, T, lane, q, tab);
        if (lane < 16) y[lane] = xj + .5f * dt * k2;
        __syncwarp();
        const float k3 = lp_rate_warp(y, i_na, sc, T, lane, q, tab);
        if (lane < 16) y[lane] = xj + dt * k3;
        __syncwarp();
        const float k4 = lp_rate_warp(y, i_na, sc, T, lane, q, tab);
        xj += dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6.0f;
        if (lane < 16) y[lane] = xj;
        __syncwarp();
    }
    if (lane < 16) x[lane] = xj;
    __syncwarp();
}

// The lane's exponential term of a Prinz substep (pz_substep), level 1 (all
// from the voltage v): gates mi[0..6] (lanes 1-7), the time constants
// mt[0..6] (8-16, the two-exponential ones split over two lanes each), gates
// hi[0..3] (17-20) and the time constants ht[0..3] (21-26). Lane 0 takes the
// logarithm of the calcium reversal. post: 0 none, 1 K1 - K2 g, 2 the
// calcium factor of mi[4].
struct PzTerm {
    LaneTerm t;
    int post;
    float k1, k2;
};
__device__ __forceinline__ PzTerm pz_term(int lane) {
    switch (lane) {
    case 1: return {{F_G, 25.5f, -5.29f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 2: return {{F_G, 27.1f, -7.2f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 3: return {{F_G, 33.0f, -8.1f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 4: return {{F_G, 27.2f, -8.7f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 5: return {{F_G, 28.3f, -12.6f, 0.0f, 1, 0}, 2, 0.0f, 0.0f};
    case 6: return {{F_G, 12.3f, -11.8f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 7: return {{F_G, 75.0f, 5.5f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 8: return {{F_G, 120.0f, -25.0f, 0.0f, 1, 0}, 1, 2.64f, 2.52f};
    case 9: return {{F_G, 68.1f, -20.5f, 0.0f, 1, 0}, 1, 43.4f, 42.6f};
    case 10: return {{F_G, 27.0f, 10.0f, 0.0f, 0, 0}, 0, 0.0f, 0.0f};
    case 11: return {{F_G, 70.0f, -13.0f, 0.0f, 0, 0}, 0, 0.0f, 0.0f};
    case 12: return {{F_G, 32.9f, -15.2f, 0.0f, 1, 0}, 1, 23.2f, 20.8f};
    case 13: return {{F_G, 46.0f, -22.7f, 0.0f, 1, 0}, 1, 180.6f, 150.2f};
    case 14: return {{F_G, 28.3f, -19.2f, 0.0f, 1, 0}, 1, 14.4f, 12.8f};
    case 15: return {{F_P, 0.0f, .086f, -14.59f, 0, 0}, 0, 0.0f, 0.0f};
    case 16: return {{F_Q, 0.0f, .0701f, -1.87f, 0, 0}, 0, 0.0f, 0.0f};
    case 17: return {{F_G, 48.9f, 5.18f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 18: return {{F_G, 32.1f, 5.5f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 19: return {{F_G, 60.0f, 6.2f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 20: return {{F_G, 56.9f, 4.9f, 0.0f, 1, 0}, 0, 0.0f, 0.0f};
    case 21: return {{F_G, 62.9f, -10.0f, 0.0f, 0, 0}, 0, 0.0f, 0.0f};
    case 22: return {{F_G, 34.9f, 3.6f, 0.0f, 0, 0}, 0, 0.0f, 0.0f};
    case 23: return {{F_G, 55.0f, -16.9f, 0.0f, 1, 0}, 1, 210.0f, 179.6f};
    case 24: return {{F_G, 55.0f, 9.0f, 0.0f, 0, 0}, 0, 0.0f, 0.0f};
    case 25: return {{F_G, 65.0f, -16.0f, 0.0f, 0, 0}, 0, 0.0f, 0.0f};
    case 26: return {{F_G, 38.9f, -26.5f, 0.0f, 1, 0}, 1, 77.2f, 58.4f};
    default: return {{F_P, 0.0f, 0.0f, -1.0f, 0, 0}, 0, 0.0f, 0.0f};  // lane 0 and idle lanes: exp(-1), unused
    }
}

// One pz_substep on u (13 floats: v, ca, m[7], h[4]) in shared memory; T
// holds the lanes' level-1 terms.
__device__ __forceinline__ void pz_substep_warp(float *u, const float *g, float ext, float clamp_ns, float clamp_rev,
                                                float *T, int lane, const PzTerm &q, const float *tab) {
    const float dt = .025f;
    const float *m = u + 2, *h = u + 9;
    const float v = u[0], ca = fmaxf(u[1], 0.000001f);
    {   // level 1: one exponential per lane, formed the same way in every lane
        const float p = q.t.form == F_G ? v + q.t.m : q.t.k * v;
        const float arg = q.t.form == F_P ? q.t.c - p : q.t.form == F_Q ? q.t.c + p : p / q.t.k;
        const float e = crexp(arg, tab);
        float t = q.t.sig ? 1.0f / (1.0f + e) : e;
        if (q.post == 1) t = q.k1 - q.k2 * t;
        else if (q.post == 2) t = (ca / (ca + 3)) * t;
        if (lane == 0) t = nsx::logf_cr(3000.0f / ca);
        T[lane] = t;
    }
    __syncwarp();
    // level 2: the voltage and calcium (lane 0), m[i] (lanes 2-8) and h[i]
    // (lanes 9-12), one exponential each
    float arg = -1.0f, gt = 0.0f, ws = 0.0f, eca = 0.0f, c1 = 0.0f, c2 = 0.0f, base = 0.0f, cur = 0.0f;
    if (lane == 0) {
        eca = (8.31451e3f * 283.0f / (2.0f * 96485.3415f)) * T[0];
        const float c[8] = {g[0] * m[0] * m[0] * m[0] * h[0], g[1] * m[1] * m[1] * m[1] * h[1],
                            g[2] * m[2] * m[2] * m[2] * h[2], g[3] * m[3] * m[3] * m[3] * h[3],
                            g[4] * m[4] * m[4] * m[4] * m[4], g[5] * m[5] * m[5] * m[5] * m[5],
                            g[6] * m[6], g[7]};
        const float rev[8] = {50, eca, eca, -80, -80, -80, -20, -50};
        gt = clamp_ns;
        ws = ext + clamp_ns * clamp_rev;
        for (int i = 0; i < 8; ++i) { gt += c[i]; ws += c[i] * rev[i]; }
        c1 = c[1];
        c2 = c[2];
        arg = -dt * gt / 628.3f;
    } else if (lane >= 2 && lane < 13) {
        const bool mg = lane < 9;
        const int i = mg ? lane - 2 : lane - 9;
        base = mg ? T[1 + i] : T[17 + i];
        cur = mg ? m[i] : h[i];
        float tau;
        if (mg) {
            if (i == 2) tau = 2.8f + 14 * (1.0f / (T[10] + T[11]));
            else if (i == 6) tau = 2.0f / (T[15] + T[16]);
            else tau = T[i < 2 ? 8 + i : 9 + i];
        } else {
            if (i == 0) tau = (1.34f / (1 + T[21])) * (1.5f + 1 / (1 + T[22]));
            else if (i == 2) tau = 120 + 300 * (1.0f / (T[24] + T[25]));
            else tau = T[i == 1 ? 23 : 26];
        }
        arg = -dt / tau;
    }
    const float e = crexp(arg, tab);
    float nv = 0.0f, nca = 0.0f;
    if (lane == 0) {
        if (fabsf(gt) < .000001f) nv = v + dt * ws / 628.3f;
        else { const float tg = ws / gt; nv = tg + (v - tg) * e; }
        const float ica = (c1 + c2) * (v - eca) / 1000000.0f;
        const float cat = .05f - 14961.0f * ica;
        nca = fmaxf(.000001f, cat + (ca - cat) * c_K.prinz_ca);
    } else if (lane >= 2 && lane < 13) {
        nv = base + (cur - base) * e;
    }
    __syncwarp();
    if (lane == 0) { u[0] = nv; u[1] = nca; }
    else if (lane >= 2 && lane < 13) u[lane] = nv;
    __syncwarp();
}

// The Prinz cell's 40 substeps of one tick on x (13 state floats); returns
// whether the voltage crossed 0 mV upwards in any substep (all lanes).
static __device__ __noinline__ bool prinz_tick_warp(float *x, const float *xg, float ext, float clamp_ns,
                                                    float clamp_rev, float *w, int lane, const float *tab) {
    float *u = w, *T = w + 16;
    const PzTerm q = pz_term(lane);
    if (lane < 13) u[lane] = x[lane];
    __syncwarp();
    bool spiked = false;
    for (int i = 0; i < 40; ++i) {
        const float before = u[0];
        pz_substep_warp(u, xg, ext, clamp_ns, clamp_rev, T, lane, q, tab);
        spiked |= before < 0 && u[0] >= 0;
    }
    if (lane < 13) x[lane] = u[lane];
    __syncwarp();
    return spiked;
}

// A warp with more LP and Prinz cells than this integrates each on its own
// lane at once (lp_integrate, pz_substep); with fewer, one after another on
// the whole warp. Measured on B200, the lanes' own integration (its
// exponentials batched, crexp_n) is faster for every count in the Gym
// engine, so the warp form is off there by default.
#ifndef NSB_WARP_CELLS_MAX
#define NSB_WARP_CELLS_MAX 0
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
