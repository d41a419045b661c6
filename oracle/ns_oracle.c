/* ORACLE — test infrastructure only (see ns_oracle.h).
 *
 * Plain-C restatement of the reference neural tick, and of the world step
 * around it (body, spatial index, bites, genome reclamation, reproduction with
 * mutation, regrowth, senses: the reference kernels run as loops in ascending
 * animal slot order). Each function cites the reference lines it follows. Arithmetic is written so every binary32
 * operation happens in the reference's order (no contraction: build with
 * -ffp-contract=off), which is what makes a bit-for-bit comparison with the
 * reference's own compiled code meaningful.
 *
 * Exp/log binding: OR_LIBM builds call glibc expf/logf wherever the reference
 * evaluates a state-dependent exponential (the reference host build does the
 * same); constant-argument exponentials, which a C compiler folds to the
 * correctly rounded value, are the correctly rounded constants in both modes.
 * The default build binds every exponential to or_cr_expf/or_cr_logf, and
 * the world step's cosf/sinf/hypotf to or_cr_cosf/or_cr_sinf/or_cr_hypotf.
 */
#include "ns_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef OR_LIBM
#define OEXP expf
#define OLOG logf
#define OCOS cosf
#define OSIN sinf
#define OHYPOT hypotf
#else
#define OEXP or_cr_expf
#define OLOG or_cr_logf
#define OCOS or_cr_cosf
#define OSIN or_cr_sinf
#define OHYPOT or_cr_hypotf
#endif

float or_bound_expf(float x) { return OEXP(x); }
float or_bound_logf(float x) { return OLOG(x); }

/* ---- units and fixed constants (src/physiology.cuh:15-25) ---------------- */
#define DT 1.0f
#define BRANCHES 4
#define E_EXC 0.0f
#define E_INH (-75.0f)
#define MOD_NE 1
#define MOD_5HT 2
#define MOD_DA 4
#define SUBSTEPS 4
#define H_SUB (DT / SUBSTEPS)

/* Correctly rounded constant exponentials, computed once (values a compiler
 * folds `expf(constant)` to). */
static float K_TP, K_TM, K_TY, K_TE;   /* profile 6 trace decays */
static float K_EXC_MS, K_INH_MS, K_EXC_SUB, K_INH_SUB, K_LTP, K_LTD, K_NE,
    K_5HT, K_LFS_THR, K_LFS_OPEN[3], K_PRINZ_CA, K_DEND_OFFSET, K_LOG_UP, K_LOG_DOWN;
static int consts_ready;

static void init_consts(void) {
    if (consts_ready) return;
    K_EXC_MS = or_cr_expf(-DT / 3.0f);        /* physiology.cuh:309 */
    K_INH_MS = or_cr_expf(-DT / 10.0f);       /* physiology.cuh:310 */
    K_EXC_SUB = or_cr_expf(-H_SUB / 3.0f);    /* physiology.cuh:371 */
    K_INH_SUB = or_cr_expf(-H_SUB / 10.0f);   /* physiology.cuh:372 */
    K_LTP = or_cr_expf(-DT / 17.0f);          /* physiology.cuh:537 */
    K_LTD = or_cr_expf(-DT / 34.0f);          /* physiology.cuh:538 */
    K_NE = or_cr_expf(-DT / 7200.0f);         /* physiology.cuh:514 */
    K_5HT = or_cr_expf(-DT / 3600.0f);        /* physiology.cuh:515 */
    K_LFS_THR = or_cr_expf(-1.0f / 10.0f);    /* physiology.cuh:266 */
    K_LFS_OPEN[0] = or_cr_expf(-1.0f / 10.0f);  /* physiology.cuh:262,271 */
    K_LFS_OPEN[1] = or_cr_expf(-1.0f / 40.0f);
    K_LFS_OPEN[2] = or_cr_expf(-1.0f / 750.0f);
    K_PRINZ_CA = or_cr_expf(-0.025f / 200.0f);  /* prinz_cell.cuh:75 */
    K_DEND_OFFSET = 5.0f / (1.0f + or_cr_expf(10.0f));  /* physiology.cuh:228 */
    K_LOG_UP = or_cr_logf(1.92f);             /* physiology.cuh:249 */
    K_LOG_DOWN = or_cr_logf(0.70f);           /* physiology.cuh:250 */
    K_TP = or_cr_expf(-DT / 16.8f);
    K_TM = or_cr_expf(-DT / 33.7f);
    K_TY = or_cr_expf(-DT / 114.0f);
    K_TE = or_cr_expf(-DT / 200.0f);
    consts_ready = 1;
}

static inline float clampf(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }

/* Decisions of the last binary32 call, read by the FP64 shadow (further down)
 * so that it follows the same spike, receptor-event and release outcomes. */
static __thread int dec_rec_event, dec_released;
static __thread unsigned dec_subspikes;

/* ---- records ------------------------------------------------------------- */
typedef struct {               /* src/physiology.cuh:29-45 */
    float cap, gl, el, vt, slope, a, tau_w, b, vr, adp_b, adp_tau;
    unsigned char type, active, modulator, inh_tx;
    float lp_scale[4];         /* src/lp_cell.cuh:19-21 */
    float prinz_g[8];          /* src/prinz_cell.cuh:17 */
    float prinz_leak;
    signed char sens;
    float rec_base, rec_gain, rec_event, rec_decay, affinity;
} ngene;

typedef struct {               /* src/physiology.cuh:50-58 */
    float v, w, adp, inh, depol, log_ampa;
    float dend[BRANCHES];
    float u[16];               /* LP x[16] | Prinz v,ca,m[7],h[4] | LFS v,thr,act[3],open[3] */
    int total;
    unsigned char spike;
    float rec_ns;
    uint32_t rec_rng;
} nstate;

typedef struct {               /* src/physiology.cuh:59-65 */
    float w0, U, trec, tfac;
    int pre, post;
    unsigned char delay, active, plast, branch, sites, receptors;
    float slow_rec, slow_depl;
} sgene;

typedef struct {               /* src/physiology.cuh:66-76 */
    float w, ru, pre_tr, post_tr, el_ltp, el_ltd, da_age, spine, st_age, pre_age, post_age;
    int64_t last;
    uint64_t ready;
    uint32_t rng;
    unsigned char arrived;
    float slow;
} sstate;

/* ---- neuron parameter profiles (src/physiology.cuh:82-176) --------------- */
static ngene blank_gene(void) {
    ngene g; memset(&g, 0, sizeof g);
    g.sens = -1; g.rec_decay = 3.0f; g.affinity = 1.0f;
    return g;
}
static ngene naud_profile(int inhibitory) {          /* 82-89 */
    ngene g = blank_gene();
    if (inhibitory) {
        g.cap = 59; g.gl = 2.9f; g.el = -62; g.vt = -42; g.slope = 3.0f;
        g.a = 1.8f; g.tau_w = 16; g.b = 61; g.vr = -54;
        g.type = 1; g.active = 1; g.inh_tx = 1;
    } else {
        g.cap = 104; g.gl = 4.3f; g.el = -65; g.vt = -52; g.slope = 0.8f;
        g.a = -0.8f; g.tau_w = 88; g.b = 65; g.vr = -53;
        g.type = 0; g.active = 1;
    }
    return g;
}
static ngene profile_for_type(unsigned char type) {  /* 94-176 */
    ngene g;
    switch (type) {
    case 0: g = naud_profile(0); g.vr = -68.0f; g.adp_b = 120.0f; g.adp_tau = 45.0f; break;
    case 1: g = naud_profile(1); break;
    case 2: g = naud_profile(1); g.type = 2;
            for (int i = 0; i < 4; ++i) g.lp_scale[i] = 1; break;
    case 3: g = naud_profile(1); g.type = 3;          /* prinz_cell.cuh:19-24 */
            g.prinz_g[0] = 400 * 628.0f; g.prinz_g[1] = 2.5f * 628;
            g.prinz_g[2] = 6 * 628.0f; g.prinz_g[3] = 50 * 628.0f;
            g.prinz_g[4] = 10 * 628.0f; g.prinz_g[5] = 100 * 628.0f;
            g.prinz_g[6] = .01f * 628; g.prinz_g[7] = 0; break;
    case 4: g = naud_profile(0); g.type = 4; g.cap = 8.7f; g.gl = 8.7f / 12.0f;
            g.el = -60.0f; g.vt = -40.0f; g.vr = -60.0f; g.a = 0; g.b = 0; break;
    case 5: g = naud_profile(0); g.type = 5; g.cap = 10.0f; g.gl = 0.5f;
            g.el = -60.0f; g.vt = -40.0f; g.vr = -60.0f; g.a = 0; g.b = 0;
            g.rec_base = 7.0f; g.rec_gain = 43.0f; g.rec_event = 2.0f; g.rec_decay = 3.0f; break;
    default: g = naud_profile(0); g.type = 6; g.cap = 1200.0f;
            g.gl = 1000.0f / 65.6f; g.el = -45.1f; g.vt = -51.8f; break;
    }
    return g;
}
static int excitatory_kind(unsigned char t) { return t == 0 || t == 4 || t == 5; }  /* 165-167 */

/* 32-bit integer hash seeding the xorshift streams (physiology.cuh:183-187, 395-399). */
static uint32_t seed_hash(uint32_t seed) {
    uint32_t x = seed ? seed : 1u;
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static uint32_t xorshift32(uint32_t x) { x ^= x << 13; x ^= x >> 17; x ^= x << 5; return x; }

/* ---- cell models ---------------------------------------------------------- */
/* LP two-compartment model (src/lp_cell.cuh:23-113). */
static void lp_initial(float *x) {
    static const float init[16] = {-56, 0, .2f, 0, 1, 0, 0, 1, 0, 0, 1, 1, 0, .04f, .01f, -56};
    memcpy(x, init, sizeof init);
}
static float lp_sig(float v, float mid, float slope) { return 1.0f / (1.0f + OEXP((v - mid) / slope)); }
static float lp_ratio(float num, float den, float lim) { return fabsf(den) < 1e-5f ? lim : num / den; }
static void lp_rates(const float *x, float i_na, const float *sc, float *d) {
    const float va = x[0], vs = x[15];
    const float na = x[1] * x[1] * x[1] * x[2] * 7.15f * (va - 50.0f);
    const float kd = x[8] * x[8] * x[8] * x[8] * 1.43f * (va + 72.0f);
    const float km = .2613041227f * x[14] * (va + 80.0f);
    const float aleak = sc[3] * .001004288227f * (va + 50.0f);
    const float cpl = .004017089073f * (vs - va);
    d[0] = (-na - kd - km - aleak + cpl) / .1148312178f;
    const float ev = OEXP(vs / 11.4866f);
    const float ghk = fabsf(vs) < .001f ? 11.4866f * (x[13] - 15123.5f)
                                        : vs * (x[13] * ev - 15123.5f) / (ev - 1.0f);
    const float ca = sc[0] * (x[3] * x[4] * .1247796343f + x[5] * .07142141077f) * .00155982f * ghk * .9f;
    const float kca = sc[1] * x[6] * x[7] * 1.663612026f * (vs + 72.0f) * .9f;
    const float amix = lp_sig(vs, 55.0f, -15.0f);
    const float ka = x[9] * x[9] * x[9] * .8008791415f * (vs + 72.0f) * (amix * x[10] + (1.0f - amix) * x[11]) * .9f;
    const float ih = sc[2] * x[12] * .0126874385f * (vs + 20.0f) * .9f;
    const float sleak = sc[3] * .0006901584324f * (vs + 50.0f);
    d[15] = (-ca - kca - ka - ih - sleak - cpl + (i_na - 2.0f) * .01222505828f) / .0543909161f;
    float a = lp_ratio(-16.64f - .32f * va, OEXP(-13.0f - va / 4.0f) - 1.0f, 1.28f);
    float b = lp_ratio(.28f * va + 7.0f, OEXP(va / 5.0f + 5.0f) - 1.0f, 1.4f);
    d[1] = a * (1.0f - x[1]) - b * x[1];
    a = .128f * OEXP(-2.66666666667f - va / 18.0f);
    b = 4.0f / (OEXP(-5.0f - va / 5.0f) + 1.0f);
    d[2] = a * (1.0f - x[2]) - b * x[2];
    a = lp_ratio(-1.6f - .032f * va, OEXP(-10.0f - va / 5.0f) - 1.0f, .16f);
    b = .5f * OEXP(-1.375f - va / 40.0f);
    d[8] = a * (1.0f - x[8]) - b * x[8];
    d[3] = (lp_sig(vs, 15.0f, -9.8f) - x[3]) * .045f;
    d[4] = (lp_sig(vs, -40.0f, 3.2f) - x[4]) * .02f * lp_sig(vs, -15.0f, -10.0f);
    d[5] = (lp_sig(vs, 29.1336f, -4.43083f) - x[5]) * .0608644f;
    const float cai = x[13];
    const float kca_inf = lp_sig(vs, -.6f * cai, -23.0f) * lp_sig(vs, -16.0f - .6f * cai, -5.0f) * cai / (2.5f + cai);
    d[6] = (kca_inf - x[6]) * .6f;
    d[7] = (.7f / (.6f + cai) - x[7]) * .035f;
    d[9] = (lp_sig(vs, -12.0f, -26.0f) - x[9]) * .14f;
    const float ainf = lp_sig(vs, -62.0f, 6.0f);
    d[10] = (ainf - x[10]) * .05f;
    d[11] = (ainf - x[11]) * .0036f * lp_sig(vs, -40.0f, -12.0f);
    d[12] = (lp_sig(vs, -70.0f, 8.0f) - x[12]) * .00033f / lp_sig(vs, -110.0f, -21.6f);
    d[13] = -.05049639866f * ca - .01729930764f * (cai - .02f);
    d[14] = (lp_sig(va, -26.9916223f, -5.957441281f) - x[14]) * .0001386796618f * lp_sig(va, -60.57875745f, -13.25674673f);
}
static void lp_integrate(float *x, float i_na, const float *sc) {  /* RK4, 20 x 0.05 ms */
    const float dt = .05f;
    for (int step = 0; step < 20; ++step) {
        float k1[16], k2[16], k3[16], k4[16], y[16];
        lp_rates(x, i_na, sc, k1);
        for (int j = 0; j < 16; ++j) y[j] = x[j] + .5f * dt * k1[j];
        lp_rates(y, i_na, sc, k2);
        for (int j = 0; j < 16; ++j) y[j] = x[j] + .5f * dt * k2[j];
        lp_rates(y, i_na, sc, k3);
        for (int j = 0; j < 16; ++j) y[j] = x[j] + dt * k3[j];
        lp_rates(y, i_na, sc, k4);
        for (int j = 0; j < 16; ++j) x[j] += dt * (k1[j] + 2 * k2[j] + 2 * k3[j] + k4[j]) / 6.0f;
    }
}

/* Prinz pacemaker (src/prinz_cell.cuh:45-121); u = {v, ca, m[7], h[4]}. */
static float pz_gate(float v, float a, float b) { return 1.0f / (1.0f + OEXP((v + a) / b)); }
static float pz_gate2(float v, float a, float b, float c, float d) { return 1.0f / (OEXP((v + a) / b) + OEXP((v + c) / d)); }
static void pz_substep(float *u, const float *g, float ext_pa, float clamp_ns, float clamp_rev) {
    const float dt = .025f;
    float *m = u + 2, *h = u + 9;
    const float v = u[0], ca = fmaxf(u[1], 0.000001f);
    const float eca = (8.31451e3f * 283.0f / (2.0f * 96485.3415f)) * OLOG(3000.0f / ca);
    const float c[8] = {g[0] * m[0] * m[0] * m[0] * h[0], g[1] * m[1] * m[1] * m[1] * h[1],
                        g[2] * m[2] * m[2] * m[2] * h[2], g[3] * m[3] * m[3] * m[3] * h[3],
                        g[4] * m[4] * m[4] * m[4] * m[4], g[5] * m[5] * m[5] * m[5] * m[5],
                        g[6] * m[6], g[7]};
    const float rev[8] = {50, eca, eca, -80, -80, -80, -20, -50};
    float gt = clamp_ns, wsum = ext_pa + clamp_ns * clamp_rev;
    for (int i = 0; i < 8; ++i) { gt += c[i]; wsum += c[i] * rev[i]; }
    if (fabsf(gt) < .000001f) u[0] = v + dt * wsum / 628.3f;
    else { const float tgt = wsum / gt; u[0] = tgt + (v - tgt) * OEXP(-dt * gt / 628.3f); }
    const float ica = (c[1] + c[2]) * (v - eca) / 1000000.0f;
    const float ca_t = .05f - 14961.0f * ica;
    u[1] = fmaxf(.000001f, ca_t + (ca - ca_t) * K_PRINZ_CA);
    const float mi[7] = {pz_gate(v, 25.5f, -5.29f), pz_gate(v, 27.1f, -7.2f), pz_gate(v, 33, -8.1f),
                         pz_gate(v, 27.2f, -8.7f), (ca / (ca + 3)) * pz_gate(v, 28.3f, -12.6f),
                         pz_gate(v, 12.3f, -11.8f), pz_gate(v, 75, 5.5f)};
    const float mt[7] = {2.64f - 2.52f * pz_gate(v, 120, -25), 43.4f - 42.6f * pz_gate(v, 68.1f, -20.5f),
                         2.8f + 14 * pz_gate2(v, 27, 10, 70, -13), 23.2f - 20.8f * pz_gate(v, 32.9f, -15.2f),
                         180.6f - 150.2f * pz_gate(v, 46, -22.7f), 14.4f - 12.8f * pz_gate(v, 28.3f, -19.2f),
                         2.0f / (OEXP(-14.59f - .086f * v) + OEXP(-1.87f + .0701f * v))};
    for (int i = 0; i < 7; ++i) m[i] = mi[i] + (m[i] - mi[i]) * OEXP(-dt / mt[i]);
    const float hi_[4] = {pz_gate(v, 48.9f, 5.18f), pz_gate(v, 32.1f, 5.5f), pz_gate(v, 60, 6.2f), pz_gate(v, 56.9f, 4.9f)};
    const float ht[4] = {(1.34f / (1 + OEXP((v + 62.9f) / -10))) * (1.5f + 1 / (1 + OEXP((v + 34.9f) / 3.6f))),
                         210 - 179.6f * pz_gate(v, 55, -16.9f), 120 + 300 * pz_gate2(v, 55, 9, 65, -16),
                         77.2f - 58.4f * pz_gate(v, 38.9f, -26.5f)};
    for (int i = 0; i < 4; ++i) h[i] = hi_[i] + (h[i] - hi_[i]) * OEXP(-dt / ht[i]);
}
static int pz_advance(float *u, const float *g, float ext_pa, float clamp_ns, float clamp_rev) {
    int spiked = 0;
    for (int i = 0; i < 40; ++i) {
        const float before = u[0];
        pz_substep(u, g, ext_pa, clamp_ns, clamp_rev);
        spiked |= before < 0 && u[0] >= 0;
    }
    return spiked;
}

/* LFS integrate-and-fire (src/physiology.cuh:258-287); u = {v, thr, act[3], open[3]}. */
static void lfs_step(const ngene *g, nstate *s, float cur, float exc, float inh) {
    static const float wt[3] = {250.0f, 10.0f, 4.0f}, op[3] = {10.0f, 40.0f, 750.0f}, cl[3] = {50.0f, 750.0f, 2000.0f};
    float *u = s->u, *act = u + 2, *open = u + 5;
    u[1] = g->vt + (u[1] - g->vt) * K_LFS_THR;
    float under = 0;
    for (int j = 0; j < 3; ++j) {
        open[j] += act[j] / op[j] - open[j] / cl[j];
        act[j] *= K_LFS_OPEN[j];
        under += wt[j] * open[j];
    }
    const float v = u[0];
    const float i = g->gl * (g->el - v) + exc * (10.0f - v) + inh * (-60.0f - v) + under * (-80.0f - v) + cur;
    u[0] = v + i / g->cap;
    s->spike = u[0] >= u[1];
    if (s->spike) {
        dec_subspikes = 1u;
        u[1] = 200.0f;
        for (int j = 0; j < 3; ++j) act[j] += 1.0f;
        ++s->total;
    }
    s->v = u[0];
}

/* ---- neuron ---------------------------------------------------------------- */
static nstate neuron_initial(const ngene *g, uint32_t seed) {     /* physiology.cuh:179-202 */
    nstate s; memset(&s, 0, sizeof s);
    s.v = g->el;
    uint32_t x = seed_hash(seed);
    s.rec_rng = x ? x : 1u;
    if (g->type == 2) { lp_initial(s.u); s.v = s.u[15] - 9.342518882f; }
    if (g->type == 3) {
        memset(s.u, 0, sizeof s.u);
        s.u[0] = -50.0f; s.u[1] = .05f;
        for (int i = 0; i < 4; ++i) s.u[9 + i] = 1.0f;
        s.v = s.u[0];
    }
    if (g->type == 6) { memset(s.u, 0, sizeof s.u); s.u[0] = g->el; s.u[1] = g->vt; }
    return s;
}

static float receptor_drive(const ngene *g, nstate *s, float level) {  /* physiology.cuh:206-219 */
    if (g->sens < 0 || g->rec_event <= 0) return 0;
    float rate = clampf(g->rec_base + g->rec_gain * level, 0, 1000);
    s->rec_rng = xorshift32(s->rec_rng);
    float u = (float)(s->rec_rng >> 8) * (1.0f / 16777216.0f);
    s->rec_ns *= OEXP(-DT / g->rec_decay);
    dec_rec_event = u < rate * (DT / 1000.0f);
    if (dec_rec_event) s->rec_ns += g->rec_event;
    return s->rec_ns * (E_EXC - s->v);
}

static float branch_gain(float gs) {                               /* physiology.cuh:226-230 */
    float regen = 5.0f / (1.0f + OEXP(-(gs - 4.0f) / 0.4f));
    return fminf(11.0f, gs + regen - K_DEND_OFFSET);
}

static void homeostasis(const ngene *g, nstate *s, float elapsed, float hz) {  /* 243-253 */
    if (g->type != 0) return;
    float ratio = clampf(hz / 0.4f, 0.0f, 2.65f);
    float change = ratio < 1.0f ? K_LOG_UP * (1.0f - ratio) : K_LOG_DOWN * ((ratio - 1.0f) / 1.65f);
    s->log_ampa = clampf(s->log_ampa + change * (elapsed / 172800000.0f), -3.0f, 3.0f);
}

/* physiology.cuh:290-374 (clamp_leak = 0, clamp_reversal = -68 as every caller passes). */
static void neuron_tick(const ngene *g, nstate *s, float cur, const float *exc_in, float inh_in) {
    const float clamp_leak = 0.0f, clamp_rev = -68.0f;
    for (int k = 0; k < BRANCHES; ++k) s->dend[k] += exc_in[k];
    float sub = fmaxf(0.0f, fminf(s->v, -50.0f) - g->el);
    s->depol += 0.1f * (sub - s->depol);
    s->inh += inh_in;
    s->spike = 0;
    dec_subspikes = 0;
    if (g->type == 6 || g->type == 2 || g->type == 3) {
        float exc = 0;
        for (int k = 0; k < BRANCHES; ++k) exc += s->dend[k];
        if (g->type == 6) {
            lfs_step(g, s, cur, exc, s->inh);
        } else if (g->type == 2) {
            float axon_before = s->u[0];
            float ext = cur + exc * (E_EXC - s->v) + s->inh * (E_INH - s->v) - clamp_leak * (s->v - clamp_rev);
            lp_integrate(s->u, ext / 1000.0f, g->lp_scale);
            s->v = s->u[15] - 9.342518882f;
            s->spike = axon_before < 0 && s->u[0] >= 0;
            s->total += s->spike;
        } else {
            const float ext = cur + exc * (E_EXC - s->v) + s->inh * (E_INH - s->v);
            s->spike = (unsigned char)pz_advance(s->u, g->prinz_g, ext, g->prinz_leak + clamp_leak, clamp_rev);
            s->total += s->spike;
            s->v = s->u[0];
        }
        for (int k = 0; k < BRANCHES; ++k) s->dend[k] *= K_EXC_MS;
        s->inh *= K_INH_MS;
        return;
    }
    for (int step = 0; step < SUBSTEPS; ++step) {
        float v = s->v;
        s->w += H_SUB * (g->a * (v - g->el) - s->w) / g->tau_w;
        float expo = clampf((v - g->vt) / g->slope, -20.0f, 10.0f);
        float soma = 0;
        for (int k = 0; k < BRANCHES; ++k) soma += g->type == 0 ? branch_gain(s->dend[k]) : s->dend[k];
        float dv = g->gl * (g->el - v) + g->gl * g->slope * OEXP(expo) + soma * (E_EXC - v) +
                   s->inh * (E_INH - v) + cur + s->adp - s->w - clamp_leak * (v - clamp_rev);
        s->v = v + H_SUB * dv / g->cap;
        if (s->v >= 0.0f) {
            dec_subspikes |= 1u << step;
            s->spike = 1; ++s->total;
            s->v = g->vr; s->w += g->b; s->adp += g->adp_b;
        }
        if (g->adp_tau > 0) s->adp *= OEXP(-H_SUB / g->adp_tau);
        for (int k = 0; k < BRANCHES; ++k) s->dend[k] *= K_EXC_SUB;
        s->inh *= K_INH_SUB;
    }
}

/* ---- synapse ---------------------------------------------------------------- */
static int sites_of(const sgene *g) { return g->sites ? (g->sites > 64 ? 64 : g->sites) : 14; }  /* 376-378 */
static float uniform24(sstate *s) { s->rng = xorshift32(s->rng); return (float)(s->rng >> 8) * (1.0f / 16777216.0f); }

static sstate synapse_initial(const sgene *g, uint32_t seed) {  /* 393-404 */
    sstate s; memset(&s, 0, sizeof s);
    uint32_t x = seed_hash(seed);
    if (!x) x = 1;
    int n = sites_of(g);
    s.w = g->w0; s.da_age = -1; s.spine = 1; s.st_age = -1;
    s.pre_age = 1000000; s.post_age = 1000000; s.last = -1000000;
    s.ready = n == 64 ? ~(uint64_t)0 : (((uint64_t)1 << n) - 1);
    s.rng = x; s.arrived = 0; s.slow = 1;
    return s;
}

static float da_window(float age) {                     /* 408-412 */
    if (age < 0 || age > 20000.0f) return 0;
    float x = age / 2000.0f;
    return x * x * x * x * OEXP(4.0f * (1.0f - x));
}
static float spine_window(float age) {                  /* 416-420 */
    if (age < 0 || age > 5000.0f) return 0;
    float x = age / 1000.0f;
    return x * x * x * OEXP(3.0f * (1.0f - x));
}

static float release(const sgene *g, sstate *s, int64_t tick) {  /* 425-454 */
    float p_rec = 0;
    if (s->last > -1000000) {
        float dt = (float)(tick - s->last) * DT;
        p_rec = 1.0f - OEXP(-dt / g->trec);
        if (g->tfac > 0) s->ru *= OEXP(-dt / g->tfac);
        if (g->slow_rec > 0) s->slow = 1.0f - (1.0f - s->slow) * OEXP(-dt / g->slow_rec);
    }
    s->ru = g->tfac > 0 ? s->ru + g->U * (1.0f - s->ru) : g->U;
    int released = 0, n = sites_of(g);
    for (int site = 0; site < n; ++site) {
        uint64_t bit = (uint64_t)1 << site;
        if (!(s->ready & bit) && uniform24(s) < p_rec) s->ready |= bit;
        if ((s->ready & bit) && uniform24(s) < s->ru) { s->ready &= ~bit; ++released; }
    }
    s->last = tick;
    dec_released = released;
    float out = s->w * (float)released / (float)n * s->slow;
    if (g->slow_rec > 0) s->slow *= 1.0f - g->slow_depl;
    return out;
}

/* physiology.cuh:459-555 with nmda/l-type/cp-AMPA/PKA all available. */
static void plasticity_tick(const sgene *g, sstate *s, int arrived, int post_spike, int pair,
                            float depol, unsigned char mod) {
    if (!g->plast || !pair) return;
    if (g->plast == 6) {
        /* No reference counterpart (the reference's profiles are 1-5): triplet
         * STDP, Pfister & Gerstner 2006 minimal all-to-all model (tau+ 16.8,
         * tau- 33.7, tau_y 114 ms, A3+ 6.5e-3, A2- 7.1e-3), written into an
         * eligibility trace (tau 200 ms) that a dopamine event applies to the
         * weight. pre_tr = r1, post_tr = o1, el_ltd = o2, el_ltp = e. */
        s->pre_tr *= K_TP; s->post_tr *= K_TM; s->el_ltd *= K_TY; s->el_ltp *= K_TE;
        s->pre_age += DT; s->post_age += DT;
        if (arrived) { s->el_ltp -= 0.0071f * s->post_tr; s->pre_tr += 1.0f; s->pre_age = 0; }
        if (post_spike) { s->el_ltp += 0.0065f * s->pre_tr * s->el_ltd; s->post_tr += 1.0f; s->el_ltd += 1.0f; s->post_age = 0; }
        if ((mod & MOD_DA) && (g->receptors & MOD_DA)) s->w += g->w0 * s->el_ltp;
        s->w = clampf(s->w, 0.0f, 2.0f * g->w0);
        return;
    }
    if (g->plast == 5) {
        if (s->st_age >= 0) { s->st_age += DT; if (s->st_age > 5000.0f) s->st_age = -1; }
        s->pre_age += DT;
        if (arrived) s->pre_age = 0;
        if (post_spike && s->pre_age <= 15.0f && s->st_age < 0) s->st_age = 0;
        if ((mod & MOD_DA) && (g->receptors & MOD_DA))
            s->spine = clampf(s->spine + 0.025f * spine_window(s->st_age), 1.0f, 2.0f);
        return;
    }
    if (g->plast == 4) {
        if (s->da_age >= 0) { s->da_age += DT; if (s->da_age > 20000.0f) s->da_age = -1; }
        s->pre_age += DT;
        if (arrived) s->pre_age = 0;
        if (post_spike && s->pre_age <= 15.0f && (s->da_age < 0 || s->da_age > 30.0f)) {
            s->da_age = 0;
            s->w -= 0.005383f * g->w0;
        }
        if ((mod & MOD_DA) && (g->receptors & MOD_DA)) {
            s->w += 0.00453f * da_window(s->da_age) * g->w0;
            s->da_age = -1;
        }
        s->w = clampf(s->w, 0.0f, 2.0f * g->w0);
        return;
    }
    if (g->plast == 3) {
        s->el_ltp *= K_NE;
        s->el_ltd *= K_5HT;
        s->pre_age += DT; s->post_age += DT;
        if (arrived) { if (s->post_age <= 15.0f) s->el_ltd += 1.0f; s->pre_age = 0; }
        if (post_spike) { if (s->pre_age <= 15.0f) s->el_ltp += 1.0f; s->post_age = 0; }
        if ((mod & MOD_NE) && (g->receptors & MOD_NE)) { s->w += 0.0048f * s->el_ltp * g->w0; s->el_ltp = 0; }
        if ((mod & MOD_5HT) && (g->receptors & MOD_5HT)) { s->w -= 0.0075f * s->el_ltd * g->w0; s->el_ltd = 0; }
        s->w = clampf(s->w, 0.0f, 2.0f * g->w0);
        return;
    }
    s->pre_tr *= K_LTP;
    s->post_tr *= K_LTD;
    s->pre_age += DT; s->post_age += DT;
    if (arrived) {
        if (s->post_age <= (g->plast == 2 ? 50.0f : 20.0f)) s->w *= 1.0f - 0.004f * s->post_tr;
        s->pre_tr += 1.0f;
        s->pre_age = 0;
    }
    if (post_spike) {
        if (s->pre_age <= 20.0f && (g->plast == 1 || depol >= 2.3f))
            s->w += 0.016f * s->pre_tr * (2.0f * g->w0 - s->w);
        s->post_tr += 1.0f;
        s->post_age = 0;
    }
    s->w = clampf(s->w, 0.0f, 2.0f * g->w0);
}

/* physiology.cuh:559-586 */
static void plasticity_quiet(const sgene *g, sstate *s, int ticks) {
    if (ticks <= 0 || !g->plast) return;
    float el = (float)ticks * DT;
    if (g->plast == 5) {
        if (s->st_age >= 0) { s->st_age += el; if (s->st_age > 5000.0f) s->st_age = -1; }
        s->pre_age += el;
    } else if (g->plast == 4) {
        if (s->da_age >= 0) { s->da_age += el; if (s->da_age > 20000.0f) s->da_age = -1; }
        s->pre_age += el;
    } else if (g->plast == 3) {
        s->el_ltp *= OEXP(-el / 7200.0f);
        s->el_ltd *= OEXP(-el / 3600.0f);
        s->pre_age += el; s->post_age += el;
    } else {
        s->pre_tr *= OEXP(-el / 17.0f);
        s->post_tr *= OEXP(-el / 34.0f);
        s->pre_age += el; s->post_age += el;
    }
}

/* ---- brain (gym_adapter/native.cpp:23-38, core.cuh:12-75) ------------------ */
#define RING 32
struct or_brain {
    int count, edges, channels, outputs, ring;
    ngene *ng; sgene *sg; nstate *ns; sstate *ss;
    int *motors, *sensory;
    uint8_t *hist;              /* count x ring spike bytes, slot tick % ring */
    float *exc, *inh; uint8_t *mod;
    uint32_t *orig_n, *orig_s;
    int64_t tick, events;
    int pulse_period;           /* global modulator pulse (0: none) */
    uint8_t pulse_mod;
    struct or_shadow *sh;       /* FP64 shadow, or NULL */
};

/* ---- FP64 shadow ----------------------------------------------------------------
 * The same equations in binary64 (decimal constants, exp/log of libm in
 * double), stepped beside the binary32 state. Every discrete outcome (spike
 * and the substep it fell in, receptor event, released site count, modulator
 * bits, the depolarisation gate of profile 2) is taken from the binary32 run,
 * so the two trajectories differ only by rounding and the tracked maxima are
 * the binary32 state's error against the FP64 model. LP and Prinz cells
 * (types 2 and 3) have no shadow. */
typedef struct { double v, w, adp, inh, depol, log_ampa, dend[BRANCHES], u[8], rec_ns; } dnstate;
typedef struct { double w, ru, pre_tr, post_tr, el_ltp, el_ltd, da_age, spine, st_age, pre_age, post_age, slow; } dsstate;
struct or_shadow {
    dnstate *n; dsstate *s; double *exc, *inh;
    double maxabs[OR_SHADOW_FIELDS], maxrel[OR_SHADOW_FIELDS];
    int64_t ticks;
};
static void sh_sync(or_brain *b);
static void sh_deliver(or_brain *b, int j, int64_t last0);
static void sh_neuron(or_brain *b, int j, const float *input, float gain);
static void sh_plast(or_brain *b, int j, int pair);
static void sh_track(or_brain *b, int tick_end);
static void sh_homeo(or_brain *b, int j, int ticks);

static int bad(char *err, int len, const char *msg) { if (err && len > 0) snprintf(err, (size_t)len, "%s", msg); return 0; }

or_brain *or_create(int count, int edges, int channels, int outputs, const float *ngr,
                    const float *sgr, const int *motors, int max_delay, char *err, int errlen) {
    init_consts();
    if (count < 1 || edges < 0 || channels < 1 || channels > 65535 || outputs < 1) {
        bad(err, errlen, "Invalid brain dimensions"); return NULL;
    }
    if (max_delay < 1 || max_delay > RING - 1) { bad(err, errlen, "Invalid delay ring"); return NULL; }
    or_brain *b = (or_brain *)calloc(1, sizeof *b);
    b->count = count; b->edges = edges; b->channels = channels; b->outputs = outputs;
    b->ring = max_delay + 1;
    b->ng = (ngene *)calloc((size_t)count, sizeof(ngene));
    b->sg = (sgene *)calloc((size_t)(edges ? edges : 1), sizeof(sgene));
    b->ns = (nstate *)calloc((size_t)count, sizeof(nstate));
    b->ss = (sstate *)calloc((size_t)(edges ? edges : 1), sizeof(sstate));
    b->motors = (int *)calloc((size_t)outputs, sizeof(int));
    b->sensory = (int *)calloc((size_t)count, sizeof(int));
    b->hist = (uint8_t *)calloc((size_t)count * RING, 1);
    b->exc = (float *)calloc((size_t)count * BRANCHES, sizeof(float));
    b->inh = (float *)calloc((size_t)count, sizeof(float));
    b->mod = (uint8_t *)calloc((size_t)count, 1);
    for (int i = 0; i < count; ++i) {                          /* native.cpp:53-66 */
        const float *p = ngr + (size_t)i * 10;
        for (int f = 0; f < 10; ++f) if (p[f] != p[f]) { bad(err, errlen, "Invalid neuron gene"); or_destroy(b); return NULL; }
        if (p[0] < 0 || p[0] > 6 || p[1] < -1 || p[1] >= channels || p[2] < 0 || p[2] > 1 || p[3] < 0 ||
            p[3] > 1 || p[4] < 0 || p[4] > 3) { bad(err, errlen, "Invalid neuron gene"); or_destroy(b); return NULL; }
        ngene g = profile_for_type((unsigned char)p[0]);
        b->sensory[i] = (int)p[1];
        g.sens = p[1] < 0 ? -1 : 0;
        g.active = (unsigned char)p[2];
        g.inh_tx = (unsigned char)p[3];
        g.modulator = (unsigned char)p[4];
        if (p[5] <= 0 || p[6] <= 0 || p[7] < -80 || p[7] > -20 || p[8] < 0 || p[9] < 0) {
            bad(err, errlen, "Invalid membrane parameters"); or_destroy(b); return NULL;
        }
        g.cap *= p[5]; g.gl *= p[6]; g.vt = p[7];
        g.rec_base = 0; g.rec_gain = p[8]; g.rec_event = p[9];
        b->ng[i] = g;
    }
    for (int i = 0; i < edges; ++i) {                          /* native.cpp:67-75 */
        const float *p = sgr + (size_t)i * 11;
        for (int f = 0; f < 11; ++f) if (p[f] != p[f]) { bad(err, errlen, "Invalid synapse gene"); or_destroy(b); return NULL; }
        if (p[0] < 0 || p[0] >= count || p[1] < 0 || p[1] >= count || p[2] < 0 || p[3] < 0 || p[3] > 1 ||
            p[4] < 1 || p[4] > max_delay || p[5] < 0 || p[5] >= BRANCHES || p[6] <= 0 || p[6] > 1 ||
            p[7] <= 0 || p[8] < 0 || p[9] < 0 || p[9] > (max_delay > 8 ? 6 : 5) || p[10] < 0 || p[10] > 7) {
            bad(err, errlen, "Invalid synapse gene"); or_destroy(b); return NULL;
        }
        sgene g; memset(&g, 0, sizeof g);
        g.pre = (int)p[0]; g.post = (int)p[1]; g.w0 = p[2];
        g.active = (unsigned char)p[3]; g.delay = (unsigned char)p[4]; g.branch = (unsigned char)p[5];
        g.U = p[6]; g.trec = p[7]; g.tfac = p[8];
        g.plast = (unsigned char)p[9]; g.receptors = (unsigned char)p[10]; g.sites = 14;
        b->sg[i] = g;
    }
    for (int i = 0; i < outputs; ++i) {
        if (motors[i] < 0 || motors[i] >= count) { bad(err, errlen, "Invalid motor index"); or_destroy(b); return NULL; }
        b->motors[i] = motors[i];
    }
    return b;
}

void or_original_indices(or_brain *b, const uint32_t *neurons, const uint32_t *synapses) {
    free(b->orig_n); free(b->orig_s);
    b->orig_n = (uint32_t *)malloc((size_t)b->count * 4);
    memcpy(b->orig_n, neurons, (size_t)b->count * 4);
    b->orig_s = NULL;
    if (b->edges) {
        b->orig_s = (uint32_t *)malloc((size_t)b->edges * 4);
        memcpy(b->orig_s, synapses, (size_t)b->edges * 4);
    }
}

void or_set_pulse(or_brain *b, int period, int mod) {
    b->pulse_period = mod ? period : 0;
    b->pulse_mod = (uint8_t)(period ? mod : 0);
}

void or_destroy(or_brain *b) {
    if (!b) return;
    free(b->ng); free(b->sg); free(b->ns); free(b->ss); free(b->motors); free(b->sensory);
    free(b->hist); free(b->exc); free(b->inh); free(b->mod); free(b->orig_n); free(b->orig_s);
    if (b->sh) { free(b->sh->n); free(b->sh->s); free(b->sh->exc); free(b->sh->inh); free(b->sh); }
    free(b);
}

void or_reset(or_brain *b, uint32_t seed) {                    /* core.cuh:25-29, native.cpp:89-94 */
    b->tick = 0;
    for (int i = 0; i < b->count; ++i) {
        uint32_t idx = b->orig_n ? b->orig_n[i] : (uint32_t)i;
        b->ns[i] = neuron_initial(&b->ng[i], seed + idx * 7919u);
        memset(b->hist + (size_t)i * RING, 0, RING);
    }
    for (int i = 0; i < b->edges; ++i) {
        uint32_t idx = b->orig_s ? b->orig_s[i] : (uint32_t)i;
        b->ss[i] = synapse_initial(&b->sg[i], seed + idx * 104729u);
    }
    if (b->sh) sh_sync(b);
}

static int edge_live(const or_brain *b, const sgene *g) {
    return g->active && b->ng[g->pre].active && b->ng[g->post].active;
}

int or_step(or_brain *b, const float *input, int ticks, float gain, float *output,
            uint8_t *raster, int stop_on_nonfinite) {                /* core.cuh:30-75 */
    int failed = 0;
    const int64_t tick0 = b->tick;
    b->events = 0;
    for (int j = 0; j < b->outputs; ++j) output[j] = 0;
    for (int t = 0; t < ticks; ++t, ++b->tick) {
        memset(b->exc, 0, sizeof(float) * (size_t)b->count * BRANCHES);
        memset(b->inh, 0, sizeof(float) * (size_t)b->count);
        memset(b->mod, 0, (size_t)b->count);
        if (b->sh) {
            memset(b->sh->exc, 0, sizeof(double) * (size_t)b->count * BRANCHES);
            memset(b->sh->inh, 0, sizeof(double) * (size_t)b->count);
        }
        for (int j = 0; j < b->edges; ++j) {                     /* delivery, edge order */
            const sgene *g = &b->sg[j]; sstate *s = &b->ss[j];
            s->arrived = 0;
            if (!edge_live(b, g)) continue;
            s->arrived = b->tick >= g->delay &&
                         b->hist[(size_t)g->pre * RING + (size_t)((b->tick - g->delay) % b->ring)];
            if (!s->arrived) continue;
            ++b->events;
            const ngene *src = &b->ng[g->pre];
            const int64_t last0 = s->last;
            float rel = (!src->inh_tx || src->modulator) ? release(g, s, b->tick) : s->w;
            if (b->sh) sh_deliver(b, j, last0);
            if (src->modulator) { if (rel > 0) b->mod[g->post] |= (uint8_t)(1u << (src->modulator - 1)); }
            else if (src->inh_tx) b->inh[g->post] += rel;
            else b->exc[(size_t)g->post * BRANCHES + g->branch] += rel * OEXP(b->ns[g->post].log_ampa);
        }
        for (int j = 0; j < b->count; ++j) {                     /* neurons, index order */
            const ngene *g = &b->ng[j]; nstate *s = &b->ns[j];
            if (g->active) {
                float cur = 0;
                if (b->sensory[j] >= 0)
                    cur = g->type == 5 ? receptor_drive(g, s, input[b->sensory[j]]) : gain * input[b->sensory[j]];
                neuron_tick(g, s, cur, b->exc + (size_t)j * BRANCHES, b->inh[j]);
                if (b->sh) sh_neuron(b, j, input, gain);
                if (!isfinite(s->v)) {
                    /* ns_step keeps its tick counter on failure (native.cpp:101-102) */
                    if (stop_on_nonfinite) { b->tick = tick0; return -1; }
                    failed = 1;
                }
            } else s->spike = 0;
            b->hist[(size_t)j * RING + (size_t)(b->tick % b->ring)] = s->spike;
            if (raster) raster[(size_t)t * b->count + j] = s->spike;
        }
        if (b->pulse_period > 0 && b->tick % b->pulse_period == 0)   /* global modulator pulse */
            for (int j = 0; j < b->count; ++j) b->mod[j] |= b->pulse_mod;
        for (int j = 0; j < b->edges; ++j) {                     /* plasticity, edge order */
            const sgene *g = &b->sg[j]; sstate *s = &b->ss[j];
            if (!edge_live(b, g)) continue;
            const ngene *a = &b->ng[g->pre], *z = &b->ng[g->post];
            int pair = !a->inh_tx && excitatory_kind(a->type) && !a->modulator && !z->inh_tx && excitatory_kind(z->type);
            plasticity_tick(g, s, s->arrived, b->ns[g->post].spike, pair, b->ns[g->post].depol, b->mod[g->post]);
            if (b->sh) sh_plast(b, j, pair);
        }
        for (int j = 0; j < b->outputs; ++j) output[j] += (float)b->ns[b->motors[j]].spike;
        if (b->sh) sh_track(b, 1);
    }
    for (int j = 0; j < b->count; ++j)                            /* homeostasis, core.cuh:71-72 */
        if (b->ng[j].active) {
            homeostasis(&b->ng[j], &b->ns[j], (float)ticks,
                        (float)b->ns[j].total * 1000.0f / (float)(ticks > b->tick ? ticks : b->tick));
            if (b->sh) sh_homeo(b, j, ticks);
        }
    if (b->sh) sh_track(b, 0);
    return failed ? -1 : 0;
}

/* ---- FP64 shadow: equations ------------------------------------------------ */
static double dclamp(double x, double lo, double hi) { return fmin(hi, fmax(lo, x)); }

static void sh_copy_neuron(dnstate *d, const nstate *s) {
    d->v = s->v; d->w = s->w; d->adp = s->adp; d->inh = s->inh; d->depol = s->depol;
    d->log_ampa = s->log_ampa; d->rec_ns = s->rec_ns;
    for (int k = 0; k < BRANCHES; ++k) d->dend[k] = s->dend[k];
    for (int k = 0; k < 8; ++k) d->u[k] = s->u[k];
}
static void sh_copy_synapse(dsstate *d, const sstate *s) {
    d->w = s->w; d->ru = s->ru; d->pre_tr = s->pre_tr; d->post_tr = s->post_tr; d->el_ltp = s->el_ltp;
    d->el_ltd = s->el_ltd; d->da_age = s->da_age; d->spine = s->spine; d->st_age = s->st_age;
    d->pre_age = s->pre_age; d->post_age = s->post_age; d->slow = s->slow;
}
static void sh_sync(or_brain *b) {
    for (int i = 0; i < b->count; ++i) sh_copy_neuron(&b->sh->n[i], &b->ns[i]);
    for (int i = 0; i < b->edges; ++i) sh_copy_synapse(&b->sh->s[i], &b->ss[i]);
}

int or_shadow_enable(or_brain *b) {
    for (int i = 0; i < b->count; ++i)
        if (b->ng[i].active && (b->ng[i].type == 2 || b->ng[i].type == 3)) return -1;
    if (!b->sh) {
        struct or_shadow *sh = (struct or_shadow *)calloc(1, sizeof *sh);
        sh->n = (dnstate *)calloc((size_t)b->count, sizeof(dnstate));
        sh->s = (dsstate *)calloc((size_t)(b->edges ? b->edges : 1), sizeof(dsstate));
        sh->exc = (double *)calloc((size_t)b->count * BRANCHES, sizeof(double));
        sh->inh = (double *)calloc((size_t)b->count, sizeof(double));
        b->sh = sh;
    }
    sh_sync(b);
    return 0;
}

/* release() (physiology.cuh:425-454) with the released site count given. */
static double sh_release(const sgene *g, dsstate *d, int64_t last0, int64_t tick, int released) {
    if (last0 > -1000000) {
        const double dt = (double)(tick - last0);
        if (g->tfac > 0) d->ru *= exp(-dt / g->tfac);
        if (g->slow_rec > 0) d->slow = 1.0 - (1.0 - d->slow) * exp(-dt / g->slow_rec);
    }
    d->ru = g->tfac > 0 ? d->ru + g->U * (1.0 - d->ru) : g->U;
    const double out = d->w * (double)released / (double)sites_of(g) * d->slow;
    if (g->slow_rec > 0) d->slow *= 1.0 - (double)g->slow_depl;
    return out;
}

static void sh_deliver(or_brain *b, int j, int64_t last0) {
    const sgene *g = &b->sg[j];
    const ngene *src = &b->ng[g->pre];
    dsstate *d = &b->sh->s[j];
    const double rel = (!src->inh_tx || src->modulator) ? sh_release(g, d, last0, b->tick, dec_released) : d->w;
    if (src->modulator) return;                 /* modulator bits come from the binary32 run */
    if (src->inh_tx) b->sh->inh[g->post] += rel;
    else b->sh->exc[(size_t)g->post * BRANCHES + g->branch] += rel * exp(b->sh->n[g->post].log_ampa);
}

static double sh_branch_gain(double gs) {
    const double regen = 5.0 / (1.0 + exp(-(gs - 4.0) / 0.4));
    return fmin(11.0, gs + regen - 5.0 / (1.0 + exp(10.0)));
}

/* neuron_tick (physiology.cuh:290-374) and lfs_advance (258-287) in binary64;
 * spikes and receptor events as decided by the binary32 step just taken. */
static void sh_neuron(or_brain *b, int j, const float *input, float gain) {
    const ngene *g = &b->ng[j];
    dnstate *d = &b->sh->n[j];
    const double *exc_in = b->sh->exc + (size_t)j * BRANCHES;
    double cur = 0;
    if (b->sensory[j] >= 0) {
        if (g->type == 5) {
            if (g->sens >= 0 && g->rec_event > 0) {
                d->rec_ns *= exp(-1.0 / g->rec_decay);
                if (dec_rec_event) d->rec_ns += g->rec_event;
                cur = d->rec_ns * (0.0 - d->v);
            }
        } else cur = (double)gain * (double)input[b->sensory[j]];
    }
    for (int k = 0; k < BRANCHES; ++k) d->dend[k] += exc_in[k];
    const double sub = fmax(0.0, fmin(d->v, -50.0) - g->el);
    d->depol += 0.1 * (sub - d->depol);
    d->inh += b->sh->inh[j];
    if (g->type == 6) {
        static const double wt[3] = {250.0, 10.0, 4.0}, op[3] = {10.0, 40.0, 750.0}, cl[3] = {50.0, 750.0, 2000.0};
        double *u = d->u, *act = u + 2, *open = u + 5, exc = 0, under = 0;
        for (int k = 0; k < BRANCHES; ++k) exc += d->dend[k];
        u[1] = g->vt + (u[1] - g->vt) * exp(-0.1);
        for (int k = 0; k < 3; ++k) {
            open[k] += act[k] / op[k] - open[k] / cl[k];
            act[k] *= exp(-1.0 / op[k]);
            under += wt[k] * open[k];
        }
        const double v = u[0];
        const double i = g->gl * (g->el - v) + exc * (10.0 - v) + d->inh * (-60.0 - v) + under * (-80.0 - v) + cur;
        u[0] = v + i / g->cap;
        if (dec_subspikes & 1u) {
            u[1] = 200.0;
            for (int k = 0; k < 3; ++k) act[k] += 1.0;
        }
        d->v = u[0];
        for (int k = 0; k < BRANCHES; ++k) d->dend[k] *= exp(-1.0 / 3.0);
        d->inh *= exp(-1.0 / 10.0);
        return;
    }
    const double h = 0.25;
    for (int step = 0; step < SUBSTEPS; ++step) {
        const double v = d->v;
        d->w += h * (g->a * (v - g->el) - d->w) / g->tau_w;
        const double expo = dclamp((v - g->vt) / g->slope, -20.0, 10.0);
        double soma = 0;
        for (int k = 0; k < BRANCHES; ++k) soma += g->type == 0 ? sh_branch_gain(d->dend[k]) : d->dend[k];
        const double dv = g->gl * (g->el - v) + (double)g->gl * g->slope * exp(expo) + soma * (0.0 - v) +
                          d->inh * (-75.0 - v) + cur + d->adp - d->w;
        d->v = v + h * dv / g->cap;
        if (dec_subspikes >> step & 1u) { d->v = g->vr; d->w += g->b; d->adp += g->adp_b; }
        if (g->adp_tau > 0) d->adp *= exp(-h / g->adp_tau);
        for (int k = 0; k < BRANCHES; ++k) d->dend[k] *= exp(-h / 3.0);
        d->inh *= exp(-h / 10.0);
    }
}

static double sh_da_window(double age) {
    if (age < 0 || age > 20000.0) return 0;
    const double x = age / 2000.0;
    return x * x * x * x * exp(4.0 * (1.0 - x));
}
static double sh_spine_window(double age) {
    if (age < 0 || age > 5000.0) return 0;
    const double x = age / 1000.0;
    return x * x * x * exp(3.0 * (1.0 - x));
}

/* plasticity_tick (physiology.cuh:459-555) in binary64. Ages are whole
 * milliseconds in both precisions, so their comparisons agree exactly; the
 * profile-2 depolarisation gate reads the binary32 depolarisation. */
static void sh_plast(or_brain *b, int j, int pair) {
    const sgene *g = &b->sg[j];
    if (!g->plast || !pair) return;
    dsstate *d = &b->sh->s[j];
    const int arrived = b->ss[j].arrived, post_spike = b->ns[g->post].spike;
    const unsigned char mod = b->mod[g->post];
    const double w0 = g->w0;
    if (g->plast == 6) {
        d->pre_tr *= exp(-1.0 / 16.8);
        d->post_tr *= exp(-1.0 / 33.7);
        d->el_ltd *= exp(-1.0 / 114.0);
        d->el_ltp *= exp(-1.0 / 200.0);
        d->pre_age += 1.0; d->post_age += 1.0;
        if (arrived) { d->el_ltp -= 0.0071 * d->post_tr; d->pre_tr += 1.0; d->pre_age = 0; }
        if (post_spike) { d->el_ltp += 0.0065 * d->pre_tr * d->el_ltd; d->post_tr += 1.0; d->el_ltd += 1.0; d->post_age = 0; }
        if ((mod & MOD_DA) && (g->receptors & MOD_DA)) d->w += w0 * d->el_ltp;
        d->w = dclamp(d->w, 0.0, 2.0 * w0);
        return;
    }
    if (g->plast == 5) {
        if (d->st_age >= 0) { d->st_age += 1.0; if (d->st_age > 5000.0) d->st_age = -1; }
        d->pre_age += 1.0;
        if (arrived) d->pre_age = 0;
        if (post_spike && d->pre_age <= 15.0 && d->st_age < 0) d->st_age = 0;
        if ((mod & MOD_DA) && (g->receptors & MOD_DA))
            d->spine = dclamp(d->spine + 0.025 * sh_spine_window(d->st_age), 1.0, 2.0);
        return;
    }
    if (g->plast == 4) {
        if (d->da_age >= 0) { d->da_age += 1.0; if (d->da_age > 20000.0) d->da_age = -1; }
        d->pre_age += 1.0;
        if (arrived) d->pre_age = 0;
        if (post_spike && d->pre_age <= 15.0 && (d->da_age < 0 || d->da_age > 30.0)) {
            d->da_age = 0;
            d->w -= 0.005383 * w0;
        }
        if ((mod & MOD_DA) && (g->receptors & MOD_DA)) {
            d->w += 0.00453 * sh_da_window(d->da_age) * w0;
            d->da_age = -1;
        }
        d->w = dclamp(d->w, 0.0, 2.0 * w0);
        return;
    }
    if (g->plast == 3) {
        d->el_ltp *= exp(-1.0 / 7200.0);
        d->el_ltd *= exp(-1.0 / 3600.0);
        d->pre_age += 1.0; d->post_age += 1.0;
        if (arrived) { if (d->post_age <= 15.0) d->el_ltd += 1.0; d->pre_age = 0; }
        if (post_spike) { if (d->pre_age <= 15.0) d->el_ltp += 1.0; d->post_age = 0; }
        if ((mod & MOD_NE) && (g->receptors & MOD_NE)) { d->w += 0.0048 * d->el_ltp * w0; d->el_ltp = 0; }
        if ((mod & MOD_5HT) && (g->receptors & MOD_5HT)) { d->w -= 0.0075 * d->el_ltd * w0; d->el_ltd = 0; }
        d->w = dclamp(d->w, 0.0, 2.0 * w0);
        return;
    }
    d->pre_tr *= exp(-1.0 / 17.0);
    d->post_tr *= exp(-1.0 / 34.0);
    d->pre_age += 1.0; d->post_age += 1.0;
    if (arrived) {
        if (d->post_age <= (g->plast == 2 ? 50.0 : 20.0)) d->w *= 1.0 - 0.004 * d->post_tr;
        d->pre_tr += 1.0;
        d->pre_age = 0;
    }
    if (post_spike) {
        if (d->pre_age <= 20.0 && (g->plast == 1 || b->ns[g->post].depol >= 2.3f))
            d->w += 0.016 * d->pre_tr * (2.0 * w0 - d->w);
        d->post_tr += 1.0;
        d->post_age = 0;
    }
    d->w = dclamp(d->w, 0.0, 2.0 * w0);
}

/* homeostatic_advance (physiology.cuh:243-253) in binary64. */
static void sh_homeo(or_brain *b, int j, int ticks) {
    const ngene *g = &b->ng[j];
    if (g->type != 0) return;
    dnstate *d = &b->sh->n[j];
    const double elapsed = ticks;
    const double hz = (double)b->ns[j].total * 1000.0 / (double)(ticks > b->tick ? ticks : b->tick);
    const double ratio = dclamp(hz / 0.4, 0.0, 2.65);
    const double change = ratio < 1.0 ? log(1.92) * (1.0 - ratio) : log(0.70) * ((ratio - 1.0) / 1.65);
    d->log_ampa = dclamp(d->log_ampa + change * (elapsed / 172800000.0), -3.0, 3.0);
}

/* Fields: see or_shadow_field. Relative error = |x32 - x64| / max(|x64|, floor). */
static const char *const SH_NAMES[OR_SHADOW_FIELDS] = {
    "V_mV", "w_adapt_pA", "adp_pA", "g_inh_nS", "g_dend_nS", "log_ampa", "depol_mV", "g_receptor_nS",
    "syn_w_nS", "syn_u", "syn_slow", "syn_pre_trace", "syn_post_trace", "syn_eligibility",
    "V_subthreshold_mV"};
static const double SH_FLOOR[OR_SHADOW_FIELDS] = {1.0, 1.0, 1.0, 1e-3, 1e-3, 1e-3, 1.0, 1e-3,
                                                 1e-3, 1e-3, 1e-3, 1e-3, 1e-3, 1e-3, 1.0};
const char *or_shadow_field(int i) { return i >= 0 && i < OR_SHADOW_FIELDS ? SH_NAMES[i] : ""; }

static void sh_err(struct or_shadow *sh, int f, float x32, double x64) {
    if (!isfinite(x32) || !isfinite(x64)) return;
    const double e = fabs((double)x32 - x64);
    const double r = e / fmax(fabs(x64), SH_FLOOR[f]);
    if (e > sh->maxabs[f]) sh->maxabs[f] = e;
    if (r > sh->maxrel[f]) sh->maxrel[f] = r;
}

static void sh_track(or_brain *b, int tick_end) {
    struct or_shadow *sh = b->sh;
    sh->ticks += tick_end;
    for (int i = 0; i < b->count; ++i) {
        const ngene *g = &b->ng[i];
        if (!g->active) continue;
        const nstate *s = &b->ns[i]; const dnstate *d = &sh->n[i];
        sh_err(sh, 0, s->v, d->v); sh_err(sh, 1, s->w, d->w);
        if (d->v < g->vt) sh_err(sh, 14, s->v, d->v); sh_err(sh, 2, s->adp, d->adp);
        sh_err(sh, 3, s->inh, d->inh);
        for (int k = 0; k < BRANCHES; ++k) sh_err(sh, 4, s->dend[k], d->dend[k]);
        sh_err(sh, 5, s->log_ampa, d->log_ampa); sh_err(sh, 6, s->depol, d->depol);
        sh_err(sh, 7, s->rec_ns, d->rec_ns);
    }
    for (int i = 0; i < b->edges; ++i) {
        if (!edge_live(b, &b->sg[i])) continue;
        const sstate *s = &b->ss[i]; const dsstate *d = &sh->s[i];
        sh_err(sh, 8, s->w, d->w); sh_err(sh, 9, s->ru, d->ru); sh_err(sh, 10, s->slow, d->slow);
        sh_err(sh, 11, s->pre_tr, d->pre_tr); sh_err(sh, 12, s->post_tr, d->post_tr);
        sh_err(sh, 13, s->el_ltp, d->el_ltp); sh_err(sh, 13, s->el_ltd, d->el_ltd);
    }
}

void or_shadow_dump(const or_brain *b, double *v, double *syn_w) {
    if (!b->sh) return;
    if (v) for (int i = 0; i < b->count; ++i) v[i] = b->sh->n[i].v;
    if (syn_w) for (int i = 0; i < b->edges; ++i) syn_w[i] = b->sh->s[i].w;
}

int64_t or_shadow_stats(const or_brain *b, double *maxabs, double *maxrel) {
    if (!b->sh) return -1;
    memcpy(maxabs, b->sh->maxabs, sizeof b->sh->maxabs);
    memcpy(maxrel, b->sh->maxrel, sizeof b->sh->maxrel);
    return b->sh->ticks;
}

static uint32_t fw(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

void or_dump(const or_brain *b, uint32_t *nw, uint32_t *sw, int64_t *tick) {
    if (tick) *tick = b->tick;
    if (nw) for (int i = 0; i < b->count; ++i) {
        const nstate *s = &b->ns[i]; uint32_t *o = nw + (size_t)i * OR_NEURON_WORDS;
        memset(o, 0, OR_NEURON_WORDS * 4);
        o[0] = fw(s->v); o[1] = fw(s->w); o[2] = fw(s->adp); o[3] = fw(s->inh);
        o[4] = fw(s->depol); o[5] = fw(s->log_ampa);
        for (int k = 0; k < 4; ++k) o[6 + k] = fw(s->dend[k]);
        for (int k = 0; k < 16; ++k) o[10 + k] = fw(s->u[k]);
        o[26] = (uint32_t)s->total; o[27] = s->spike; o[28] = fw(s->rec_ns); o[29] = s->rec_rng;
        uint32_t h = 0;   /* bit k = spike at tick - 1 - k, k < ring-1 (the readable window) */
        for (int k = 0; k < b->ring - 1 && k < 31; ++k) {
            int64_t t = b->tick - 1 - k;
            if (t < 0) break;
            if (b->hist[(size_t)i * RING + (size_t)(t % b->ring)]) h |= 1u << k;
        }
        o[30] = h;
    }
    if (sw) for (int i = 0; i < b->edges; ++i) {
        const sstate *s = &b->ss[i]; uint32_t *o = sw + (size_t)i * OR_SYNAPSE_WORDS;
        memset(o, 0, OR_SYNAPSE_WORDS * 4);
        o[0] = fw(s->w); o[1] = fw(s->ru); o[2] = fw(s->pre_tr); o[3] = fw(s->post_tr);
        o[4] = fw(s->el_ltp); o[5] = fw(s->el_ltd); o[6] = fw(s->da_age); o[7] = fw(s->spine);
        o[8] = fw(s->st_age); o[9] = fw(s->pre_age); o[10] = fw(s->post_age);
        o[11] = (uint32_t)(uint64_t)s->last; o[12] = (uint32_t)((uint64_t)s->last >> 32);
        o[13] = (uint32_t)s->ready; o[14] = (uint32_t)(s->ready >> 32);
        o[15] = s->rng; o[16] = s->arrived; o[17] = fw(s->slow);
    }
}

int or_count(const or_brain *b) { return b->count; }
int or_edges(const or_brain *b) { return b->edges; }
int64_t or_last_events(const or_brain *b) { return b->events; }

/* ---- reference protocol checks ------------------------------------------------
 * Restated from tests/physiology.cpp, tests/event_synapses.cpp and
 * tests/cuda_relay_parity.cu; the Python test applies the same windows. */
static int step_current_spikes(const ngene *g, float pa, int *first_isi, int *last_isi) {
    nstate s = neuron_initial(g, 1);
    const float none[4] = {0, 0, 0, 0};
    int n = 0, prev2 = -1, prev = -1;
    *first_isi = *last_isi = 0;
    for (int t = 0; t < 2000; ++t) {
        neuron_tick(g, &s, pa, none, 0);
        if (s.spike) {
            if (n == 1) *first_isi = t - prev;
            prev2 = prev; prev = t; ++n;
            if (n >= 2) *last_isi = prev - prev2;
        }
    }
    return n;
}
static float stdp_pairs(int interval, int exc_target, unsigned char prof, float depol, int pairs) {
    sgene g; memset(&g, 0, sizeof g);
    g.w0 = 1.0f; g.U = 0.55f; g.trec = 450.0f; g.active = 1; g.delay = 1; g.plast = prof; g.sites = 14;
    sstate s = synapse_initial(&g, 1);
    for (int t = 0; t < pairs * 1000; ++t) {
        int ph = t % 1000;
        plasticity_tick(&g, &s, ph == 100, ph == 100 + interval, exc_target, depol, 0);
    }
    return s.w;
}
int or_protocols(float *out, int n) {
    init_consts();
    float r[40]; memset(r, 0, sizeof r);
    int fi, li;
    ngene rs = naud_profile(0), cna = naud_profile(1);
    r[0] = (float)step_current_spikes(&rs, 130, &fi, &li); r[1] = (float)fi; r[2] = (float)li;
    r[3] = (float)step_current_spikes(&cna, 150, &fi, &li); r[4] = (float)fi; r[5] = (float)li;
    r[6] = (float)step_current_spikes(&rs, 0, &fi, &li);
    /* release means (physiology.cpp:177-192) */
    sgene dep; memset(&dep, 0, sizeof dep);
    dep.w0 = 1.0f; dep.U = 0.55f; dep.trec = 450.0f; dep.active = 1; dep.delay = 1; dep.sites = 14;
    double first = 0, second = 0, rec = 0;
    for (int trial = 1; trial <= 10000; ++trial) {
        sstate s = synapse_initial(&dep, (uint32_t)trial);
        first += release(&dep, &s, 0); second += release(&dep, &s, 50); rec += release(&dep, &s, 2050);
    }
    r[7] = (float)(first / 10000); r[8] = (float)(second / 10000); r[9] = (float)(rec / 10000);
    /* STDP pairs (physiology.cpp:226-239) */
    r[10] = stdp_pairs(10, 1, 1, 0, 60); r[11] = stdp_pairs(-10, 1, 1, 0, 60);
    r[12] = stdp_pairs(50, 1, 1, 0, 60); r[13] = stdp_pairs(-50, 1, 1, 0, 60);
    r[14] = stdp_pairs(10, 0, 1, 0, 60);
    r[15] = stdp_pairs(10, 1, 2, 0, 50); r[16] = stdp_pairs(10, 1, 2, 3, 50);
    /* homeostasis 48 h (physiology.cpp:288-315) */
    nstate q = neuron_initial(&rs, 1), c = q, a = q;
    for (int h = 0; h < 48; ++h) {
        homeostasis(&rs, &q, 3600000.0f, 0.0f);
        homeostasis(&rs, &c, 3600000.0f, 0.4f);
        homeostasis(&rs, &a, 3600000.0f, 1.06f);
    }
    r[17] = (float)exp((double)q.log_ampa); r[18] = (float)exp((double)c.log_ampa); r[19] = (float)exp((double)a.log_ampa);
    /* quiet-jump agreement (event_synapses.cpp:25-60): max relative difference */
    float worst = 0;
    for (int prof = 1; prof <= 5; ++prof) {
        sgene g; memset(&g, 0, sizeof g);
        g.plast = (unsigned char)prof; g.w0 = 1.0f; g.receptors = MOD_NE | MOD_5HT | MOD_DA;
        sstate reg = synapse_initial(&g, 1), ev = reg;
        int last = -1;
        for (int t = 0; t < 8192; ++t) {
            int arr = t % 23 == 4 || t % 137 == 5, post = t % 29 == 8 || t % 137 == 9;
            unsigned char m = 0;
            if (t % 67 == 13) m |= MOD_NE;
            if (t % 71 == 17) m |= MOD_5HT;
            if (t % 73 == 21) m |= MOD_DA;
            plasticity_tick(&g, &reg, arr, post, 1, 3.0f, m);
            if (arr || post || m) {
                plasticity_quiet(&g, &ev, t - last - 1);
                plasticity_tick(&g, &ev, arr, post, 1, 3.0f, m);
                last = t;
            }
            if (t % 16 == 15) {
                plasticity_quiet(&g, &ev, t - last);
                last = t;
                const float *x = &reg.w, *y = &ev.w;
                for (int f = 0; f < 11; ++f) {
                    float den = fmaxf(1.0f, fmaxf(fabsf(x[f]), fabsf(y[f])));
                    float d = fabsf(x[f] - y[f]) / den;
                    if (d > worst) worst = d;
                }
            }
        }
    }
    r[20] = worst;
    /* CPU relay (cuda_relay_parity.cu:15-40) */
    ngene l5 = profile_for_type(0);
    nstate cell = neuron_initial(&l5, 19);
    sgene orn; memset(&orn, 0, sizeof orn);
    orn.w0 = 29.0f / (60.0f * 0.75f); orn.U = 0.75f; orn.trec = 50.0f; orn.sites = 50;
    orn.slow_rec = 7500.0f; orn.slow_depl = 0.023f;
    sstate rel = synapse_initial(&orn, 31);
    float peak = l5.el, released = 0; int arrivals = 0;
    for (int t = 0; t < 2000; ++t) {
        float e[4] = {0, 0, 0, 0};
        if (t % 137 == 0) { e[0] = release(&orn, &rel, t); released += e[0]; ++arrivals; }
        neuron_tick(&l5, &cell, 0, e, 0);
        peak = fmaxf(peak, cell.v);
    }
    r[21] = (float)arrivals; r[22] = released; r[23] = peak; r[24] = cell.v; r[25] = (float)cell.total;
    int m = n < 40 ? n : 40;
    memcpy(out, r, (size_t)m * sizeof(float));
    return m;
}

/* ---- World neural stage (src/main.cu:659-801, 1287-1300) ------------------------
 * The reference world loop runs, per tick, synapse_delivery over every occupied
 * synapse slot, neuron_step over every occupied neuron slot, then
 * synapse_plasticity (src/main.cu:2696-2728; the fused
 * synapse_plasticity_delivery kernel is plasticity(tick - 1) followed by
 * delivery(tick) per synapse, the same sequence). Its per-branch sums are
 * float atomics; this restatement fixes their order: each animal's synapse
 * list order (the order of the animal's synapse_head/synapse_next chain).
 * Trace float sums (observer-only) are fixed as: per neuron over the step in
 * tick order, then added per motor port in the animal's neuron list order. */
typedef struct {                   /* src/main.cu:81-91 */
    float x, y, heading, energy, health, fullness, pain;
    float taste[4];
    float muscle[3];
    unsigned long long rng;
    int id, parent_id, generation, age, alive;
    int neuron_head, synapse_head, neuron_count, synapse_count;
    int ports[24];
    struct {                       /* src/main.cu:66-74 */
        int opportunities[3][2][3];
        int accepted[3][2][3];
        int empty_steps[3][2], empty_eat[3][2];
        float approach_progress[3][3];
        float approach_travel[3][3];
        int first_b_age, offspring, death_cause;
    } behavior;
} or_animal;
typedef struct {                   /* src/main.cu:96-104 */
    int id, assigned, frozen, initial_age, initial_offspring;
    int final_age, final_offspring, alive, death_cause;
    int neurons, synapses, generation;
    float initial_energy, initial_health;
    int64_t start_step, observed_step, death_step;
} or_cohort;

#define W_S 19
#define W_M 5
#define W_HIST 9
#define W_CONTACT 16

static int or_w_frozen(const or_world_pools *w, int a) {       /* src/main.cu:142-146 */
    const or_animal *A = (const or_animal *)w->animals;
    const or_cohort *C = (const or_cohort *)w->plasticity_cohort;
    return C && a >= 0 && C[a].assigned && C[a].frozen && C[a].id == A[a].id;
}

/* An edge delivers when active, owned endpoints of the same animal, genes active
 * (src/main.cu:700-704). */
static int or_w_valid(const or_world_pools *w, int a, const sgene *g) {
    const ngene *NG = (const ngene *)w->neurons;
    if (!g->active || g->pre < 0 || g->post < 0 || g->pre >= w->neuron_capacity || g->post >= w->neuron_capacity)
        return 0;
    return w->neuron_owner[g->pre] == a && w->neuron_owner[g->post] == a && NG[g->pre].active && NG[g->post].active;
}

int or_world_step(const or_world_pools *w, int64_t step) {
    init_consts();
    const or_animal *A = (const or_animal *)w->animals;
    const ngene *NG = (const ngene *)w->neurons;
    nstate *NS = (nstate *)w->neuron_state;
    const sgene *SG = (const sgene *)w->synapses;
    sstate *SS = (sstate *)w->synapse_state;
    const int P = w->animal_capacity, NC = w->neuron_capacity;
    const int64_t first = (step - 1) * 16;
    float *tx = NULL, *ti = NULL;
    const int tr = w->trace_animal;
    if (tr >= 0 && tr < P && A[tr].alive == 1) {
        tx = (float *)calloc((size_t)NC, sizeof(float));
        ti = (float *)calloc((size_t)NC, sizeof(float));
    }
    /* gene checks the engine enforces on live edges */
    for (int a = 0; a < P; ++a) {
        if (A[a].alive != 1) continue;
        for (int e = A[a].synapse_head; e >= 0; e = w->synapse_next[e]) {
            const sgene *g = &SG[e];
            if (!or_w_valid(w, a, g)) continue;
            if (g->delay < 1 || g->delay > 8 || g->branch > 3 || g->plast > 7 || NG[g->pre].modulator > 3) {
                free(tx); free(ti);
                return -1;
            }
        }
    }
    for (int t = 0; t < 16; ++t) {
        const int64_t tick = first + t;
        for (int a = 0; a < P; ++a) {                                  /* delivery, src/main.cu:659-708 */
            if (A[a].alive != 1) continue;
            for (int e = A[a].synapse_head; e >= 0; e = w->synapse_next[e]) {
                const sgene *g = &SG[e];
                sstate *s = &SS[e];
                if (!or_w_valid(w, a, g)) continue;
                s->arrived = tick >= g->delay &&
                             w->spike_history[(size_t)((tick - g->delay) % W_HIST) * NC + (size_t)g->pre];
                if (!s->arrived) continue;
                const ngene *src = &NG[g->pre];
                const float rel = (!src->inh_tx || src->modulator) ? release(g, s, tick) : s->w;
                const int motor = w->neuron_port[g->post] - W_S;
                const int traced = a == tr && motor >= 0 && motor < W_M;
                if (src->modulator) {
                    if (rel > 0) {
                        unsigned long long *q = &w->mod_event_tick[(size_t)g->post * 6 + (size_t)(src->modulator - 1) * 2 +
                                                                   (size_t)(tick & 1)];
                        if (*q < (unsigned long long)(tick + 1)) *q = (unsigned long long)(tick + 1);
                    }
                } else if (!src->inh_tx) {
                    if (traced) {
                        w->trace_exc_arrivals[motor] += 1;
                        if (rel > 0) w->trace_exc_releases[motor] += 1;
                        tx[g->post] += rel;
                    }
                    w->pending_exc[(size_t)g->post * 4 + g->branch] += rel * OEXP(NS[g->post].log_ampa);
                } else {
                    if (traced) {
                        w->trace_inh_arrivals[motor] += 1;
                        ti[g->post] += rel;
                    }
                    w->pending_inh[g->post] += rel;
                }
            }
        }
        for (int a = 0; a < P; ++a) {                                  /* neurons, src/main.cu:710-746 */
            if (A[a].alive != 1) continue;
            for (int n = A[a].neuron_head; n >= 0; n = w->neuron_next[n]) {
                const ngene *g = &NG[n];
                if (!g->active) continue;
                nstate *s = &NS[n];
                float exc[4];
                for (int k = 0; k < 4; ++k) { exc[k] = w->pending_exc[(size_t)n * 4 + k]; w->pending_exc[(size_t)n * 4 + k] = 0; }
                const float inh = w->pending_inh[n];
                w->pending_inh[n] = 0;
                const int port = w->neuron_port[n];
                float cur = 0.0f;
                if (g->sens >= 0 && g->sens < W_S) {
                    const float level = (w->silence_senses || (w->silence_contact && g->sens >= W_CONTACT))
                                            ? 0.0f : w->senses[(size_t)a * W_S + (size_t)g->sens];
                    cur = g->type == 5 && g->sens < 6 ? receptor_drive(g, s, level) : level * 230.0f;
                }
                neuron_tick(g, s, cur, exc, inh);
                if (a == tr && port >= W_S && port < W_S + W_M)
                    w->trace_peak_mv[port - W_S] = fmaxf(w->trace_peak_mv[port - W_S], s->v);
                if (s->spike && port >= W_S && port < W_S + W_M) w->motors[(size_t)a * W_M + (size_t)(port - W_S)] += 1;
                w->spike_history[(size_t)(tick % W_HIST) * NC + (size_t)n] = s->spike;
            }
        }
        for (int a = 0; a < P; ++a) {                                  /* plasticity, src/main.cu:748-767 */
            if (A[a].alive != 1 || or_w_frozen(w, a)) continue;
            for (int e = A[a].synapse_head; e >= 0; e = w->synapse_next[e]) {
                const sgene *g = &SG[e];
                if (!or_w_valid(w, a, g)) continue;
                const ngene *x = &NG[g->pre], *z = &NG[g->post];
                const int pair = !x->inh_tx && excitatory_kind(x->type) && x->modulator == 0 && !z->inh_tx &&
                                 excitatory_kind(z->type);
                const size_t target = (size_t)g->post * 6 + (size_t)(tick & 1);
                unsigned char mod = 0;
                if (w->mod_event_tick[target] == (unsigned long long)(tick + 1)) mod |= MOD_NE;
                if (w->mod_event_tick[target + 2] == (unsigned long long)(tick + 1)) mod |= MOD_5HT;
                if (w->mod_event_tick[target + 4] == (unsigned long long)(tick + 1)) mod |= MOD_DA;
                plasticity_tick(g, &SS[e], SS[e].arrived, NS[g->post].spike, pair, NS[g->post].depol, mod);
            }
        }
    }
    if (tx) {
        for (int n = A[tr].neuron_head; n >= 0; n = w->neuron_next[n]) {
            const int port = w->neuron_port[n];
            if (port < W_S || port >= W_S + W_M || !NG[n].active) continue;
            w->trace_exc_ns[port - W_S] += tx[n];
            w->trace_inh_ns[port - W_S] += ti[n];
        }
        free(tx); free(ti);
    }
    return 0;
}

void or_world_homeostasis(const or_world_pools *w) {          /* src/main.cu:1287-1300 */
    init_consts();
    const or_animal *A = (const or_animal *)w->animals;
    const ngene *NG = (const ngene *)w->neurons;
    nstate *NS = (nstate *)w->neuron_state;
    for (int i = 0; i < w->neuron_capacity; ++i) {
        const int a = w->neuron_owner[i];
        if (a < 0 || a >= w->animal_capacity) continue;
        if (A[a].alive != 1 || !NG[i].active || or_w_frozen(w, a)) continue;
        const float elapsed = fmaxf(16.0f, (float)A[a].age * 16.0f);
        homeostasis(&NG[i], &NS[i], 16.0f, (float)NS[i].total * 1000.0f / elapsed);
    }
}

void or_records(const or_brain *b, void *neuron_genes, void *neuron_states, void *synapse_genes,
                void *synapse_states) {
    if (neuron_genes) memcpy(neuron_genes, b->ng, sizeof(ngene) * (size_t)b->count);
    if (neuron_states) memcpy(neuron_states, b->ns, sizeof(nstate) * (size_t)b->count);
    if (synapse_genes) memcpy(synapse_genes, b->sg, sizeof(sgene) * (size_t)b->edges);
    if (synapse_states) memcpy(synapse_states, b->ss, sizeof(sstate) * (size_t)b->edges);
}

int or_world_layout(uint64_t *out) {
    const uint64_t v[14] = {sizeof(or_animal), sizeof(or_cohort), sizeof(ngene), sizeof(nstate), sizeof(sgene),
                            sizeof(sstate), offsetof(or_animal, id), offsetof(or_animal, age),
                            offsetof(or_animal, alive), offsetof(or_animal, neuron_head),
                            offsetof(or_animal, synapse_head), offsetof(or_animal, neuron_count),
                            offsetof(or_animal, synapse_count), offsetof(or_cohort, frozen)};
    for (int i = 0; i < 14; ++i) out[i] = v[i];
    return 14;
}


/* ---- world ecology (src/main.cu:612-657, 1138-1338) ------------------------
 * The reference kernels restated as loops over animal slots in ascending
 * order (cells for regrowth): one thread after another, which fixes the
 * outcome of every contended step (harvests, spatial list order, bites,
 * record indices) as that sequential execution. */
#define W_W 128
#define W_H 128
#define W_CELLS (W_W * W_H)

typedef struct {                   /* src/main.cu:85-90 */
    or_animal body;
    int64_t death_step;
    int active_neurons, active_synapses, modulatory_neurons, plastic_synapses;
    float mean_abs_weight_change;
} or_life;
typedef struct {                   /* src/main.cu:91-95 */
    int64_t step;
    int attacker_id, prey_id;
    float x, y;
} or_bite;

static float or_clamp(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }
static int or_cell(float x, float y) {                         /* src/main.cu:347-351 */
    int ix = (int)floorf(or_clamp(x, 0.0f, W_W - 0.001f));
    int iy = (int)floorf(or_clamp(y, 0.0f, W_H - 0.001f));
    return iy * W_W + ix;
}
static unsigned long long or_random64(unsigned long long *s) {  /* src/main.cu:331-346 */
    *s ^= *s >> 12; *s ^= *s << 25; *s ^= *s >> 27;
    return *s * 2685821657736338717ULL;
}
static float or_uniform(unsigned long long *s) {
    return (float)((or_random64(s) >> 40) * (1.0 / 16777216.0));
}
static unsigned long long or_seed_for(unsigned long long seed, unsigned long long i) {
    unsigned long long x = seed + 0x9e3779b97f4a7c15ULL * (i + 1);
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return (x ^ (x >> 31)) | 1ULL;
}
static int or_excitatory(unsigned char t) { return t == 0 || t == 4 || t == 5; }

static void or_index(const or_world_pools *w, const or_world_eco *x) {   /* src/main.cu:612-617 */
    const or_animal *A = (const or_animal *)w->animals;
    for (int c = 0; c < W_CELLS; ++c) x->cell_head[c] = -1;
    for (int a = 0; a < w->animal_capacity; ++a) {
        if (A[a].alive != 1) continue;
        int c = or_cell(A[a].x, A[a].y);
        x->cell_next[a] = x->cell_head[c];
        x->cell_head[c] = a;
    }
}

static void or_body(const or_world_pools *w, const or_world_eco *x, int a) {   /* src/main.cu:1146-1249 */
    or_animal *A = (or_animal *)w->animals;
    const ngene *NG = (const ngene *)w->neurons;
    or_animal b = A[a];
    const int age_bin = b.age < 100 ? 0 : (b.age < 300 ? 1 : 2);
    const int hungry = b.energy < 16.0f;
    const float old_x = b.x, old_y = b.y;
    int *mo = w->motors + (size_t)a * W_M;
    float force[3];
    for (int m = 0; m < 3; ++m)
        force[m] = x->instant_motors ? mo[m] / (float)16
                                     : (b.muscle[m] = fminf(1.0f, b.muscle[m] * 0.92311635f + mo[m] * 0.30f));
    float thrust = force[0], left = force[1], right = force[2];
    int eat = mo[3] > 0;
    x->bite_intent[a] = mo[4] > 0;
    if (b.id < x->initial_count && b.age < 100) {
        ++*x->founder_observed_steps;
        for (int m = 0; m < W_M; ++m)
            if (mo[m] > 0) ++x->founder_motor_steps[m];
    }
    for (int m = 0; m < W_M; ++m) mo[m] = 0;
    b.heading += (right - left) * 1.2f;
    b.x = or_clamp(b.x + OCOS(b.heading) * thrust * 1.5f, 0, W_W - 0.001f);
    b.y = or_clamp(b.y + OSIN(b.heading) * thrust * 1.5f, 0, W_H - 0.001f);
    float travel = OHYPOT(b.x - old_x, b.y - old_y);
    if (hungry && travel > 0.0001f) {
        float nearest[3] = {1e9f, 1e9f, 1e9f};
        float target_x[3] = {0, 0, 0}, target_y[3] = {0, 0, 0};
        int cx = (int)old_x, cy = (int)old_y;
        for (int dy = -4; dy <= 4; ++dy) {
            int y = cy + dy;
            if (y < 0 || y >= W_H) continue;
            for (int dx = -4; dx <= 4; ++dx) {
                int xx = cx + dx;
                if (xx < 0 || xx >= W_W || x->food[y * W_W + xx] <= 0) continue;
                int kind = x->kind[y * W_W + xx];
                float fx = xx + 0.5f, fy = y + 0.5f;
                float distance = (fx - old_x) * (fx - old_x) + (fy - old_y) * (fy - old_y);
                if (distance < nearest[kind]) {
                    nearest[kind] = distance;
                    target_x[kind] = fx;
                    target_y[kind] = fy;
                }
            }
        }
        for (int kind = 0; kind < 3; ++kind)
            if (nearest[kind] < 1e9f) {
                b.behavior.approach_progress[age_bin][kind] +=
                    sqrtf(nearest[kind]) - OHYPOT(target_x[kind] - b.x, target_y[kind] - b.y);
                b.behavior.approach_travel[age_bin][kind] += travel;
            }
    }
    int active_neurons = 0;
    for (int n = b.neuron_head; n >= 0; n = w->neuron_next[n]) active_neurons += NG[n].active;
    b.energy -= 0.003f + active_neurons * 0.00002f + thrust * 0.02f + (x->bite_intent[a] ? 0.02f : 0.0f);
    b.fullness = fmaxf(0, b.fullness - 0.05f);
    b.pain *= 0.8f;
    for (int k = 0; k < 4; ++k) b.taste[k] *= 0.7f;
    int food_cell = or_cell(old_x, old_y);
    int food_offered = x->food[food_cell] > 0;
    if (food_offered) {
        int kind = x->kind[food_cell];
        ++b.behavior.opportunities[age_bin][hungry ? 0 : 1][kind];
    } else {
        ++b.behavior.empty_steps[age_bin][hungry ? 0 : 1];
        b.behavior.empty_eat[age_bin][hungry ? 0 : 1] += eat;
    }
    if (eat && x->food[food_cell] > 0) {                       /* harvest */
        --x->food[food_cell];
        int kind = x->kind[food_cell];
        if (!food_offered) ++b.behavior.opportunities[age_bin][hungry ? 0 : 1][kind];
        ++b.behavior.accepted[age_bin][hungry ? 0 : 1][kind];
        if (kind == 1 && b.behavior.first_b_age == 0) b.behavior.first_b_age = b.age + 1;
        b.taste[kind] = 1;
        b.fullness += 1;
        if (kind == 0) b.energy = fminf(30, b.energy + 4);
        if (kind == 1) { b.energy = fminf(30, b.energy + 2); b.health -= 1.4f; b.pain += 1.4f; }
        if (b.fullness > 8) { b.health -= 0.8f; b.pain += 0.8f; }
    }
    if (b.energy <= 0) { b.energy = 0; b.health -= 0.15f; b.pain += 0.15f; }
    ++b.age;
    if (b.health <= 0 || b.age >= 10000) {
        b.behavior.death_cause = b.age >= 10000 ? 4 : (b.energy <= 0 ? 2 : 3);
        b.alive = 0;
        ++*x->deaths;
    }
    A[a] = b;
}

void or_world_body_step(const or_world_pools *w, const or_world_eco *x, int64_t step) {
    or_animal *A = (or_animal *)w->animals;
    const int P = w->animal_capacity;
    for (int a = 0; a < P; ++a)
        if (A[a].alive == 1) or_body(w, x, a);
    or_index(w, x);
    or_bite *events = (or_bite *)x->bite_events;
    for (int a = 0; a < P; ++a) {                              /* src/main.cu:1251-1276 */
        if (A[a].alive != 1 || !x->bite_intent[a]) continue;
        int c = or_cell(A[a].x, A[a].y);
        for (int prey = x->cell_head[c]; prey >= 0; prey = x->cell_next[prey]) {
            if (prey == a || A[prey].alive != 1) continue;
            float previous = A[prey].health;
            A[prey].health = previous + -2.0f;
            A[prey].pain += 2.0f;
            ++*x->bites;
            if (events) {
                int event = (*x->bite_event_count)++;
                if (event < 2 * P) {
                    or_bite e = {step, A[a].id, A[prey].id, A[prey].x, A[prey].y};
                    events[event] = e;
                }
            }
            if (previous <= 2.0f && A[prey].alive == 1) {
                A[prey].alive = -2;
                A[a].energy += fmaxf(0.0f, A[prey].energy) * 0.45f;
                A[a].taste[3] = 1.0f;
                A[a].fullness += 1.0f;
            }
            break;
        }
    }
    for (int a = 0; a < P; ++a) {                              /* src/main.cu:1278-1285 */
        if (A[a].alive != -2) continue;
        A[a].behavior.death_cause = 1;
        A[a].alive = 0;
        ++*x->deaths;
        ++*x->predation_deaths;
    }
}

void or_world_reclaim(const or_world_pools *w, const or_world_eco *x, int64_t step) {   /* 1302-1338 */
    or_animal *A = (or_animal *)w->animals;
    const ngene *NG = (const ngene *)w->neurons;
    const sgene *SG = (const sgene *)w->synapses;
    const sstate *SS = (const sstate *)w->synapse_state;
    int *nowner = (int *)w->neuron_owner, *sowner = (int *)w->synapse_owner;
    for (int a = 0; a < w->animal_capacity; ++a) {
        if (A[a].alive != 0) continue;
        or_animal body = A[a];
        if (body.neuron_head < 0 && body.synapse_head < 0) continue;
        int index = (*x->life_count)++;
        if (x->life_records && index < x->life_capacity) {
            or_life rec;
            memset(&rec, 0, sizeof rec);
            rec.body = body;
            rec.death_step = step;
            for (int n = body.neuron_head; n >= 0; n = w->neuron_next[n]) {
                rec.active_neurons += NG[n].active;
                rec.modulatory_neurons += NG[n].active && NG[n].modulator != 0;
            }
            float total = 0;
            for (int e = body.synapse_head; e >= 0; e = w->synapse_next[e]) {
                const sgene *g = &SG[e];
                int active = g->active && NG[g->pre].active && NG[g->post].active;
                rec.active_synapses += active;
                rec.plastic_synapses += active && g->plast != 0 && !NG[g->pre].inh_tx &&
                                        or_excitatory(NG[g->pre].type) && NG[g->pre].modulator == 0 &&
                                        !NG[g->post].inh_tx && or_excitatory(NG[g->post].type);
                if (active) total += fabsf(SS[e].w - g->w0);
            }
            rec.mean_abs_weight_change = rec.active_synapses > 0 ? total / rec.active_synapses : 0;
            ((or_life *)x->life_records)[index] = rec;
        }
        for (int e = body.synapse_head; e >= 0;) {             /* release_genome, 436-454 */
            int next = w->synapse_next[e];
            sowner[e] = -1;
            x->synapse_used[e / 32] &= ~(1u << (e % 32));
            e = next;
        }
        for (int n = body.neuron_head; n >= 0;) {
            int next = w->neuron_next[n];
            nowner[n] = -1;
            x->neuron_used[n / 32] &= ~(1u << (n % 32));
            n = next;
        }
        body.neuron_head = body.synapse_head = -1;
        body.neuron_count = body.synapse_count = 0;
        for (int p = 0; p < W_S + W_M; ++p) body.ports[p] = -1;
        A[a] = body;
    }
}

void or_world_regrow_and_sense(const or_world_pools *w, const or_world_eco *x, int64_t step,
                               unsigned long long seed, float renewal) {
    for (int c = 0; c < W_CELLS; ++c) {                        /* regrow, 1138-1144 */
        if (x->food[c] != 0) continue;
        unsigned long long rng = or_seed_for(seed + (unsigned long long)step, (unsigned long long)c);
        if (or_uniform(&rng) < renewal) x->food[c] = 1;
    }
    or_index(w, x);
    const or_animal *A = (const or_animal *)w->animals;
    float *senses = (float *)w->senses;
    for (int a = 0; a < w->animal_capacity; ++a) {             /* update_senses, 619-657 */
        if (A[a].alive != 1) continue;
        or_animal b = A[a];
        float *out = senses + (size_t)a * W_S;
        for (int s = 0; s < 6; ++s) {
            float angle = b.heading + (s % 3 - 1) * 0.7f;
            float level = 0;
            for (int range = 1; range <= 4; ++range) {
                int c = or_cell(b.x + OCOS(angle) * range, b.y + OSIN(angle) * range);
                if (x->kind[c] == s / 3 && x->food[c] > 0) level += 0.25f;
            }
            out[s] = or_clamp(level, 0, 1);
        }
        out[6] = or_clamp((16.0f - b.energy) / 16.0f, 0, 1);
        out[7] = or_clamp(b.fullness / 8.0f, 0, 1);
        out[8] = or_clamp(b.pain / 3.0f, 0, 1);
        for (int k = 0; k < 3; ++k) out[9 + k] = or_clamp(b.taste[k], 0, 1);
        for (int direction = 0; direction < 3; ++direction) {
            float angle = b.heading + (direction - 1) * 0.7f;
            float level = 0;
            for (int range = 1; range <= 4; ++range) {
                int c = or_cell(b.x + OCOS(angle) * range, b.y + OSIN(angle) * range);
                for (int other = x->cell_head[c]; other >= 0; other = x->cell_next[other])
                    if (other != a && A[other].alive == 1) level += 0.25f;
            }
            out[12 + direction] = or_clamp(level, 0, 1);
        }
        out[15] = or_clamp(b.taste[3], 0, 1);
        int contact = or_cell(b.x, b.y);
        for (int kind = 0; kind < 3; ++kind)
            out[W_CONTACT + kind] = x->food[contact] > 0 && x->kind[contact] == kind ? 1.0f : 0.0f;
    }
}

/* ---- reproduction with mutation (src/main.cu:364-454, 464-525, 1340-1737) --
 * Parents (alive, energy >= 22 when the step starts) reproduce one after
 * another in ascending slot order; every slot claim runs alone. */
#define W_D 8
static int or_randint(unsigned long long *s, int size) { return (int)(or_uniform(s) * size); }

static int or_claim(uint32_t *used, int capacity, int hint) {   /* claim_slot, 364-385 */
    int words = (capacity + 31) / 32;
    int start = hint % words;
    for (int off = 0; off < words; ++off) {
        int w = (start + off) % words;
        uint32_t occ = used[w];
        if (~occ) {
            int bit = __builtin_ctz(~occ);
            int slot = w * 32 + bit;
            if (slot < capacity) { used[w] = occ | (1u << bit); return slot; }
            return -1;
        }
    }
    return -1;
}
static void or_release(uint32_t *used, int slot) { used[slot / 32] &= ~(1u << (slot % 32)); }

typedef struct { const or_world_pools *w; const or_world_eco *x; } or_rw;

static void or_init_neuron(or_rw r, int n, int owner, int port, const ngene *g, int next, uint32_t seed) {
    const or_world_pools *w = r.w;
    ((int *)w->neuron_owner)[n] = owner;
    ((int *)w->neuron_next)[n] = next;
    ((int *)w->neuron_port)[n] = port;
    ((ngene *)w->neurons)[n] = *g;
    ((nstate *)w->neuron_state)[n] = neuron_initial(g, seed);
    for (int b = 0; b < 4; ++b) w->pending_exc[(size_t)n * 4 + b] = 0;
    w->pending_inh[n] = 0;
    for (int k = 0; k < 6; ++k) w->mod_event_tick[(size_t)n * 6 + k] = 0;
    for (int h = 0; h < W_HIST; ++h) w->spike_history[(size_t)h * w->neuron_capacity + n] = 0;
}
static void or_init_synapse(or_rw r, int e, int owner, const sgene *g, int next, unsigned long long *rng) {
    const or_world_pools *w = r.w;
    ((int *)w->synapse_owner)[e] = owner;
    ((int *)w->synapse_next)[e] = next;
    ((sgene *)w->synapses)[e] = *g;
    ((sstate *)w->synapse_state)[e] = synapse_initial(g, (uint32_t)or_random64(rng));
}
static void or_release_genome(or_rw r, or_animal *body) {            /* 436-454 */
    const or_world_pools *w = r.w;
    for (int e = body->synapse_head; e >= 0;) {
        int next = w->synapse_next[e];
        ((int *)w->synapse_owner)[e] = -1;
        or_release(r.x->synapse_used, e);
        e = next;
    }
    for (int n = body->neuron_head; n >= 0;) {
        int next = w->neuron_next[n];
        ((int *)w->neuron_owner)[n] = -1;
        or_release(r.x->neuron_used, n);
        n = next;
    }
    body->neuron_head = body->synapse_head = -1;
    body->neuron_count = body->synapse_count = 0;
    for (int p = 0; p < W_S + W_M; ++p) body->ports[p] = -1;
}
static int or_neuron_at(or_rw r, const or_animal *b, int ordinal) {
    int n = b->neuron_head;
    for (int j = 0; j < ordinal && n >= 0; ++j) n = r.w->neuron_next[n];
    return n;
}
static int or_synapse_at(or_rw r, const or_animal *b, int ordinal) {
    int e = b->synapse_head;
    for (int j = 0; j < ordinal && e >= 0; ++j) e = r.w->synapse_next[e];
    return e;
}
static int or_random_hidden(or_rw r, const or_animal *b, unsigned long long *rng) {
    int hidden = b->neuron_count - (W_S + W_M);
    if (hidden <= 0) return -1;
    int ordinal = or_randint(rng, hidden);
    for (int n = b->neuron_head; n >= 0; n = r.w->neuron_next[n])
        if (r.w->neuron_port[n] < 0 && ordinal-- == 0) return n;
    return -1;
}
static void or_random_synapse(or_rw r, sgene *g, int animal, unsigned long long *rng) {   /* 464-525 */
    const or_world_pools *w = r.w;
    const ngene *NG = (const ngene *)w->neurons;
    or_animal body = ((or_animal *)w->animals)[animal];
    int active_sources = 0;
    float target_weight = 0;
    for (int n = body.neuron_head; n >= 0; n = w->neuron_next[n]) {
        if (!NG[n].active) continue;
        ++active_sources;
        int port = w->neuron_port[n];
        if (port < 0 || port >= W_S) target_weight += NG[n].affinity;
    }
    g->pre = body.ports[0];
    int source_choice = or_randint(rng, active_sources);
    for (int n = body.neuron_head; n >= 0; n = w->neuron_next[n])
        if (NG[n].active && source_choice-- == 0) { g->pre = n; break; }
    g->post = body.ports[W_S + or_randint(rng, W_M)];
    float target_choice = or_uniform(rng) * target_weight;
    for (int n = body.neuron_head; n >= 0; n = w->neuron_next[n]) {
        int port = w->neuron_port[n];
        if (!NG[n].active || (port >= 0 && port < W_S)) continue;
        target_choice -= NG[n].affinity;
        if (target_choice <= 0) { g->post = n; break; }
    }
    g->delay = (unsigned char)(1 + or_randint(rng, W_D));
    g->branch = (unsigned char)or_randint(rng, 4);
    g->w0 = 0.5f + or_uniform(rng) * 3.5f;
    g->U = 0.55f;
    g->trec = 450.0f;
    g->tfac = 0;
    g->sites = 14;
    if (NG[g->pre].type == 5) {
        g->w0 = 29.0f / (60.0f * 0.75f);
        g->U = 0.75f;
        g->trec = 50.0f;
        g->sites = 50;
        g->slow_rec = 7500.0f;
        g->slow_depl = 0.023f;
    }
    if (NG[g->pre].type == 0 && NG[g->post].type == 1) {
        g->U = 0.1f;
        g->trec = 30.0f;
        g->tfac = 1700.0f;
    }
    float draw = or_uniform(rng);
    g->plast = draw < 0.05f ? 5 : (draw < 0.10f ? 4 : (draw < 0.20f ? 3 : 2));
    g->receptors = g->plast == 3 ? (MOD_NE | MOD_5HT) : (g->plast >= 4 ? 4 : 0);
    g->active = 1;
}
static void or_remove_synapse(or_rw r, or_animal *body, int target) {   /* 1357-1372 */
    int *next = (int *)r.w->synapse_next;
    int previous = -1;
    for (int e = body->synapse_head; e >= 0; e = next[e]) {
        if (e != target) { previous = e; continue; }
        int nx = next[e];
        if (previous < 0) body->synapse_head = nx; else next[previous] = nx;
        --body->synapse_count;
        ((int *)r.w->synapse_owner)[e] = -1;
        or_release(r.x->synapse_used, e);
        return;
    }
}
static void or_remove_hidden(or_rw r, or_animal *body, int target) {    /* 1374-1395 */
    const sgene *SG = (const sgene *)r.w->synapses;
    int *nnext = (int *)r.w->neuron_next;
    if (target < 0 || r.w->neuron_port[target] >= 0) return;
    for (int e = body->synapse_head; e >= 0;) {
        int nx = r.w->synapse_next[e];
        if (SG[e].pre == target || SG[e].post == target) or_remove_synapse(r, body, e);
        e = nx;
    }
    int previous = -1;
    for (int n = body->neuron_head; n >= 0; n = nnext[n]) {
        if (n != target) { previous = n; continue; }
        int nx = nnext[n];
        if (previous < 0) body->neuron_head = nx; else nnext[previous] = nx;
        --body->neuron_count;
        ((int *)r.w->neuron_owner)[n] = -1;
        or_release(r.x->neuron_used, n);
        return;
    }
}
static int or_random_afferent(or_rw r, const or_animal *b, unsigned long long *rng) {
    const ngene *NG = (const ngene *)r.w->neurons;
    for (int attempt = 0; attempt < 12; ++attempt) {
        int n = or_random_hidden(r, b, rng);
        if (n >= 0 && NG[n].sens >= 0) return n;
    }
    return -1;
}

static void or_mutate(or_rw r, int child, unsigned long long *rng) {    /* 1401-1660 */
    const or_world_pools *w = r.w;
    or_animal *A = (or_animal *)w->animals;
    ngene *NG = (ngene *)w->neurons;
    sgene *SG = (sgene *)w->synapses;
    const int NC = w->neuron_capacity, EC = w->synapse_capacity;
    int mutations = 1 + or_randint(rng, 4);
    for (int m = 0; m < mutations; ++m) {
        int choice = or_randint(rng, 12);
        or_animal body = A[child];
        int n = or_random_hidden(r, &body, rng);
        int e = body.synapse_count ? or_synapse_at(r, &body, or_randint(rng, body.synapse_count)) : -1;
        if (choice == 0) {
            float action = or_uniform(rng);
            if (action < 1.0f / 3.0f) {
                int added = or_claim(r.x->neuron_used, NC, child * 131 + body.neuron_count);
                int incoming = added >= 0 ? or_claim(r.x->synapse_used, EC, child * 257 + body.synapse_count) : -1;
                int outgoing = incoming >= 0 ? or_claim(r.x->synapse_used, EC, child * 257 + body.synapse_count + 1) : -1;
                if (added >= 0 && incoming >= 0 && outgoing >= 0 && e >= 0) {
                    int template_e = e;
                    for (int attempt = 0; attempt < 8; ++attempt) {
                        int cand = or_synapse_at(r, &body, or_randint(rng, body.synapse_count));
                        sgene cg = SG[cand];
                        if (cg.active && NG[cg.pre].active && NG[cg.post].active) { template_e = cand; break; }
                    }
                    unsigned char type = (unsigned char)or_randint(rng, 7);
                    ngene g = profile_for_type(type);
                    g.modulator = or_uniform(rng) < 0.12f ? (unsigned char)(1 + or_randint(rng, 3)) : 0;
                    or_init_neuron(r, added, child, -1, &g, body.neuron_head, (uint32_t)or_random64(rng));
                    body.neuron_head = added;
                    ++body.neuron_count;
                    sgene first = SG[template_e], second = first;
                    first.post = added;
                    second.pre = added;
                    first.active = second.active = 1;
                    or_init_synapse(r, incoming, child, &first, body.synapse_head, rng);
                    body.synapse_head = incoming;
                    or_init_synapse(r, outgoing, child, &second, body.synapse_head, rng);
                    body.synapse_head = outgoing;
                    body.synapse_count += 2;
                    A[child] = body;
                } else {
                    if (outgoing >= 0) or_release(r.x->synapse_used, outgoing);
                    if (incoming >= 0) or_release(r.x->synapse_used, incoming);
                    if (added >= 0) or_release(r.x->neuron_used, added);
                }
            } else if (action < 2.0f / 3.0f) {
                if (n >= 0) { or_remove_hidden(r, &body, n); A[child] = body; }
            } else if (n >= 0) NG[n].active ^= 1;
        } else if (choice == 1 && n >= 0) {
            unsigned char active = NG[n].active;
            unsigned char type = (unsigned char)or_randint(rng, 7);
            unsigned char modulator = NG[n].modulator, inh = NG[n].inh_tx;
            float affinity = NG[n].affinity;
            NG[n] = profile_for_type(type);
            NG[n].active = active;
            NG[n].modulator = modulator;
            NG[n].inh_tx = inh;
            NG[n].affinity = affinity;
        } else if (choice == 2) {
            int target = or_uniform(rng) < 0.2f ? body.ports[W_S + or_randint(rng, W_M)] : n;
            if (target < 0) continue;
            ngene *g = &NG[target];
            if (g->type == 2) {
                int channel = or_randint(rng, 4);
                g->lp_scale[channel] = or_clamp(g->lp_scale[channel] * (0.9f + or_uniform(rng) * 0.2f), 0.2f, 3.0f);
            } else if (g->type == 3) {
                int channel = or_randint(rng, 9);
                float *c = channel == 8 ? &g->prinz_leak : &g->prinz_g[channel];
                *c = or_clamp((*c + (channel >= 7 ? 2.0f : 0.0f)) * (0.9f + or_uniform(rng) * 0.2f), 0.0f,
                              channel >= 7 ? 200.0f : 500000.0f);
            } else if (g->type == 5) {
                int parameter = or_randint(rng, 4);
                if (parameter == 0) g->rec_base = or_clamp(g->rec_base + (or_uniform(rng) - 0.5f) * 2, 0, 30);
                if (parameter == 1) g->rec_gain = or_clamp(g->rec_gain + (or_uniform(rng) - 0.5f) * 10, 0, 300);
                if (parameter == 2) g->rec_event = or_clamp(g->rec_event * (0.9f + or_uniform(rng) * 0.2f), 0.5f, 6);
                if (parameter == 3) g->rec_decay = or_clamp(g->rec_decay * (0.9f + or_uniform(rng) * 0.2f), 1, 20);
            } else {
                g->vt = or_clamp(g->vt + (or_uniform(rng) - 0.5f) * 2, -60, -35);
            }
        } else if (choice == 3) {
            float action = or_uniform(rng);
            if (action < 1.0f / 3.0f) {
                int added = or_claim(r.x->synapse_used, EC, child * 257 + body.synapse_count);
                if (added >= 0) {
                    sgene g; memset(&g, 0, sizeof g);
                    or_random_synapse(r, &g, child, rng);
                    or_init_synapse(r, added, child, &g, body.synapse_head, rng);
                    body.synapse_head = added;
                    ++body.synapse_count;
                    A[child] = body;
                }
            } else if (action < 2.0f / 3.0f) {
                if (e >= 0) { or_remove_synapse(r, &body, e); A[child] = body; }
            } else if (e >= 0) SG[e].active ^= 1;
        } else if (choice == 4 && e >= 0) {
            or_random_synapse(r, &SG[e], child, rng);
        } else if (choice == 5 && e >= 0) {
            sgene *g = &SG[e];
            g->w0 = or_clamp(g->w0 + (or_uniform(rng) - 0.5f) * 0.5f, 0.1f, 8);
            g->sites = (unsigned char)or_clamp(g->sites + (or_uniform(rng) < 0.5f ? -1 : 1), 1, 64);
        } else if (choice == 6 && e >= 0) {
            sgene *g = &SG[e];
            g->plast = (unsigned char)or_randint(rng, 6);
            g->receptors = g->plast == 3 ? (unsigned char)(1 + or_randint(rng, 3)) : (g->plast >= 4 ? 4 : 0);
            g->U = or_clamp(g->U + (or_uniform(rng) - 0.5f) * 0.1f, 0.02f, 0.8f);
            g->trec = or_clamp(g->trec + (or_uniform(rng) - 0.5f) * 50, 20, 1000);
            if (or_uniform(rng) < 0.15f) {
                g->slow_rec = g->slow_rec == 0 ? 7500.0f :
                    (or_uniform(rng) < 0.1f ? 0.0f : or_clamp(g->slow_rec + (or_uniform(rng) - 0.5f) * 500, 1000.0f, 20000.0f));
                g->slow_depl = g->slow_rec == 0 ? 0.0f :
                    or_clamp(g->slow_depl + (or_uniform(rng) - 0.5f) * 0.01f, 0.0f, 0.1f);
            }
        } else if (choice == 7 && e >= 0) {
            sgene *g = &SG[e];
            g->delay = (unsigned char)(1 + or_randint(rng, W_D));
            g->tfac = g->tfac == 0 ? 500.0f + or_uniform(rng) * 3500.0f
                    : (or_uniform(rng) < 0.1f ? 0.0f : or_clamp(g->tfac + (or_uniform(rng) - 0.5f) * 200, 100, 4000));
            if (n >= 0) NG[n].b = or_clamp(NG[n].b + (or_uniform(rng) - 0.5f) * 5, 0, 150);
        } else if (choice == 8 && n >= 0) {
            ngene *g = &NG[n];
            if (g->type == 0) {
                g->adp_b = or_clamp(g->adp_b + (or_uniform(rng) - 0.5f) * 20, 0, 200);
                g->adp_tau = or_clamp(g->adp_tau + (or_uniform(rng) - 0.5f) * 10, 10, 150);
            }
        } else if (choice == 9 && n >= 0) {
            if (NG[n].type != 5 && or_uniform(rng) < 0.5f) NG[n].modulator = (unsigned char)or_randint(rng, 4);
            else NG[n].inh_tx ^= 1;
        } else if (choice == 10) {
            float action = or_uniform(rng);
            int afferent = or_random_afferent(r, &body, rng);
            if (action < 0.5f) {
                int added = or_claim(r.x->neuron_used, NC, child * 131 + body.neuron_count);
                int outgoing = added >= 0 ? or_claim(r.x->synapse_used, EC, child * 257 + body.synapse_count) : -1;
                if (added >= 0 && outgoing >= 0) {
                    int target = body.ports[W_S + or_randint(rng, W_M)];
                    for (int attempt = 0; attempt < 8; ++attempt) {
                        int cand = or_neuron_at(r, &body, or_randint(rng, body.neuron_count));
                        if (w->neuron_port[cand] < 0 || w->neuron_port[cand] >= W_S) { target = cand; break; }
                    }
                    int source = afferent >= 0 && or_uniform(rng) < 0.5f ? afferent : body.ports[or_randint(rng, W_S)];
                    ngene g = NG[source];
                    g.modulator = 0;
                    g.active = 1;
                    or_init_neuron(r, added, child, -1, &g, body.neuron_head, (uint32_t)or_random64(rng));
                    body.neuron_head = added;
                    ++body.neuron_count;
                    sgene edge; memset(&edge, 0, sizeof edge);
                    edge.pre = added;
                    edge.post = target;
                    edge.delay = (unsigned char)(1 + or_randint(rng, W_D));
                    edge.branch = (unsigned char)or_randint(rng, 4);
                    edge.w0 = g.type == 5 ? 29.0f / (60.0f * 0.75f) : 1.0f;
                    edge.U = g.type == 5 ? 0.75f : 0.55f;
                    edge.trec = g.type == 5 ? 50.0f : 450.0f;
                    edge.sites = g.type == 5 ? 50 : 14;
                    edge.slow_rec = g.type == 5 ? 7500.0f : 0.0f;
                    edge.slow_depl = g.type == 5 ? 0.023f : 0.0f;
                    edge.active = 1;
                    or_init_synapse(r, outgoing, child, &edge, body.synapse_head, rng);
                    body.synapse_head = outgoing;
                    ++body.synapse_count;
                    A[child] = body;
                } else {
                    if (outgoing >= 0) or_release(r.x->synapse_used, outgoing);
                    if (added >= 0) or_release(r.x->neuron_used, added);
                }
            } else if (action < 0.75f && afferent >= 0) {
                or_remove_hidden(r, &body, afferent);
                A[child] = body;
            } else if (afferent >= 0) {
                ngene *g = &NG[afferent];
                int channel = or_randint(rng, W_S);
                unsigned char active = g->active, inh = g->inh_tx;
                float affinity = g->affinity;
                if (g->type == 5 && channel >= 6) *g = profile_for_type(0);
                else if (g->type != 5 && channel < 6) *g = profile_for_type(5);
                g->sens = (signed char)channel;
                g->active = active;
                g->inh_tx = inh;
                g->affinity = affinity;
            }
        } else if (choice == 11) {
            int target = or_uniform(rng) < 0.3f ? body.ports[W_S + or_randint(rng, W_M)] : n;
            if (target >= 0)
                NG[target].affinity = or_clamp(NG[target].affinity * (or_uniform(rng) < 0.5f ? 0.5f : 2.0f),
                                               0.125f, 256.0f);
        }
    }
}

static void or_reproduce_one(or_rw r, int a) {                           /* 1662-1737 */
    const or_world_pools *w = r.w;
    const or_world_eco *x = r.x;
    or_animal *A = (or_animal *)w->animals;
    const int P = w->animal_capacity;
    or_animal parent = A[a];
    unsigned long long rng = parent.rng;
    int start = or_randint(&rng, P);
    int child = -1;
    for (int j = 0; j < P; ++j) {
        int cand = (start + j) % P;
        if (A[cand].alive == 0) { A[cand].alive = -1; child = cand; break; }
    }
    if (child < 0) { A[a].rng = rng; return; }
    or_animal nb; memset(&nb, 0, sizeof nb);
    nb.neuron_head = nb.synapse_head = -1;
    for (int p = 0; p < W_S + W_M; ++p) nb.ports[p] = -1;
    nb.x = or_clamp(parent.x + (or_uniform(&rng) - 0.5f) * 2, 0, W_W - 0.001f);
    nb.y = or_clamp(parent.y + (or_uniform(&rng) - 0.5f) * 2, 0, W_H - 0.001f);
    nb.heading = or_uniform(&rng) * 2 * 3.14159265358979323846f;
    nb.energy = 8;
    nb.health = 10;
    nb.generation = parent.generation + 1;
    int complete = 1;
    for (int old = parent.neuron_head; old >= 0; old = w->neuron_next[old]) {
        int n = or_claim(x->neuron_used, w->neuron_capacity, child * 131 + nb.neuron_count);
        if (n < 0) { complete = 0; break; }
        int port = w->neuron_port[old];
        ngene g = ((const ngene *)w->neurons)[old];
        or_init_neuron(r, n, child, port, &g, nb.neuron_head, (uint32_t)or_random64(&rng));
        x->neuron_clone[old] = n;
        nb.neuron_head = n;
        ++nb.neuron_count;
        if (port >= 0) nb.ports[port] = n;
    }
    if (complete)
        for (int old = parent.synapse_head; old >= 0; old = w->synapse_next[old]) {
            int e = or_claim(x->synapse_used, w->synapse_capacity, child * 257 + nb.synapse_count);
            if (e < 0) { complete = 0; break; }
            sgene g = ((const sgene *)w->synapses)[old];
            g.pre = x->neuron_clone[g.pre];
            g.post = x->neuron_clone[g.post];
            or_init_synapse(r, e, child, &g, nb.synapse_head, &rng);
            nb.synapse_head = e;
            ++nb.synapse_count;
        }
    if (!complete) {
        or_release_genome(r, &nb);
        A[child].alive = 0;
        A[a].rng = rng;
        return;
    }
    nb.id = (*x->next_id)++;
    nb.parent_id = parent.id;
    nb.alive = -1;
    A[child] = nb;
    or_mutate(r, child, &rng);
    nb = A[child];
    for (int n = nb.neuron_head; n >= 0; n = w->neuron_next[n])
        ((nstate *)w->neuron_state)[n] = neuron_initial(&((const ngene *)w->neurons)[n], (uint32_t)or_random64(&rng));
    for (int e = nb.synapse_head; e >= 0; e = w->synapse_next[e])
        ((sstate *)w->synapse_state)[e] = synapse_initial(&((const sgene *)w->synapses)[e], (uint32_t)or_random64(&rng));
    for (int s = 0; s < W_S; ++s) ((float *)w->senses)[(size_t)child * W_S + s] = 0;
    for (int m = 0; m < W_M; ++m) w->motors[(size_t)child * W_M + m] = 0;
    nb.rng = rng;
    A[child] = nb;
    parent.energy -= 10;
    ++parent.behavior.offspring;
    parent.rng = rng;
    A[a] = parent;
    A[child].alive = 1;
    ++*x->births;
}

void or_world_reproduce(const or_world_pools *w, const or_world_eco *x) {
    const or_animal *A = (const or_animal *)w->animals;
    const int P = w->animal_capacity;
    unsigned char *parent = (unsigned char *)calloc((size_t)P, 1);
    for (int a = 0; a < P; ++a) parent[a] = A[a].alive == 1 && A[a].energy >= 22;
    or_rw r = {w, x};
    for (int a = 0; a < P; ++a)
        if (parent[a]) or_reproduce_one(r, a);
    free(parent);
}
