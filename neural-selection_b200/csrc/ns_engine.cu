// B200 neural-tick engine: planner, persistent fused tick kernel, reset and
// state readback.
//
// Work decomposition. Synapses are partitioned by their POSTsynaptic neuron:
// the thread that owns neuron j also owns every synapse onto j, stored
// contiguously in ascending original edge order. Within one tick that thread
// (1) delivers its incoming spikes — arrival test against a shared-memory
// ring of spike bitmasks, stochastic release, and accumulation per dendritic
// branch in ascending edge order, the reference's summation order
// (gym_adapter/core.cuh:37-47, gym_adapter/gpu.cu:41-47); (2) integrates the
// neuron; (3) publishes its spike with a warp ballot into the ring; and
// (4) applies plasticity to its incoming synapses. Every input of (1), (2),
// (4) is either its own state or a spike bit from an earlier tick, so one
// __syncthreads per tick is the only synchronisation and no float atomics
// exist. All ticks of a call run inside one launch: the CTA keeps neuron state
// in registers and the spike ring in shared memory for the whole call.
//
// Work units. Brains of at most `block` neurons are packed (best-fit
// decreasing) into units of at most `block` neurons, one neuron per thread.
// A larger brain is a unit of its own; its threads step several neurons each,
// keeping neuron state in global memory (L2-resident during the call). A
// persistent grid pulls units from an atomic queue, largest first.
//
// Plasticity is applied lazily and exactly: a synapse is updated at each tick
// where it has an arrival, a postsynaptic spike or a relevant modulator event;
// the quiet ticks in between are replayed operation by operation
// (plasticity_quiet), and a final pass at the end of the call brings every
// plastic synapse to the last tick. The results equal tick-by-tick updating.
#include "ns_engine.h"
#include "ns_internal.h"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <stdexcept>

#include "ns_crmath.h"
#include "ns_layout.h"
#include "ns_physio.cuh"
#include "ns_reset.cuh"

namespace nsb {

#ifndef NSB_MIN_CTAS
#define NSB_MIN_CTAS 3   // CTAs per SM the light kernel's register budget is sized for
#endif

__device__ __forceinline__ uint32_t rotl32(uint32_t x, uint32_t r) { return __funnelshift_l(x, x, r); }
__device__ __forceinline__ uint32_t rotr32(uint32_t x, uint32_t r) { return __funnelshift_r(x, x, r); }

// Arrival of synapse with meta m at local tick t (gym_adapter/core.cuh:40).
__device__ __forceinline__ bool arrives(uint32_t m, int t, int64_t tick0, const uint32_t *hist, int hw) {
    if (!(m & M_LIVE)) return false;
    const int d = (int)((m >> M_DELAY_SHIFT) & 31u);
    if (tick0 + t < d) return false;
    const uint32_t pre = m & M_PRE_MASK;
    return (hist[((t - d) & 31) * hw + (pre >> 5)] >> (pre & 31u)) & 1u;
}

__device__ __forceinline__ void load_plast(const uint32_t *z, SynPlast &p) {
    p.w = __uint_as_float(z[Z_W]); p.pre_tr = __uint_as_float(z[Z_PRETR]); p.post_tr = __uint_as_float(z[Z_POSTTR]);
    p.eltp = __uint_as_float(z[Z_ELTP]); p.eltd = __uint_as_float(z[Z_ELTD]); p.da_age = __uint_as_float(z[Z_DAAGE]);
    p.spine = __uint_as_float(z[Z_SPINE]); p.st_age = __uint_as_float(z[Z_STAGE]);
    p.pre_age = __uint_as_float(z[Z_PREAGE]); p.post_age = __uint_as_float(z[Z_POSTAGE]);
}
__device__ __forceinline__ void store_plast(uint32_t *z, const SynPlast &p) {
    z[Z_W] = __float_as_uint(p.w); z[Z_PRETR] = __float_as_uint(p.pre_tr); z[Z_POSTTR] = __float_as_uint(p.post_tr);
    z[Z_ELTP] = __float_as_uint(p.eltp); z[Z_ELTD] = __float_as_uint(p.eltd); z[Z_DAAGE] = __float_as_uint(p.da_age);
    z[Z_SPINE] = __float_as_uint(p.spine); z[Z_STAGE] = __float_as_uint(p.st_age);
    z[Z_PREAGE] = __float_as_uint(p.pre_age); z[Z_POSTAGE] = __float_as_uint(p.post_age);
}

__device__ __forceinline__ void load_neuron(const uint32_t *r, NeuronRegs &s, float &log_ampa, uint32_t &hist) {
    const uint4 *q = reinterpret_cast<const uint4 *>(r);
    uint4 a = q[0], b = q[1], c = q[2], d = q[3];
    s.v = __uint_as_float(a.x); s.w = __uint_as_float(a.y); s.adp = __uint_as_float(a.z); s.inh = __uint_as_float(a.w);
    s.depol = __uint_as_float(b.x); log_ampa = __uint_as_float(b.y); s.rec_ns = __uint_as_float(b.z); s.rng = b.w;
    s.d0 = __uint_as_float(c.x); s.d1 = __uint_as_float(c.y); s.d2 = __uint_as_float(c.z); s.d3 = __uint_as_float(c.w);
    s.total = (int)d.x; s.spike = d.y; hist = d.z;
}
__device__ __forceinline__ void store_neuron(uint32_t *r, const NeuronRegs &s, float log_ampa, uint32_t hist,
                                             uint32_t pad) {
    uint4 *q = reinterpret_cast<uint4 *>(r);
    q[0] = make_uint4(__float_as_uint(s.v), __float_as_uint(s.w), __float_as_uint(s.adp), __float_as_uint(s.inh));
    q[1] = make_uint4(__float_as_uint(s.depol), __float_as_uint(log_ampa), __float_as_uint(s.rec_ns), s.rng);
    q[2] = make_uint4(__float_as_uint(s.d0), __float_as_uint(s.d1), __float_as_uint(s.d2), __float_as_uint(s.d3));
    q[3] = make_uint4((uint32_t)s.total, s.spike, hist, pad);
}

__device__ __forceinline__ void load_gene(const float4 *g4, float (&g)[16]) {
    float4 a = g4[0], b = g4[1], c = g4[2], d = g4[3];
    g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w; g[4] = b.x; g[5] = b.y; g[6] = b.z; g[7] = b.w;
    g[8] = c.x; g[9] = c.y; g[10] = c.z; g[11] = c.w; g[12] = d.x; g[13] = d.y; g[14] = d.z; g[15] = d.w;
}

// Stochastic release of one arriving synapse (event path).
__device__ __forceinline__ float release_event(uint32_t *sstate, const uint32_t *sgene, int e, int64_t tick,
                                               const float *tab) {
    uint32_t *z = sstate + (size_t)e * Z_WORDS;
    const float *y = reinterpret_cast<const float *>(sgene + (size_t)e * Y_WORDS);
    SynRelease r;
    r.w = __uint_as_float(z[Z_W]); r.ru = __uint_as_float(z[Z_RU]); r.slow = __uint_as_float(z[Z_SLOW]);
    r.ready = ((uint64_t)z[Z_READYHI] << 32) | z[Z_READYLO];
    r.rng = z[Z_RNG]; r.last = (int)z[Z_LAST];
    const float rel = release(y, r, tick, tab);
    z[Z_RU] = __float_as_uint(r.ru); z[Z_SLOW] = __float_as_uint(r.slow);
    z[Z_READYLO] = (uint32_t)r.ready; z[Z_READYHI] = (uint32_t)(r.ready >> 32);
    z[Z_RNG] = r.rng; z[Z_LAST] = (uint32_t)r.last;
    return rel;
}

// One tick's synaptic input of a postsynaptic neuron.
struct Delivered {
    float e0, e1, e2, e3, inh;
    uint32_t mod;
    int narr;
};

// Fixed points of the input-free tick. A tick integrates a neuron from the
// words below (voltage, adaptation, afterdepolarisation, inhibitory and
// dendritic conductances, depolarisation trace) plus its input; the spike
// word is written, never read, and a neuron without an input channel draws no
// receptor events. So when a tick without input (no applied current, every
// branch sum and the inhibitory sum exactly +0) leaves these words bit for
// bit as they were and emits no spike, every later tick without input leaves
// them unchanged too, and is skipped until an input arrives. The results are
// those of integrating every tick; non-finite voltages and the LP, Prinz and
// LFS cells, whose state lives elsewhere, are never treated as fixed.
__device__ __forceinline__ bool no_input(uint32_t flags, const Delivered &d) {
    return !(flags & NF_HAS_INPUT) &&
           (__float_as_uint(d.e0) | __float_as_uint(d.e1) | __float_as_uint(d.e2) | __float_as_uint(d.e3) |
            __float_as_uint(d.inh)) == 0u;
}
// Does the integrated state s leave the neuron record r (not yet overwritten)
// as it was, with no spike and a finite voltage?
__device__ __forceinline__ bool unchanged(const uint32_t *r, const NeuronRegs &s) {
    const uint4 *q = reinterpret_cast<const uint4 *>(r);
    const uint4 a = q[0], b = q[1], c = q[2];
    return ((a.x ^ __float_as_uint(s.v)) | (a.y ^ __float_as_uint(s.w)) | (a.z ^ __float_as_uint(s.adp)) |
            (a.w ^ __float_as_uint(s.inh)) | (b.x ^ __float_as_uint(s.depol)) | (c.x ^ __float_as_uint(s.d0)) |
            (c.y ^ __float_as_uint(s.d1)) | (c.z ^ __float_as_uint(s.d2)) | (c.w ^ __float_as_uint(s.d3))) == 0u &&
           s.spike == 0u && isfinite(s.v);
}

// Delivery for one postsynaptic neuron at local tick t: arrival test,
// stochastic release and per-branch accumulation in ascending edge order.
__device__ __forceinline__ Delivered deliver(const Pools &P, int ib, int ie, int e0, const uint32_t *meta,
                                             const uint32_t *hist, int t, int64_t tick0, float ampa,
                                             const float *tab) {
    Delivered d = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u, 0};
    const int64_t tick = tick0 + t;
    for (int e = ib; e < ie; ++e) {
        const uint32_t m = meta[e - e0];
        if (!arrives(m, t, tick0, hist, P.hw)) continue;
        ++d.narr;
        const uint32_t kind = (m >> M_KIND_SHIFT) & 3u;
        if (kind == KIND_INH) {             // inhibitory source: weight, no release
            d.inh += __uint_as_float(P.sstate[(size_t)e * Z_WORDS + Z_W]);
            continue;
        }
        const float rel = release_event(P.sstate, P.sgene, e, tick, tab);
        if (kind == KIND_MOD) {
            if (rel > 0) d.mod |= 1u << ((m >> M_MODID_SHIFT) & 3u);
        } else {
            const float c = rel * ampa;
            switch ((m >> M_BRANCH_SHIFT) & 3u) {
            case 0: d.e0 += c; break;
            case 1: d.e1 += c; break;
            case 2: d.e2 += c; break;
            default: d.e3 += c; break;
            }
        }
    }
    return d;
}

// Warp-cooperative delivery: every lane of the warp calls this for its own
// neuron (ib == ie for lanes with nothing to deliver). Arrivals are found per
// lane, compacted into the warp's event list (each lane's events contiguous
// and in ascending edge order), released by all 32 lanes in parallel, and
// then summed by their owner in ascending edge order, so the result equals
// deliver() bit for bit while the release work runs at full SIMD width. A
// warp with more than kEvCap arrivals in one tick falls back to deliver().
constexpr int kEvCap = 128;
__device__ __forceinline__ Delivered deliver_warp(const Pools &P, int ib, int ie, int e0, const uint32_t *meta,
                                                  const uint32_t *hist, int t, int64_t tick0, float ampa,
                                                  const float *tab, int *s_e, uint32_t *s_v, int lane) {
    Delivered d = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u, 0};
    uint32_t amask = 0;
    int cnt = 0;
    for (int e = ib; e < ie; ++e)
        if (arrives(meta[e - e0], t, tick0, hist, P.hw)) {
            if (e - ib < 32) amask |= 1u << (e - ib);
            ++cnt;
        }
    if (__ballot_sync(0xffffffffu, cnt != 0) == 0u) return d;   // no arrival in the warp (the common case)
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return d;
    if (total > kEvCap) return deliver(P, ib, ie, e0, meta, hist, t, tick0, ampa, tab);
    d.narr = cnt;
    const int off = incl - cnt;
    const uint32_t tk = (uint32_t)(tick0 + t);   // below 2^31 (checked per call)
    int k = off;
    for (uint32_t mm = amask; mm; mm &= mm - 1u) {
        s_e[k] = ib + __ffs(mm) - 1;
        s_v[k] = tk;
        ++k;
    }
    for (int e = ib + 32; k < off + cnt; ++e)
        if (arrives(meta[e - e0], t, tick0, hist, P.hw)) {
            s_e[k] = e;
            s_v[k] = tk;
            ++k;
        }
    __syncwarp();
    for (int i = lane; i < total; i += 32) {
        const int e = s_e[i];
        const uint32_t m = meta[e - e0];
        float v;
        if (((m >> M_KIND_SHIFT) & 3u) == KIND_INH) v = __uint_as_float(P.sstate[(size_t)e * Z_WORDS + Z_W]);
        else v = release_event(P.sstate, P.sgene, e, (int64_t)s_v[i], tab);
        s_v[i] = __float_as_uint(v);
    }
    __syncwarp();
    for (int i = off; i < off + cnt; ++i) {
        const uint32_t m = meta[s_e[i] - e0];
        const float v = __uint_as_float(s_v[i]);
        const uint32_t kind = (m >> M_KIND_SHIFT) & 3u;
        if (kind == KIND_INH) {
            d.inh += v;
        } else if (kind == KIND_MOD) {
            if (v > 0) d.mod |= 1u << ((m >> M_MODID_SHIFT) & 3u);
        } else {
            const float c = v * ampa;
            switch ((m >> M_BRANCH_SHIFT) & 3u) {
            case 0: d.e0 += c; break;
            case 1: d.e1 += c; break;
            case 2: d.e2 += c; break;
            default: d.e3 += c; break;
            }
        }
    }
    __syncwarp();
    return d;
}

// Integration of one neuron with this tick's synaptic input. HEAVY builds
// also integrate the LP, Prinz and LFS cell types (out-of-line calls, which
// cost registers, so units without such cells use the light build).
template <bool HEAVY>
__device__ __forceinline__ void integrate(const Pools &P, int n, uint32_t flags, const Delivered &d, float level,
                                          float gain, NeuronRegs &s, int *status, const float *tab) {
    float g[16];
    load_gene(P.ngene + (size_t)n * 4, g);
    const uint32_t type = flags & NF_TYPE_MASK;
    float cur = 0.0f;
    if (flags & NF_HAS_INPUT) cur = type == 5 ? receptor_drive(g, flags, s, level) : gain * level;
    if (HEAVY && (type == 2 || type == 3 || type == 6)) {
        const int xidx = P.nxidx[n];
        s = heavy_tick(reinterpret_cast<const float *>(P.ngene + (size_t)n * 4), type, P.xgene + (size_t)xidx * 16,
                       P.xstate + (size_t)xidx * 16, s, cur, d.e0, d.e1, d.e2, d.e3, d.inh, tab);
    } else {
        adex_tick(g, type, flags, s, cur, d.e0, d.e1, d.e2, d.e3, d.inh, tab);
    }
    if (!isfinite(s.v)) *status = -1;
}

// Plasticity for the incoming synapses of one neuron at local tick t (runs
// only on ticks with an arrival, a postsynaptic spike or a modulator event).
__device__ __forceinline__ void plasticity_events(uint32_t *sstate, const uint32_t *sgene, int16_t *slastp, int hw,
                                                  int ib, int ie, int e0, const uint32_t *meta, const uint32_t *hist,
                                                  int t, int64_t tick0, bool post, uint32_t mod, float depol,
                                                  const float *tab) {
    for (int e = ib; e < ie; ++e) {
        const uint32_t m = meta[e - e0];
        if (!(m & M_PLASTIC)) continue;
        const bool arr = arrives(m, t, tick0, hist, hw);
        const uint32_t prof = m >> M_PROF_SHIFT;
        uint32_t receptors = 0;
        if (mod) receptors = (sgene[(size_t)e * Y_WORDS + Y_INFO] >> 8) & 0xffu;
        if (!arr && !post && !mod_relevant(prof, receptors, mod)) continue;
        const float w0 = __uint_as_float(sgene[(size_t)e * Y_WORDS + Y_W0]);
        uint32_t *z = sstate + (size_t)e * Z_WORDS;
        SynPlast p;
        load_plast(z, p);
        const int last = slastp[e];
        plasticity_quiet(prof, w0, p, t - last - 1);
        plasticity_tick(prof, receptors, w0, p, arr, post, depol, mod, tab);
        store_plast(z, p);
        slastp[e] = (int16_t)t;
    }
}

// End of call for the incoming synapses of one neuron: bring plastic synapses
// to the last tick and record the last tick's arrivals.
__device__ __forceinline__ void finish_synapses(const Pools &P, int ib, int ie, int e0, const uint32_t *meta,
                                                const uint32_t *hist, int ticks, int64_t tick0) {
    for (int e = ib; e < ie; ++e) {
        const uint32_t m = meta[e - e0];
        P.sarrived[e] = arrives(m, ticks - 1, tick0, hist, P.hw) ? 1 : 0;
        if (m & M_PLASTIC) {
            const int last = P.slastp[e];
            const int q = ticks - 1 - last;
            if (q > 0) {
                uint32_t *z = P.sstate + (size_t)e * Z_WORDS;
                SynPlast p;
                load_plast(z, p);
                plasticity_quiet(m >> M_PROF_SHIFT, __uint_as_float(P.sgene[(size_t)e * Y_WORDS + Y_W0]), p, q);
                store_plast(z, p);
            }
            if (last >= 0) P.slastp[e] = -1;
        }
    }
}

extern __shared__ __align__(16) unsigned char g_smem[];

// A heavy unit's pool of pending LP and Prinz cells (one entry per thread at
// most). The counter alternates between two words from call to call, so that
// each pooling needs only its two barriers: a call reads n[p] between them and
// clears n[p ^ 1], which the previous call read and the next call fills.
template <int NT> struct UnitHeavyPool {
    int n[2];
    int xidx[NT];
    float ext[NT];
    float res[NT];       // LP: the axon voltage before the tick; Prinz: 1 when it spiked
    uint8_t type[NT];
};

// One launch steps every unit of [unit_begin, unit_end) through `ticks`
// ticks. Units are pulled from `queue` (reset to 0 before the launch).
template <bool HEAVY, bool COOP>
__global__ void __launch_bounds__(256, HEAVY ? 1 : NSB_MIN_CTAS) tick_kernel(Pools P, int unit_begin, int unit_end, int *queue,
                                                   const float *__restrict__ input,
                                                   const uint8_t *__restrict__ mask, float *__restrict__ output,
                                                   int *__restrict__ status, int ticks, float gain) {
    float *tab = reinterpret_cast<float *>(g_smem);                      // 2^(j/128) hi/lo pairs
    uint32_t *s_meta = reinterpret_cast<uint32_t *>(g_smem + 1024);       // P.meta_cap
    uint32_t *hist = s_meta + P.meta_cap;                                   // 32 * hw
    int *cnt = reinterpret_cast<int *>(hist + 32 * P.hw);                // 32 * hw (spike counts)
    int64_t *s_tick = reinterpret_cast<int64_t *>(cnt + 32 * P.hw);      // kMaxUnitBrains
    int *s_mask = reinterpret_cast<int *>(s_tick + kMaxUnitBrains);
    int *s_bid = s_mask + kMaxUnitBrains;                                 // caller brain index
    int *s_ev = s_bid + kMaxUnitBrains;                                   // 8 warps x kEvCap event synapses
    uint32_t *s_evv = reinterpret_cast<uint32_t *>(s_ev + 8 * kEvCap);    // 8 warps x kEvCap tick / value
    float *s_heavy = reinterpret_cast<float *>(s_evv + 8 * kEvCap);       // 8 warps x kHeavyWarpScratch
    __shared__ int s_unit;
    __shared__ unsigned long long s_events;
    __shared__ UnitHeavyPool<HEAVY ? 256 : 1> s_pool;

    const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = bs >> 5;
    int hcall = 0;   // poolings so far (HEAVY)
    {
        const float *src = nsx::exp2f_table();
        for (int i = tid; i < 256; i += bs) tab[i] = src[i];
        if (HEAVY && tid == 0) s_pool.n[0] = s_pool.n[1] = 0;
    }
    for (;;) {
        if (tid == 0) { s_unit = unit_begin + atomicAdd(queue, 1); s_events = 0; }
        __syncthreads();
        const int u = s_unit;
        if (u >= unit_end) break;
        const int4 U = P.units[u];
        const int2 UB = P.unitb[u];
        const int n0 = U.x, nn = U.y, e0 = U.z, ne = U.w, b0 = UB.x, nb = UB.y;
        for (int i = tid; i < nb; i += bs) {
            const int b = P.ubrain[b0 + i];
            s_bid[i] = b;
            const int64_t t0 = P.btick[b];
            s_tick[i] = t0;
            // last-arrival ticks are stored as int32: refuse to step past 2^31
            const bool in_range = t0 + (int64_t)ticks < 2147483647ll;
            s_mask[i] = mask[b] && in_range;
            status[b] = in_range ? 0 : -2;
        }
        const bool meta_smem = ne <= P.meta_cap;
        if (meta_smem)
            for (int k = tid; k < ne; k += bs) s_meta[k] = P.smeta[e0 + k];
        const uint32_t *meta = meta_smem ? s_meta : P.smeta + e0;
        // A unit whose brains are all masked off does no work: outputs 0.
        if (!__syncthreads_or(tid < nb && s_mask[tid] != 0)) {
            for (int i = tid; i < nb * P.outputs; i += bs)
                output[(size_t)s_bid[i / P.outputs] * P.outputs + (i % P.outputs)] = 0.0f;
            continue;
        }
        const int slots = (nn + bs - 1) / bs;
        int my_events = 0;
        // Each thread steps neurons j = sl0*bs + tid, sl0 < slots; their state
        // stays in global memory (L1/L2-resident for the call). The per-call
        // AMPA scale exp(log_ampa) is kept in the record's spare word.
        for (int sl0 = 0; sl0 < slots; ++sl0) {
            const int j = sl0 * bs + tid;
            const bool has = j < nn;
            const uint32_t flags = has ? P.nflags[n0 + j] : 0u;
            const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
            const bool run = has && s_mask[bi] != 0;
            uint32_t h0 = 0;
            if (run) {
                uint32_t *r = P.nstate + (size_t)(n0 + j) * S_WORDS;
                h0 = r[S_HIST];
                r[S_PAD] = __float_as_uint(crexp(__uint_as_float(r[S_LOGAMPA]), tab));
            }
            const uint32_t rot = run ? rotr32(h0, (uint32_t)(s_tick[bi] & 31)) : 0u;
            for (int sl = 0; sl < 32; ++sl) {
                const uint32_t w = __ballot_sync(0xffffffffu, (rot >> sl) & 1u);
                if (lane == 0) hist[sl * P.hw + sl0 * nwarp + warp] = w;
            }
            if (has) cnt[j] = 0;
        }
        __syncthreads();
        uint32_t fixed = 0;   // bit sl0: this thread's neuron of slot sl0 is at a fixed point (see unchanged)
        for (int t = 0; t < ticks; ++t) {
            for (int sl0 = 0; sl0 < slots; ++sl0) {
                const int j = sl0 * bs + tid;
                const int n = n0 + j;
                const uint32_t flags = j < nn ? P.nflags[n] : 0u;
                const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
                const bool run = j < nn && s_mask[bi] != 0;
                uint32_t spike = 0;
                int ib = 0, ie = 0;
                int64_t tick0 = 0;
                float ampa = 0.0f;
                if (run) {
                    tick0 = s_tick[bi];
                    ib = P.inptr[n];
                    ie = P.inptr[n + 1];
                    ampa = __uint_as_float(P.nstate[(size_t)n * S_WORDS + S_PAD]);
                }
                const bool dlv = run && (flags & NF_ACTIVE);
                Delivered d = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u, 0};
                if (COOP)
                    d = deliver_warp(P, dlv ? ib : 0, dlv ? ie : 0, e0, meta, hist, t, tick0, ampa, tab,
                                     s_ev + warp * kEvCap, s_evv + warp * kEvCap, lane);
                else if (dlv)
                    d = deliver(P, ib, ie, e0, meta, hist, t, tick0, ampa, tab);
                uint32_t *r = P.nstate + (size_t)n * S_WORDS;
                const uint32_t type = flags & NF_TYPE_MASK;
                const uint32_t bit = sl0 < 32 ? 1u << sl0 : 0u;
                uint32_t mod = d.mod;
                float depol = 0.0f;
                // HEAVY: an LP or Prinz cell whose model runs on the whole warp
                bool pending = false;
                NeuronRegs s;
                float log_ampa = 0.0f, ext = 0.0f;
                uint32_t hw0 = 0;
                int xidx = 0;
                if (run) {
                    const bool quiet = no_input(flags, d) && !(HEAVY && (type == 2 || type == 3 || type == 6));
                    if (P.pulse_period > 0 && (tick0 + t) % P.pulse_period == 0) mod |= P.pulse_mod;
                    const bool plast = (flags & NF_PLASTIC_IN) && (mod || d.narr);
                    if (quiet && (fixed & bit)) {
                        // a fixed point without input: the record stays as it is
                        depol = plast ? __uint_as_float(r[S_DEPOL]) : 0.0f;
                    } else {
                        load_neuron(r, s, log_ampa, hw0);
                        if (flags & NF_ACTIVE) {
                            const float level =
                                (flags & NF_HAS_INPUT) ? input[(size_t)s_bid[bi] * P.channels + P.nsens[n]] : 0.0f;
                            if (HEAVY && (type == 2 || type == 3)) {
                                const float *g = reinterpret_cast<const float *>(P.ngene + (size_t)n * 4);
                                const float cur = (flags & NF_HAS_INPUT) ? gain * level : 0.0f;
                                ext = heavy_pre(g, type, s, cur, d.e0, d.e1, d.e2, d.e3, d.inh);
                                xidx = P.nxidx[n];
                                pending = true;
                            } else {
                                integrate<HEAVY>(P, n, flags, d, level, gain, s, status + s_bid[bi], tab);
                            }
                        } else {
                            s.spike = 0;
                        }
                        if (!pending) {
                            fixed = quiet && unchanged(r, s) ? fixed | bit : fixed & ~bit;
                            // the record's spare word keeps the call's AMPA scale
                            store_neuron(r, s, log_ampa, hw0, r[S_PAD]);
                            spike = s.spike;
                            depol = s.depol;
                        }
                    }
                }
                if (HEAVY) {
                    // The unit's pending LP and Prinz cells: a warp that owned
                    // several would step them one after another while the rest
                    // of the CTA waited, so the CTA pools them and the warps take
                    // the pool round-robin, each cell on all 32 lanes; with more
                    // than wc cells per warp on average, each cell runs on its
                    // owner lane at once instead.
                    float axon_before = 0.0f;
                    bool spiked = false;
                    const int p = hcall & 1;
                    ++hcall;
                    int k = 0;
                    if (pending) {
                        k = atomicAdd(&s_pool.n[p], 1);
                        s_pool.xidx[k] = xidx;
                        s_pool.ext[k] = ext;
                        s_pool.type[k] = (uint8_t)type;
                    }
                    __syncthreads();
                    const int np = s_pool.n[p];
                    if (tid == 0) s_pool.n[p ^ 1] = 0;
                    const int wc = P.warp_cells >= 0 ? P.warp_cells : kWarpCellsMax;
                    const bool lanes = np > wc * nwarp;
                    if (lanes) {
                        if (pending)
                            axon_before = heavy_model_lane(type, P.xstate + (size_t)xidx * 16,
                                                           P.xgene + (size_t)xidx * 16, ext, spiked, tab);
                    } else {
                        for (int e = warp; e < np; e += nwarp) {
                            const int xi = s_pool.xidx[e];
                            const uint32_t ty = s_pool.type[e];
                            const float ex = s_pool.ext[e];
                            float *x = P.xstate + (size_t)xi * 16;
                            const float *xg = P.xgene + (size_t)xi * 16;
                            if (ty == 2) {
                                const float ab = x[0];
                                lp_integrate_warp(x, ex / 1000.0f, xg, s_heavy + warp * kHeavyWarpScratch, lane, tab);
                                if (lane == 0) s_pool.res[e] = ab;
                            } else {
                                const bool sp = prinz_tick_warp(x, xg, ex, xg[8] + 0.0f, -68.0f,
                                                                s_heavy + warp * kHeavyWarpScratch, lane, tab);
                                if (lane == 0) s_pool.res[e] = sp ? 1.0f : 0.0f;
                            }
                            __syncwarp();
                        }
                    }
                    __syncthreads();
                    if (pending && !lanes) {
                        axon_before = type == 2 ? s_pool.res[k] : 0.0f;
                        spiked = type == 3 && s_pool.res[k] != 0.0f;
                    }
                    if (pending) {
                        heavy_post(type, s, P.xstate + (size_t)xidx * 16, axon_before, spiked);
                        if (!isfinite(s.v)) status[s_bid[bi]] = -1;
                        fixed &= ~bit;
                        store_neuron(r, s, log_ampa, hw0, r[S_PAD]);
                        spike = s.spike;
                        depol = s.depol;
                    }
                }
                if (run) {
                    if ((flags & NF_PLASTIC_IN) && (spike || mod || d.narr))
                        plasticity_events(P.sstate, P.sgene, P.slastp, P.hw, ib, ie, e0, meta, hist, t, tick0,
                                          spike != 0, mod, depol, tab);
                    cnt[j] += (int)spike;
                    my_events += d.narr;
                }
                const uint32_t w = __ballot_sync(0xffffffffu, spike);
                if (lane == 0) hist[(t & 31) * P.hw + sl0 * nwarp + warp] = w;
            }
            __syncthreads();
        }
        for (int sl0 = 0; sl0 < slots; ++sl0) {
            const int j = sl0 * bs + tid;
            if (j >= nn) continue;
            const int n = n0 + j;
            const uint32_t flags = P.nflags[n];
            const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
            if (!s_mask[bi]) continue;
            const int64_t tick0 = s_tick[bi];
            uint32_t *r = P.nstate + (size_t)n * S_WORDS;
            float la = __uint_as_float(r[S_LOGAMPA]);
            if (flags & NF_ACTIVE) {
                const int total = (int)r[S_TOTAL];
                const int64_t t1 = tick0 + ticks;
                la = homeostasis(flags & NF_TYPE_MASK, la, (float)ticks,
                                 (float)total * 1000.0f / (float)(ticks > t1 ? (int64_t)ticks : t1));
            }
            uint32_t L = 0;
            const int word = sl0 * nwarp + warp;
            for (int sl = 0; sl < 32; ++sl) L |= ((hist[sl * P.hw + word] >> lane) & 1u) << sl;
            r[S_LOGAMPA] = __float_as_uint(la);
            r[S_HIST] = rotl32(L, (uint32_t)(tick0 & 31));
            r[S_PAD] = 0u;
            finish_synapses(P, P.inptr[n], P.inptr[n + 1], e0, meta, hist, ticks, tick0);
        }
        __syncthreads();
        // ---- motor outputs (spikes per call) and tick counters --------------------
        for (int i = tid; i < nb * P.outputs; i += bs) {
            const int bi = i / P.outputs, b = s_bid[bi];
            output[(size_t)b * P.outputs + (i - bi * P.outputs)] =
                s_mask[bi] ? (float)cnt[P.bmotor[(size_t)b * P.outputs + (i - bi * P.outputs)] - n0] : 0.0f;
        }
        for (int i = tid; i < nb; i += bs)
            if (s_mask[i]) P.btick[s_bid[i]] = s_tick[i] + ticks;
        if (P.events) {
            unsigned long long v = (unsigned long long)my_events;
            for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0 && v) atomicAdd(&s_events, v);
            __syncthreads();
            if (tid == 0 && s_events) atomicAdd(P.events, s_events);
        }
        __syncthreads();
    }
}

// ---- light units with a per-tick integration list ---------------------------------
// The light kernel splits each tick in two phases. Phase A: every thread
// delivers the input of its own neurons (in ascending edge order, as above)
// and decides whether each needs integrating; a neuron at a fixed point of
// the input-free tick (see unchanged) with no input this tick does not, and
// its plasticity, if an arrival or modulator calls for it, runs right there
// with no postsynaptic spike. Neurons that do need integrating are appended,
// with their delivered input, to a shared-memory list. Phase B: the CTA's
// threads integrate the list, one entry each, so the integrations run at
// full warp width however the needy neurons are spread over the unit; a
// spike sets its bit in the current ring slot (atomicOr), which phase A of
// the next tick reads. Each neuron's arithmetic is the same as when its owner
// integrates it, so the results are identical bit for bit. Units above
// kListCap neurons run the two phases per chunk of kListCap neurons.
constexpr int kListCap = 768;

#ifndef NSB_LIST_MIN_CTAS
#define NSB_LIST_MIN_CTAS NSB_MIN_CTAS
#endif
template <bool COOP>
__global__ void __launch_bounds__(256, NSB_LIST_MIN_CTAS) tick_kernel_list(Pools P, int unit_begin, int unit_end,
                                                                      int *queue, const float *__restrict__ input,
                                                                      const uint8_t *__restrict__ mask,
                                                                      float *__restrict__ output,
                                                                      int *__restrict__ status, int ticks,
                                                                      float gain) {
    float *tab = reinterpret_cast<float *>(g_smem);                      // 2^(j/128) hi/lo pairs
    uint32_t *s_meta = reinterpret_cast<uint32_t *>(g_smem + 1024);       // P.meta_cap
    uint32_t *hist = s_meta + P.meta_cap;                                   // 32 * hw
    int *cnt = reinterpret_cast<int *>(hist + 32 * P.hw);                // 32 * hw (spike counts)
    uint32_t *s_fixed = reinterpret_cast<uint32_t *>(cnt + 32 * P.hw);   // hw: neuron at a fixed point
    int64_t *s_tick = reinterpret_cast<int64_t *>(s_fixed + ((P.hw + 1) & ~1));   // kMaxUnitBrains
    int *s_mask = reinterpret_cast<int *>(s_tick + kMaxUnitBrains);
    int *s_bid = s_mask + kMaxUnitBrains;                                 // caller brain index
    int *s_ev = s_bid + kMaxUnitBrains;                                   // 8 warps x kEvCap event synapses
    uint32_t *s_evv = reinterpret_cast<uint32_t *>(s_ev + 8 * kEvCap);    // 8 warps x kEvCap tick / value
    int *l_j = reinterpret_cast<int *>(s_evv + 8 * kEvCap);              // the list: neuron, input, mod | narr << 8
    float *l_e0 = reinterpret_cast<float *>(l_j + kListCap), *l_e1 = l_e0 + kListCap, *l_e2 = l_e1 + kListCap,
          *l_e3 = l_e2 + kListCap, *l_inh = l_e3 + kListCap;
    uint32_t *l_mn = reinterpret_cast<uint32_t *>(l_inh + kListCap);
    // units of up to kListCap neurons: flags, incoming-segment starts and the
    // call's AMPA scale of every neuron, staged for the call
    uint32_t *s_nf = l_mn + kListCap;
    int *s_ip = reinterpret_cast<int *>(s_nf + kListCap);                 // kListCap + 1
    float *s_amp = reinterpret_cast<float *>(s_ip + kListCap + 1);
    __shared__ int s_unit, s_count[2];
    __shared__ unsigned long long s_events;

    const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = bs >> 5;
    const int spc = kListCap / bs;                                         // slots per chunk
    {
        const float *src = nsx::exp2f_table();
        for (int i = tid; i < 256; i += bs) tab[i] = src[i];
    }
    for (;;) {
        if (tid == 0) { s_unit = unit_begin + atomicAdd(queue, 1); s_events = 0; s_count[0] = s_count[1] = 0; }
        __syncthreads();
        const int u = s_unit;
        if (u >= unit_end) break;
        const int4 U = P.units[u];
        const int2 UB = P.unitb[u];
        const int n0 = U.x, nn = U.y, e0 = U.z, ne = U.w, b0 = UB.x, nb = UB.y;
        for (int i = tid; i < nb; i += bs) {
            const int b = P.ubrain[b0 + i];
            s_bid[i] = b;
            const int64_t t0 = P.btick[b];
            s_tick[i] = t0;
            // last-arrival ticks are stored as int32: refuse to step past 2^31
            const bool in_range = t0 + (int64_t)ticks < 2147483647ll;
            s_mask[i] = mask[b] && in_range;
            status[b] = in_range ? 0 : -2;
        }
        const bool meta_smem = ne <= P.meta_cap;
        if (meta_smem)
            for (int k = tid; k < ne; k += bs) s_meta[k] = P.smeta[e0 + k];
        const uint32_t *meta = meta_smem ? s_meta : P.smeta + e0;
        for (int w = tid; w < P.hw; w += bs) s_fixed[w] = 0u;
        const bool stage = nn <= kListCap;
        if (stage) {
            for (int j = tid; j < nn; j += bs) {
                s_nf[j] = P.nflags[n0 + j];
                s_ip[j] = P.inptr[n0 + j];
            }
            if (tid == 0) s_ip[nn] = P.inptr[n0 + nn];
        }
        // A unit whose brains are all masked off does no work: outputs 0.
        if (!__syncthreads_or(tid < nb && s_mask[tid] != 0)) {
            for (int i = tid; i < nb * P.outputs; i += bs)
                output[(size_t)s_bid[i / P.outputs] * P.outputs + (i % P.outputs)] = 0.0f;
            continue;
        }
        const int slots = (nn + bs - 1) / bs;
        int my_events = 0;
        for (int sl0 = 0; sl0 < slots; ++sl0) {
            const int j = sl0 * bs + tid;
            const bool has = j < nn;
            const uint32_t flags = has ? P.nflags[n0 + j] : 0u;
            const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
            const bool run = has && s_mask[bi] != 0;
            uint32_t h0 = 0;
            if (run) {
                uint32_t *r = P.nstate + (size_t)(n0 + j) * S_WORDS;
                h0 = r[S_HIST];
                const float amp = crexp(__uint_as_float(r[S_LOGAMPA]), tab);
                r[S_PAD] = __float_as_uint(amp);
                if (stage) s_amp[j] = amp;
            }
            const uint32_t rot = run ? rotr32(h0, (uint32_t)(s_tick[bi] & 31)) : 0u;
            for (int sl = 0; sl < 32; ++sl) {
                const uint32_t w = __ballot_sync(0xffffffffu, (rot >> sl) & 1u);
                if (lane == 0) hist[sl * P.hw + sl0 * nwarp + warp] = w;
            }
            if (has) cnt[j] = 0;
        }
        __syncthreads();
        int seq = 0;   // chunks run so far (the list counter alternates between two words)
        for (int t = 0; t < ticks; ++t) {
            for (int c0 = 0; c0 < slots; c0 += spc, ++seq) {
                const int par = seq & 1;
                if (tid == 0) s_count[par ^ 1] = 0;                      // the next chunk's counter
                // ---- phase A: delivery and the integration list --------------------
                for (int sl0 = c0; sl0 < min(slots, c0 + spc); ++sl0) {
                    const int j = sl0 * bs + tid;
                    const int n = n0 + j;
                    const uint32_t flags = j < nn ? (stage ? s_nf[j] : P.nflags[n]) : 0u;
                    const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
                    const bool run = j < nn && s_mask[bi] != 0;
                    if (lane == 0) hist[(t & 31) * P.hw + sl0 * nwarp + warp] = 0u;   // filled in phase B
                    int ib = 0, ie = 0;
                    int64_t tick0 = 0;
                    float ampa = 0.0f;
                    if (run) {
                        tick0 = s_tick[bi];
                        if (stage) {
                            ib = s_ip[j];
                            ie = s_ip[j + 1];
                            ampa = s_amp[j];
                        } else {
                            ib = P.inptr[n];
                            ie = P.inptr[n + 1];
                            ampa = __uint_as_float(P.nstate[(size_t)n * S_WORDS + S_PAD]);
                        }
                    }
                    const bool dlv = run && (flags & NF_ACTIVE);
                    Delivered d = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u, 0};
                    if (COOP)
                        d = deliver_warp(P, dlv ? ib : 0, dlv ? ie : 0, e0, meta, hist, t, tick0, ampa, tab,
                                         s_ev + warp * kEvCap, s_evv + warp * kEvCap, lane);
                    else if (dlv)
                        d = deliver(P, ib, ie, e0, meta, hist, t, tick0, ampa, tab);
                    bool need = false;
                    uint32_t mod = d.mod;
                    if (run) {
                        if (P.pulse_period > 0 && (tick0 + t) % P.pulse_period == 0) mod |= P.pulse_mod;
                        my_events += d.narr;
                        if (no_input(flags, d) && ((s_fixed[j >> 5] >> (j & 31)) & 1u)) {
                            // a fixed point without input: the record stays as it is, no spike
                            if ((flags & NF_PLASTIC_IN) && (mod || d.narr))
                                plasticity_events(P.sstate, P.sgene, P.slastp, P.hw, ib, ie, e0, meta, hist, t,
                                                  tick0, false, mod,
                                                  __uint_as_float(P.nstate[(size_t)n * S_WORDS + S_DEPOL]), tab);
                        } else {
                            need = true;
                        }
                    }
                    const uint32_t nm = __ballot_sync(0xffffffffu, need);
                    int base = 0;
                    if (lane == 0 && nm) base = atomicAdd(&s_count[par], __popc(nm));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (need) {
                        const int k = base + __popc(nm & ((1u << lane) - 1u));
                        l_j[k] = j;
                        l_e0[k] = d.e0; l_e1[k] = d.e1; l_e2[k] = d.e2; l_e3[k] = d.e3; l_inh[k] = d.inh;
                        l_mn[k] = mod | ((uint32_t)d.narr << 8);
                    }
                }
                __syncthreads();
                // ---- phase B: the list's integrations, one per thread ---------------
                const int count = s_count[par];
                for (int k = tid; k < count; k += bs) {
                    const int j = l_j[k];
                    const int n = n0 + j;
                    const uint32_t flags = stage ? s_nf[j] : P.nflags[n];
                    const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
                    const uint32_t mn = l_mn[k];
                    const Delivered d = {l_e0[k], l_e1[k], l_e2[k], l_e3[k], l_inh[k], mn & 0xffu, (int)(mn >> 8)};
                    uint32_t *r = P.nstate + (size_t)n * S_WORDS;
                    NeuronRegs s;
                    float log_ampa;
                    uint32_t hw0;
                    load_neuron(r, s, log_ampa, hw0);
                    if (flags & NF_ACTIVE) {
                        const float level =
                            (flags & NF_HAS_INPUT) ? input[(size_t)s_bid[bi] * P.channels + P.nsens[n]] : 0.0f;
                        integrate<false>(P, n, flags, d, level, gain, s, status + s_bid[bi], tab);
                    } else {
                        s.spike = 0;
                    }
                    if (no_input(flags, d) && unchanged(r, s)) atomicOr(&s_fixed[j >> 5], 1u << (j & 31));
                    else atomicAnd(&s_fixed[j >> 5], ~(1u << (j & 31)));
                    // the record's spare word keeps the call's AMPA scale
                    store_neuron(r, s, log_ampa, hw0, r[S_PAD]);
                    if (s.spike) {
                        atomicOr(&hist[(t & 31) * P.hw + (j >> 5)], 1u << (j & 31));
                        ++cnt[j];
                    }
                    if ((flags & NF_PLASTIC_IN) && (s.spike || d.mod || d.narr))
                        plasticity_events(P.sstate, P.sgene, P.slastp, P.hw, stage ? s_ip[j] : P.inptr[n],
                                          stage ? s_ip[j + 1] : P.inptr[n + 1], e0, meta, hist, t, s_tick[bi],
                                          s.spike != 0, d.mod, s.depol, tab);
                }
                __syncthreads();
            }
        }
        for (int sl0 = 0; sl0 < slots; ++sl0) {
            const int j = sl0 * bs + tid;
            if (j >= nn) continue;
            const int n = n0 + j;
            const uint32_t flags = P.nflags[n];
            const int bi = (int)((flags >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
            if (!s_mask[bi]) continue;
            const int64_t tick0 = s_tick[bi];
            uint32_t *r = P.nstate + (size_t)n * S_WORDS;
            float la = __uint_as_float(r[S_LOGAMPA]);
            if (flags & NF_ACTIVE) {
                const int total = (int)r[S_TOTAL];
                const int64_t t1 = tick0 + ticks;
                la = homeostasis(flags & NF_TYPE_MASK, la, (float)ticks,
                                 (float)total * 1000.0f / (float)(ticks > t1 ? (int64_t)ticks : t1));
            }
            uint32_t L = 0;
            const int word = sl0 * nwarp + warp;
            for (int sl = 0; sl < 32; ++sl) L |= ((hist[sl * P.hw + word] >> lane) & 1u) << sl;
            r[S_LOGAMPA] = __float_as_uint(la);
            r[S_HIST] = rotl32(L, (uint32_t)(tick0 & 31));
            r[S_PAD] = 0u;
            finish_synapses(P, P.inptr[n], P.inptr[n + 1], e0, meta, hist, ticks, tick0);
        }
        __syncthreads();
        // ---- motor outputs (spikes per call) and tick counters --------------------
        for (int i = tid; i < nb * P.outputs; i += bs) {
            const int bi = i / P.outputs, b = s_bid[bi];
            output[(size_t)b * P.outputs + (i - bi * P.outputs)] =
                s_mask[bi] ? (float)cnt[P.bmotor[(size_t)b * P.outputs + (i - bi * P.outputs)] - n0] : 0.0f;
        }
        for (int i = tid; i < nb; i += bs)
            if (s_mask[i]) P.btick[s_bid[i]] = s_tick[i] + ticks;
        if (P.events) {
            unsigned long long v = (unsigned long long)my_events;
            for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0 && v) atomicAdd(&s_events, v);
            __syncthreads();
            if (tid == 0 && s_events) atomicAdd(P.events, s_events);
        }
        __syncthreads();
    }
}

// ---- big brains: one brain per thread-block cluster -------------------------------
// A brain above the CTA unit size is stepped by a cluster of C CTAs (C = 2, 4
// or 8, from the launch). CTA rank r owns the brain's neurons [r*per,
// min(nn, (r+1)*per)) with per a multiple of 32, so every spike-ring word has
// one owner; each CTA caches the synapse meta words of its own neurons in
// shared memory and keeps a full copy of the brain's spike ring, to which the
// owner of each word writes its ballots (its own copy and, through
// distributed shared memory, every other rank's). One cluster barrier per
// tick replaces the CTA barrier of tick_kernel: tick t+1 reads only ring
// slots of earlier ticks, which the barrier has made visible everywhere.
// Every rank takes the same number of cluster barriers: the unit index comes
// from rank 0 through distributed shared memory, and the mask, tick and tick
// count that decide the work are the same values for every rank.
template <bool COOP>
__global__ void __launch_bounds__(256, NSB_MIN_CTAS) tick_kernel_cluster(Pools P, int unit_begin, int unit_end,
                                                                         int *queue, const float *__restrict__ input,
                                                                         const uint8_t *__restrict__ mask,
                                                                         float *__restrict__ output,
                                                                         int *__restrict__ status, int ticks,
                                                                         float gain) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    float *tab = reinterpret_cast<float *>(g_smem);                      // 2^(j/128) hi/lo pairs
    uint32_t *s_meta = reinterpret_cast<uint32_t *>(g_smem + 1024);       // P.meta_cap
    uint32_t *hist = s_meta + P.meta_cap;                                   // 32 * hw
    int *cnt = reinterpret_cast<int *>(hist + 32 * P.hw);                // 32 * hw (own neurons' spike counts)
    int *s_ev = cnt + 32 * P.hw;                                          // 8 warps x kEvCap
    uint32_t *s_evv = reinterpret_cast<uint32_t *>(s_ev + 8 * kEvCap);
    __shared__ int s_unit;
    __shared__ unsigned long long s_events;

    const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5;
    {
        const float *src = nsx::exp2f_table();
        for (int i = tid; i < 256; i += bs) tab[i] = src[i];
    }
    for (;;) {
        if (tid == 0) {
            if (rank == 0) s_unit = unit_begin + atomicAdd(queue, 1);
            s_events = 0;
        }
        cluster.sync();
        const int u = *cluster.map_shared_rank(&s_unit, 0);
        cluster.sync();                                  // rank 0's s_unit is read before it changes
        if (u >= unit_end) break;
        const int4 U = P.units[u];
        const int n0 = U.x, nn = U.y;
        const int b = P.ubrain[P.unitb[u].x];           // a big unit holds one brain
        const int64_t tick0 = P.btick[b];
        const bool in_range = tick0 + (int64_t)ticks < 2147483647ll;
        const bool run = mask[b] && in_range;
        if (rank == 0 && tid == 0) status[b] = in_range ? 0 : -2;
        if (!run) {
            if (rank == 0)
                for (int i = tid; i < P.outputs; i += bs) output[(size_t)b * P.outputs + i] = 0.0f;
            continue;
        }
        const int per = (((nn + C - 1) / C) + 31) & ~31;
        const int lo = min(nn, rank * per), hi = min(nn, lo + per);
        const int e0 = P.inptr[n0 + lo], e1 = P.inptr[n0 + hi];
        const bool meta_smem = e1 - e0 <= P.meta_cap;
        if (meta_smem)
            for (int k = tid; k < e1 - e0; k += bs) s_meta[k] = P.smeta[e0 + k];
        const uint32_t *meta = meta_smem ? s_meta : P.smeta + e0;
        const int slots = (hi - lo + bs - 1) / bs;
        int my_events = 0;
        for (int sl0 = 0; sl0 < slots; ++sl0) {
            const int j = lo + sl0 * bs + tid;
            const bool has = j < hi;
            uint32_t h0 = 0;
            if (has) {
                uint32_t *r = P.nstate + (size_t)(n0 + j) * S_WORDS;
                h0 = r[S_HIST];
                r[S_PAD] = __float_as_uint(crexp(__uint_as_float(r[S_LOGAMPA]), tab));
            }
            const uint32_t rot = has ? rotr32(h0, (uint32_t)(tick0 & 31)) : 0u;
            const int word = (lo >> 5) + sl0 * (bs >> 5) + warp;
            const bool word_in = lo + sl0 * bs + warp * 32 < hi;
            for (int sl = 0; sl < 32; ++sl) {
                const uint32_t w = __ballot_sync(0xffffffffu, (rot >> sl) & 1u);
                if (lane == 0 && word_in)
                    for (int q = 0; q < C; ++q) *cluster.map_shared_rank(hist + sl * P.hw + word, q) = w;
            }
            if (has) cnt[j - lo] = 0;
        }
        cluster.sync();
        uint32_t fixed = 0;   // bit sl0: this thread's neuron of slot sl0 is at a fixed point (see unchanged)
        for (int t = 0; t < ticks; ++t) {
            for (int sl0 = 0; sl0 < slots; ++sl0) {
                const int j = lo + sl0 * bs + tid;
                const int n = n0 + j;
                const bool has = j < hi;
                const uint32_t flags = has ? P.nflags[n] : 0u;
                uint32_t spike = 0;
                int ib = 0, ie = 0;
                float ampa = 0.0f;
                if (has) {
                    ib = P.inptr[n];
                    ie = P.inptr[n + 1];
                    ampa = __uint_as_float(P.nstate[(size_t)n * S_WORDS + S_PAD]);
                }
                const bool dlv = has && (flags & NF_ACTIVE);
                Delivered d = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u, 0};
                if (COOP)
                    d = deliver_warp(P, dlv ? ib : 0, dlv ? ie : 0, e0, meta, hist, t, tick0, ampa, tab,
                                     s_ev + warp * kEvCap, s_evv + warp * kEvCap, lane);
                else if (dlv)
                    d = deliver(P, ib, ie, e0, meta, hist, t, tick0, ampa, tab);
                if (has) {
                    uint32_t *r = P.nstate + (size_t)n * S_WORDS;
                    const bool quiet = no_input(flags, d);
                    const uint32_t bit = sl0 < 32 ? 1u << sl0 : 0u;
                    uint32_t mod = d.mod;
                    if (P.pulse_period > 0 && (tick0 + t) % P.pulse_period == 0) mod |= P.pulse_mod;
                    const bool plast = (flags & NF_PLASTIC_IN) && (mod || d.narr);
                    float depol;
                    if (quiet && (fixed & bit)) {
                        depol = plast ? __uint_as_float(r[S_DEPOL]) : 0.0f;
                    } else {
                        NeuronRegs s;
                        float log_ampa;
                        uint32_t hw0;
                        load_neuron(r, s, log_ampa, hw0);
                        if (flags & NF_ACTIVE) {
                            const float level =
                                (flags & NF_HAS_INPUT) ? input[(size_t)b * P.channels + P.nsens[n]] : 0.0f;
                            integrate<false>(P, n, flags, d, level, gain, s, status + b, tab);
                        } else {
                            s.spike = 0;
                        }
                        fixed = quiet && unchanged(r, s) ? fixed | bit : fixed & ~bit;
                        store_neuron(r, s, log_ampa, hw0, r[S_PAD]);
                        spike = s.spike;
                        depol = s.depol;
                    }
                    if ((flags & NF_PLASTIC_IN) && (spike || mod || d.narr))
                        plasticity_events(P.sstate, P.sgene, P.slastp, P.hw, ib, ie, e0, meta, hist, t, tick0,
                                          spike != 0, mod, depol, tab);
                    cnt[j - lo] += (int)spike;
                    my_events += d.narr;
                }
                const uint32_t w = __ballot_sync(0xffffffffu, spike);
                const int word = (lo >> 5) + sl0 * (bs >> 5) + warp;
                if (lane == 0 && lo + sl0 * bs + warp * 32 < hi)
                    for (int q = 0; q < C; ++q) *cluster.map_shared_rank(hist + (t & 31) * P.hw + word, q) = w;
            }
            cluster.sync();
        }
        for (int sl0 = 0; sl0 < slots; ++sl0) {
            const int j = lo + sl0 * bs + tid;
            if (j >= hi) continue;
            const int n = n0 + j;
            const uint32_t flags = P.nflags[n];
            uint32_t *r = P.nstate + (size_t)n * S_WORDS;
            float la = __uint_as_float(r[S_LOGAMPA]);
            if (flags & NF_ACTIVE) {
                const int total = (int)r[S_TOTAL];
                const int64_t t1 = tick0 + ticks;
                la = homeostasis(flags & NF_TYPE_MASK, la, (float)ticks,
                                 (float)total * 1000.0f / (float)(ticks > t1 ? (int64_t)ticks : t1));
            }
            uint32_t L = 0;
            const int word = j >> 5;
            for (int sl = 0; sl < 32; ++sl) L |= ((hist[sl * P.hw + word] >> lane) & 1u) << sl;
            r[S_LOGAMPA] = __float_as_uint(la);
            r[S_HIST] = rotl32(L, (uint32_t)(tick0 & 31));
            r[S_PAD] = 0u;
            finish_synapses(P, P.inptr[n], P.inptr[n + 1], e0, meta, hist, ticks, tick0);
        }
        __syncthreads();
        for (int k = tid; k < P.outputs; k += bs) {
            const int m = P.bmotor[(size_t)b * P.outputs + k] - n0;
            if (m >= lo && m < hi) output[(size_t)b * P.outputs + k] = (float)cnt[m - lo];
        }
        if (rank == 0 && tid == 0) P.btick[b] = tick0 + ticks;
        if (P.events) {
            unsigned long long v = (unsigned long long)my_events;
            for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0 && v) atomicAdd(&s_events, v);
            __syncthreads();
            if (tid == 0 && s_events) atomicAdd(P.events, s_events);
        }
        cluster.sync();                                  // ring copies are free for the next unit
    }
}

// ---- reset (gym_adapter/gpu.cu:18-23 with physiology.cuh:179-202, 393-404) --------
__global__ void reset_neurons(Pools P, const int *nbrain, const uint32_t *norig, const uint8_t *mask,
                              const uint32_t *seeds, int n_neurons) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_neurons; n += gridDim.x * blockDim.x) {
        const int b = nbrain[n];
        if (!mask[b]) continue;
        const int xi = P.nxidx[n];
        init_neuron(P.nstate + (size_t)n * S_WORDS, xi >= 0 ? P.xstate + (size_t)xi * 16 : nullptr,
                    P.ngene + (size_t)n * 4, P.nflags[n], seeds[b], norig[n]);
    }
}

__global__ void reset_synapses(Pools P, const int *sbrain, const uint32_t *sorig, const uint8_t *mask,
                               const uint32_t *seeds, int n_synapses) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_synapses; e += gridDim.x * blockDim.x) {
        const int b = sbrain[e];
        if (!mask[b]) continue;
        init_synapse(P.sstate + (size_t)e * Z_WORDS, P.sgene + (size_t)e * Y_WORDS, seeds[b], sorig[e]);
        P.sarrived[e] = 0;
    }
}

__global__ void reset_ticks(int64_t *btick, const uint8_t *mask, int n) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < n && mask[b]) btick[b] = 0;
}

// ---- host side ------------------------------------------------------------------
PhysConst make_constants() {
    PhysConst K;
    K.exc_ms = nsx::expf_cr(-1.0f / 3.0f);
    K.inh_ms = nsx::expf_cr(-1.0f / 10.0f);
    K.exc_sub = nsx::expf_cr(-0.25f / 3.0f);
    K.inh_sub = nsx::expf_cr(-0.25f / 10.0f);
    K.ltp = nsx::expf_cr(-1.0f / 17.0f);
    K.ltd = nsx::expf_cr(-1.0f / 34.0f);
    K.ne = nsx::expf_cr(-1.0f / 7200.0f);
    K.sht = nsx::expf_cr(-1.0f / 3600.0f);
    K.lfs_thr = nsx::expf_cr(-1.0f / 10.0f);
    K.lfs_open[0] = nsx::expf_cr(-1.0f / 10.0f);
    K.lfs_open[1] = nsx::expf_cr(-1.0f / 40.0f);
    K.lfs_open[2] = nsx::expf_cr(-1.0f / 750.0f);
    K.prinz_ca = nsx::expf_cr(-0.025f / 200.0f);
    K.dend_offset = 5.0f / (1.0f + nsx::expf_cr(10.0f));
    K.log_up = nsx::logf_cr(1.92f);
    K.log_down = nsx::logf_cr(0.70f);
    K.tp = nsx::expf_cr(-1.0f / 16.8f);
    K.tm = nsx::expf_cr(-1.0f / 33.7f);
    K.ty = nsx::expf_cr(-1.0f / 114.0f);
    K.te = nsx::expf_cr(-1.0f / 200.0f);
    return K;
}

int spike_words(int max_unit_neurons, int block) {
    // Whole CTA-sized neuron slots: a big unit's threads write one word per
    // warp per slot.
    return ((std::max(max_unit_neurons, block) + block - 1) / block) * (block / 32);
}

// Dynamic shared memory of the light (list) kernel.
int tick_smem_bytes(int hw, int meta_cap) {
    return 1024 + (meta_cap + 32 * hw * 2 + ((hw + 1) & ~1)) * 4 + kMaxUnitBrains * 8 + 2 * kMaxUnitBrains * 4 +
           8 * kEvCap * 8 + kListCap * 7 * 4 + (3 * kListCap + 1) * 4;
}

// Dynamic shared memory of the heavy kernel for hw ring words.
static int heavy_smem_bytes(int hw, int meta_cap = kMetaCap) {
    return 1024 + (meta_cap + 32 * hw * 2) * 4 + kMaxUnitBrains * 8 + 2 * kMaxUnitBrains * 4 + 8 * kEvCap * 8 +
           8 * kHeavyWarpScratch * 4;
}

// The kernels' dynamic shared memory limit is a process-wide attribute: it is
// set to the device's opt-in maximum, so that engines of different shapes in
// one process never lower it under one another's launches.
template <class K> static void allow_dynamic_smem(K kernel, int optin) {
    cudaFuncAttributes fa;
    NSB_CHECK(cudaFuncGetAttributes(&fa, kernel));
    NSB_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   optin - (int)fa.sharedSizeBytes));
}

static void set_tick_smem(int) {
    int dev = 0, optin = 0;
    NSB_CHECK(cudaGetDevice(&dev));
    NSB_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    allow_dynamic_smem(tick_kernel_list<false>, optin);
    allow_dynamic_smem(tick_kernel_list<true>, optin);
    allow_dynamic_smem(tick_kernel<false, false>, optin);
    allow_dynamic_smem(tick_kernel<false, true>, optin);
    allow_dynamic_smem(tick_kernel<true, false>, optin);
    allow_dynamic_smem(tick_kernel_cluster<false>, optin);
    allow_dynamic_smem(tick_kernel_cluster<true>, optin);
}

// Dynamic shared memory of the cluster kernel for hw ring words.
static int cluster_smem_bytes(int hw, int meta_cap = kMetaCap) {
    return 1024 + (meta_cap + 64 * hw) * 4 + 8 * kEvCap * 8;
}

static cudaLaunchConfig_t cluster_config(int C, int clusters, int block, int smem, cudaStream_t s,
                                         cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * clusters), 1, 1);
    cfg.blockDim = dim3((unsigned)block, 1, 1);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// Occupancy queries for the autotuner: 0 when the shape cannot run (the
// query's error, if any, is cleared so that it does not surface later).
static int clusters_resident(int C, int block, int smem) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config(C, 1, block, smem, nullptr, attr);
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveClusters(&a, tick_kernel_cluster<false>, &cfg) != cudaSuccess ||
        cudaOccupancyMaxActiveClusters(&b, tick_kernel_cluster<true>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return std::min(a, b);
}
template <class K> static int ctas_resident(K kernel, int block, int smem) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, block, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ;
}

static void launch_cluster(bool coop, int C, int clusters, int block, int smem, cudaStream_t s, const Pools &P,
                           int ub, int ue, int *queue, const float *input, const uint8_t *mask, float *output,
                           int *status, int ticks, float gain) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = cluster_config(C, clusters, block, smem, s, attr);
    if (coop)
        NSB_CHECK(cudaLaunchKernelEx(&cfg, tick_kernel_cluster<true>, P, ub, ue, queue, input, mask, output, status,
                                     ticks, gain));
    else
        NSB_CHECK(cudaLaunchKernelEx(&cfg, tick_kernel_cluster<false>, P, ub, ue, queue, input, mask, output, status,
                                     ticks, gain));
}

// Light units in either delivery mode (serial per lane, or warp-cooperative).
static void launch_light(bool coop, int grid, int block, int smem, cudaStream_t s, const Pools &P, int ub, int ue,
                         int *queue, const float *input, const uint8_t *mask, float *output, int *status, int ticks,
                         float gain) {
    if (coop)
        tick_kernel_list<true><<<grid, block, smem, s>>>(P, ub, ue, queue, input, mask, output, status, ticks, gain);
    else
        tick_kernel_list<false><<<grid, block, smem, s>>>(P, ub, ue, queue, input, mask, output, status, ticks, gain);
}

void prepare_tick_kernels(int smem) {
    set_tick_smem(smem);
    const PhysConst K = make_constants();
    NSB_CHECK(cudaMemcpyToSymbol(c_K, &K, sizeof(PhysConst)));
}

int serve_smem_bytes(int hw, int meta_cap) { return heavy_smem_bytes(hw, meta_cap); }

int tick_occupancy(int block, int smem) {
    int occ = 0;
    NSB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, tick_kernel<false, true>, block, smem));
    return std::max(occ, 1);
}

// The serving loop's units hold one brain each, of up to 4,096 dense
// neurons: the per-thread kernel with warp-cooperative delivery steps them
// fastest (the autotuner's choice for that population in static batches).
void launch_tick_light(const Pools &P, int n_units, int grid, int block, int smem, int *queue, const float *input,
                       const uint8_t *mask, float *output, int *status, int ticks, float gain, cudaStream_t stream) {
    NSB_CHECK(cudaMemsetAsync(queue, 0, sizeof(int), stream));
    if (n_units > 0)
        tick_kernel<false, true><<<grid, block, smem, stream>>>(P, 0, n_units, queue, input, mask, output, status,
                                                                ticks, gain);
    NSB_CHECK(cudaGetLastError());
}

template <class T> T *Engine::alloc(size_t n) {
    T *p = nullptr;
    if (n == 0) n = 1;
    NSB_CHECK(cudaMalloc(reinterpret_cast<void **>(&p), n * sizeof(T)));
    allocations_.push_back(p);
    return p;
}

static bool excitatory_type(unsigned char t) { return t == 0 || t == 4 || t == 5; }

Plan make_plan(const std::vector<BrainSpec> &brains, int channels, int outputs, int max_delay, int unit_cap,
               bool cluster_big, int heavy_target) {
    Plan p;
    const int n_brains = (int)brains.size();
    // ---- validate and size ----
    long long nsum = 0, esum = 0;
    for (const auto &b : brains) {
        if (b.count < 1 || b.edges < 0) throw std::runtime_error("Invalid brain dimensions");
        if (b.count > kMaxBrainNeurons) throw std::runtime_error("Brain exceeds 16384 neurons");
        for (int j = 0; j < b.edges; ++j) {
            const auto &c = b.conns[j];
            if (c.pre < 0 || c.pre >= b.count || c.post < 0 || c.post >= b.count)
                throw std::runtime_error("Invalid synapse gene");
            if (c.delay > max_delay || c.delay < 1) throw std::runtime_error("Synapse delay exceeds the delay ring");
        }
        for (int j = 0; j < outputs; ++j)
            if (b.motors[j] < 0 || b.motors[j] >= b.count) throw std::runtime_error("Invalid motor index");
        nsum += b.count; esum += b.edges;
    }
    if (nsum > (1ll << 30) || esum > (1ll << 30)) throw std::runtime_error("Pool exceeds 2^30 entries");
    p.n_neurons = (int)nsum; p.n_synapses = (int)esum;

    // ---- work units ------------------------------------------------------------
    // Brains with LP/Prinz/LFS cells go to units of their own (stepped by the
    // heavy kernel). Within each group a brain above the group's unit capacity
    // is a unit of its own; smaller brains are packed best-fit decreasing. The
    // heavy kernel runs one CTA per SM and its cell models are long chains per
    // lane, so its units are sized to spread the heavy neurons over
    // heavy_target SMs rather than filled to unit_cap.
    auto is_heavy_type = [](unsigned char t) { return t == 2 || t == 3 || t == 6; };
    std::vector<char> brain_heavy(n_brains, 0);
    long long heavy_neurons = 0;
    for (int b = 0; b < n_brains; ++b)
        for (int j = 0; j < brains[b].count; ++j)
            if (is_heavy_type(brains[b].genes[j].type)) { brain_heavy[b] = 1; heavy_neurons += brains[b].count; break; }
    const int heavy_cap = heavy_target > 0
        ? (int)std::min<long long>(unit_cap, std::max<long long>(1, (heavy_neurons + heavy_target - 1) / heavy_target))
        : unit_cap;
    std::vector<std::vector<int>> unit_brains;
    std::vector<int> unit_fill;
    std::vector<char> unit_heavy;
    for (int group = 0; group < 2; ++group) {
        const int cap = group ? heavy_cap : unit_cap;
        std::vector<int> order;
        for (int b = 0; b < n_brains; ++b)
            if (brain_heavy[b] == group) order.push_back(b);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return brains[a].count > brains[b].count; });
        std::multimap<int, int> open;   // remaining capacity -> unit
        for (int b : order) {
            const int n = brains[b].count;
            if (n > cap) {
                unit_brains.push_back({b}); unit_fill.push_back(n); unit_heavy.push_back((char)group);
                continue;
            }
            auto it = open.lower_bound(n);
            if (it != open.end()) {
                const int uidx = it->second;
                open.erase(it);
                unit_brains[uidx].push_back(b);
                unit_fill[uidx] += n;
                const int rem = cap - unit_fill[uidx];
                if (rem > 0 && (int)unit_brains[uidx].size() < kMaxUnitBrains) open.emplace(rem, uidx);
            } else {
                unit_brains.push_back({b}); unit_fill.push_back(n); unit_heavy.push_back((char)group);
                const int rem = cap - n;
                if (rem > 0) open.emplace(rem, (int)unit_brains.size() - 1);
            }
        }
    }
    // Queue order: light units stepped by clusters of 8, 4 and 2 CTAs (one
    // brain above the CTA unit size each), light units of one CTA, heavy
    // units; by neuron count descending within each group.
    auto group_of = [&](int u) {
        if (unit_heavy[u]) return 4;
        if (!cluster_big || unit_fill[u] <= unit_cap) return 3;
        if (unit_fill[u] <= 2 * unit_cap) return 2;
        if (unit_fill[u] <= 4 * unit_cap) return 1;
        return 0;
    };
    std::vector<int> uorder(unit_brains.size());
    std::iota(uorder.begin(), uorder.end(), 0);
    std::stable_sort(uorder.begin(), uorder.end(), [&](int a, int b) {
        const int ga = group_of(a), gb = group_of(b);
        if (ga != gb) return ga < gb;
        return unit_fill[a] > unit_fill[b];
    });
    p.n_units = (int)unit_brains.size();
    p.n_light_units = 0;
    for (int u : uorder) {
        const int g = group_of(u);
        p.n_light_units += g < 4 ? 1 : 0;
        if (g < 3) ++p.n_cluster[g];
        int &mx = g < 3 ? p.max_big : (g == 3 ? p.max_small : p.max_heavy);
        mx = std::max(mx, unit_fill[u]);
    }

    // ---- per-brain bookkeeping (caller order) ----
    auto &h_noff_ = p.noff, &h_soff_ = p.soff, &h_npos_ = p.npos, &h_spos_ = p.spos, &h_bunit_ = p.bunit;
    h_noff_.assign(n_brains + 1, 0);
    h_soff_.assign(n_brains + 1, 0);
    for (int b = 0; b < n_brains; ++b) {
        h_noff_[b + 1] = h_noff_[b] + brains[b].count;
        h_soff_[b + 1] = h_soff_[b] + brains[b].edges;
    }
    h_npos_.assign(p.n_neurons, 0);
    h_spos_.assign(p.n_synapses, 0);
    h_bunit_.assign(n_brains, 0);
    p.units.assign(p.n_units, make_int4(0, 0, 0, 0));
    p.unitb.assign(p.n_units, make_int2(0, 0));
    auto &h_units_ = p.units;
    auto &unitb = p.unitb;
    auto &brain_order = p.brain_order;   // unit brain lists (caller indices), pool order

    // ---- per-neuron and per-synapse records ----
    const int n_neurons = p.n_neurons, n_synapses = p.n_synapses;
    auto &ngene = p.ngene, &xgene = p.xgene;
    auto &h_nflags_ = p.nflags, &norig = p.norig, &smeta = p.smeta, &sgene = p.sgene, &sorig = p.sorig;
    auto &nsens = p.nsens, &nbrain = p.nbrain, &h_nxidx_ = p.nxidx, &inptr = p.inptr, &sbrain = p.sbrain,
         &bmotor = p.bmotor;
    ngene.assign((size_t)n_neurons * 16, 0.0f);
    h_nflags_.assign(n_neurons, 0);
    nsens.assign(n_neurons, 0); nbrain.assign(n_neurons, 0);
    h_nxidx_.assign(n_neurons, -1);
    norig.assign(n_neurons, 0);
    inptr.assign(n_neurons + 1, 0);
    smeta.assign(n_synapses, 0); sgene.assign((size_t)n_synapses * Y_WORDS, 0); sorig.assign(n_synapses, 0);
    sbrain.assign(n_synapses, 0);
    bmotor.assign((size_t)n_brains * outputs, 0);

    int ncur = 0, ecur = 0;
    for (int ui = 0; ui < p.n_units; ++ui) {
        const auto &ub = unit_brains[uorder[ui]];
        const int un0 = ncur, ue0 = ecur;
        unitb[ui] = make_int2((int)brain_order.size(), (int)ub.size());
        // Neuron order inside the unit: active before inactive, then by cell
        // class (type 0 | types 1,4 | type 5 | LP | Prinz | LFS), then by which
        // dendritic branches receive excitatory synapses, so that a warp's
        // lanes take the same path through the integrator.
        struct Key { int inactive, cls, bmask, slot, j; };
        std::vector<Key> keys;
        for (int slot = 0; slot < (int)ub.size(); ++slot) {
            const int b = ub[slot];
            const BrainSpec &B = brains[b];
            h_bunit_[b] = ui;
            brain_order.push_back(b);
            std::vector<int> bmask(B.count, 0);
            for (int j = 0; j < B.edges; ++j) {
                const ref::SynapseGene &C = B.conns[j];
                const ref::NeuronGene &A = B.genes[C.pre], &Z = B.genes[C.post];
                if (C.active && A.active && Z.active && !A.modulator && !A.inh_tx) bmask[C.post] |= 1 << (C.branch & 3);
            }
            for (int j = 0; j < B.count; ++j) {
                const unsigned char t = B.genes[j].type;
                // LP, Prinz and LFS cells each in a class of their own, so a
                // warp's cells run one model at a time instead of diverging
                const int cls = t == 2 ? 3 : t == 3 ? 4 : t == 6 ? 5 : (t == 0 ? 0 : (t == 5 ? 2 : 1));
                keys.push_back({B.genes[j].active ? 0 : 1, cls, t == 0 ? bmask[j] : 0, slot, j});
            }
        }
        std::stable_sort(keys.begin(), keys.end(), [](const Key &a, const Key &b) {
            if (a.inactive != b.inactive) return a.inactive < b.inactive;
            if (a.cls != b.cls) return a.cls < b.cls;
            if (a.bmask != b.bmask) return a.bmask < b.bmask;
            if (a.slot != b.slot) return a.slot < b.slot;
            return a.j < b.j;
        });
        for (size_t q = 0; q < keys.size(); ++q) {
            const int b = ub[keys[q].slot];
            h_npos_[h_noff_[b] + keys[q].j] = un0 + (int)q;
        }
        // neuron records
        for (size_t q = 0; q < keys.size(); ++q) {
            const int slot = keys[q].slot, j = keys[q].j, b = ub[slot];
            const BrainSpec &B = brains[b];
            const ref::NeuronGene &G = B.genes[j];
            const int n = un0 + (int)q;
            float *g = &ngene[(size_t)n * 16];
            g[G_CAP] = G.cap; g[G_GL] = G.gl; g[G_EL] = G.el; g[G_VT] = G.vt;
            g[G_SLOPE] = G.slope; g[G_A] = G.a; g[G_TAUW] = G.tau_w; g[G_B] = G.b;
            g[G_VR] = G.vr; g[G_ADPB] = G.adp_b;
            g[G_ADPDECAY] = G.adp_tau > 0 ? nsx::expf_cr(-0.25f / G.adp_tau) : 1.0f;
            g[G_GLSLOPE] = G.gl * G.slope;
            g[G_RECBASE] = G.rec_base; g[G_RECGAIN] = G.rec_gain; g[G_RECEVENT] = G.rec_event;
            g[G_RECDECAY] = nsx::expf_cr(-1.0f / G.rec_decay);
            if (G.type > 6) throw std::runtime_error("Invalid neuron gene");
            uint32_t f = (uint32_t)G.type;
            if (G.active) f |= NF_ACTIVE;
            if (G.inh_tx) f |= NF_INH;
            f |= (uint32_t)(G.modulator & 3u) << NF_MOD_SHIFT;
            if (G.sensory_channel >= 0) f |= NF_GENE_SENS;
            if (G.adp_tau > 0) f |= NF_ADP;
            const int sens = B.sensory ? B.sensory[j] : -1;
            if (sens >= 0) {
                if (sens >= channels) throw std::runtime_error("Invalid neuron gene");
                f |= NF_HAS_INPUT;
            }
            if (excitatory_type(G.type)) f |= NF_EXC_TYPE;
            f |= (uint32_t)slot << NF_SLOT_SHIFT;
            h_nflags_[n] = f;
            nsens[n] = sens;
            nbrain[n] = b;
            norig[n] = B.orig_n ? B.orig_n[j] : (uint32_t)j;
            if (is_heavy_type(G.type)) {
                h_nxidx_[n] = p.n_heavy++;
                float xg[16] = {};
                if (G.type == 2) { xg[0] = G.lp.calcium; xg[1] = G.lp.calcium_k; xg[2] = G.lp.h; xg[3] = G.lp.leak; }
                if (G.type == 3) { for (int r = 0; r < 8; ++r) xg[r] = G.prinz.g[r]; xg[8] = G.prinz_leak; }
                xgene.insert(xgene.end(), xg, xg + 16);
            }
        }
        // synapses: grouped by postsynaptic pool position, then original edge order
        struct SKey { int post, j, b; };
        std::vector<SKey> sk;
        for (int slot = 0; slot < (int)ub.size(); ++slot) {
            const int b = ub[slot];
            for (int j = 0; j < brains[b].edges; ++j)
                sk.push_back({h_npos_[h_noff_[b] + brains[b].conns[j].post], j, b});
        }
        std::stable_sort(sk.begin(), sk.end(), [](const SKey &a, const SKey &b) {
            return a.post != b.post ? a.post < b.post : a.j < b.j;
        });
        for (size_t q = 0; q < sk.size(); ++q) {
            const int b = sk[q].b, j = sk[q].j;
            const BrainSpec &B = brains[b];
            const ref::SynapseGene &C = B.conns[j];
            const int e = ue0 + (int)q;
            h_spos_[h_soff_[b] + j] = e;
            const ref::NeuronGene &A = B.genes[C.pre], &Z = B.genes[C.post];
            const bool live = C.active && A.active && Z.active;
            const bool pair = !A.inh_tx && excitatory_type(A.type) && !A.modulator && !Z.inh_tx &&
                              excitatory_type(Z.type);
            const uint32_t kind = A.modulator ? KIND_MOD : (A.inh_tx ? KIND_INH : KIND_EXC);
            const int pre_local = h_npos_[h_noff_[b] + C.pre] - un0;
            if (pre_local > 0xffff) throw std::runtime_error("Unit exceeds 65536 neurons");
            if (C.plasticity > 7) throw std::runtime_error("Invalid synapse gene");
            uint32_t m = (uint32_t)pre_local | ((uint32_t)C.delay << M_DELAY_SHIFT) |
                         ((uint32_t)(C.branch & 3u) << M_BRANCH_SHIFT) | (kind << M_KIND_SHIFT) |
                         ((uint32_t)((A.modulator ? A.modulator - 1 : 0) & 3u) << M_MODID_SHIFT) |
                         ((uint32_t)C.plasticity << M_PROF_SHIFT);
            if (live) m |= M_LIVE;
            if (live && C.plasticity && pair) {
                m |= M_PLASTIC;
                h_nflags_[sk[q].post] |= NF_PLASTIC_IN;
            }
            smeta[e] = m;
            const int sites = C.sites ? (C.sites > 64 ? 64 : C.sites) : 14;
            uint32_t *y = &sgene[(size_t)e * Y_WORDS];
            const float yf[8] = {C.w0, C.U, C.trec, C.tfac, C.slow_rec, C.slow_depl, 0.0f, 0.0f};
            std::memcpy(y, yf, sizeof yf);
            y[Y_INFO] = (uint32_t)sites | ((uint32_t)C.receptors << 8);
            sorig[e] = B.orig_s ? B.orig_s[j] : (uint32_t)j;
            sbrain[e] = b;
        }
        // incoming segment starts
        int cursor = ue0;
        size_t q = 0;
        for (int n = un0; n < un0 + (int)keys.size(); ++n) {
            inptr[n] = cursor;
            while (q < sk.size() && sk[q].post == n) { ++q; ++cursor; }
        }
        ncur += (int)keys.size();
        ecur += (int)sk.size();
        h_units_[ui] = make_int4(un0, ncur - un0, ue0, ecur - ue0);
        p.max_unit_neurons = std::max(p.max_unit_neurons, ncur - un0);
        if (ncur - un0 > unit_cap) ++p.n_big_units;
        p.max_unit_brains = std::max(p.max_unit_brains, (int)ub.size());
    }
    inptr[n_neurons] = n_synapses;
    for (int b = 0; b < n_brains; ++b)
        for (int j = 0; j < outputs; ++j)
            bmotor[(size_t)b * outputs + j] = h_npos_[h_noff_[b] + brains[b].motors[j]];
    return p;
}

Engine::Engine(const std::vector<BrainSpec> &brains, int channels, int outputs, const EngineConfig &cfg) {
    if (brains.empty()) throw std::runtime_error("Empty GPU batch");
    if (cfg.max_delay < 1 || cfg.max_delay > kMaxDelay) throw std::runtime_error("Invalid delay ring");
    if (cfg.block != 128 && cfg.block != 256) throw std::runtime_error("Invalid CUDA block size");
    n_brains_ = (int)brains.size();
    channels_ = channels; outputs_ = outputs; max_delay_ = cfg.max_delay; block_ = cfg.block;
    count_events_ = cfg.count_events;
    warp_cells_ = cfg.warp_cells;
    unit_cap_ = block_ * (cfg.unit_slots > 0 ? cfg.unit_slots : 3);
    int dev0 = 0, sms0 = 0;
    NSB_CHECK(cudaGetDevice(&dev0));
    NSB_CHECK(cudaDeviceGetAttribute(&sms0, cudaDevAttrMultiProcessorCount, dev0));
    Plan p = make_plan(brains, channels, outputs, max_delay_, unit_cap_, cfg.cluster_big == 1, sms0);
    if (cfg.unit_slots <= 0 && p.n_light_units < sms0 * NSB_MIN_CTAS) {
        // A batch too small to fill the GPU: one neuron per thread, so each
        // unit's tick is one neuron update long instead of three.
        unit_cap_ = block_;
        p = make_plan(brains, channels, outputs, max_delay_, unit_cap_, cfg.cluster_big == 1, sms0);
    }
    if (cfg.cluster_big < 0 && p.n_big_units > 0 && p.n_light_units < sms0 * NSB_MIN_CTAS)
        p = make_plan(brains, channels, outputs, max_delay_, unit_cap_, true, sms0);
    n_neurons_ = p.n_neurons; n_synapses_ = p.n_synapses; n_units_ = p.n_units; n_light_units_ = p.n_light_units;
    n_big_units_ = p.n_big_units; n_heavy_ = p.n_heavy; max_unit_neurons_ = p.max_unit_neurons;
    max_unit_brains_ = p.max_unit_brains;
    h_noff_ = std::move(p.noff); h_soff_ = std::move(p.soff); h_npos_ = std::move(p.npos);
    h_spos_ = std::move(p.spos); h_bunit_ = std::move(p.bunit); h_units_ = p.units;
    h_nflags_ = p.nflags; h_nxidx_ = p.nxidx;
    const auto &ngene = p.ngene, &xgene = p.xgene;
    const auto &norig = p.norig, &smeta = p.smeta, &sgene = p.sgene, &sorig = p.sorig;
    const auto &nsens = p.nsens, &nbrain = p.nbrain, &inptr = p.inptr, &sbrain = p.sbrain, &bmotor = p.bmotor;
    const auto &unitb = p.unitb;
    const auto &brain_order = p.brain_order;
    hw_ = spike_words(max_unit_neurons_, block_);
    coop_ = n_synapses_ >= 4ll * n_neurons_;
    // Light units are in queue order by size, largest first; a unit above the
    // unit size holds one brain. Buckets by size class, then the heavy units.
    const bool clustered = cfg.cluster_big == 1 ||
                           (cfg.cluster_big < 0 && p.n_big_units > 0 && p.n_light_units < sms0 * NSB_MIN_CTAS);
    buckets_.assign(kBuckets, Bucket{});
    {
        auto bucket_of = [&](int nn) { return nn > 4 * unit_cap_ ? 0 : nn > 2 * unit_cap_ ? 1 : nn > unit_cap_ ? 2 : 3; };
        for (int b = 0; b < kBuckets; ++b) buckets_[b].ub = buckets_[b].ue = b == kBucketHeavy ? n_light_units_ : 0;
        int cur = -1;
        for (int u = 0; u < n_light_units_; ++u) {
            const int b = bucket_of(p.units[u].y);
            if (b < cur) throw std::runtime_error("Work units out of size order");
            if (b != cur) { buckets_[b].ub = u; cur = b; }
            buckets_[b].ue = u + 1;
        }
        buckets_[kBucketHeavy].ub = n_light_units_;
        buckets_[kBucketHeavy].ue = n_units_;
        buckets_[kBucketHeavy].heavy = true;
        for (int b = 0; b < kBuckets; ++b) {
            Bucket &B = buckets_[b];
            if (B.ue < B.ub) B.ue = B.ub;
            for (int u = B.ub; u < B.ue; ++u) {
                B.max_neurons = std::max(B.max_neurons, p.units[u].y);
                B.max_synapses = std::max(B.max_synapses, p.units[u].w);
            }
            B.cluster_size = b < 3 ? kClusterSizes[b] : 1;
            B.cfg.block = block_;
            B.cfg.coop = b == kBucketHeavy ? 0 : (int)coop_;
            B.cfg.cluster = b < 3 && clustered ? B.cluster_size : 1;
            B.cfg.meta_cap = kMetaCap;
        }
    }

    // ---- device allocation and upload ----
    NSB_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    auto up = [&](auto *dst, const auto &src) {
        NSB_CHECK(cudaMemcpy(dst, src.data(), src.size() * sizeof(src[0]), cudaMemcpyHostToDevice));
    };
    d_ngene_ = alloc<float>(ngene.size()); up(d_ngene_, ngene);
    d_nflags_ = alloc<uint32_t>(n_neurons_); up(d_nflags_, h_nflags_);
    d_nsens_ = alloc<int>(n_neurons_); up(d_nsens_, nsens);
    d_nxidx_ = alloc<int>(n_neurons_); up(d_nxidx_, h_nxidx_);
    d_xgene_ = alloc<float>(std::max<size_t>(xgene.size(), 16)); if (!xgene.empty()) up(d_xgene_, xgene);
    d_xstate_ = alloc<float>((size_t)std::max(n_heavy_, 1) * 16);
    NSB_CHECK(cudaMemset(d_xstate_, 0, (size_t)std::max(n_heavy_, 1) * 16 * sizeof(float)));
    d_nstate_ = alloc<uint32_t>((size_t)n_neurons_ * S_WORDS);
    NSB_CHECK(cudaMemset(d_nstate_, 0, (size_t)n_neurons_ * S_WORDS * 4));
    d_inptr_ = alloc<int>(n_neurons_ + 1); up(d_inptr_, inptr);
    d_smeta_ = alloc<uint32_t>(n_synapses_); if (n_synapses_) up(d_smeta_, smeta);
    d_sgene_ = alloc<uint32_t>((size_t)n_synapses_ * Y_WORDS); if (n_synapses_) up(d_sgene_, sgene);
    d_sstate_ = alloc<uint32_t>((size_t)n_synapses_ * Z_WORDS);
    NSB_CHECK(cudaMemset(d_sstate_, 0, (size_t)std::max(n_synapses_, 1) * Z_WORDS * 4));
    d_sarrived_ = alloc<uint8_t>(n_synapses_);
    NSB_CHECK(cudaMemset(d_sarrived_, 0, std::max(n_synapses_, 1)));
    d_slastp_ = alloc<int16_t>(n_synapses_);
    NSB_CHECK(cudaMemset(d_slastp_, 0xff, (size_t)std::max(n_synapses_, 1) * 2));
    d_btick_ = alloc<int64_t>(n_brains_); NSB_CHECK(cudaMemset(d_btick_, 0, n_brains_ * sizeof(int64_t)));
    d_bmotor_ = alloc<int>(std::max<size_t>(bmotor.size(), 1)); up(d_bmotor_, bmotor);
    d_ubrain_ = alloc<int>(n_brains_); up(d_ubrain_, brain_order);
    d_units_ = alloc<int4>(n_units_); up(d_units_, h_units_);
    d_unitb_ = alloc<int2>(n_units_); up(d_unitb_, unitb);
    d_queue_ = alloc<int>(8);
    d_events_ = alloc<unsigned long long>(1); NSB_CHECK(cudaMemset(d_events_, 0, 8));
    d_input_ = alloc<float>((size_t)n_brains_ * channels);
    NSB_CHECK(cudaMemset(d_input_, 0, (size_t)n_brains_ * channels * 4));
    d_mask_ = alloc<uint8_t>(n_brains_); NSB_CHECK(cudaMemset(d_mask_, 1, n_brains_));
    d_output_ = alloc<float>((size_t)n_brains_ * outputs);
    d_status_ = alloc<int>(n_brains_);
    d_seeds_ = alloc<uint32_t>(n_brains_);
    d_rmask_ = alloc<uint8_t>(n_brains_);
    d_nbrain_ = alloc<int>(n_neurons_); up(d_nbrain_, nbrain);
    d_norig_ = alloc<uint32_t>(n_neurons_); up(d_norig_, norig);
    d_sbrain_ = alloc<int>(n_synapses_); if (n_synapses_) up(d_sbrain_, sbrain);
    d_sorig_ = alloc<uint32_t>(n_synapses_); if (n_synapses_) up(d_sorig_, sorig);
    h_tick_.assign(n_brains_, 0);

    // ---- launch shape ----
    set_tick_smem(0);
    int dev = 0, optin = 0;
    NSB_CHECK(cudaGetDevice(&dev));
    NSB_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
    NSB_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    smem_optin_ = optin - 1024;      // room for the kernels' static shared memory
    ctas_cap_ = cfg.ctas_per_sm;
    for (int b = 0; b < kBuckets; ++b) {
        Bucket &B = buckets_[b];
        if (!shape_bucket(B) && B.cfg.cluster > 1) {   // clusters that cannot run: one CTA per brain
            B.cfg.cluster = 1;
            if (!shape_bucket(B)) throw std::runtime_error("Work unit exceeds the device's shared memory");
        } else if (B.units() && B.grid == 0) {
            throw std::runtime_error("Work unit exceeds the device's shared memory");
        }
    }
    for (int b = 0; b < kBuckets; ++b) {
        NSB_CHECK(cudaStreamCreateWithFlags(&bstream_[b], cudaStreamNonBlocking));
        NSB_CHECK(cudaEventCreateWithFlags(&join_[b], cudaEventDisableTiming));
    }
    NSB_CHECK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    K_ = make_constants();
    NSB_CHECK(cudaMemcpyToSymbol(c_K, &K_, sizeof(PhysConst)));
}

Engine::~Engine() {
    for (auto &g : graphs_) cudaGraphExecDestroy(g.exec);
    for (void *p : allocations_) cudaFree(p);
    for (int b = 0; b < kBuckets; ++b) {
        if (bstream_[b]) cudaStreamDestroy(bstream_[b]);
        if (join_[b]) cudaEventDestroy(join_[b]);
    }
    if (fork_) cudaEventDestroy(fork_);
    if (stream_) cudaStreamDestroy(stream_);
}

Stats Engine::stats() const {
    const Bucket &B = buckets_[kBucketPacked];
    const int occ = B.units() ? ctas_resident(tick_kernel_list<false>, B.cfg.block, B.smem) : 0;
    return Stats{n_brains_, n_units_, n_big_units_, n_neurons_, n_synapses_, n_heavy_, max_unit_neurons_,
                 B.grid, B.cfg.block, B.smem, occ};
}

bool Engine::shape_bucket(Bucket &B) const {
    const BucketConfig &c = B.cfg;
    if (c.block != 128 && c.block != 256) return false;
    if (c.meta_cap < 0 || c.meta_cap % 32 != 0) return false;
    if (B.heavy && (c.coop || c.cluster != 1 || !c.list)) return false;
    if (c.list != 0 && c.list != 1) return false;
    if (c.cluster != 1 && c.cluster != B.cluster_size) return false;
    B.hw = spike_words(B.max_neurons, c.block);
    if (B.units() == 0) {
        B.smem = 0;
        B.grid = 0;
        return true;
    }
    if (B.heavy) {
        B.smem = heavy_smem_bytes(B.hw, c.meta_cap);
        const int occ = B.smem <= smem_optin_ ? ctas_resident(tick_kernel<true, false>, c.block, B.smem) : 0;
        B.grid = std::min(B.units(), sms_ * occ);
    } else if (c.cluster > 1) {
        B.smem = cluster_smem_bytes(B.hw, c.meta_cap);
        B.grid = B.smem <= smem_optin_ ? std::min(B.units(), clusters_resident(c.cluster, c.block, B.smem)) : 0;
    } else if (!c.list) {
        B.smem = heavy_smem_bytes(B.hw, c.meta_cap);
        int occ = B.smem <= smem_optin_ ? std::min(ctas_resident(tick_kernel<false, false>, c.block, B.smem),
                                                   ctas_resident(tick_kernel<false, true>, c.block, B.smem))
                                        : 0;
        if (ctas_cap_ > 0) occ = std::min(occ, ctas_cap_);
        B.grid = std::min(B.units(), sms_ * occ);
    } else {
        B.smem = tick_smem_bytes(B.hw, c.meta_cap);
        int occ = B.smem <= smem_optin_ ? std::min(ctas_resident(tick_kernel_list<false>, c.block, B.smem),
                                                   ctas_resident(tick_kernel_list<true>, c.block, B.smem))
                                        : 0;
        if (ctas_cap_ > 0) occ = std::min(occ, ctas_cap_);
        B.grid = std::min(B.units(), sms_ * occ);
    }
    return B.grid > 0;
}

void Engine::set_bucket(int b, const BucketConfig &cfg) {
    if (b < 0 || b >= kBuckets) throw std::runtime_error("Invalid bucket");
    Bucket B = buckets_[b];
    B.cfg = cfg;
    if (!shape_bucket(B)) throw std::runtime_error("Bucket configuration cannot run on this device");
    NSB_CHECK(cudaDeviceSynchronize());
    buckets_[b] = B;
    drop_graphs();
}

void Engine::drop_graphs() {
    for (auto &g : graphs_) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
}

Pools Engine::pools(bool events) const {
    Pools P;
    P.ngene = reinterpret_cast<const float4 *>(d_ngene_); P.nflags = d_nflags_; P.nsens = d_nsens_;
    P.nxidx = d_nxidx_; P.xgene = d_xgene_; P.xstate = d_xstate_; P.nstate = d_nstate_; P.inptr = d_inptr_;
    P.smeta = d_smeta_; P.sgene = d_sgene_; P.sstate = d_sstate_; P.sarrived = d_sarrived_; P.slastp = d_slastp_;
    P.btick = d_btick_; P.bmotor = d_bmotor_; P.units = d_units_; P.unitb = d_unitb_; P.ubrain = d_ubrain_;
    P.channels = channels_; P.outputs = outputs_; P.hw = hw_;
    P.events = events ? d_events_ : nullptr;
    P.pulse_period = pulse_period_;
    P.pulse_mod = pulse_mod_;
    P.warp_cells = warp_cells_;
    return P;
}

// One bucket's kernel over its units.
void Engine::launch_bucket(const Bucket &B, const Pools &P0, int *queue, const float *d_input, const uint8_t *d_mask,
                           int ticks, float gain, float *d_output, int *d_status, cudaStream_t stream) const {
    Pools P = P0;
    P.hw = B.hw;
    P.meta_cap = B.cfg.meta_cap;
    if (B.heavy)
        tick_kernel<true, false><<<B.grid, B.cfg.block, B.smem, stream>>>(P, B.ub, B.ue, queue, d_input, d_mask,
                                                                           d_output, d_status, ticks, gain);
    else if (B.cfg.cluster > 1)
        launch_cluster(B.cfg.coop != 0, B.cfg.cluster, B.grid, B.cfg.block, B.smem, stream, P, B.ub, B.ue, queue,
                       d_input, d_mask, d_output, d_status, ticks, gain);
    else if (!B.cfg.list && B.cfg.coop)
        tick_kernel<false, true><<<B.grid, B.cfg.block, B.smem, stream>>>(P, B.ub, B.ue, queue, d_input, d_mask,
                                                                           d_output, d_status, ticks, gain);
    else if (!B.cfg.list)
        tick_kernel<false, false><<<B.grid, B.cfg.block, B.smem, stream>>>(P, B.ub, B.ue, queue, d_input, d_mask,
                                                                            d_output, d_status, ticks, gain);
    else
        launch_light(B.cfg.coop != 0, B.grid, B.cfg.block, B.smem, stream, P, B.ub, B.ue, queue, d_input, d_mask,
                     d_output, d_status, ticks, gain);
}

// Every bucket of a step, each on its own stream so that the buckets run
// side by side: the big-brain and heavy buckets are launched first, the
// packed bucket (on the caller's stream) fills the rest of the GPU.
// queue: 8 counters, zeroed here.
void Engine::launch_groups(const Pools &P, int *queue, const float *d_input, const uint8_t *d_mask, int ticks,
                           float gain, float *d_output, int *d_status, cudaStream_t stream) {
    NSB_CHECK(cudaMemsetAsync(queue, 0, 8 * sizeof(int), stream));
    int active = 0;
    for (const Bucket &B : buckets_) active += B.units() > 0;
    bool forked[kBuckets] = {};
    if (active > 1) NSB_CHECK(cudaEventRecord(fork_, stream));
    for (int b = 0; b < kBuckets; ++b) {
        const Bucket &B = buckets_[b];
        if (!B.units() || (active > 1 && b == kBucketPacked)) continue;
        cudaStream_t s = stream;
        if (active > 1) {
            s = bstream_[b];
            NSB_CHECK(cudaStreamWaitEvent(s, fork_, 0));
            forked[b] = true;
        }
        launch_bucket(B, P, queue + b, d_input, d_mask, ticks, gain, d_output, d_status, s);
        if (forked[b]) NSB_CHECK(cudaEventRecord(join_[b], s));
    }
    if (active > 1 && buckets_[kBucketPacked].units())
        launch_bucket(buckets_[kBucketPacked], P, queue + kBucketPacked, d_input, d_mask, ticks, gain, d_output,
                      d_status, stream);
    for (int b = 0; b < kBuckets; ++b)
        if (forked[b]) NSB_CHECK(cudaStreamWaitEvent(stream, join_[b], 0));
    NSB_CHECK(cudaGetLastError());
}

void Engine::launch(const float *d_input, const uint8_t *d_mask, int ticks, float gain, float *d_output,
                    int *d_status, cudaStream_t stream) {
    launch_groups(pools(count_events_), d_queue_, d_input, d_mask, ticks, gain, d_output, d_status, stream);
}

// ---- allocation-free step ----------------------------------------------------
// For callers that may not allocate device memory when they step: processes
// whose device memory all belongs to another allocator (a host application's
// memory pool, a framework that owns the GPU heap) or that run under a
// no-allocation rule once started. The tick kernel's scratch memory — the
// work-queue counters and the per-synapse record of the last tick at which
// plasticity was applied — comes from this file-scope array instead of
// engine-allocated buffers. Every GPU that loads this library holds the array
// (256 B + 2 B x kNoAllocMaxSynapses = 4 MiB + 256 B) until the process exits.
constexpr int kNoAllocMaxSynapses = 2097152;
constexpr size_t kNoAllocScratchBytes = 256 + sizeof(int16_t) * (size_t)kNoAllocMaxSynapses;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device, looked up once
// per device and kept for the life of the process (the host-side name is only
// a stand-in for the device array). The cache assumes the device's primary
// context lives as long: after a cudaDeviceReset the address would be stale.
static unsigned char *noalloc_scratch_address() {
    static std::mutex lock;
    static unsigned char *addr[64] = {};
    int dev = 0;
    NSB_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("Device index outside the scratch table");
    std::lock_guard<std::mutex> guard(lock);
    if (!addr[dev]) {
        void *ptr = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (rc != cudaSuccess)
            throw std::runtime_error(std::string("CUDA: scratch address lookup failed: ") + cudaGetErrorString(rc));
        addr[dev] = static_cast<unsigned char *>(ptr);
    }
    return addr[dev];
}

void Engine::step_noalloc(const float *d_input, const uint8_t *d_mask, int ticks, float gain, float *d_output,
                          int *d_status, cudaStream_t stream) {
    if (ticks < 1 || ticks > 10000 || !std::isfinite(gain) || gain < 0)
        throw std::runtime_error("Invalid neural integration interval");
    if (n_synapses_ > kNoAllocMaxSynapses)
        throw std::runtime_error("Batch has " + std::to_string(n_synapses_) +
                                 " synapses; the allocation-free step supports at most 2097152");
    unsigned char *scratch = noalloc_scratch_address();
    int *queue = reinterpret_cast<int *>(scratch);
    int16_t *lastp = reinterpret_cast<int16_t *>(scratch + 256);
    cudaStream_t s = stream ? stream : stream_;
    // The array keeps the previous call's contents: the plasticity
    // bookkeeping is reset to -1 ("none this call") here, the queue counters
    // to 0 by launch_groups.
    // (launch_groups clears its eight queue counters at the start of the array.)
    NSB_CHECK(cudaMemsetAsync(lastp, 0xff, sizeof(int16_t) * (size_t)std::max(n_synapses_, 1), s));
    // Arrivals are counted into the engine's existing counter (no allocation).
    Pools P = pools(count_events_);
    P.slastp = lastp;
    launch_groups(P, queue, d_input, d_mask, ticks, gain, d_output, d_status, s);
}

void Engine::step_device(const float *d_input, const uint8_t *d_mask, int ticks, float gain, float *d_output,
                         int *d_status, cudaStream_t stream) {
    if (ticks < 1 || ticks > 10000 || !std::isfinite(gain) || gain < 0)
        throw std::runtime_error("Invalid neural integration interval");
    launch(d_input, d_mask, ticks, gain, d_output, d_status, stream ? stream : stream_);
}

void Engine::step_host(const float *input, const uint8_t *mask, int ticks, float gain, float *output, int *status) {
    if (ticks < 1 || ticks > 10000 || !std::isfinite(gain) || gain < 0)
        throw std::runtime_error("Invalid neural integration interval");
    // An observation outside [0, 1] is invalid; NaN and the infinities fail
    // one of the two comparisons. The row test has no branch, so it vectorises.
    for (int i = 0; i < n_brains_; ++i) {
        if (!mask[i]) continue;
        const float *row = input + (size_t)i * channels_;
        bool ok = true;
        for (int j = 0; j < channels_; ++j) ok &= (row[j] >= 0.0f) & (row[j] <= 1.0f);
        if (!ok) throw std::runtime_error("Invalid encoded observation");
    }
    NSB_CHECK(cudaMemcpyAsync(d_input_, input, (size_t)n_brains_ * channels_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
    NSB_CHECK(cudaMemcpyAsync(d_mask_, mask, n_brains_, cudaMemcpyHostToDevice, stream_));
    step_graph(ticks, gain, stream_);          // the step's launches, replayed from the captured graph
    NSB_CHECK(cudaMemcpyAsync(output, d_output_, (size_t)n_brains_ * outputs_ * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    NSB_CHECK(cudaMemcpyAsync(status, d_status_, n_brains_ * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    NSB_CHECK(cudaStreamSynchronize(stream_));
    for (int i = 0; i < n_brains_; ++i)
        if (mask[i] && status[i] != -2) h_tick_[i] += ticks;
}

void Engine::set_global_modulation(int period, uint32_t mod) {
    if (period < 0 || mod > 7u) throw std::runtime_error("Invalid modulator pulse");
    NSB_CHECK(cudaDeviceSynchronize());
    drop_graphs();
    pulse_period_ = mod ? period : 0;
    pulse_mod_ = period ? mod : 0u;
}

void Engine::set_cooperative(bool coop) {
    NSB_CHECK(cudaStreamSynchronize(stream_));
    NSB_CHECK(cudaDeviceSynchronize());
    for (int b = 0; b < kBuckets; ++b)
        if (!buckets_[b].heavy) buckets_[b].cfg.coop = coop ? 1 : 0;
    coop_ = coop;
    drop_graphs();
}

bool Engine::autotune(int ticks, float gain, cudaStream_t stream) {
    if (ticks < 1 || ticks > 10000 || !std::isfinite(gain) || gain < 0)
        throw std::runtime_error("Invalid neural integration interval");
    if (n_light_units_ == 0) return cooperative();
    cudaStream_t s = stream ? stream : stream_;
    NSB_CHECK(cudaDeviceSynchronize());
    // Back up everything a step writes.
    struct Buf { void *dev; size_t bytes; void *copy; };
    std::vector<Buf> bufs = {
        {d_nstate_, (size_t)n_neurons_ * S_WORDS * 4, nullptr},
        {d_sstate_, (size_t)n_synapses_ * Z_WORDS * 4, nullptr},
        {d_sarrived_, (size_t)n_synapses_, nullptr},
        {d_slastp_, (size_t)n_synapses_ * 2, nullptr},
        {d_xstate_, (size_t)std::max(n_heavy_, 1) * 16 * 4, nullptr},
        {d_btick_, (size_t)n_brains_ * 8, nullptr},
        {d_output_, (size_t)n_brains_ * outputs_ * 4, nullptr},
        {d_status_, (size_t)n_brains_ * 4, nullptr},
        {d_events_, 8, nullptr},
    };
    for (auto &b : bufs) {
        if (b.bytes == 0) continue;
        NSB_CHECK(cudaMalloc(&b.copy, b.bytes));
        NSB_CHECK(cudaMemcpyAsync(b.copy, b.dev, b.bytes, cudaMemcpyDeviceToDevice, s));
    }
    auto restore = [&]() {
        for (auto &b : bufs)
            if (b.copy) NSB_CHECK(cudaMemcpyAsync(b.dev, b.copy, b.bytes, cudaMemcpyDeviceToDevice, s));
    };
    cudaEvent_t e0, e1;
    NSB_CHECK(cudaEventCreate(&e0));
    NSB_CHECK(cudaEventCreate(&e1));
    const Pools P = pools(count_events_);
    // Times a bucket alone: one warm-up launch and three timed ones from the
    // same restored state for every candidate.
    // Times whole steps (every bucket, side by side, as a real step runs):
    // one warm-up step and three timed ones from the same restored state.
    auto time_step = [&]() {
        restore();
        for (int k = 0; k < 4; ++k) {
            if (k == 1) NSB_CHECK(cudaEventRecord(e0, s));
            launch_groups(P, d_queue_, d_input_, d_mask_, ticks, gain, d_output_, d_status_, s);
        }
        NSB_CHECK(cudaEventRecord(e1, s));
        NSB_CHECK(cudaEventSynchronize(e1));
        NSB_CHECK(cudaGetLastError());
        float ms = 0;
        NSB_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        return ms;
    };
    // Coordinate descent: one bucket at a time (the packed bucket first, then
    // the big-brain buckets), each candidate timed in the whole step, kept
    // when it saves more than 1 %; at most two passes.
    float best_ms = time_step();
    // First the whole-batch switches: every light bucket on per-thread
    // integration, and every big-brain bucket on one CTA per brain (a
    // descent one bucket at a time can stop short of these).
    for (int sw = 0; sw < 2; ++sw) {
        const std::vector<Bucket> saved = buckets_;
        bool ok = true, any = false;
        for (int b = 0; b < kBuckets && ok; ++b) {
            Bucket &B = buckets_[b];
            if (B.heavy || B.units() == 0) continue;
            if (sw == 0 && B.cfg.list) { B.cfg.list = 0; B.cfg.cluster = 1; any = true; }
            if (sw == 1 && B.cfg.cluster > 1) { B.cfg.cluster = 1; any = true; }
            ok = shape_bucket(B);
        }
        if (!any || !ok) { buckets_ = saved; continue; }
        const float ms = time_step();
        if (ms < 0.99f * best_ms) best_ms = ms;
        else buckets_ = saved;
    }
    const int order[4] = {kBucketPacked, 2, 1, 0};
    for (int pass = 0; pass < 2; ++pass) {
        bool changed = false;
        for (int b : order) {
            Bucket &cur = buckets_[b];
            if (cur.heavy || cur.units() == 0) continue;
            // staging depths: the default, and exactly the bucket's largest
            // unit (less shared memory per CTA, or no global meta reads)
            std::vector<int> caps = {kMetaCap};
            const int fit = std::min((cur.max_synapses + 31) & ~31, 32768);
            if (fit != kMetaCap) caps.push_back(fit);
            std::vector<BucketConfig> cands;
            for (int block : {256, 128})
                for (int coop : {0, 1})
                    for (int cap : caps) {
                        cands.push_back(BucketConfig{block, coop, 1, cap, 1});
                        cands.push_back(BucketConfig{block, coop, 1, cap, 0});
                        if (cur.cluster_size > 1) cands.push_back(BucketConfig{block, coop, cur.cluster_size, cap, 1});
                    }
            for (const BucketConfig &c : cands) {
                if (c.block == cur.cfg.block && c.coop == cur.cfg.coop && c.cluster == cur.cfg.cluster &&
                    c.meta_cap == cur.cfg.meta_cap && c.list == cur.cfg.list)
                    continue;
                const Bucket saved = cur;
                cur.cfg = c;
                if (!shape_bucket(cur)) { cur = saved; continue; }
                const float ms = time_step();
                if (ms < 0.99f * best_ms) { best_ms = ms; changed = true; }
                else cur = saved;
            }
        }
        if (!changed) break;
    }
    restore();
    NSB_CHECK(cudaStreamSynchronize(s));
    for (auto &b : bufs)
        if (b.copy) cudaFree(b.copy);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    coop_ = cooperative();
    drop_graphs();
    return coop_;
}

void Engine::step_graph(int ticks, float gain, cudaStream_t stream) {
    if (ticks < 1 || ticks > 10000 || !std::isfinite(gain) || gain < 0)
        throw std::runtime_error("Invalid neural integration interval");
    cudaStream_t s = stream ? stream : stream_;
    for (auto &g : graphs_)
        if (g.ticks == ticks && g.gain == gain) {
            NSB_CHECK(cudaGraphLaunch(g.exec, s));
            return;
        }
    cudaGraph_t graph;
    NSB_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    launch(d_input_, d_mask_, ticks, gain, d_output_, d_status_, s);
    NSB_CHECK(cudaStreamEndCapture(s, &graph));
    cudaGraphExec_t exec;
    NSB_CHECK(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    graphs_.push_back({ticks, gain, exec});
    NSB_CHECK(cudaGraphLaunch(exec, s));
}

void Engine::reset_host(const uint8_t *mask, const uint32_t *seeds) {
    NSB_CHECK(cudaMemcpyAsync(d_rmask_, mask, n_brains_, cudaMemcpyHostToDevice, stream_));
    NSB_CHECK(cudaMemcpyAsync(d_seeds_, seeds, n_brains_ * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_));
    const Pools P = pools(false);
    reset_neurons<<<sms_ * 8, 256, 0, stream_>>>(P, d_nbrain_, d_norig_, d_rmask_, d_seeds_, n_neurons_);
    if (n_synapses_) reset_synapses<<<sms_ * 8, 256, 0, stream_>>>(P, d_sbrain_, d_sorig_, d_rmask_, d_seeds_, n_synapses_);
    reset_ticks<<<(n_brains_ + 255) / 256, 256, 0, stream_>>>(d_btick_, d_rmask_, n_brains_);
    NSB_CHECK(cudaGetLastError());
    NSB_CHECK(cudaStreamSynchronize(stream_));
    for (int i = 0; i < n_brains_; ++i)
        if (mask[i]) h_tick_[i] = 0;
}

void Engine::set_tick(int brain, int64_t tick) {
    if (brain < 0 || brain >= n_brains_) throw std::runtime_error("Invalid brain index");
    NSB_CHECK(cudaStreamSynchronize(stream_));
    NSB_CHECK(cudaMemcpy(d_btick_ + brain, &tick, 8, cudaMemcpyHostToDevice));
    h_tick_[brain] = tick;
}

unsigned long long Engine::take_events() {
    unsigned long long v = 0;
    NSB_CHECK(cudaDeviceSynchronize());
    NSB_CHECK(cudaMemcpy(&v, d_events_, 8, cudaMemcpyDeviceToHost));
    NSB_CHECK(cudaMemset(d_events_, 0, 8));
    return v;
}

void Engine::dump(int brain, uint32_t *nw, uint32_t *sw, int64_t *tick) {
    if (brain < 0 || brain >= n_brains_) throw std::runtime_error("Invalid brain index");
    NSB_CHECK(cudaDeviceSynchronize());
    const int4 U = h_units_[h_bunit_[brain]];
    const int un0 = U.x, unn = U.y, ue0 = U.z, une = U.w;
    const int nn = h_noff_[brain + 1] - h_noff_[brain], ne = h_soff_[brain + 1] - h_soff_[brain];
    std::vector<uint32_t> rec((size_t)unn * S_WORDS), srec((size_t)std::max(une, 1) * Z_WORDS);
    std::vector<uint8_t> arr(std::max(une, 1));
    int64_t t = 0;
    NSB_CHECK(cudaMemcpy(rec.data(), d_nstate_ + (size_t)un0 * S_WORDS, rec.size() * 4, cudaMemcpyDeviceToHost));
    if (une) {
        NSB_CHECK(cudaMemcpy(srec.data(), d_sstate_ + (size_t)ue0 * Z_WORDS, (size_t)une * Z_WORDS * 4, cudaMemcpyDeviceToHost));
        NSB_CHECK(cudaMemcpy(arr.data(), d_sarrived_ + ue0, une, cudaMemcpyDeviceToHost));
    }
    NSB_CHECK(cudaMemcpy(&t, d_btick_ + brain, 8, cudaMemcpyDeviceToHost));
    if (tick) *tick = t;
    if (nw) {
        for (int j = 0; j < nn; ++j) {
            const int n = h_npos_[h_noff_[brain] + j];
            const uint32_t *r = &rec[(size_t)(n - un0) * S_WORDS];
            uint32_t *o = nw + (size_t)j * kDumpNeuronWords;
            std::memset(o, 0, kDumpNeuronWords * 4);
            o[0] = r[S_V]; o[1] = r[S_W]; o[2] = r[S_ADP]; o[3] = r[S_INH]; o[4] = r[S_DEPOL]; o[5] = r[S_LOGAMPA];
            o[6] = r[S_D0]; o[7] = r[S_D1]; o[8] = r[S_D2]; o[9] = r[S_D3];
            const int xi = h_nxidx_[n];
            if (xi >= 0) NSB_CHECK(cudaMemcpy(o + 10, d_xstate_ + (size_t)xi * 16, 64, cudaMemcpyDeviceToHost));
            o[26] = r[S_TOTAL]; o[27] = r[S_SPIKE]; o[28] = r[S_RECNS]; o[29] = r[S_RECRNG];
            uint32_t h = 0;
            for (int k = 0; k < max_delay_ && k < 31; ++k) {
                const int64_t tau = t - 1 - k;
                if (tau < 0) break;
                if ((r[S_HIST] >> (tau & 31)) & 1u) h |= 1u << k;
            }
            o[30] = h;
        }
    }
    if (sw) {
        for (int j = 0; j < ne; ++j) {
            const int e = h_spos_[h_soff_[brain] + j] - ue0;
            const uint32_t *z = &srec[(size_t)e * Z_WORDS];
            uint32_t *o = sw + (size_t)j * kDumpSynapseWords;
            std::memset(o, 0, kDumpSynapseWords * 4);
            for (int k = 0; k < 11; ++k) o[k] = z[k];   // w .. post_age share the order
            const int64_t last = (int32_t)z[Z_LAST];
            o[11] = (uint32_t)(uint64_t)last; o[12] = (uint32_t)((uint64_t)last >> 32);
            o[13] = z[Z_READYLO]; o[14] = z[Z_READYHI]; o[15] = z[Z_RNG]; o[16] = arr[e]; o[17] = z[Z_SLOW];
        }
    }
}

void Engine::export_state(int brain, ref::NeuronState *neurons, ref::SynapseState *synapses,
                          unsigned char (*history)[9], int64_t *tick_out) {
    if (brain < 0 || brain >= n_brains_) throw std::runtime_error("Invalid brain index");
    NSB_CHECK(cudaDeviceSynchronize());
    const int4 U = h_units_[h_bunit_[brain]];
    const int un0 = U.x, unn = U.y, ue0 = U.z, une = U.w;
    const int nn = h_noff_[brain + 1] - h_noff_[brain], ne = h_soff_[brain + 1] - h_soff_[brain];
    std::vector<uint32_t> rec((size_t)unn * S_WORDS), srec((size_t)std::max(une, 1) * Z_WORDS);
    std::vector<uint8_t> arr(std::max(une, 1));
    int64_t tick = 0;
    NSB_CHECK(cudaMemcpy(rec.data(), d_nstate_ + (size_t)un0 * S_WORDS, rec.size() * 4, cudaMemcpyDeviceToHost));
    if (une) {
        NSB_CHECK(cudaMemcpy(srec.data(), d_sstate_ + (size_t)ue0 * Z_WORDS, (size_t)une * Z_WORDS * 4, cudaMemcpyDeviceToHost));
        NSB_CHECK(cudaMemcpy(arr.data(), d_sarrived_ + ue0, une, cudaMemcpyDeviceToHost));
    }
    NSB_CHECK(cudaMemcpy(&tick, d_btick_ + brain, 8, cudaMemcpyDeviceToHost));
    auto uf = [](uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; };
    for (int j = 0; j < nn; ++j) {
        const int n = h_npos_[h_noff_[brain] + j];
        const uint32_t *r = &rec[(size_t)(n - un0) * S_WORDS];
        ref::NeuronState s;
        std::memset(&s, 0, sizeof s);
        s.v = uf(r[S_V]); s.w = uf(r[S_W]); s.adp = uf(r[S_ADP]); s.inh = uf(r[S_INH]); s.depol = uf(r[S_DEPOL]);
        s.log_ampa = uf(r[S_LOGAMPA]); s.rec_ns = uf(r[S_RECNS]); s.rec_rng = r[S_RECRNG];
        s.dend[0] = uf(r[S_D0]); s.dend[1] = uf(r[S_D1]); s.dend[2] = uf(r[S_D2]); s.dend[3] = uf(r[S_D3]);
        s.total = (int)r[S_TOTAL]; s.spike = (unsigned char)r[S_SPIKE];
        const int xi = h_nxidx_[n];
        if (xi >= 0) NSB_CHECK(cudaMemcpy(s.cell, d_xstate_ + (size_t)xi * 16, 64, cudaMemcpyDeviceToHost));
        neurons[j] = s;
        if (history) {
            std::memset(history[j], 0, 9);
            for (int k = 1; k <= 9; ++k) {
                const int64_t tau = tick - k;
                if (tau < 0) break;
                history[j][tau % 9] = (unsigned char)((r[S_HIST] >> (tau & 31)) & 1u);
            }
        }
    }
    for (int j = 0; j < ne; ++j) {
        const int e = h_spos_[h_soff_[brain] + j] - ue0;
        const uint32_t *z = &srec[(size_t)e * Z_WORDS];
        ref::SynapseState s;
        std::memset(&s, 0, sizeof s);
        s.w = uf(z[Z_W]); s.ru = uf(z[Z_RU]); s.pre_tr = uf(z[Z_PRETR]); s.post_tr = uf(z[Z_POSTTR]);
        s.eltp = uf(z[Z_ELTP]); s.eltd = uf(z[Z_ELTD]); s.da_age = uf(z[Z_DAAGE]); s.spine = uf(z[Z_SPINE]);
        s.st_age = uf(z[Z_STAGE]); s.pre_age = uf(z[Z_PREAGE]); s.post_age = uf(z[Z_POSTAGE]);
        s.last = (int64_t)(int32_t)z[Z_LAST];
        s.ready = ((uint64_t)z[Z_READYHI] << 32) | z[Z_READYLO];
        s.rng = z[Z_RNG];
        s.arrived = arr[e];
        s.slow = uf(z[Z_SLOW]);
        synapses[j] = s;
    }
    if (tick_out) *tick_out = tick;
}

void Engine::load_state(int brain, const ref::NeuronState *neurons, const ref::SynapseState *synapses,
                        const unsigned char (*history)[9], int64_t tick) {
    if (brain < 0 || brain >= n_brains_) throw std::runtime_error("Invalid brain index");
    if (tick < 0 || tick >= 2147483647ll) throw std::runtime_error("Tick outside the engine range");
    NSB_CHECK(cudaDeviceSynchronize());
    const int4 U = h_units_[h_bunit_[brain]];
    const int un0 = U.x, unn = U.y, ue0 = U.z, une = U.w;
    const int nn = h_noff_[brain + 1] - h_noff_[brain], ne = h_soff_[brain + 1] - h_soff_[brain];
    std::vector<uint32_t> rec((size_t)unn * S_WORDS), srec((size_t)std::max(une, 1) * Z_WORDS);
    std::vector<uint8_t> arr(std::max(une, 1));
    NSB_CHECK(cudaMemcpy(rec.data(), d_nstate_ + (size_t)un0 * S_WORDS, rec.size() * 4, cudaMemcpyDeviceToHost));
    if (une) {
        NSB_CHECK(cudaMemcpy(srec.data(), d_sstate_ + (size_t)ue0 * Z_WORDS, (size_t)une * Z_WORDS * 4, cudaMemcpyDeviceToHost));
        NSB_CHECK(cudaMemcpy(arr.data(), d_sarrived_ + ue0, une, cudaMemcpyDeviceToHost));
    }
    auto fw = [](float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; };
    for (int j = 0; j < nn; ++j) {
        const ref::NeuronState &s = neurons[j];
        const int n = h_npos_[h_noff_[brain] + j];
        uint32_t *r = &rec[(size_t)(n - un0) * S_WORDS];
        std::memset(r, 0, S_WORDS * 4);
        r[S_V] = fw(s.v); r[S_W] = fw(s.w); r[S_ADP] = fw(s.adp); r[S_INH] = fw(s.inh); r[S_DEPOL] = fw(s.depol);
        r[S_LOGAMPA] = fw(s.log_ampa); r[S_RECNS] = fw(s.rec_ns); r[S_RECRNG] = s.rec_rng;
        r[S_D0] = fw(s.dend[0]); r[S_D1] = fw(s.dend[1]); r[S_D2] = fw(s.dend[2]); r[S_D3] = fw(s.dend[3]);
        r[S_TOTAL] = (uint32_t)s.total; r[S_SPIKE] = s.spike;
        uint32_t h = 0;
        if (history)
            for (int k = 1; k <= 9; ++k) {
                const int64_t tau = tick - k;
                if (tau < 0) break;
                if (history[j][tau % 9]) h |= 1u << (tau & 31);
            }
        r[S_HIST] = h;
        const int xi = h_nxidx_[n];
        if (xi >= 0) NSB_CHECK(cudaMemcpy(d_xstate_ + (size_t)xi * 16, s.cell, 64, cudaMemcpyHostToDevice));
    }
    for (int j = 0; j < ne; ++j) {
        const ref::SynapseState &s = synapses[j];
        const int e = h_spos_[h_soff_[brain] + j] - ue0;
        uint32_t *z = &srec[(size_t)e * Z_WORDS];
        const float f[11] = {s.w, s.ru, s.pre_tr, s.post_tr, s.eltp, s.eltd, s.da_age, s.spine, s.st_age, s.pre_age, s.post_age};
        for (int k = 0; k < 11; ++k) z[k] = fw(f[k]);
        z[Z_SLOW] = fw(s.slow);
        z[Z_READYLO] = (uint32_t)s.ready; z[Z_READYHI] = (uint32_t)(s.ready >> 32);
        z[Z_RNG] = s.rng;
        const int64_t last = s.last < -1000000 ? -1000000 : s.last;
        if (last >= 2147483647ll) throw std::runtime_error("Last arrival outside the engine range");
        z[Z_LAST] = (uint32_t)(int32_t)last;
        arr[e] = s.arrived;
    }
    NSB_CHECK(cudaMemcpy(d_nstate_ + (size_t)un0 * S_WORDS, rec.data(), rec.size() * 4, cudaMemcpyHostToDevice));
    if (une) {
        NSB_CHECK(cudaMemcpy(d_sstate_ + (size_t)ue0 * Z_WORDS, srec.data(), (size_t)une * Z_WORDS * 4, cudaMemcpyHostToDevice));
        NSB_CHECK(cudaMemcpy(d_sarrived_ + ue0, arr.data(), une, cudaMemcpyHostToDevice));
    }
    NSB_CHECK(cudaMemcpy(d_btick_ + brain, &tick, 8, cudaMemcpyHostToDevice));
    h_tick_[brain] = tick;
}

}  // namespace nsb
