// World neural stage on the world simulator's own pools (CUDA, sm_100a).
//
// Replaces the neural part of the reference world loop
// (mixic/neural-selection src/main.cu:2634-2728: CUB slot selection, a
// device-to-host count read, then 16 ticks of synapse_delivery /
// synapse_plasticity_delivery / neuron_step / synapse_plasticity, or the
// brain_block_step tiers) and its homeostasis launches (2751-2758). It reads
// and writes the simulator's Device pools in place, in the reference record
// layouts (ns_refabi.h), with the semantics of src/main.cu:659-801.
//
// Design:
//  * Device-resident compiled brains. An animal's neuron and synapse lists are
//    fixed from birth to death (built by init_animals / reproduce, released
//    by release_genome, src/main.cu:413-452). The first step after a birth
//    compiles the animal once, on the device (world_compile: list walk, slot
//    sort, owner/activity checks, a stable CSR of live synapses by
//    post-synaptic neuron), into an arena keyed by (animal slot, animal id).
//    Later steps read the compiled CSR with coalesced loads. Selection is a
//    list of living animals that CTAs claim a few at a time: no CUB pass, no
//    host round trip inside the step.
//  * A tick runs in five barrier-separated phases over a unit: arrival test
//    of every live synapse against the 9-tick spike-history ring; release of
//    the arriving synapses from a compacted event list; per post-synaptic
//    neuron (one thread each), the arriving inputs summed in list order (the
//    per-branch sums of src/main.cu:680-690 in a fixed order instead of float
//    atomics) and the integration; compaction of plasticity events; their
//    plasticity, quiet ticks since the last update replayed exactly.
//  * Small animals are packed into units of up to 256 neurons (one CTA,
//    neuron genes, ring and CSR in shared memory, neuron state in registers);
//    larger animals run one per CTA, largest first, with their per-neuron
//    arrays in a global scratch slab and the CSR read in place from the
//    arena. Animals with LP, Prinz or LFS cells run in separate heavy builds
//    of both kernels, so the light builds keep a small register budget.
//  * Synapse state stays in the SynapseState records and is updated in place
//    only when a synapse releases or its plasticity catches up.
// Arithmetic is the engine's (ns_physio.cuh): bit-identical to the oracle.
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ns_b200.h"
#include "ns_internal.h"
#include "ns_physio.cuh"
#include "ns_refabi.h"

namespace nsb {
void set_error(const char *message);   // ns_abi.cu

namespace {

constexpr int kS = 19, kM = 5, kHist = 9, kTicks = 16, kContact = 16;
#ifndef NSB_WORLD_BLOCK
#define NSB_WORLD_BLOCK 256
#endif
#ifndef NSB_WORLD_EDGES
#define NSB_WORLD_EDGES 2048
#endif
constexpr int kBlock = NSB_WORLD_BLOCK;      // small units: one thread per neuron
constexpr int kUnitEdges = NSB_WORLD_EDGES;  // live synapses of a small unit (shared memory)
constexpr int kUnitAnimals = 32;
constexpr int kBigBlock = 256;
constexpr int kBigClasses = 4;       // big animals by size: above 2,048, 1,024, 512 neurons, the rest
constexpr int kCompileWarps = 4;     // compile kernel: warps per CTA, one animal per warp at a time

// World neuron flags: bits 0-11 as the engine's NF_* (type, active,
// inhibitory, modulator, gene sensory channel, ADP), plus:
enum : uint32_t {
    WF_MOTOR_SHIFT = 12,      // bits 12-14: motor index + 1 (port 19..23), 0 otherwise
    WF_RECEPTOR = 1u << 15,   // type 5 on a receptor channel (< 6): receptor events
    WF_SENSE = 1u << 16,      // reads a world sense channel (0..18)
    WF_TRACED = 1u << 17,     // motor neuron of the traced animal
};
// Step status bits (reported by the host as errors).
enum : int { ST_LIST = 1, ST_SIZE = 2, ST_GENE = 4, ST_ARENA = 8 };
// Unit animal flags.
enum : int { UA_FROZEN = 1, UA_TRACED = 2 };

struct WorldArgs {
    const ref::Animal *animals;
    const ref::PlasticityCohort *cohort;
    const ref::NeuronGene *ngene;
    const ref::SynapseGene *sgene;
    ref::NeuronState *nstate;
    ref::SynapseState *sstate;
    float *pexc, *pinh;
    const float *senses;
    unsigned long long *modtick;
    unsigned char *hist;
    const int *nowner, *sowner, *nnext, *snext, *nport;
    int *motors;
    int *tr_ea, *tr_er, *tr_ia;
    float *tr_en, *tr_in, *tr_pk;
    int trace, sil_senses, sil_contact;
    int P, ncap, ecap;
    int warp_cells;    // LP and Prinz cells per warp, on average, up to which heavy_cells_cta uses whole warps
};

// Compiled-brain cache, one entry per animal slot. Region layout at arena +
// off (ints): nslot[nn] (list order), inptr[nn + 1] (animal-local CSR
// offsets), cmeta[nl], cslot[nl] (live synapses grouped by post-synaptic
// neuron, list order within a neuron).
struct Cache {
    int *id, *nn, *ne, *nl, *off, *cap;
    int *hv;           // 1: the animal has an active LP, Prinz or LFS cell
    int *arena;
    long long arena_cap;
    unsigned long long *bump;
};

// Per-warp compile scratch.
struct Scratch {
    int *elist;        // max_e (list order synapse slots)
    uint32_t *tmeta;   // max_e
    int *tpost;        // max_e (-1: not live)
    int *skey, *sval;  // pow2(max_n) sorted (slot, local)
    int *cnt;          // max_n
    int max_n, max_e, pow2n;
};

struct Counters {
    unsigned long long animals, neurons, synapses, events;
};

__device__ __forceinline__ bool frozen_animal(const WorldArgs &d, int a) {
    if (!d.cohort || a < 0) return false;
    const ref::PlasticityCohort &r = d.cohort[a];
    return r.assigned && r.frozen && r.id == d.animals[a].id;
}
__device__ __forceinline__ bool exc_type(uint32_t t) { return t == 0 || t == 4 || t == 5; }

__device__ __forceinline__ bool compiled(const WorldArgs &d, const Cache &c, int a) {
    const ref::Animal &A = d.animals[a];
    return c.id[a] == A.id && c.nn[a] == A.neuron_count && c.ne[a] == A.synapse_count && c.off[a] >= 0;
}

// ---- selection: animals whose compiled brain is missing or stale --------------
// Also lists every living animal (order irrelevant: animals do not interact
// within the neural stage).
__global__ void world_select(WorldArgs d, Cache c, int *list, int *count, int *alive, int *nalive) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < d.P; a += gridDim.x * blockDim.x) {
        if (d.animals[a].alive != 1) continue;
        alive[atomicAdd(nalive, 1)] = a;
        if (!compiled(d, c, a)) list[atomicAdd(count, 1)] = a;
    }
}

// ---- compile: one warp per animal ---------------------------------------------------
__device__ int find_slot(const int *key, const int *val, int n2, int slot) {
    int lo = 0, hi = n2;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key[mid] < slot) lo = mid + 1; else hi = mid;
    }
    return lo < n2 && key[lo] == slot ? val[lo] : -1;
}

__device__ void compile_animal(const WorldArgs &d, const Cache &c, const Scratch &s, int a, int lane, int *status) {
    const unsigned FULL = 0xffffffffu;
    const ref::Animal &A = d.animals[a];
    const int nn = A.neuron_count, ne = A.synapse_count;
    if (nn < 0 || ne < 0 || nn > s.max_n || ne > s.max_e) {
        if (lane == 0) atomicOr(status, ST_SIZE);
        return;
    }
    const int need = 2 * nn + 1 + 2 * ne;
    int off = -1, bad = 0;
    if (lane == 0) {
        if (c.off[a] >= 0 && c.cap[a] >= need) {
            off = c.off[a];
        } else {
            const unsigned long long o = atomicAdd(c.bump, (unsigned long long)need);
            if ((long long)(o + need) <= c.arena_cap) {
                off = (int)o;
                c.cap[a] = need;
            }
        }
        if (off < 0) {
            atomicOr(status, ST_ARENA);
        } else {
            c.id[a] = INT_MIN;     // invalid while rewritten
            c.off[a] = off;
            int *nslot = c.arena + off;
            int k = 0;
            for (int q = A.neuron_head; q >= 0 && k <= nn; q = d.nnext[q]) {
                if (q >= d.ncap) { bad = 1; break; }
                if (k < nn) nslot[k] = q;
                ++k;
            }
            if (k != nn) bad = 1;
            k = 0;
            for (int q = A.synapse_head; q >= 0 && k <= ne && !bad; q = d.snext[q]) {
                if (q >= d.ecap) { bad = 1; break; }
                if (k < ne) s.elist[k] = q;
                ++k;
            }
            if (k != ne) bad = 1;
            if (bad) atomicOr(status, ST_LIST);
        }
    }
    off = __shfl_sync(FULL, off, 0);
    bad = __shfl_sync(FULL, bad, 0);
    if (off < 0 || bad) return;
    __syncwarp();
    int *nslot = c.arena + off;
    int *inptr = nslot + nn;
    // sort (slot, local) by slot: bitonic over pow2 >= nn
    int n2 = 1;
    while (n2 < nn) n2 <<= 1;
    for (int i = lane; i < n2; i += 32) {
        s.skey[i] = i < nn ? nslot[i] : INT_MAX;
        s.sval[i] = i < nn ? i : -1;
    }
    for (int i = lane; i < nn; i += 32) s.cnt[i] = 0;
    __syncwarp();
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < n2; i += 32) {
                const int p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const int ki = s.skey[i], kp = s.skey[p];
                    if ((ki > kp) == up) {
                        s.skey[i] = kp; s.skey[p] = ki;
                        const int v = s.sval[i]; s.sval[i] = s.sval[p]; s.sval[p] = v;
                    }
                }
            }
            __syncwarp();
        }
    // synapses: endpoints, liveness, meta, counts per post
    int gbad = 0;
    for (int j = lane; j < ne; j += 32) {
        const ref::SynapseGene &G = d.sgene[s.elist[j]];
        const int lp = (G.pre >= 0 && G.pre < d.ncap) ? find_slot(s.skey, s.sval, n2, G.pre) : -1;
        const int lq = (G.post >= 0 && G.post < d.ncap) ? find_slot(s.skey, s.sval, n2, G.post) : -1;
        bool live = false;
        uint32_t m = 0;
        if (lp >= 0 && lq >= 0 && G.active) {
            const ref::NeuronGene &P = d.ngene[G.pre], &Z = d.ngene[G.post];
            if (P.active && Z.active) {
                live = true;
                if (G.delay < 1 || G.delay > 8 || G.branch > 3 || G.plasticity > 7 || P.modulator > 3) gbad = 1;
                const uint32_t kind = P.modulator ? KIND_MOD : (P.inh_tx ? KIND_INH : KIND_EXC);
                const bool pair = !P.inh_tx && exc_type(P.type) && !P.modulator && !Z.inh_tx && exc_type(Z.type);
                m = (uint32_t)lp | ((uint32_t)G.delay << M_DELAY_SHIFT) | ((uint32_t)(G.branch & 3u) << M_BRANCH_SHIFT) |
                    (kind << M_KIND_SHIFT) | ((uint32_t)((P.modulator ? P.modulator - 1 : 0) & 3u) << M_MODID_SHIFT) |
                    M_LIVE | ((uint32_t)(G.plasticity & 7u) << M_PROF_SHIFT);
                if (G.plasticity && pair) m |= M_PLASTIC;
            }
        }
        s.tmeta[j] = m;
        s.tpost[j] = live ? lq : -1;
        if (live) atomicAdd(&s.cnt[lq], 1);
    }
    if (__any_sync(FULL, gbad)) {
        if (lane == 0) atomicOr(status, ST_GENE);
        return;
    }
    __syncwarp();
    // exclusive scan of counts -> inptr (animal-local)
    int carry = 0;
    for (int base = 0; base < nn; base += 32) {
        const int i = base + lane;
        const int v = i < nn ? s.cnt[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        if (i < nn) { inptr[i] = carry + x - v; s.cnt[i] = carry + x - v; }
        carry += __shfl_sync(FULL, x, 31);
    }
    if (lane == 0) inptr[nn] = carry;
    const int nl = carry;
    int hv = 0;
    for (int k = lane; k < nn; k += 32) {
        const ref::NeuronGene &G = d.ngene[nslot[k]];
        if (G.active && (G.type == 2 || G.type == 3 || G.type == 6)) hv = 1;
    }
    hv = __any_sync(FULL, hv) ? 1 : 0;
    int *cmeta = inptr + nn + 1;
    int *cslot = cmeta + nl;
    __syncwarp();
    // stable placement by post (list order within a neuron)
    for (int base = 0; base < ne; base += 32) {
        const int j = base + lane;
        const int post = j < ne ? s.tpost[j] : -1;
        const int key = post >= 0 ? post : -2 - lane;      // distinct keys for lanes without a live synapse
        const unsigned peers = __match_any_sync(FULL, key);
        if (post >= 0) {
            const int rank = __popc(peers & ((1u << lane) - 1u));
            const int pos = s.cnt[post] + rank;
            cmeta[pos] = (int)s.tmeta[j];
            cslot[pos] = s.elist[j];
        }
        __syncwarp();
        if (post >= 0 && lane == 31 - __clz(peers)) s.cnt[post] += __popc(peers);
        __syncwarp();
    }
    __syncwarp();
    if (lane == 0) {
        c.nn[a] = nn; c.ne[a] = ne; c.nl[a] = nl; c.hv[a] = hv;
        __threadfence();
        c.id[a] = A.id;
    }
}

__global__ void __launch_bounds__(32 * kCompileWarps) world_compile(WorldArgs d, Cache c, const int *list,
                                                                    const int *count, Scratch s, int *status) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kCompileWarps + (threadIdx.x >> 5);
    const int nw = gridDim.x * kCompileWarps;
    Scratch w = s;
    w.elist += (size_t)gw * s.max_e;
    w.tmeta += (size_t)gw * s.max_e;
    w.tpost += (size_t)gw * s.max_e;
    w.skey += (size_t)gw * s.pow2n;
    w.sval += (size_t)gw * s.pow2n;
    w.cnt += (size_t)gw * s.max_n;
    const int n = *count;
    for (int i = gw; i < n; i += nw) compile_animal(d, c, w, list[i], lane, status);
}

// ---- the ticks ------------------------------------------------------------------------
// Per-unit arrays (shared memory for small units, a global slab for big ones).
struct UnitMem {
    float *gene;       // [16][gs] engine gene records, word-major
    int gs;
    uint32_t *nflag;
    float *cur;        // receptor level, or level x 230 pA
    float *scale;      // exp(log AMPA scale) of the post-synaptic neuron
    float *ndepol;     // this tick's recent depolarisation per neuron
    float *rel;        // this tick's released conductance (or weight) per arriving synapse
    float *trx, *tri;  // per-neuron trace sums (traced animal)
    const int *inptr;  // unit CSR offsets
    const uint32_t *cmeta;
    const int *cslot;
    int *ev;           // event list: arrivals, then plasticity events
    int *counters;     // [0] arrivals, [1] plasticity events
    const int *nslot;
    uint16_t *cpost;   // post-synaptic neuron of each synapse (unit-local)
    uint16_t *ring;    // spike history bits: bit k = history slot k
    uint8_t *carr;     // this tick's arrival flag per synapse
    int8_t *clast;     // tick of the synapse's last plasticity update (-1: none this step)
    uint8_t *nspk;     // this tick's spike per neuron
    uint8_t *nmod;     // this tick's modulator bits per neuron
};
constexpr uint32_t WF_FROZEN = 1u << 18;   // the neuron's animal is a frozen plasticity cohort

struct TraceRegs {
    int ea, er, ia;
    float en, in, pk;
};

__device__ __forceinline__ void gene_record(const ref::NeuronGene &G, float *g, int stride, const float *tab) {
    g[G_CAP * stride] = G.cap; g[G_GL * stride] = G.gl; g[G_EL * stride] = G.el; g[G_VT * stride] = G.vt;
    g[G_SLOPE * stride] = G.slope; g[G_A * stride] = G.a; g[G_TAUW * stride] = G.tau_w; g[G_B * stride] = G.b;
    g[G_VR * stride] = G.vr; g[G_ADPB * stride] = G.adp_b;
    g[G_ADPDECAY * stride] = G.adp_tau > 0 ? crexp(-0.25f / G.adp_tau, tab) : 1.0f;
    g[G_GLSLOPE * stride] = G.gl * G.slope;
    g[G_RECBASE * stride] = G.rec_base; g[G_RECGAIN * stride] = G.rec_gain; g[G_RECEVENT * stride] = G.rec_event;
    g[G_RECDECAY * stride] = crexp(-1.0f / G.rec_decay, tab);
}

// Static per-neuron setup for neuron n of animal a (pool slot `slot`); also
// marks the neuron's incoming synapses with their post-synaptic index.
__device__ __forceinline__ void setup_neuron(const WorldArgs &d, const UnitMem &U, int n, int slot, int a,
                                             bool traced, bool frozen, const float *tab) {
    const ref::NeuronGene &G = d.ngene[slot];
    gene_record(G, U.gene + n, U.gs, tab);
    uint32_t f = (uint32_t)(G.type & 7u);
    if (G.active) f |= NF_ACTIVE;
    if (G.inh_tx) f |= NF_INH;
    f |= (uint32_t)(G.modulator & 3u) << NF_MOD_SHIFT;
    if (G.sensory_channel >= 0) f |= NF_GENE_SENS;
    if (G.adp_tau > 0) f |= NF_ADP;
    if (exc_type(G.type)) f |= NF_EXC_TYPE;
    if (frozen) f |= WF_FROZEN;
    const int port = d.nport[slot];
    if (port >= kS && port < kS + kM) {
        f |= (uint32_t)(port - kS + 1) << WF_MOTOR_SHIFT;
        if (traced) f |= WF_TRACED;
    }
    float cur = 0.0f;
    const int ch = G.sensory_channel;
    if (ch >= 0 && ch < kS) {
        f |= WF_SENSE;
        const float level = (d.sil_senses || (d.sil_contact && ch >= kContact)) ? 0.0f
                                                                                 : d.senses[(size_t)a * kS + ch];
        if (G.type == 5 && ch < 6) { f |= WF_RECEPTOR; cur = level; }
        else cur = level * 230.0f;
    }
    U.nflag[n] = f;
    U.cur[n] = cur;
    U.scale[n] = crexp(d.nstate[slot].log_ampa, tab);
    uint16_t r = 0;
    for (int k = 0; k < kHist; ++k)
        if (d.hist[(size_t)k * d.ncap + slot]) r |= (uint16_t)(1u << k);
    U.ring[n] = r;
    U.trx[n] = 0.0f;
    U.tri[n] = 0.0f;
    for (int p = U.inptr[n]; p < U.inptr[n + 1]; ++p) {
        U.cpost[p] = (uint16_t)n;
        U.carr[p] = 0;
        U.clast[p] = -1;
    }
}

__device__ __forceinline__ void load_regs(const ref::NeuronState &S, NeuronRegs &s) {
    s.v = S.v; s.w = S.w; s.adp = S.adp; s.inh = S.inh; s.depol = S.depol; s.rec_ns = S.rec_ns; s.rng = S.rec_rng;
    s.d0 = S.dend[0]; s.d1 = S.dend[1]; s.d2 = S.dend[2]; s.d3 = S.dend[3];
    s.total = S.total; s.spike = S.spike;
}
__device__ __forceinline__ void store_regs(ref::NeuronState &S, const NeuronRegs &s) {
    S.v = s.v; S.w = s.w; S.adp = s.adp; S.inh = s.inh; S.depol = s.depol; S.rec_ns = s.rec_ns; S.rec_rng = s.rng;
    S.dend[0] = s.d0; S.dend[1] = s.d1; S.dend[2] = s.d2; S.dend[3] = s.d3;
    S.total = s.total; S.spike = (unsigned char)s.spike;
}

__device__ __forceinline__ float release_world(const WorldArgs &d, int slot, int64_t tick, const float *tab) {
    const ref::SynapseGene &G = d.sgene[slot];
    ref::SynapseState &Z = d.sstate[slot];
    const int sites = G.sites ? (G.sites > 64 ? 64 : G.sites) : 14;
    float y[8];
    y[Y_W0] = G.w0; y[Y_U] = G.U; y[Y_TREC] = G.trec; y[Y_TFAC] = G.tfac;
    y[Y_SLOWREC] = G.slow_rec; y[Y_SLOWDEPL] = G.slow_depl;
    y[Y_INFO] = __uint_as_float((uint32_t)sites);
    y[Y_PAD] = 0.0f;
    SynReleaseT<int64_t> r;
    r.w = Z.w; r.ru = Z.ru; r.slow = Z.slow; r.ready = Z.ready; r.rng = Z.rng; r.last = Z.last;
    const float v = release(y, r, tick, tab);
    Z.ru = r.ru; Z.slow = r.slow; Z.ready = r.ready; Z.rng = r.rng; Z.last = r.last;
    return v;
}

__device__ __forceinline__ void load_plast_ref(const ref::SynapseState &Z, SynPlast &p) {
    p.w = Z.w; p.pre_tr = Z.pre_tr; p.post_tr = Z.post_tr; p.eltp = Z.eltp; p.eltd = Z.eltd; p.da_age = Z.da_age;
    p.spine = Z.spine; p.st_age = Z.st_age; p.pre_age = Z.pre_age; p.post_age = Z.post_age;
}
__device__ __forceinline__ void store_plast_ref(ref::SynapseState &Z, const SynPlast &p) {
    Z.w = p.w; Z.pre_tr = p.pre_tr; Z.post_tr = p.post_tr; Z.eltp = p.eltp; Z.eltd = p.eltd; Z.da_age = p.da_age;
    Z.spine = p.spine; Z.st_age = p.st_age; Z.pre_age = p.pre_age; Z.post_age = p.post_age;
}

// One tick runs in five barrier-separated phases over the unit:
//   1 arrival test of every live synapse (ring of the source neuron at
//     tick - delay), arriving synapses appended to the event list;
//   2 release of the arriving synapses, one per thread (independent per
//     synapse; inhibitory sources deliver their weight);
//   3 per neuron: the arriving inputs summed in list order, integration,
//     motor/trace/ring updates;
//   4 plasticity events (arrival, post-synaptic spike or a relevant
//     modulator) appended to the event list;
//   5 plasticity of those synapses, quiet ticks since the last update replayed
//     first.
__device__ __forceinline__ void phase_arrivals(const UnitMem &U, int ne, int cur9, int64_t tick, int tid, int bs) {
    for (int p = tid; p < ne; p += bs) {
        const uint32_t m = U.cmeta[p];
        const int dl = (int)((m >> M_DELAY_SHIFT) & 31u);
        int r = cur9 - dl;
        if (r < 0) r += kHist;
        const bool arr = tick >= dl && ((U.ring[m & M_PRE_MASK] >> r) & 1u);
        U.carr[p] = arr ? 1 : 0;
        if (arr) U.ev[atomicAdd(&U.counters[0], 1)] = p;
    }
}

__device__ __forceinline__ void phase_release(const WorldArgs &d, const UnitMem &U, int64_t tick, int tid, int bs,
                                              const float *tab) {
    const int n = U.counters[0];
    for (int i = tid; i < n; i += bs) {
        const int p = U.ev[i];
        const int es = U.cslot[p];
        U.rel[p] = ((U.cmeta[p] >> M_KIND_SHIFT) & 3u) == KIND_INH ? d.sstate[es].w : release_world(d, es, tick, tab);
    }
}

// An LP or Prinz cell waiting for its warp (HEAVY builds): its slot, type,
// external current and this tick's modulator bits.
struct HeavyJob {
    int pending;
    uint32_t type;
    int slot;
    float ext;
    uint32_t mod;
};

// The end of phase 3 for neuron n: motor counts, trace peak, spike ring and
// the per-tick records plasticity reads.
__device__ __forceinline__ void phase_neuron_tail(const UnitMem &U, int n, int cur9, const NeuronRegs &s,
                                                  uint32_t mod, int *motor_cnt, TraceRegs &tr) {
    const uint32_t f = U.nflag[n];
    const bool traced = (f & WF_TRACED) != 0;
    const int motor = (int)((f >> WF_MOTOR_SHIFT) & 7u) - 1;
    if (motor >= 0) {
        if (traced) tr.pk = fmaxf(tr.pk, s.v);
        if (s.spike) atomicAdd(&motor_cnt[motor], 1);
    }
    const uint16_t bit = (uint16_t)(1u << cur9);
    U.ring[n] = s.spike ? (uint16_t)(U.ring[n] | bit) : (uint16_t)(U.ring[n] & ~bit);
    U.nspk[n] = s.spike ? 1 : 0;
    U.nmod[n] = (uint8_t)mod;
    U.ndepol[n] = s.depol;
}

// Phase 3 for neuron n (state in s). In HEAVY builds an LP or Prinz cell
// stops after heavy_pre with `job` pending: heavy_cells_cta runs its model
// on the whole warp and phase_neuron_tail finishes it.
template <bool HEAVY>
__device__ __forceinline__ void phase_neuron(const WorldArgs &d, const UnitMem &U, int n, int t, int64_t tick,
                                             int cur9, NeuronRegs &s, int *motor_cnt, TraceRegs &tr,
                                             const float *tab, HeavyJob &job) {
    const uint32_t f = U.nflag[n];
    if (!(f & NF_ACTIVE)) return;
    const int slot = U.nslot[n];
    const int ib = U.inptr[n], ie = U.inptr[n + 1];
    float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f, e3 = 0.0f, inh = 0.0f;
    if (t == 0) {    // input left pending from before the step (zero in a running world)
        e0 = d.pexc[(size_t)slot * 4 + 0]; e1 = d.pexc[(size_t)slot * 4 + 1];
        e2 = d.pexc[(size_t)slot * 4 + 2]; e3 = d.pexc[(size_t)slot * 4 + 3];
        inh = d.pinh[slot];
    }
    uint32_t mod = 0;
    const float scale = U.scale[n];
    const bool traced = (f & WF_TRACED) != 0;
    for (int p = ib; p < ie; ++p) {
        if (!U.carr[p]) continue;
        const uint32_t m = U.cmeta[p];
        const float v = U.rel[p];
        const uint32_t kind = (m >> M_KIND_SHIFT) & 3u;
        if (kind == KIND_INH) {
            inh += v;
            if (traced) { ++tr.ia; tr.in += v; }
        } else if (kind == KIND_MOD) {
            if (v > 0) {
                const uint32_t id = (m >> M_MODID_SHIFT) & 3u;
                mod |= 1u << id;
                unsigned long long &q = d.modtick[(size_t)slot * 6 + id * 2 + (uint32_t)(tick & 1)];
                if (q < (unsigned long long)(tick + 1)) q = (unsigned long long)(tick + 1);
            }
        } else {
            if (traced) { ++tr.ea; if (v > 0) ++tr.er; tr.en += v; }
            const float c = v * scale;
            switch ((m >> M_BRANCH_SHIFT) & 3u) {
            case 0: e0 += c; break;
            case 1: e1 += c; break;
            case 2: e2 += c; break;
            default: e3 += c; break;
            }
        }
    }
    // integration (src/main.cu:710-746)
    float g[16];
#pragma unroll
    for (int w = 0; w < 16; ++w) g[w] = U.gene[w * U.gs + n];
    const uint32_t type = f & NF_TYPE_MASK;
    float cur = 0.0f;
    if (f & WF_SENSE) cur = (f & WF_RECEPTOR) ? receptor_drive(g, f, s, U.cur[n]) : U.cur[n];
    if (HEAVY && (type == 2 || type == 3)) {
        job = HeavyJob{1, type, slot, heavy_pre(g, type, s, cur, e0, e1, e2, e3, inh), mod};
        return;
    }
    if (HEAVY && type == 6) {
        float xg[16] = {};
        float gg[16];
        for (int k = 0; k < 16; ++k) gg[k] = g[k];
        s = heavy_tick(gg, type, xg, d.nstate[slot].cell, s, cur, e0, e1, e2, e3, inh, tab);
    } else {
        adex_tick(g, type, f, s, cur, e0, e1, e2, e3, inh, tab);
    }
    phase_neuron_tail(U, n, cur9, s, mod, motor_cnt, tr);
}

// A world step's time is set by its slowest warp: a warp that owns five LP
// cells and steps them one after another takes five times as long as one that
// owns one, while the rest of its CTA waits at the next barrier. So the CTA
// pools its pending LP and Prinz cells (heavy_cells_cta): the warps take the
// pool round-robin and step each cell on all 32 lanes (lp_integrate_warp,
// prinz_tick_warp), or, with more than kWorldWarpCellsMax cells per warp on
// average (where one cell per lane at once costs less), every cell runs on
// its owner lane (heavy_model_lane).
#ifndef NSB_WORLD_WARP_CELLS_MAX
#define NSB_WORLD_WARP_CELLS_MAX 3
#endif
constexpr int kWorldWarpCellsMax = NSB_WORLD_WARP_CELLS_MAX;

// The CTA's pool of pending LP and Prinz cells (one entry per thread at most).
// The counter alternates between two words from call to call, so that each
// call needs only its two barriers: a call reads n[p] between them and clears
// n[p ^ 1], which the previous call read and the next call fills.
template <int NT> struct HeavyPool {
    int n[2];
    int slot[NT];
    float ext[NT];
    float res[NT];       // LP: the axon voltage before the tick; Prinz: 1 when it spiked
    uint8_t type[NT];
};

// The cell model of pending cells between heavy_pre and heavy_post. All
// threads of the CTA call it together, `call` counting the calls (the same in
// every thread); w is the warp's kHeavyWarpScratch + 16 floats of shared
// memory. The owner thread then completes heavy_tick's arithmetic.
template <int NT>
__device__ __forceinline__ void heavy_cells_cta(const WorldArgs &d, const HeavyJob &job, NeuronRegs &s,
                                                HeavyPool<NT> &pool, float *w, int tid, int call,
                                                const float *tab) {
    const int lane = tid & 31, warp = tid >> 5, nwarps = NT / 32, p = call & 1;
    int k = 0;
    if (job.pending) {
        k = atomicAdd(&pool.n[p], 1);
        pool.slot[k] = job.slot;
        pool.ext[k] = job.ext;
        pool.type[k] = (uint8_t)job.type;
    }
    __syncthreads();
    const int n = pool.n[p];
    if (tid == 0) pool.n[p ^ 1] = 0;
    if (n > d.warp_cells * nwarps) {   // many cells: each on its owner lane at once
        if (job.pending) {
            const ref::NeuronGene &G = d.ngene[job.slot];
            float xg[16] = {};
            if (job.type == 2) { xg[0] = G.lp.calcium; xg[1] = G.lp.calcium_k; xg[2] = G.lp.h; xg[3] = G.lp.leak; }
            else { for (int q = 0; q < 8; ++q) xg[q] = G.prinz.g[q]; xg[8] = G.prinz_leak; }
            float *x = d.nstate[job.slot].cell;
            bool spiked = false;
            const float ab = heavy_model_lane(job.type, x, xg, job.ext, spiked, tab);
            heavy_post(job.type, s, x, ab, spiked);
        }
        __syncthreads();
        return;
    }
    for (int e = warp; e < n; e += nwarps) {
        const int slot = pool.slot[e];
        const uint32_t ty = pool.type[e];
        const float ex = pool.ext[e];
        const ref::NeuronGene &G = d.ngene[slot];
        float *xg = w + kHeavyWarpScratch;
        if (lane < 16) {
            float v = 0.0f;
            if (ty == 2) v = lane == 0 ? G.lp.calcium : lane == 1 ? G.lp.calcium_k : lane == 2 ? G.lp.h
                                                      : lane == 3 ? G.lp.leak : 0.0f;
            else v = lane < 8 ? G.prinz.g[lane] : lane == 8 ? G.prinz_leak : 0.0f;
            xg[lane] = v;
        }
        __syncwarp();
        float *x = d.nstate[slot].cell;
        if (ty == 2) {
            const float ab = x[0];
            lp_integrate_warp(x, ex / 1000.0f, xg, w, lane, tab);
            if (lane == 0) pool.res[e] = ab;
        } else {
            const bool sp = prinz_tick_warp(x, xg, ex, xg[8] + 0.0f, -68.0f, w, lane, tab);
            if (lane == 0) pool.res[e] = sp ? 1.0f : 0.0f;
        }
        __syncwarp();
    }
    __syncthreads();
    if (job.pending)
        heavy_post(job.type, s, d.nstate[job.slot].cell, job.type == 2 ? pool.res[k] : 0.0f,
                   job.type == 3 && pool.res[k] != 0.0f);
}

__device__ __forceinline__ void phase_plastic_events(const WorldArgs &d, const UnitMem &U, int ne, int tid, int bs) {
    for (int p = tid; p < ne; p += bs) {
        const uint32_t m = U.cmeta[p];
        if (!(m & M_PLASTIC)) continue;
        const int post = U.cpost[p];
        if (U.nflag[post] & WF_FROZEN) continue;
        const uint32_t mod = U.nmod[post];
        bool ev = U.carr[p] || U.nspk[post];
        if (!ev && mod) ev = mod_relevant(m >> M_PROF_SHIFT, d.sgene[U.cslot[p]].receptors, mod);
        if (ev) U.ev[atomicAdd(&U.counters[1], 1)] = p;
    }
}

__device__ __forceinline__ void phase_plasticity(const WorldArgs &d, const UnitMem &U, int t, int tid, int bs,
                                                 const float *tab) {
    const int n = U.counters[1];
    for (int i = tid; i < n; i += bs) {
        const int p = U.ev[i];
        const uint32_t m = U.cmeta[p];
        const int post = U.cpost[p];
        const int es = U.cslot[p];
        const ref::SynapseGene &G = d.sgene[es];
        const uint32_t mod = U.nmod[post];
        const uint32_t receptors = mod ? (uint32_t)G.receptors : 0u;
        const uint32_t prof = m >> M_PROF_SHIFT;
        const float w0 = G.w0;
        ref::SynapseState &Z = d.sstate[es];
        SynPlast pl;
        load_plast_ref(Z, pl);
        plasticity_quiet(prof, w0, pl, t - U.clast[p] - 1);
        plasticity_tick(prof, receptors, w0, pl, U.carr[p] != 0, U.nspk[post] != 0, U.ndepol[post], mod, tab);
        store_plast_ref(Z, pl);
        U.clast[p] = (int8_t)t;
    }
}

// End of the step for neuron n: state, cleared accumulators, history.
__device__ __forceinline__ void finish_neuron(const WorldArgs &d, const UnitMem &U, int n, const NeuronRegs &s) {
    if (!(U.nflag[n] & NF_ACTIVE)) return;
    const int slot = U.nslot[n];
    store_regs(d.nstate[slot], s);
    for (int b = 0; b < 4; ++b) d.pexc[(size_t)slot * 4 + b] = 0.0f;
    d.pinh[slot] = 0.0f;
    const uint16_t r = U.ring[n];
    for (int k = 0; k < kHist; ++k) d.hist[(size_t)k * d.ncap + slot] = (unsigned char)((r >> k) & 1u);
}
// End of the step for every synapse: the last tick's arrival flag, plasticity
// caught up to the last tick.
__device__ __forceinline__ void finish_synapses(const WorldArgs &d, const UnitMem &U, int ne, int tid, int bs) {
    for (int p = tid; p < ne; p += bs) {
        const uint32_t m = U.cmeta[p];
        const int es = U.cslot[p];
        d.sstate[es].arrived = U.carr[p];
        if ((m & M_PLASTIC) && !(U.nflag[U.cpost[p]] & WF_FROZEN)) {
            const int q = kTicks - 1 - U.clast[p];
            if (q > 0) {
                ref::SynapseState &Z = d.sstate[es];
                SynPlast pl;
                load_plast_ref(Z, pl);
                plasticity_quiet(m >> M_PROF_SHIFT, d.sgene[es].w0, pl, q);
                store_plast_ref(Z, pl);
            }
        }
    }
}

// Global float max (trace peak); order-independent.
__device__ __forceinline__ void atomic_fmax(float *p, float v) {
    unsigned int *u = reinterpret_cast<unsigned int *>(p);
    unsigned int old = *u;
    while (true) {
        const float cur = __uint_as_float(old);
        const float nv = fmaxf(cur, v);
        if (__float_as_uint(nv) == old) break;
        const unsigned int got = atomicCAS(u, old, __float_as_uint(nv));
        if (got == old) break;
        old = got;
    }
}

extern __shared__ __align__(16) unsigned char w_smem[];

// Animals taken from the living list per claim, in the light and heavy builds
// alike: a CTA keeps what it claims, so larger claims let a few CTAs take a
// population whose animals are mostly of one build.
constexpr int kClaim = 4;

// Small units: animals with at most kBlock neurons and kUnitEdges live
// synapses, packed in claim order. The light instantiation takes the animals
// without LP, Prinz or LFS cells (no heavy-cell code: three CTAs per SM) and
// appends the larger animals to `big`; the heavy one takes the rest.
// MINB: CTAs per SM the register budget is sized for (the light kernel is
// built for 3, at 79 registers, and for 2, at about 100, which steps each
// unit faster when there are few units per CTA slot).
// CTAs per SM of the heavy instantiations (their LP and Prinz cell models
// need the registers).
#ifndef NSB_WORLD_HEAVY_MINB
#define NSB_WORLD_HEAVY_MINB 2
#endif
constexpr int kHeavyMinb = NSB_WORLD_HEAVY_MINB;

template <bool HEAVY, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) world_tick_small(WorldArgs d, Cache c, int64_t first_tick,
                                                              const int *alive, const int *nalive, int *queue,
                                                              int *big, int *big_count, int *status,
                                                              Counters *stats) {
    float *tab = reinterpret_cast<float *>(w_smem);                         // 256
    float *gene = tab + 256;                                                // 16 x kBlock
    uint32_t *nflag = reinterpret_cast<uint32_t *>(gene + 16 * kBlock);     // kBlock
    float *curv = reinterpret_cast<float *>(nflag + kBlock);
    float *scale = curv + kBlock;
    float *trx = scale + kBlock;
    float *tri = trx + kBlock;
    float *ndepol = tri + kBlock;
    float *rel = ndepol + kBlock;                                           // kUnitEdges
    int *nslot = reinterpret_cast<int *>(rel + kUnitEdges);                 // kBlock
    int *inptr = nslot + kBlock;                                            // kBlock + 4
    uint32_t *cmeta = reinterpret_cast<uint32_t *>(inptr + kBlock + 4);     // kUnitEdges
    int *cslot = reinterpret_cast<int *>(cmeta + kUnitEdges);
    int *ev = cslot + kUnitEdges;                                           // kUnitEdges
    uint16_t *cpost = reinterpret_cast<uint16_t *>(ev + kUnitEdges);        // kUnitEdges
    uint16_t *ring = cpost + kUnitEdges;                                    // kBlock
    uint8_t *nani = reinterpret_cast<uint8_t *>(ring + kBlock);             // kBlock
    uint8_t *nspk = nani + kBlock;                                          // kBlock
    uint8_t *nmod = nspk + kBlock;                                          // kBlock
    uint8_t *carr = nmod + kBlock;                                          // kUnitEdges
    int8_t *clast = reinterpret_cast<int8_t *>(carr + kUnitEdges);          // kUnitEdges
    __shared__ int ua_a[kUnitAnimals], ua_n0[kUnitAnimals + 1], ua_e0[kUnitAnimals + 1], ua_f[kUnitAnimals];
    __shared__ int ua_motor[kUnitAnimals * kM];
    __shared__ int q_a[32], q_nn[32], q_nl[32];
    __shared__ int q_n, q_i, q_done, s_nu, s_ntot, s_etot;
    __shared__ int s_cnt[2];
    __shared__ unsigned long long s_events;
    __shared__ float s_hscr[HEAVY ? (kBlock / 32) * (kHeavyWarpScratch + 16) : 1];   // warp scratch of LP/Prinz cells
    __shared__ HeavyPool<HEAVY ? kBlock : 32> s_pool;

    const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5;
    int hcall = 0;
    {
        const float *src = nsx::exp2f_table();
        for (int i = tid; i < 256; i += bs) tab[i] = src[i];
    }
    if (tid == 0) { q_n = 0; q_i = 0; q_done = 0; s_pool.n[0] = s_pool.n[1] = 0; }
    __syncthreads();
    const int n_alive = *nalive;
    UnitMem U;
    U.gene = gene; U.gs = kBlock; U.nflag = nflag; U.cur = curv; U.scale = scale; U.ndepol = ndepol; U.rel = rel;
    U.trx = trx; U.tri = tri; U.inptr = inptr; U.cmeta = cmeta; U.cslot = cslot; U.ev = ev; U.counters = s_cnt;
    U.nslot = nslot; U.cpost = cpost; U.ring = ring; U.carr = carr; U.clast = clast; U.nspk = nspk; U.nmod = nmod;
    const int base9 = (int)(first_tick % kHist);
    for (;;) {
        // ---- form the next unit (warp 0) ----
        if (warp == 0) {
            int nu = 0, ntot = 0, etot = 0;
            for (;;) {
                if (q_i >= q_n && !q_done) {
                    int base = 0;
                    if (lane == 0) base = atomicAdd(queue, kClaim);
                    base = __shfl_sync(0xffffffffu, base, 0);
                    bool ok = false;
                    int a = -1, nn = 0, nl = 0;
                    if (lane < (kClaim) && base + lane < n_alive) {
                        a = alive[base + lane];
                        if (!compiled(d, c, a)) {
                            if (!HEAVY) atomicOr(status, ST_LIST);    // compile failed (its own bit is set too)
                        } else {
                            nn = c.nn[a]; nl = c.nl[a];
                            if (nn > kBlock || nl > kUnitEdges) {
                                if (!HEAVY) {
                                    const int k = nn > 2048 ? 0 : nn > 1024 ? 1 : nn > 512 ? 2 : 3;
                                    big[(size_t)k * d.P + atomicAdd(&big_count[k], 1)] = a;
                                }
                            } else {
                                ok = nn > 0 && (c.hv[a] != 0) == HEAVY;
                            }
                        }
                    }
                    const unsigned mk = __ballot_sync(0xffffffffu, ok);
                    if (ok) {
                        const int pos = __popc(mk & ((1u << lane) - 1u));
                        q_a[pos] = a; q_nn[pos] = nn; q_nl[pos] = nl;
                    }
                    __syncwarp();
                    if (lane == 0) { q_n = __popc(mk); q_i = 0; if (base + (kClaim) >= n_alive) q_done = 1; }
                    __syncwarp();
                    continue;
                }
                if (q_i >= q_n) break;
                const int i = q_i, nn = q_nn[i], nl = q_nl[i];
                if (nu < kUnitAnimals && ntot + nn <= kBlock && etot + nl <= kUnitEdges) {
                    __syncwarp();                                   // every lane has read q_i
                    if (lane == 0) {
                        ua_a[nu] = q_a[i]; ua_n0[nu] = ntot; ua_e0[nu] = etot;
                        q_i = i + 1;
                    }
                    ++nu; ntot += nn; etot += nl;
                    __syncwarp();
                } else {
                    break;
                }
            }
            if (lane == 0) {
                s_nu = nu; s_ntot = ntot; s_etot = etot; ua_n0[nu] = ntot; ua_e0[nu] = etot;
                s_events = 0; s_cnt[0] = 0; s_cnt[1] = 0;
            }
        }
        __syncthreads();
        const int nu = s_nu, ntot = s_ntot, etot = s_etot;
        if (nu == 0) break;
        // ---- load the compiled animals ----
        for (int i = 0; i < nu; ++i) {
            const int a = ua_a[i], n0 = ua_n0[i], e0 = ua_e0[i];
            const int nn = ua_n0[i + 1] - n0, nl = ua_e0[i + 1] - e0;
            const int *R = c.arena + c.off[a];
            for (int k = tid; k < nn; k += bs) { nslot[n0 + k] = R[k]; nani[n0 + k] = (uint8_t)i; }
            for (int k = tid; k <= nn; k += bs) inptr[n0 + k] = e0 + R[nn + k];
            const int *Mt = R + 2 * nn + 1;
            for (int k = tid; k < nl; k += bs) {
                cmeta[e0 + k] = (uint32_t)Mt[k] + (uint32_t)n0;    // pre index: animal-local -> unit-local
                cslot[e0 + k] = Mt[nl + k];
            }
            if (tid < kM) ua_motor[i * kM + tid] = 0;
            if (tid == 0) ua_f[i] = (frozen_animal(d, a) ? UA_FROZEN : 0) | (a == d.trace ? UA_TRACED : 0);
        }
        __syncthreads();
        NeuronRegs s = {};
        TraceRegs tr = {0, 0, 0, 0.0f, 0.0f, -INFINITY};
        if (tid < ntot) {
            const int i = nani[tid];
            setup_neuron(d, U, tid, nslot[tid], ua_a[i], (ua_f[i] & UA_TRACED) != 0, (ua_f[i] & UA_FROZEN) != 0, tab);
            load_regs(d.nstate[nslot[tid]], s);
        }
        __syncthreads();
        int narr = 0;
        for (int t = 0; t < kTicks; ++t) {
            const int cur9 = (base9 + t) % kHist;
            const int64_t tick = first_tick + t;
            phase_arrivals(U, etot, cur9, tick, tid, bs);
            __syncthreads();
            if (tid == 0) { narr += s_cnt[0]; s_cnt[1] = 0; }
            phase_release(d, U, tick, tid, bs, tab);
            __syncthreads();
            if (tid == 0) s_cnt[0] = 0;
            HeavyJob job = {};
            if (tid < ntot) phase_neuron<HEAVY>(d, U, tid, t, tick, cur9, s, &ua_motor[nani[tid] * kM], tr, tab, job);
            if (HEAVY) {
                heavy_cells_cta(d, job, s, s_pool, s_hscr + warp * (kHeavyWarpScratch + 16), tid, hcall++, tab);
                if (job.pending) phase_neuron_tail(U, tid, cur9, s, job.mod, &ua_motor[nani[tid] * kM], tr);
            }
            __syncthreads();
            phase_plastic_events(d, U, etot, tid, bs);
            __syncthreads();
            phase_plasticity(d, U, t, tid, bs, tab);
            __syncthreads();
        }
        finish_synapses(d, U, etot, tid, bs);
        if (tid < ntot) {
            finish_neuron(d, U, tid, s);
            const uint32_t f = nflag[tid];
            if (f & WF_TRACED) {
                const int m = (int)((f >> WF_MOTOR_SHIFT) & 7u) - 1;
                if (tr.ea) atomicAdd(&d.tr_ea[m], tr.ea);
                if (tr.er) atomicAdd(&d.tr_er[m], tr.er);
                if (tr.ia) atomicAdd(&d.tr_ia[m], tr.ia);
                atomic_fmax(&d.tr_pk[m], tr.pk);
                trx[tid] = tr.en;
                tri[tid] = tr.in;
            }
        }
        if (tid == 0 && narr) s_events = (unsigned long long)narr;
        __syncthreads();
        if (tid < nu) {
            const int a = ua_a[tid];
            for (int m = 0; m < kM; ++m)
                if (ua_motor[tid * kM + m]) atomicAdd(&d.motors[(size_t)a * kM + m], ua_motor[tid * kM + m]);
            if (ua_f[tid] & UA_TRACED) {
                // trace sums: neurons in list order, one add per motor port
                for (int n = ua_n0[tid]; n < ua_n0[tid + 1]; ++n) {
                    const uint32_t f = nflag[n];
                    if (!(f & WF_TRACED) || !(f & NF_ACTIVE)) continue;
                    const int m = (int)((f >> WF_MOTOR_SHIFT) & 7u) - 1;
                    d.tr_en[m] += trx[n];
                    d.tr_in[m] += tri[n];
                }
            }
        }
        if (tid == 0) {
            atomicAdd(&stats->animals, (unsigned long long)nu);
            atomicAdd(&stats->neurons, (unsigned long long)ntot);
            atomicAdd(&stats->synapses, (unsigned long long)etot);
            atomicAdd(&stats->events, s_events);
        }
        __syncthreads();
    }
}

// Big animals: one per CTA, per-neuron and per-synapse arrays and the
// neurons' register state in a global slab, CSR read in place from the arena.
struct BigSlab {
    float *gene;        // [16][max_n]
    uint32_t *nflag;
    float *cur, *scale, *trx, *tri, *ndepol;
    uint16_t *ring;
    uint8_t *nspk, *nmod;
    float *rel;         // max_e
    int *ev;            // max_e
    uint16_t *cpost;    // max_e
    uint8_t *carr;      // max_e
    int8_t *clast;      // max_e
    uint32_t *regs;     // [14][max_n] NeuronRegs words and the trace peak
    int max_n, max_e;
};

__device__ __forceinline__ void slab_load(const BigSlab &B, int n, NeuronRegs &s) {
    const int M = B.max_n;
    s.v = __uint_as_float(B.regs[0 * M + n]); s.w = __uint_as_float(B.regs[1 * M + n]);
    s.adp = __uint_as_float(B.regs[2 * M + n]); s.inh = __uint_as_float(B.regs[3 * M + n]);
    s.depol = __uint_as_float(B.regs[4 * M + n]); s.rec_ns = __uint_as_float(B.regs[5 * M + n]);
    s.rng = B.regs[6 * M + n];
    s.d0 = __uint_as_float(B.regs[7 * M + n]); s.d1 = __uint_as_float(B.regs[8 * M + n]);
    s.d2 = __uint_as_float(B.regs[9 * M + n]); s.d3 = __uint_as_float(B.regs[10 * M + n]);
    s.total = (int)B.regs[11 * M + n]; s.spike = B.regs[12 * M + n];
}
__device__ __forceinline__ void slab_store(const BigSlab &B, int n, const NeuronRegs &s) {
    const int M = B.max_n;
    B.regs[0 * M + n] = __float_as_uint(s.v); B.regs[1 * M + n] = __float_as_uint(s.w);
    B.regs[2 * M + n] = __float_as_uint(s.adp); B.regs[3 * M + n] = __float_as_uint(s.inh);
    B.regs[4 * M + n] = __float_as_uint(s.depol); B.regs[5 * M + n] = __float_as_uint(s.rec_ns);
    B.regs[6 * M + n] = s.rng;
    B.regs[7 * M + n] = __float_as_uint(s.d0); B.regs[8 * M + n] = __float_as_uint(s.d1);
    B.regs[9 * M + n] = __float_as_uint(s.d2); B.regs[10 * M + n] = __float_as_uint(s.d3);
    B.regs[11 * M + n] = (uint32_t)s.total; B.regs[12 * M + n] = s.spike;
}

// Big animals of one class (HEAVY: with an active LP, Prinz or LFS cell),
// one per 256-thread CTA; each class has its own claim counter.
template <bool HEAVY>
__global__ void __launch_bounds__(kBigBlock, HEAVY ? kHeavyMinb : 3) world_tick_big(WorldArgs d, Cache c, int64_t first_tick,
                                                                          const int *big, const int *big_count,
                                                                          int *queue, BigSlab slab, Counters *stats) {
    float *tab = reinterpret_cast<float *>(w_smem);
    __shared__ int s_i, s_motor[kM], s_cnt[2];
    __shared__ unsigned long long s_events;
    __shared__ float s_hscr[HEAVY ? (kBigBlock / 32) * (kHeavyWarpScratch + 16) : 1];   // warp scratch of LP/Prinz cells
    __shared__ HeavyPool<HEAVY ? kBigBlock : 32> s_pool;
    const int tid = threadIdx.x, bs = blockDim.x;
    int hcall = 0;
    {
        const float *src = nsx::exp2f_table();
        for (int i = tid; i < 256; i += bs) tab[i] = src[i];
        if (tid == 0) s_pool.n[0] = s_pool.n[1] = 0;
    }
    BigSlab B = slab;
    const size_t sn = (size_t)blockIdx.x, MN = (size_t)slab.max_n, ME = (size_t)slab.max_e;
    B.gene += sn * 16 * MN; B.nflag += sn * MN; B.cur += sn * MN; B.scale += sn * MN; B.trx += sn * MN;
    B.tri += sn * MN; B.ndepol += sn * MN; B.ring += sn * MN; B.nspk += sn * MN; B.nmod += sn * MN;
    B.rel += sn * ME; B.ev += sn * ME; B.cpost += sn * ME; B.carr += sn * ME; B.clast += sn * ME;
    B.regs += sn * 14 * MN;
    int nbig = 0;
    for (int k = 0; k < kBigClasses; ++k) nbig += big_count[k];
    const int base9 = (int)(first_tick % kHist);
    for (;;) {
        if (tid == 0) {
            int a = -1;
            for (;;) {
                int i = atomicAdd(queue, 1), k = 0;
                if (i >= nbig) break;
                while (i >= big_count[k]) { i -= big_count[k]; ++k; }
                a = big[(size_t)k * d.P + i];
                if ((c.hv[a] != 0) == HEAVY) break;
                a = -1;
            }
            s_i = a; s_events = 0; s_cnt[0] = 0; s_cnt[1] = 0;
        }
        if (tid < kM) s_motor[tid] = 0;
        __syncthreads();
        const int a = s_i;
        if (a < 0) break;
        const int nn = c.nn[a], nl = c.nl[a];
        const int *R = c.arena + c.off[a];
        const bool fz = frozen_animal(d, a), traced = a == d.trace;
        UnitMem U;
        U.gene = B.gene; U.gs = B.max_n; U.nflag = B.nflag; U.cur = B.cur; U.scale = B.scale; U.ndepol = B.ndepol;
        U.rel = B.rel; U.trx = B.trx; U.tri = B.tri; U.inptr = R + nn;
        U.cmeta = reinterpret_cast<const uint32_t *>(R + 2 * nn + 1); U.cslot = R + 2 * nn + 1 + nl;
        U.ev = B.ev; U.counters = s_cnt; U.nslot = R; U.cpost = B.cpost; U.ring = B.ring; U.carr = B.carr;
        U.clast = B.clast; U.nspk = B.nspk; U.nmod = B.nmod;
        for (int n = tid; n < nn; n += bs) {
            setup_neuron(d, U, n, R[n], a, traced, fz, tab);
            NeuronRegs s;
            load_regs(d.nstate[R[n]], s);
            slab_store(B, n, s);
            B.regs[13 * MN + n] = __float_as_uint(-INFINITY);
        }
        __syncthreads();
        int narr = 0;
        for (int t = 0; t < kTicks; ++t) {
            const int cur9 = (base9 + t) % kHist;
            const int64_t tick = first_tick + t;
            phase_arrivals(U, nl, cur9, tick, tid, bs);
            __syncthreads();
            if (tid == 0) { narr += s_cnt[0]; s_cnt[1] = 0; }
            phase_release(d, U, tick, tid, bs, tab);
            __syncthreads();
            if (tid == 0) s_cnt[0] = 0;
            for (int nb0 = 0; nb0 < nn; nb0 += bs) {    // the same trip count for every thread (warp cells)
                const int n = nb0 + tid;
                if (!HEAVY && n >= nn) break;
                NeuronRegs s = {};
                TraceRegs tr = {0, 0, 0, 0.0f, 0.0f, -INFINITY};
                HeavyJob job = {};
                if (n < nn) {
                    slab_load(B, n, s);
                    tr = TraceRegs{0, 0, 0, B.trx[n], B.tri[n], __uint_as_float(B.regs[13 * MN + n])};
                    phase_neuron<HEAVY>(d, U, n, t, tick, cur9, s, s_motor, tr, tab, job);
                }
                if (HEAVY) {
                    heavy_cells_cta(d, job, s, s_pool, s_hscr + (tid >> 5) * (kHeavyWarpScratch + 16), tid, hcall++,
                                    tab);
                    if (job.pending) phase_neuron_tail(U, n, cur9, s, job.mod, s_motor, tr);
                }
                if (n >= nn) continue;
                slab_store(B, n, s);
                if (tr.ea || tr.er || tr.ia) {
                    const int m = (int)((U.nflag[n] >> WF_MOTOR_SHIFT) & 7u) - 1;
                    if (tr.ea) atomicAdd(&d.tr_ea[m], tr.ea);
                    if (tr.er) atomicAdd(&d.tr_er[m], tr.er);
                    if (tr.ia) atomicAdd(&d.tr_ia[m], tr.ia);
                }
                B.trx[n] = tr.en; B.tri[n] = tr.in;
                B.regs[13 * MN + n] = __float_as_uint(tr.pk);
            }
            __syncthreads();
            phase_plastic_events(d, U, nl, tid, bs);
            __syncthreads();
            phase_plasticity(d, U, t, tid, bs, tab);
            __syncthreads();
        }
        finish_synapses(d, U, nl, tid, bs);
        for (int n = tid; n < nn; n += bs) {
            NeuronRegs s;
            slab_load(B, n, s);
            finish_neuron(d, U, n, s);
            const uint32_t f = U.nflag[n];
            if (f & WF_TRACED) {
                const int m = (int)((f >> WF_MOTOR_SHIFT) & 7u) - 1;
                atomic_fmax(&d.tr_pk[m], __uint_as_float(B.regs[13 * MN + n]));
            }
        }
        if (tid == 0) s_events = (unsigned long long)narr;
        __syncthreads();
        if (tid == 0) {
            for (int m = 0; m < kM; ++m)
                if (s_motor[m]) atomicAdd(&d.motors[(size_t)a * kM + m], s_motor[m]);
            if (traced)
                for (int n = 0; n < nn; ++n) {
                    const uint32_t f = U.nflag[n];
                    if (!(f & WF_TRACED) || !(f & NF_ACTIVE)) continue;
                    const int m = (int)((f >> WF_MOTOR_SHIFT) & 7u) - 1;
                    d.tr_en[m] += B.trx[n];
                    d.tr_in[m] += B.tri[n];
                }
            atomicAdd(&stats->animals, 1ull);
            atomicAdd(&stats->neurons, (unsigned long long)nn);
            atomicAdd(&stats->synapses, (unsigned long long)nl);
            atomicAdd(&stats->events, s_events);
        }
        __syncthreads();
    }
}

// Homeostasis (src/main.cu:1287-1300) over every owned neuron slot.
__global__ void world_homeostasis(WorldArgs d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.ncap; i += gridDim.x * blockDim.x) {
        const int a = d.nowner[i];
        if (a < 0 || a >= d.P) continue;
        const ref::Animal &A = d.animals[a];
        if (A.alive != 1 || frozen_animal(d, a)) continue;
        const ref::NeuronGene &G = d.ngene[i];
        if (!G.active || G.type != 0) continue;
        ref::NeuronState &S = d.nstate[i];
        const float elapsed = fmaxf(16.0f, (float)A.age * 16.0f);
        const float hz = (float)S.total * 1000.0f / elapsed;
        S.log_ampa = homeostasis(0u, S.log_ampa, 16.0f, hz);
    }
}

template <class T> T *dev_alloc(std::vector<void *> &owned, size_t n) {
    T *p = nullptr;
    NSB_CHECK(cudaMalloc(reinterpret_cast<void **>(&p), sizeof(T) * (n ? n : 1)));
    owned.push_back(p);
    return p;
}

}  // namespace

// Host side of one world stage.
class WorldStage {
public:
    WorldStage(const NsbWorldPools &p, int max_n, int max_e) {
        if (!p.animals || !p.neurons || !p.synapses || !p.neuron_state || !p.synapse_state || !p.pending_exc ||
            !p.pending_inh || !p.senses || !p.mod_event_tick || !p.spike_history || !p.neuron_owner ||
            !p.synapse_owner || !p.neuron_next || !p.synapse_next || !p.neuron_port || !p.motors ||
            !p.trace_exc_arrivals || !p.trace_exc_releases || !p.trace_inh_arrivals || !p.trace_exc_ns ||
            !p.trace_inh_ns || !p.trace_peak_mv)
            throw std::runtime_error("Missing world pool pointer");
        if (p.animal_capacity <= 0 || p.neuron_capacity <= 0 || p.synapse_capacity <= 0)
            throw std::runtime_error("Invalid world pool capacity");
        if (max_n <= 0) max_n = 4096;
        if (max_e <= 0) max_e = 65536;
        if (max_n > 65535) throw std::runtime_error("Brain neuron maximum above 65535");
        d_.animals = static_cast<const ref::Animal *>(p.animals);
        d_.cohort = static_cast<const ref::PlasticityCohort *>(p.plasticity_cohort);
        d_.ngene = static_cast<const ref::NeuronGene *>(p.neurons);
        d_.sgene = static_cast<const ref::SynapseGene *>(p.synapses);
        d_.nstate = static_cast<ref::NeuronState *>(p.neuron_state);
        d_.sstate = static_cast<ref::SynapseState *>(p.synapse_state);
        d_.pexc = p.pending_exc; d_.pinh = p.pending_inh; d_.senses = p.senses;
        d_.modtick = p.mod_event_tick; d_.hist = p.spike_history;
        d_.nowner = p.neuron_owner; d_.sowner = p.synapse_owner; d_.nnext = p.neuron_next;
        d_.snext = p.synapse_next; d_.nport = p.neuron_port; d_.motors = p.motors;
        d_.tr_ea = p.trace_exc_arrivals; d_.tr_er = p.trace_exc_releases; d_.tr_ia = p.trace_inh_arrivals;
        d_.tr_en = p.trace_exc_ns; d_.tr_in = p.trace_inh_ns; d_.tr_pk = p.trace_peak_mv;
        d_.trace = p.trace_animal; d_.sil_senses = p.silence_senses; d_.sil_contact = p.silence_contact;
        d_.P = p.animal_capacity; d_.ncap = p.neuron_capacity; d_.ecap = p.synapse_capacity;
        d_.warp_cells = kWorldWarpCellsMax;
        if (const char *wc = std::getenv("NSB_WORLD_WARP_CELLS")) d_.warp_cells = std::atoi(wc);
        int dev = 0;
        NSB_CHECK(cudaGetDevice(&dev));
        NSB_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
        const PhysConst K = make_constants();
        NSB_CHECK(cudaMemcpyToSymbol(c_K, &K, sizeof(PhysConst)));
        // tab, gene records, 6 per-neuron floats, rel, nslot, inptr, cmeta, cslot,
        // ev, cpost, ring, 3 per-neuron bytes, carr, clast
        small_smem_ = 256 * 4 + 16 * kBlock * 4 + 6 * kBlock * 4 + kUnitEdges * 4 + kBlock * 4 + (kBlock + 4) * 4 +
                      3 * kUnitEdges * 4 + kUnitEdges * 2 + kBlock * 2 + 3 * kBlock + 2 * kUnitEdges;
        int occ = 0;
        NSB_CHECK(cudaFuncSetAttribute(world_tick_small<false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       small_smem_));
        NSB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, world_tick_small<false, 3>, kBlock, small_smem_));
        small_grid_ = sms_ * std::max(occ, 1);
        NSB_CHECK(cudaFuncSetAttribute(world_tick_small<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       small_smem_));
        NSB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, world_tick_small<false, 2>, kBlock, small_smem_));
        small2_grid_ = sms_ * std::max(occ, 1);
        NSB_CHECK(cudaFuncSetAttribute(world_tick_small<true, kHeavyMinb>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       small_smem_));
        NSB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, world_tick_small<true, kHeavyMinb>, kBlock, small_smem_));
        heavy_grid_ = sms_ * std::max(occ, 1);
        NSB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, world_tick_big<false>, kBigBlock, 1024));
        big_grid_ = sms_ * std::max(occ, 1);
        NSB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, world_tick_big<true>, kBigBlock, 1024));
        big_heavy_grid_ = sms_ * std::max(occ, 1);
        compile_grid_ = sms_;
        const size_t P = (size_t)d_.P;
        c_.id = dev_alloc<int>(owned_, P); c_.nn = dev_alloc<int>(owned_, P); c_.ne = dev_alloc<int>(owned_, P);
        c_.nl = dev_alloc<int>(owned_, P); c_.off = dev_alloc<int>(owned_, P); c_.cap = dev_alloc<int>(owned_, P);
        c_.hv = dev_alloc<int>(owned_, P);
        c_.arena_cap = 2 * (2LL * d_.ncap + (long long)d_.P + 2LL * d_.ecap);
        c_.arena = dev_alloc<int>(owned_, (size_t)c_.arena_cap);
        c_.bump = dev_alloc<unsigned long long>(owned_, 1);
        reset_cache();
        int pow2n = 1;
        while (pow2n < max_n) pow2n <<= 1;
        const size_t cw = (size_t)compile_grid_ * kCompileWarps;
        s_.max_n = max_n; s_.max_e = max_e; s_.pow2n = pow2n;
        s_.elist = dev_alloc<int>(owned_, cw * max_e);
        s_.tmeta = dev_alloc<uint32_t>(owned_, cw * max_e);
        s_.tpost = dev_alloc<int>(owned_, cw * max_e);
        s_.skey = dev_alloc<int>(owned_, cw * pow2n);
        s_.sval = dev_alloc<int>(owned_, cw * pow2n);
        s_.cnt = dev_alloc<int>(owned_, cw * max_n);
        const size_t bg = (size_t)std::max(big_grid_, big_heavy_grid_);   // one slab per CTA
        b_.max_n = max_n; b_.max_e = max_e;
        b_.gene = dev_alloc<float>(owned_, bg * 16 * max_n);
        b_.nflag = dev_alloc<uint32_t>(owned_, bg * max_n);
        b_.cur = dev_alloc<float>(owned_, bg * max_n);
        b_.scale = dev_alloc<float>(owned_, bg * max_n);
        b_.trx = dev_alloc<float>(owned_, bg * max_n);
        b_.tri = dev_alloc<float>(owned_, bg * max_n);
        b_.ndepol = dev_alloc<float>(owned_, bg * max_n);
        b_.ring = dev_alloc<uint16_t>(owned_, bg * max_n);
        b_.nspk = dev_alloc<uint8_t>(owned_, bg * max_n);
        b_.nmod = dev_alloc<uint8_t>(owned_, bg * max_n);
        b_.rel = dev_alloc<float>(owned_, bg * max_e);
        b_.ev = dev_alloc<int>(owned_, bg * max_e);
        b_.cpost = dev_alloc<uint16_t>(owned_, bg * max_e);
        b_.carr = dev_alloc<uint8_t>(owned_, bg * max_e);
        b_.clast = dev_alloc<int8_t>(owned_, bg * max_e);
        b_.regs = dev_alloc<uint32_t>(owned_, bg * 14 * max_n);
        list_ = dev_alloc<int>(owned_, P);
        alive_ = dev_alloc<int>(owned_, P);
        big_ = dev_alloc<int>(owned_, (size_t)kBigClasses * P);
        // 0 compile count, 1 light queue, 3 light big queue, 4 status, 5 living animals, 6 heavy queue,
        // 7 heavy big queue, 8..11 big animals per size class
        ints_ = dev_alloc<int>(owned_, kInts);
        stats_ = dev_alloc<Counters>(owned_, 1);
        NSB_CHECK(cudaMallocHost(&h_ints_, kInts * sizeof(int)));
        NSB_CHECK(cudaMallocHost(&h_stats_, sizeof(Counters)));
        NSB_CHECK(cudaMallocHost(&h_bump_, sizeof(unsigned long long)));
        NSB_CHECK(cudaDeviceSynchronize());
    }
    ~WorldStage() {
        for (void *q : owned_) cudaFree(q);
        if (h_ints_) cudaFreeHost(h_ints_);
        if (h_stats_) cudaFreeHost(h_stats_);
        if (h_bump_) cudaFreeHost(h_bump_);
    }

    void neural_step(int64_t step) {
        if (step < 1) throw std::runtime_error("Invalid world step");
        const int64_t first_tick = (step - 1) * kTicks;
        cudaStream_t st = 0;
        NSB_CHECK(cudaMemsetAsync(ints_, 0, kInts * sizeof(int), st));
        NSB_CHECK(cudaMemsetAsync(stats_, 0, sizeof(Counters), st));
        world_select<<<std::max(1, std::min((d_.P + 255) / 256, sms_ * 8)), 256, 0, st>>>(d_, c_, list_, ints_,
                                                                                            alive_, ints_ + 5);
        world_compile<<<compile_grid_, 32 * kCompileWarps, 0, st>>>(d_, c_, list_, ints_, s_, ints_ + 4);
        // Few units per CTA slot (judged by the previous step's neurons): the
        // 2-CTA build steps each unit faster; otherwise the 3-CTA build.
        const bool few = last_.neurons > 0 && (long long)last_.neurons < 2LL * small_grid_ * kBlock;
        if (few)
            world_tick_small<false, 2><<<small2_grid_, kBlock, small_smem_, st>>>(
                d_, c_, first_tick, alive_, ints_ + 5, ints_ + 1, big_, ints_ + 8, ints_ + 4, stats_);
        else
            world_tick_small<false, 3><<<small_grid_, kBlock, small_smem_, st>>>(
                d_, c_, first_tick, alive_, ints_ + 5, ints_ + 1, big_, ints_ + 8, ints_ + 4, stats_);
        world_tick_small<true, kHeavyMinb><<<heavy_grid_, kBlock, small_smem_, st>>>(d_, c_, first_tick, alive_, ints_ + 5,
                                                                           ints_ + 6, big_, ints_ + 8, ints_ + 4, stats_);
        world_tick_big<false><<<big_grid_, kBigBlock, 1024, st>>>(d_, c_, first_tick, big_, ints_ + 8, ints_ + 3, b_,
                                                                 stats_);
        world_tick_big<true><<<big_heavy_grid_, kBigBlock, 1024, st>>>(d_, c_, first_tick, big_, ints_ + 8, ints_ + 7,
                                                                       b_, stats_);
        NSB_CHECK(cudaGetLastError());
        NSB_CHECK(cudaMemcpyAsync(h_ints_, ints_, kInts * sizeof(int), cudaMemcpyDeviceToHost, st));
        NSB_CHECK(cudaMemcpyAsync(h_stats_, stats_, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        NSB_CHECK(cudaMemcpyAsync(h_bump_, c_.bump, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        NSB_CHECK(cudaStreamSynchronize(st));
        last_ = *h_stats_;
        const int status = h_ints_[4];
        const unsigned long long used = *h_bump_;
        if (status & ST_ARENA || (long long)used > c_.arena_cap / 2) reset_cache();
        if (status & ST_SIZE) throw std::runtime_error("Animal brain larger than the world stage's maximum");
        if (status & ST_GENE) throw std::runtime_error("Invalid synapse gene in a living animal");
        if (status & ST_ARENA) throw std::runtime_error("Compiled-brain arena exhausted; retry the step");
        if (status & ST_LIST) throw std::runtime_error("Animal neuron/synapse lists disagree with its counts");
    }

    // Launched on the legacy default stream, ordered before the caller's next
    // launches there, as the reference's own homeostasis launches are.
    void homeostasis_step() {
        world_homeostasis<<<sms_ * 8, 256, 0, 0>>>(d_);
        NSB_CHECK(cudaGetLastError());
    }

    void stats(long long *out) const {
        out[0] = (long long)last_.animals; out[1] = (long long)last_.neurons;
        out[2] = (long long)last_.synapses; out[3] = (long long)last_.events;
    }

private:
    void reset_cache() {
        NSB_CHECK(cudaMemset(c_.id, 0xff, sizeof(int) * d_.P));    // -1: nothing compiled
        NSB_CHECK(cudaMemset(c_.off, 0xff, sizeof(int) * d_.P));
        NSB_CHECK(cudaMemset(c_.cap, 0, sizeof(int) * d_.P));
        NSB_CHECK(cudaMemset(c_.bump, 0, sizeof(unsigned long long)));
    }

    WorldArgs d_{};
    Cache c_{};
    Scratch s_{};
    BigSlab b_{};
    std::vector<void *> owned_;
    int *list_ = nullptr, *alive_ = nullptr, *big_ = nullptr, *ints_ = nullptr, *h_ints_ = nullptr;
    Counters *stats_ = nullptr, *h_stats_ = nullptr, last_{};
    unsigned long long *h_bump_ = nullptr;
    int sms_ = 148, small_smem_ = 0, small_grid_ = 0, small2_grid_ = 0, heavy_grid_ = 0, big_grid_ = 0;
    int big_heavy_grid_ = 0;
    static constexpr int kInts = 16;
    int compile_grid_ = 0;
};

}  // namespace nsb

extern "C" {

void *nsb_world_create(const NsbWorldPools *pools, int max_brain_neurons, int max_brain_synapses) {
    try {
        if (!pools) throw std::runtime_error("Missing world pools");
        return new nsb::WorldStage(*pools, max_brain_neurons, max_brain_synapses);
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return nullptr;
    }
}

void nsb_world_destroy(void *world) { delete static_cast<nsb::WorldStage *>(world); }

int nsb_world_neural_step(void *world, int64_t step) {
    try {
        if (!world) throw std::runtime_error("Invalid world handle");
        static_cast<nsb::WorldStage *>(world)->neural_step(step);
        return 0;
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return -1;
    }
}

int nsb_world_homeostasis(void *world) {
    try {
        if (!world) throw std::runtime_error("Invalid world handle");
        static_cast<nsb::WorldStage *>(world)->homeostasis_step();
        return 0;
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return -1;
    }
}

int nsb_world_stats(void *world, long long *out) {
    if (!world || !out) return -1;
    static_cast<nsb::WorldStage *>(world)->stats(out);
    return 0;
}

int nsb_world_layout(uint64_t *out) {
    if (!out) return -1;
    using nsb::ref::Animal;
    using nsb::ref::PlasticityCohort;
    const uint64_t v[10] = {sizeof(Animal), sizeof(PlasticityCohort), offsetof(Animal, id), offsetof(Animal, age),
                            offsetof(Animal, alive), offsetof(Animal, neuron_head), offsetof(Animal, synapse_head),
                            offsetof(Animal, neuron_count), offsetof(Animal, synapse_count),
                            offsetof(PlasticityCohort, frozen)};
    for (int i = 0; i < 10; ++i) out[i] = v[i];
    return 10;
}

}  // extern "C"
