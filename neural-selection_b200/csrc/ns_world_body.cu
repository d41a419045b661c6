// World ecology stage: the world simulator's per-step body, predation, genome
// reclamation, reproduction with mutation, food regrowth and senses
// (mixic/neural-selection src/main.cu:364-525, 612-657 and 1138-1737), on the
// simulator's own pools: the neural pools of NsbWorldPools plus the food
// grid, spatial index, slot bitmaps and counters of NsbWorldEcology.
//
// Order of one world step in the reference host loop (src/main.cu:2745-2770),
// with the calls that replace each part:
//   body_step, spatial reset, index_animals, bite_animals, finish_predation
//                                                  nsb_world_body_step
//   homeostasis                                    nsb_world_homeostasis
//   reclaim_dead_genomes                           nsb_world_reclaim
//   reproduce                                      nsb_world_reproduce
//   (cohort observation: the caller's)
//   regrow, spatial reset, index_animals, update_senses
//                                                  nsb_world_regrow_and_sense
//
// Semantics. The reference runs each kernel one thread per animal (per cell
// for regrowth) with atomics: food harvests, the spatial index's list order,
// bites, and the slots of life records and bite events, so under contention
// its results depend on thread timing. This stage computes the outcome of one
// fixed legal execution: each kernel as if its threads ran one after another
// in ascending animal slot order. It is computed in parallel:
//   - harvests: an animal finds the food of its cell reduced by the eaters of
//     lower slot in that cell (stock s, k such eaters: max(0, s - k)), which
//     is what a slot-ordered sequence of harvests leaves; its 9 x 9 food scan
//     reads the same quantity for each cell;
//   - spatial index: each cell's list runs from the highest slot down, as
//     ascending pushes onto the list head leave it (one warp ranks a cell);
//   - bites only touch animals of the attacker's own cell, so each cell's
//     attackers run in slot order on one thread, cells in parallel;
//   - bite events and life records take consecutive indices in slot order
//     (a scan over the animal slots);
//   - births: parents one after another in slot order, each birth's slot
//     claims as claim_slot run alone (below, reproduction).
// Arithmetic: cosf, sinf and hypotf are the correctly rounded nsx functions,
// sqrtf and division are IEEE (no contraction), so the results are those of
// the reference's kernels built with IEEE arithmetic and the same correctly
// rounded functions, bit for bit.
#include <cuda_runtime.h>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ns_b200.h"
#include "ns_crmath.h"
#include "ns_internal.h"
#include "ns_refabi.h"

namespace nsb {
void set_error(const char *message);   // ns_abi.cu

namespace {

constexpr int kS = 19, kM = 5, kTicks = 16, kContact = 16;
constexpr int kW = 128, kH = 128, kCells = kW * kH;
constexpr float kBodyUpkeep = 0.003f;
constexpr float kNeuronUpkeep = 0.00002f;
constexpr float kBiteDamage = 2.0f;
constexpr float kBiteCost = 0.02f;
constexpr float kMeatFraction = 0.45f;
constexpr float kMuscleDecay = 0.92311635f;   // exp(-16 / 200)
constexpr float kMuscleTwitch = 0.30f;
constexpr int kMaxAge = 10000;
// Status bits, reported by the host as errors.
enum : int { ES_LIST = 1, ES_SLOT = 2, ES_KIND = 4 };

struct Eco {
    ref::Animal *animals;
    ref::NeuronGene *ngene;
    ref::SynapseGene *sgene;
    ref::SynapseState *sstate;
    int *nowner, *sowner;
    int *nnext, *snext;
    float *senses;
    int *motors;
    int *food, *kind, *cell_head, *cell_next;
    unsigned char *bite_intent;
    uint32_t *nused, *sused;
    int *f_motor, *f_observed, *deaths, *pred_deaths, *bites;
    ref::LifeRecord *life;
    int *life_count;
    ref::BiteEvent *bite_events;
    int *bite_count;
    int initial_count, instant_motors, life_capacity;
    int P, ncap, ecap;
    // scratch
    int *ecnt, *estart, *efill, *elist;          // eaters by food cell (slot order not kept)
    int *acnt, *astart, *afill, *alist, *asort;  // living animals by cell; asort: highest slot first
    unsigned char *flag;                         // per animal: bit, or reclaimed
    int *prey, *rank, *base;                     // base[0]: first index of this call's records
    int *active;                                 // active neurons per animal
    // reclamation: per reclaimed animal its synapse slots (gathered by owner)
    // and the life record's sums
    int *goff, *gcount, *gslot, *dead, *stmp;
    int *r_as, *r_ps, *r_an, *r_mn, *r_nc;
    float *r_total;
    // reproduction: the pools a birth writes, the parents' lists in list
    // order, the child's lists (tail first: the last entry is the head)
    ref::NeuronState *nstate;
    int *nport;
    float *pexc, *pinh;
    unsigned long long *modtick;
    unsigned char *hist;
    int *neuron_clone, *births, *next_id;
    const ref::NeuronGene *profiles;             // initial_profile(0..6)
    unsigned char *pflag;
    int *prank, *parents, *pn_off, *ps_off, *pn_cnt, *ps_cnt, *pn_tmp, *ps_tmp;
    int *pn_g, *ps_g, *pn_list, *ps_list;
    int *cn, *cs;
    uint32_t *nseed, *sseed;
    const unsigned long long *jump;              // [kJumpLevels][64]: columns of M^(2^j), M the xorshift64 step
    int *status;
};

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(hi, fmaxf(lo, x)); }
__device__ __forceinline__ int cell_of(float x, float y) {
    const int ix = (int)floorf(clampf(x, 0.0f, (float)kW - 0.001f));
    const int iy = (int)floorf(clampf(y, 0.0f, (float)kH - 0.001f));
    return iy * kW + ix;
}
// xorshift64* and the seed hash of src/main.cu:331-346.
__device__ __forceinline__ unsigned long long random64(unsigned long long &s) {
    s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
    return s * 2685821657736338717ULL;
}
__device__ __forceinline__ float uniform(unsigned long long &s) {
    return (float)((random64(s) >> 40) * (1.0 / 16777216.0));
}
__device__ __forceinline__ unsigned long long seed_for(unsigned long long seed, unsigned long long i) {
    unsigned long long x = seed + 0x9e3779b97f4a7c15ULL * (i + 1);
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return (x ^ (x >> 31)) | 1ULL;
}
__device__ __forceinline__ bool excitatory(unsigned char t) { return t == 0 || t == 4 || t == 5; }

// Food of cell c at animal a's turn: the stock minus the harvests of the
// cell's eaters of lower slot (each takes one unit while any is left).
__device__ int food_at(const Eco &e, int c, int a) {
    const int f0 = e.food[c];
    if (f0 <= 0) return f0;
    const int n = e.ecnt[c];
    if (!n) return f0;
    const int *l = e.elist + e.estart[c];
    int k = 0;
    for (int i = 0; i < n; ++i) k += l[i] < a;
    return k >= f0 ? 0 : f0 - k;
}

// ---- cell and slot scans (one CTA of 1024 threads) ------------------------------
// out[i] = sum of in[0..i). With `accumulate`, base_out
// receives *accumulate and *accumulate grows by the total.
template <class T>
__global__ void __launch_bounds__(1024) eco_scan(const T *in, int n, int *out, int *accumulate, int *base_out) {
    constexpr int kPer = 8, kChunk = 1024 * kPer;
    __shared__ int buf[kChunk];
    __shared__ int warp_sum[32];
    __shared__ int carry;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) carry = 0;
    for (int chunk = 0; chunk < n; chunk += kChunk) {
        for (int k = 0; k < kPer; ++k) {                 // coalesced loads
            const int i = chunk + k * 1024 + t;
            buf[k * 1024 + t] = i < n ? (int)in[i] : 0;
        }
        __syncthreads();
        int v[kPer], s = 0;
        for (int k = 0; k < kPer; ++k) {
            v[k] = buf[t * kPer + k];
            s += v[k];
        }
        int x = s;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = warp_sum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sum[lane] = w;
        }
        __syncthreads();
        int b = carry + x - s + (warp ? warp_sum[warp - 1] : 0);
        for (int k = 0; k < kPer; ++k) {
            buf[t * kPer + k] = b;
            b += v[k];
        }
        __syncthreads();
        for (int k = 0; k < kPer; ++k) {                 // coalesced stores
            const int i = chunk + k * 1024 + t;
            if (i < n) out[i] = buf[k * 1024 + t];
        }
        if (t == 0) carry += warp_sum[31];
        __syncthreads();
    }
    if (t == 0 && accumulate) {
        base_out[0] = *accumulate;
        *accumulate += carry;
    }
}

// ---- body step (src/main.cu:1146-1249) -------------------------------------------
__global__ void eco_count_eaters(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        if (A.alive != 1 || e.motors[(size_t)a * kM + 3] <= 0) continue;
        atomicAdd(&e.ecnt[cell_of(A.x, A.y)], 1);
    }
}
__global__ void eco_place_eaters(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        if (A.alive != 1 || e.motors[(size_t)a * kM + 3] <= 0) continue;
        const int c = cell_of(A.x, A.y);
        e.elist[e.estart[c] + atomicAdd(&e.efill[c], 1)] = a;
    }
}

// Active neurons of each living animal (its upkeep): over the neuron slots by
// owner, which the simulator keeps equal to list membership (initialize_neuron
// and release_genome / remove_hidden_neuron set and clear both together). An
// integer sum, so the slot order of the additions does not matter.
__global__ void eco_count_active(Eco e) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < e.ncap; n += gridDim.x * blockDim.x) {
        const int a = e.nowner[n];
        if (a < 0 || a >= e.P) continue;
        const int on = e.ngene[n].active;
        if (on && e.animals[a].alive == 1) atomicAdd(&e.active[a], on);
    }
}

__global__ void __launch_bounds__(128) eco_body(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        if (e.animals[a].alive != 1) continue;
        ref::Animal b = e.animals[a];
        ref::Behavior &bh = b.behavior;
        const int age_bin = b.age < 100 ? 0 : (b.age < 300 ? 1 : 2);
        const bool hungry = b.energy < 16.0f;
        const float old_x = b.x, old_y = b.y;
        int *mo = e.motors + (size_t)a * kM;
        float force[3];
        for (int m = 0; m < 3; ++m)
            force[m] = e.instant_motors ? (float)mo[m] / (float)kTicks
                                        : (b.muscle[m] = fminf(1.0f, b.muscle[m] * kMuscleDecay +
                                                                     (float)mo[m] * kMuscleTwitch));
        const float thrust = force[0], left = force[1], right = force[2];
        const bool eat = mo[3] > 0;
        const bool bite = mo[4] > 0;
        e.bite_intent[a] = bite;
        if (b.id < e.initial_count && b.age < 100) {
            atomicAdd(e.f_observed, 1);
            for (int m = 0; m < kM; ++m)
                if (mo[m] > 0) atomicAdd(&e.f_motor[m], 1);
        }
        for (int m = 0; m < kM; ++m) mo[m] = 0;
        b.heading += (right - left) * 1.2f;
        b.x = clampf(b.x + nsx::cosf_cr(b.heading) * thrust * 1.5f, 0.0f, (float)kW - 0.001f);
        b.y = clampf(b.y + nsx::sinf_cr(b.heading) * thrust * 1.5f, 0.0f, (float)kH - 0.001f);
        const float travel = nsx::hypotf_cr(b.x - old_x, b.y - old_y);
        if (hungry && travel > 0.0001f) {
            float nearest[3] = {1e9f, 1e9f, 1e9f};
            float tx[3] = {0.0f, 0.0f, 0.0f}, ty[3] = {0.0f, 0.0f, 0.0f};
            const int cx = (int)old_x, cy = (int)old_y;
            for (int dy = -4; dy <= 4; ++dy) {
                const int y = cy + dy;
                if (y < 0 || y >= kH) continue;
                int f[9], n[9];                                   // the row's stocks and eaters, loaded first
#pragma unroll
                for (int i = 0; i < 9; ++i) {
                    const int x = cx - 4 + i;
                    const bool in = x >= 0 && x < kW;
                    f[i] = in ? e.food[y * kW + x] : 0;
                    n[i] = in ? e.ecnt[y * kW + x] : 0;
                }
#pragma unroll
                for (int i = 0; i < 9; ++i) {
                    const int x = cx - 4 + i;
                    if (x < 0 || x >= kW || f[i] <= 0) continue;
                    const int c = y * kW + x;
                    if (n[i] && food_at(e, c, a) <= 0) continue;
                    const int kind = e.kind[c];
                    if (kind < 0 || kind > 2) { atomicOr(e.status, ES_KIND); continue; }
                    const float fx = x + 0.5f, fy = y + 0.5f;
                    const float distance = (fx - old_x) * (fx - old_x) + (fy - old_y) * (fy - old_y);
                    if (distance < nearest[kind]) {
                        nearest[kind] = distance;
                        tx[kind] = fx;
                        ty[kind] = fy;
                    }
                }
            }
            for (int kind = 0; kind < 3; ++kind)
                if (nearest[kind] < 1e9f) {
                    bh.approach_progress[age_bin][kind] += sqrtf(nearest[kind]) -
                                                           nsx::hypotf_cr(tx[kind] - b.x, ty[kind] - b.y);
                    bh.approach_travel[age_bin][kind] += travel;
                }
        }
        const int active = e.active[a];
        b.energy -= kBodyUpkeep + (float)active * kNeuronUpkeep + thrust * 0.02f + (bite ? kBiteCost : 0.0f);
        b.fullness = fmaxf(0.0f, b.fullness - 0.05f);
        b.pain *= 0.8f;
        for (int k = 0; k < 4; ++k) b.taste[k] *= 0.7f;
        // Feed at the cell sensed before this decision; the harvest succeeds
        // exactly when food is left at this animal's turn.
        const int fc = cell_of(old_x, old_y);
        const bool offered = food_at(e, fc, a) > 0;
        const int hb = hungry ? 0 : 1;
        int fkind = 0;
        if (offered) {
            fkind = e.kind[fc];
            if (fkind < 0 || fkind > 2) { atomicOr(e.status, ES_KIND); fkind = 0; }
            ++bh.opportunities[age_bin][hb][fkind];
        } else {
            ++bh.empty_steps[age_bin][hb];
            bh.empty_eat[age_bin][hb] += eat;
        }
        if (eat && offered) {
            ++bh.accepted[age_bin][hb][fkind];
            if (fkind == 1 && bh.first_b_age == 0) bh.first_b_age = b.age + 1;
            b.taste[fkind] = 1;
            b.fullness += 1;
            if (fkind == 0) b.energy = fminf(30, b.energy + 4);
            if (fkind == 1) { b.energy = fminf(30, b.energy + 2); b.health -= 1.4f; b.pain += 1.4f; }
            if (b.fullness > 8) { b.health -= 0.8f; b.pain += 0.8f; }
        }
        if (b.energy <= 0) { b.energy = 0; b.health -= 0.15f; b.pain += 0.15f; }
        ++b.age;
        if (b.health <= 0 || b.age >= kMaxAge) {
            bh.death_cause = b.age >= kMaxAge ? 4 : (b.energy <= 0 ? 2 : 3);
            b.alive = 0;
            atomicAdd(e.deaths, 1);
        }
        e.animals[a] = b;
    }
}

// Stock after every eater of the cell had its turn.
__global__ void eco_commit_food(Eco e) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kCells; c += gridDim.x * blockDim.x) {
        const int f0 = e.food[c], n = e.ecnt[c];
        if (f0 > 0 && n > 0) e.food[c] = n >= f0 ? 0 : f0 - n;
    }
}

// ---- spatial index (src/main.cu:612-617) -----------------------------------------
__global__ void eco_count_cells(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        if (A.alive == 1) atomicAdd(&e.acnt[cell_of(A.x, A.y)], 1);
    }
}
__global__ void eco_place_cells(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        if (A.alive != 1) continue;
        const int c = cell_of(A.x, A.y);
        e.alist[e.astart[c] + atomicAdd(&e.afill[c], 1)] = a;
    }
}
// One warp per cell: rank each member by the number of higher slots, then link
// the list highest slot first (cell_next of animals not alive is untouched).
__global__ void eco_link_cells(Eco e) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * blockDim.x / 32;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) / 32; c < kCells; c += warps) {
        const int n = e.acnt[c], s = e.astart[c];
        for (int i = lane; i < n; i += 32) {
            const int a = e.alist[s + i];
            int r = 0;
            for (int j = 0; j < n; ++j) r += e.alist[s + j] > a;
            e.asort[s + r] = a;
        }
        __syncwarp();
        for (int i = lane; i < n; i += 32) e.cell_next[e.asort[s + i]] = i + 1 < n ? e.asort[s + i + 1] : -1;
        if (lane == 0) e.cell_head[c] = n ? e.asort[s] : -1;
    }
}

// ---- predation (src/main.cu:1251-1285) --------------------------------------------
// One thread per cell: the cell's attackers in ascending slot order, each
// biting the first other living member in list order.
__global__ void eco_bites(Eco e) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kCells; c += gridDim.x * blockDim.x) {
        const int n = e.acnt[c];
        if (n < 2) continue;
        const int *list = e.asort + e.astart[c];
        for (int i = n - 1; i >= 0; --i) {
            const int a = list[i];
            if (e.animals[a].alive != 1 || !e.bite_intent[a]) continue;
            for (int j = 0; j < n; ++j) {
                const int prey = list[j];
                if (prey == a || e.animals[prey].alive != 1) continue;
                ref::Animal &p = e.animals[prey];
                const float previous = p.health;
                p.health = previous + -kBiteDamage;
                p.pain = p.pain + kBiteDamage;
                e.flag[a] = 1;
                e.prey[a] = prey;
                if (previous <= kBiteDamage) {
                    p.alive = -2;
                    ref::Animal &q = e.animals[a];
                    q.energy = q.energy + fmaxf(0.0f, p.energy) * kMeatFraction;
                    q.taste[3] = 1.0f;
                    q.fullness = q.fullness + 1.0f;
                }
                break;
            }
        }
    }
}
__global__ void eco_bite_events(Eco e, int64_t step) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        if (!e.flag[a]) continue;
        atomicAdd(e.bites, 1);
        if (!e.bite_events) continue;
        const int event = e.base[0] + e.rank[a];
        if (event < 2 * e.P) {
            const ref::Animal &p = e.animals[e.prey[a]];
            e.bite_events[event] = ref::BiteEvent{step, e.animals[a].id, p.id, p.x, p.y};
        }
    }
}
__global__ void eco_finish_predation(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        if (e.animals[a].alive != -2) continue;
        e.animals[a].behavior.death_cause = 1;
        e.animals[a].alive = 0;
        atomicAdd(e.deaths, 1);
        atomicAdd(e.pred_deaths, 1);
    }
}

// ---- genome reclamation (src/main.cu:1302-1338, 436-454) ------------------------
// Reclamation. Counts and releases do not depend on list order, so they run
// over the pool slots by owner (the simulator keeps owner equal to list
// membership). Only the life record's float sum of weight changes follows
// the synapse list order: each reclaimed animal's list is ranked in shared
// memory by pointer jumping (Wyllie's list ranking) and the values are added
// in that order.
constexpr int kRankCap = 4096;                  // synapses ranked in shared memory; longer lists are walked
constexpr int kRankSmem = (2 * kRankCap) * 8 + kRankCap * (4 + 16 + 4 + 1) + 64;

__device__ __forceinline__ int dead_count(const Eco &e) { return e.rank[e.P - 1] + e.flag[e.P - 1]; }

__global__ void eco_reclaim_flags(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        const bool f = A.alive == 0 && (A.neuron_head >= 0 || A.synapse_head >= 0);
        e.flag[a] = f;
        const bool sane = A.synapse_count >= 0 && A.synapse_count <= e.ecap;
        if (f && !sane) atomicOr(e.status, ES_LIST);
        e.stmp[a] = f && sane ? A.synapse_count : 0;
    }
}
__global__ void eco_reclaim_list(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        if (!e.flag[a]) continue;
        e.dead[e.rank[a]] = a;
        e.gcount[a] = e.r_as[a] = e.r_ps[a] = e.r_an[a] = e.r_mn[a] = e.r_nc[a] = 0;
        e.r_total[a] = 0.0f;
    }
}
// Synapse slots of reclaimed animals: gathered (in no particular order) and released.
__global__ void eco_gather_synapses(Eco e) {
    if (dead_count(e) == 0) return;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < e.ecap; s += gridDim.x * blockDim.x) {
        const int a = e.sowner[s];
        if (a < 0 || a >= e.P || !e.flag[a]) continue;
        const int pos = atomicAdd(&e.gcount[a], 1);
        const int at = e.goff[a] + pos;
        if (pos < e.stmp[a] && at >= 0 && at < e.ecap) e.gslot[at] = s;
        e.sowner[s] = -1;
        atomicAnd(&e.sused[s / 32], ~(1u << (s % 32)));
    }
}
// Neuron slots of reclaimed animals: the record's counts, and released.
__global__ void eco_release_neurons(Eco e) {
    if (dead_count(e) == 0) return;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < e.ncap; n += gridDim.x * blockDim.x) {
        const int a = e.nowner[n];
        if (a < 0 || a >= e.P || !e.flag[a]) continue;
        const ref::NeuronGene &g = e.ngene[n];
        atomicAdd(&e.r_nc[a], 1);
        if (g.active) atomicAdd(&e.r_an[a], g.active);
        if (g.active && g.modulator != 0) atomicAdd(&e.r_mn[a], 1);
        e.nowner[n] = -1;
        atomicAnd(&e.nused[n / 32], ~(1u << (n % 32)));
    }
}

// Contribution of synapse slot s to the life record (src/main.cu:1317-1328).
__device__ __forceinline__ bool synapse_terms(const Eco &e, int s, bool &plastic, float &change) {
    const ref::SynapseGene &g = e.sgene[s];
    plastic = false;
    change = 0.0f;
    if ((unsigned)g.pre >= (unsigned)e.ncap || (unsigned)g.post >= (unsigned)e.ncap) {
        atomicOr(e.status, ES_SLOT);
        return false;
    }
    const ref::NeuronGene &pre = e.ngene[g.pre], &post = e.ngene[g.post];
    const bool live = g.active && pre.active && post.active;
    plastic = live && g.plasticity != 0 && !pre.inh_tx && excitatory(pre.type) && pre.modulator == 0 &&
              !post.inh_tx && excitatory(post.type);
    if (live) change = fabsf(e.sstate[s].w - g.w0);
    return live;
}
__device__ __forceinline__ uint32_t slot_hash(int slot, int bits) {
    return ((uint32_t)slot * 0x9E3779B1u) >> (32 - bits);
}

// One CTA per reclaimed animal (grid-stride over the list of reclaimed animals).
__global__ void __launch_bounds__(256) eco_rank_synapses(Eco e) {
    extern __shared__ __align__(16) unsigned char sm[];
    int *hkey = reinterpret_cast<int *>(sm);                 // 2 kRankCap: slot -> index table
    int *hval = hkey + 2 * kRankCap;
    int *slot = hval + 2 * kRankCap;                         // kRankCap each
    int *succ0 = slot + kRankCap, *succ1 = succ0 + kRankCap;
    int *dist0 = succ1 + kRankCap, *dist1 = dist0 + kRankCap;
    float *val = reinterpret_cast<float *>(dist1 + kRankCap);
    unsigned char *live = reinterpret_cast<unsigned char *>(val + kRankCap);
    __shared__ int bad, head_index, n_live, n_plastic;
    const int nd = dead_count(e);
    for (int d = blockIdx.x; d < nd; d += gridDim.x) {
        const int a = e.dead[d];
        const ref::Animal &A = e.animals[a];
        const int M = e.stmp[a];
        if (threadIdx.x == 0) {
            bad = e.gcount[a] != M || e.goff[a] < 0 || e.goff[a] > e.ecap - M;
            head_index = -1;
            n_live = n_plastic = 0;
        }
        __syncthreads();
        if (bad || M == 0) {
            if (threadIdx.x == 0 && bad) atomicOr(e.status, ES_LIST);
            __syncthreads();
            continue;
        }
        if (M > kRankCap) {                                   // long list: walked by one thread
            if (threadIdx.x == 0) {
                int k = 0, nl = 0, np = 0;
                float total = 0;
                for (int s = A.synapse_head; s >= 0 && k <= M; s = e.snext[s], ++k) {
                    if (s >= e.ecap) { atomicOr(e.status, ES_SLOT); break; }
                    bool pl;
                    float ch;
                    if (synapse_terms(e, s, pl, ch)) { ++nl; total += ch; }
                    np += pl;
                }
                if (k != M) atomicOr(e.status, ES_LIST);
                e.r_as[a] = nl; e.r_ps[a] = np; e.r_total[a] = total;
            }
            __syncthreads();
            continue;
        }
        int bits = 1;
        while ((1 << bits) < 2 * M) ++bits;
        const int T = 1 << bits;
        for (int i = threadIdx.x; i < T; i += blockDim.x) hkey[i] = -1;
        __syncthreads();
        const int *gs = e.gslot + e.goff[a];
        for (int i = threadIdx.x; i < M; i += blockDim.x) {
            const int k = gs[i];
            slot[i] = k;
            uint32_t h = slot_hash(k, bits);
            for (int probe = 0; probe < T; ++probe, h = (h + 1) & (T - 1))
                if (atomicCAS(&hkey[h], -1, k) == -1) { hval[h] = i; break; }
        }
        __syncthreads();
        auto lookup = [&](int k) {
            uint32_t h = slot_hash(k, bits);
            for (int probe = 0; probe < T; ++probe, h = (h + 1) & (T - 1)) {
                const int key = hkey[h];
                if (key == k) return hval[h];
                if (key == -1) return -1;
            }
            return -1;
        };
        for (int i = threadIdx.x; i < M; i += blockDim.x) {
            const int nx = e.snext[slot[i]];
            const int j = nx < 0 ? -1 : lookup(nx);
            if (nx >= 0 && j < 0) bad = 1;                    // successor outside this animal's slots
            succ0[i] = j;
            dist0[i] = j >= 0;
        }
        if (threadIdx.x == 0) head_index = A.synapse_head < 0 ? -1 : lookup(A.synapse_head);
        __syncthreads();
        int *sa = succ0, *sb = succ1, *da = dist0, *db = dist1;
        for (int span = 1; span < M; span <<= 1) {            // pointer jumping: hops to the list end
            for (int i = threadIdx.x; i < M; i += blockDim.x) {
                const int j = sa[i];
                db[i] = j >= 0 ? da[i] + da[j] : da[i];
                sb[i] = j >= 0 ? sa[j] : -1;
            }
            __syncthreads();
            int *t = sa; sa = sb; sb = t;
            t = da; da = db; db = t;
        }
        // a single chain of M entries from the head: the head is M - 1 hops from the end
        if (bad || head_index < 0 || da[head_index] != M - 1) {
            if (threadIdx.x == 0) atomicOr(e.status, ES_LIST);
            __syncthreads();
            continue;
        }
        for (int i = threadIdx.x; i < M; i += blockDim.x) {
            const int p = M - 1 - da[i];                      // list position
            bool pl;
            float ch;
            const bool lv = synapse_terms(e, slot[i], pl, ch);
            val[p] = ch;
            live[p] = lv;
            if (lv) atomicAdd(&n_live, 1);
            if (pl) atomicAdd(&n_plastic, 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float total = 0;
            for (int p = 0; p < M; ++p)
                if (live[p]) total += val[p];
            e.r_as[a] = n_live; e.r_ps[a] = n_plastic; e.r_total[a] = total;
        }
        __syncthreads();
    }
}

__global__ void eco_reclaim_finish(Eco e, int64_t step) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        if (!e.flag[a]) continue;
        ref::Animal &A = e.animals[a];
        if (e.r_nc[a] != A.neuron_count) atomicOr(e.status, ES_LIST);
        const int index = e.base[0] + e.rank[a];
        if (e.life && index < e.life_capacity) {
            ref::LifeRecord &rec = e.life[index];
            rec.body = A;
            rec.death_step = step;
            rec.active_neurons = e.r_an[a];
            rec.active_synapses = e.r_as[a];
            rec.modulatory_neurons = e.r_mn[a];
            rec.plastic_synapses = e.r_ps[a];
            rec.mean_abs_weight_change = e.r_as[a] > 0 ? e.r_total[a] / e.r_as[a] : 0;
        }
        A.neuron_head = A.synapse_head = -1;
        A.neuron_count = A.synapse_count = 0;
        for (int p = 0; p < kS + kM; ++p) A.ports[p] = -1;
    }
}

// ---- regrowth and senses (src/main.cu:1138-1144, 619-657) ------------------------
__global__ void eco_regrow(Eco e, int64_t step, unsigned long long seed, float renewal) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kCells; c += gridDim.x * blockDim.x) {
        if (e.food[c] != 0) continue;
        unsigned long long rng = seed_for(seed + (unsigned long long)step, (unsigned long long)c);
        if (uniform(rng) < renewal) e.food[c] = 1;
    }
}

__global__ void __launch_bounds__(128) eco_senses(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        if (A.alive != 1) continue;
        const float x = A.x, y = A.y, heading = A.heading;
        float *out = e.senses + (size_t)a * kS;
        for (int s = 0; s < 6; ++s) {
            const float angle = heading + (s % 3 - 1) * 0.7f;
            const float ca = nsx::cosf_cr(angle), sa = nsx::sinf_cr(angle);
            float level = 0;
            for (int range = 1; range <= 4; ++range) {
                const int c = cell_of(x + ca * range, y + sa * range);
                if (e.kind[c] == s / 3 && e.food[c] > 0) level += 0.25f;
            }
            out[s] = clampf(level, 0, 1);
        }
        out[6] = clampf((16.0f - A.energy) / 16.0f, 0, 1);
        out[7] = clampf(A.fullness / 8.0f, 0, 1);
        out[8] = clampf(A.pain / 3.0f, 0, 1);
        for (int k = 0; k < 3; ++k) out[9 + k] = clampf(A.taste[k], 0, 1);
        for (int direction = 0; direction < 3; ++direction) {
            const float angle = heading + (direction - 1) * 0.7f;
            const float ca = nsx::cosf_cr(angle), sa = nsx::sinf_cr(angle);
            float level = 0;
            for (int range = 1; range <= 4; ++range) {
                const int c = cell_of(x + ca * range, y + sa * range);
                const int *list = e.asort + e.astart[c];
                for (int j = 0, n = e.acnt[c]; j < n; ++j)
                    if (list[j] != a && e.animals[list[j]].alive == 1) level += 0.25f;
            }
            out[12 + direction] = clampf(level, 0, 1);
        }
        out[15] = clampf(A.taste[3], 0, 1);
        const int cc = cell_of(x, y);
        for (int kind = 0; kind < 3; ++kind)
            out[kContact + kind] = e.food[cc] > 0 && e.kind[cc] == kind ? 1.0f : 0.0f;
    }
}

// ---- reproduction with mutation (src/main.cu:364-525, 1340-1737) ----------------
// Parents (alive, energy >= 22 when the step starts) reproduce one after
// another in ascending slot order, each birth complete (copy, mutation, new
// states) before the next, every slot claim as claim_slot run alone. A birth
// is one CTA: the parent's lists come ranked in list order (gathered by owner,
// ranked in shared memory as for reclamation); claims run 256 at a time in
// parallel when each lands in its own hint word (claims in distinct words do
// not see each other, so the result is that of the sequence), otherwise one
// after another with the CTA searching for the first free word; the birth's
// RNG draws are taken in parallel by jumping ahead in the stream, and the
// records written in parallel; mutation runs on one thread over array copies
// of the child's lists, keeping the linked lists in global memory exactly as
// the reference's list surgery leaves them.
constexpr int kGrowth = 64;                      // list entries mutation may add (4 x at most 2)
constexpr int kD = 8;

__device__ __forceinline__ int randint(unsigned long long &s, int size) { return (int)(uniform(s) * size); }
// The xorshift64 state step (src/main.cu:331-334, before the output multiply)
// is linear over GF(2): s' = M s. Columns of M^(2^j) let a thread reach the
// state k steps ahead in log2(k) matrix-vector products, so the draws of a
// birth are taken in parallel, each thread a contiguous run of the stream,
// with the values the sequence gives.
constexpr int kJumpLevels = 24;                  // jumps up to 2^24 draws
__device__ __forceinline__ unsigned long long jump_state(const unsigned long long *jump, unsigned long long s,
                                                         unsigned k) {
    for (int level = 0; k; ++level, k >>= 1) {
        if (!(k & 1u)) continue;
        const unsigned long long *col = jump + level * 64;
        unsigned long long acc[4] = {0, 0, 0, 0};
#pragma unroll
        for (int b = 0; b < 64; ++b) acc[b & 3] ^= col[b] & (0ull - ((s >> b) & 1ull));
        s = (acc[0] ^ acc[1]) ^ (acc[2] ^ acc[3]);
    }
    return s;
}
// The draws k < count after state s0, (uint32)random64 each: k < na to
// a[k], the rest to b[k - na]. All threads; each takes a contiguous run. The
// state after the last draw goes to *final.
__device__ void parallel_draws(const unsigned long long *jump, unsigned long long s0, int na, uint32_t *a, int nb,
                               uint32_t *b, unsigned long long *final) {
    const int count = na + nb;
    const int chunk = (count + blockDim.x - 1) / blockDim.x;
    const int k0 = threadIdx.x * chunk, k1 = min(count, k0 + chunk);
    if (count == 0 && threadIdx.x == 0) *final = s0;
    if (k0 >= k1) return;
    unsigned long long st = jump_state(jump, s0, (unsigned)k0);
    for (int k = k0; k < k1; ++k) {
        const uint32_t v = (uint32_t)random64(st);
        if (k < na) a[k] = v;
        else b[k - na] = v;
    }
    if (k1 == count) *final = st;
}
__device__ __forceinline__ uint32_t state_hash(uint32_t seed) {
    uint32_t x = seed ? seed : 1u;
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
// initialize_neuron / initial_neuron_state (src/main.cu:408-422, src/physiology.cuh:179-202).
__device__ void birth_state(const Eco &e, int n, uint32_t seed) {
    const ref::NeuronGene &g = e.ngene[n];
    ref::NeuronState s;
    memset(&s, 0, sizeof s);
    s.v = g.el;
    const uint32_t x = state_hash(seed);
    s.rec_rng = x ? x : 1u;
    if (g.type == 2) {
        const float init[16] = {-56, 0, .2f, 0, 1, 0, 0, 1, 0, 0, 1, 1, 0, .04f, .01f, -56};
        for (int k = 0; k < 16; ++k) s.cell[k] = init[k];
        s.v = s.cell[15] - 9.342518882f;
    } else if (g.type == 3) {
        s.cell[0] = -50.0f; s.cell[1] = .05f;
        for (int k = 0; k < 4; ++k) s.cell[9 + k] = 1.0f;
        s.v = s.cell[0];
    } else if (g.type == 6) {
        s.cell[0] = g.el;
        s.cell[1] = g.vt;
    }
    e.nstate[n] = s;
}
__device__ void birth_neuron(const Eco &e, int n, int owner, int port, const ref::NeuronGene &g, int next,
                             uint32_t seed) {
    e.nowner[n] = owner;
    e.nnext[n] = next;
    e.nport[n] = port;
    e.ngene[n] = g;
    birth_state(e, n, seed);
    for (int b = 0; b < 4; ++b) e.pexc[(size_t)n * 4 + b] = 0;
    e.pinh[n] = 0;
    for (int k = 0; k < 6; ++k) e.modtick[(size_t)n * 6 + k] = 0;
    for (int h = 0; h < 9; ++h) e.hist[(size_t)h * e.ncap + n] = 0;
}
// initial_synapse_state (src/physiology.cuh:393-404).
__device__ void birth_synapse_state(const Eco &e, int s, uint32_t seed) {
    const ref::SynapseGene &g = e.sgene[s];
    uint32_t x = state_hash(seed);
    if (!x) x = 1;
    const int n = g.sites ? (g.sites > 64 ? 64 : g.sites) : 14;
    ref::SynapseState z;
    memset(&z, 0, sizeof z);
    z.w = g.w0;
    z.da_age = -1; z.spine = 1; z.st_age = -1;
    z.pre_age = 1000000; z.post_age = 1000000;
    z.last = -1000000;
    z.ready = n == 64 ? ~0ull : ((1ull << n) - 1ull);
    z.rng = x;
    z.slow = 1;
    e.sstate[s] = z;
}
__device__ void birth_synapse(const Eco &e, int s, int owner, const ref::SynapseGene &g, int next, uint32_t seed) {
    e.sowner[s] = owner;
    e.snext[s] = next;
    e.sgene[s] = g;
    birth_synapse_state(e, s, seed);
}
// claim_slot run alone (src/main.cu:364-385).
__device__ int claim_one(uint32_t *used, int capacity, int hint) {
    const int words = (capacity + 31) / 32;
    const int start = hint % words;
    for (int off = 0; off < words; ++off) {
        const int w = (start + off) % words;
        const uint32_t occ = used[w];
        if (~occ) {
            const int bit = __ffs(~occ) - 1;
            const int slot = w * 32 + bit;
            if (slot >= capacity) return -1;
            used[w] = occ | (1u << bit);
            return slot;
        }
    }
    return -1;
}
__device__ __forceinline__ void release_one(uint32_t *used, int slot) { used[slot >> 5] &= ~(1u << (slot & 31)); }

// Claims for hints hint0 + k, k < K, in order, into out[k]; the number that
// succeeded (K, or the index of the first failure). All threads of the CTA.
__device__ int claim_run(uint32_t *used, int capacity, int hint0, int K, int *out) {
    __shared__ int fail_at, found_off;
    const int words = (capacity + 31) / 32;
    const int t = threadIdx.x;
    int done = 0;
    while (done < K) {
        const int B = min(min((int)blockDim.x, K - done), words);
        int mine = -1;
        bool flag = false;
        if (t < B) {
            const int w = (hint0 + done + t) % words;
            const uint32_t occ = used[w];
            if (~occ) {
                const int slot = w * 32 + __ffs(~occ) - 1;
                if (slot < capacity) mine = slot;
                else flag = true;
            } else {
                flag = true;
            }
        }
        if (__syncthreads_or(flag)) {
            // one claim after another; the CTA searches 256 words at a time
            // for the first word with a free bit, as claim_slot scans from its hint
            if (t == 0) fail_at = -1;
            for (int i = 0; i < B; ++i) {
                const int start = (hint0 + done + i) % words;
                if (t == 0) found_off = INT_MAX;
                __syncthreads();
                for (int base = 0; base < words; base += blockDim.x) {
                    const int off = base + t;
                    const bool hit = off < words && ~used[(start + off) % words];
                    if (hit) atomicMin(&found_off, off);
                    if (__syncthreads_or(hit)) break;          // the same answer for every thread
                }
                if (t == 0) {
                    int slot = -1;
                    if (found_off != INT_MAX) {
                        const int w = (start + found_off) % words;
                        const uint32_t occ = used[w];
                        const int cand = w * 32 + __ffs(~occ) - 1;
                        if (cand < capacity) {
                            used[w] = occ | (1u << (cand & 31));
                            slot = cand;
                        }
                    }
                    out[done + i] = slot;
                    if (slot < 0) fail_at = done + i;
                }
                __syncthreads();
                if (fail_at >= 0) return fail_at;
            }
        } else {
            if (t < B) {
                used[mine >> 5] |= 1u << (mine & 31);     // each lane owns its word in this round
                out[done + t] = mine;
            }
            __syncthreads();
        }
        done += B;
    }
    return K;
}

__global__ void eco_parent_flags(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        const ref::Animal &A = e.animals[a];
        const bool f = A.alive == 1 && A.energy >= 22;
        // (a birth draws one value per neuron and synapse, twice; the jump
        // tables reach 2^kJumpLevels draws)
        const bool sane = A.neuron_count >= 0 && A.neuron_count <= e.ncap && A.synapse_count >= 0 &&
                          A.synapse_count <= e.ecap &&
                          (long long)A.neuron_count + A.synapse_count + 2 * kGrowth < (1ll << kJumpLevels);
        if (f && !sane) atomicOr(e.status, ES_LIST);
        e.pflag[a] = f && sane;
        e.pn_tmp[a] = f && sane ? A.neuron_count : 0;
        e.ps_tmp[a] = f && sane ? A.synapse_count : 0;
    }
}
__device__ __forceinline__ int parent_count(const Eco &e) { return e.prank[e.P - 1] + e.pflag[e.P - 1]; }
__global__ void eco_parent_list(Eco e) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < e.P; a += gridDim.x * blockDim.x) {
        if (!e.pflag[a]) continue;
        e.parents[e.prank[a]] = a;
        e.pn_cnt[a] = e.ps_cnt[a] = 0;
    }
}
__global__ void eco_gather_parents(Eco e) {
    if (parent_count(e) == 0) return;
    const int stride = gridDim.x * blockDim.x;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < e.ncap; n += stride) {
        const int a = e.nowner[n];
        if (a < 0 || a >= e.P || !e.pflag[a]) continue;
        const int pos = atomicAdd(&e.pn_cnt[a], 1), at = e.pn_off[a] + pos;
        if (pos < e.pn_tmp[a] && at >= 0 && at < e.ncap) e.pn_g[at] = n;
    }
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < e.ecap; s += stride) {
        const int a = e.sowner[s];
        if (a < 0 || a >= e.P || !e.pflag[a]) continue;
        const int pos = atomicAdd(&e.ps_cnt[a], 1), at = e.ps_off[a] + pos;
        if (pos < e.ps_tmp[a] && at >= 0 && at < e.ecap) e.ps_g[at] = s;
    }
}
// Ranks one list of M slots gathered at g (in any order) whose head is `head`
// and successors next[]: out[k] = the k-th slot in list order. All threads;
// returns whether the slots form exactly that list. Lists above kRankCap are
// walked by one thread.
__device__ bool rank_list(const int *g, int M, int head, const int *next, int cap, int *out, unsigned char *sm) {
    __shared__ int r_bad, r_head;
    int *hkey = reinterpret_cast<int *>(sm);
    int *hval = hkey + 2 * kRankCap;
    int *slot = hval + 2 * kRankCap;
    int *succ0 = slot + kRankCap, *succ1 = succ0 + kRankCap;
    int *dist0 = succ1 + kRankCap, *dist1 = dist0 + kRankCap;
    __syncthreads();
    if (threadIdx.x == 0) { r_bad = 0; r_head = -1; }
    if (M > kRankCap) {
        if (threadIdx.x == 0) {
            int k = 0;
            for (int s = head; s >= 0 && k <= M; s = next[s], ++k) {
                if (s >= cap) { r_bad = 1; break; }
                if (k < M) out[k] = s;
            }
            if (k != M) r_bad = 1;
        }
        __syncthreads();
        return !r_bad;
    }
    if (M == 0) {
        __syncthreads();
        return head < 0;
    }
    int bits = 1;
    while ((1 << bits) < 2 * M) ++bits;
    const int T = 1 << bits;
    for (int i = threadIdx.x; i < T; i += blockDim.x) hkey[i] = -1;
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        const int k = g[i];
        slot[i] = k;
        uint32_t h = slot_hash(k, bits);
        for (int probe = 0; probe < T; ++probe, h = (h + 1) & (T - 1))
            if (atomicCAS(&hkey[h], -1, k) == -1) { hval[h] = i; break; }
    }
    __syncthreads();
    auto lookup = [&](int k) {
        uint32_t h = slot_hash(k, bits);
        for (int probe = 0; probe < T; ++probe, h = (h + 1) & (T - 1)) {
            const int key = hkey[h];
            if (key == k) return hval[h];
            if (key == -1) return -1;
        }
        return -1;
    };
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        const int nx = next[slot[i]];
        const int j = nx < 0 ? -1 : lookup(nx);
        if (nx >= 0 && j < 0) r_bad = 1;
        succ0[i] = j;
        dist0[i] = j >= 0;
    }
    if (threadIdx.x == 0) r_head = head < 0 ? -1 : lookup(head);
    __syncthreads();
    int *sa = succ0, *sb = succ1, *da = dist0, *db = dist1;
    for (int span = 1; span < M; span <<= 1) {
        for (int i = threadIdx.x; i < M; i += blockDim.x) {
            const int j = sa[i];
            db[i] = j >= 0 ? da[i] + da[j] : da[i];
            sb[i] = j >= 0 ? sa[j] : -1;
        }
        __syncthreads();
        int *tmp = sa; sa = sb; sb = tmp;
        tmp = da; da = db; db = tmp;
    }
    const bool ok = !r_bad && r_head >= 0 && da[r_head] == M - 1;
    if (ok)
        for (int i = threadIdx.x; i < M; i += blockDim.x) out[M - 1 - da[i]] = slot[i];
    __syncthreads();
    return ok;
}
__global__ void __launch_bounds__(256) eco_rank_parents(Eco e) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int np = parent_count(e);
    for (int q = blockIdx.x; q < np; q += gridDim.x) {
        const int a = e.parents[q];
        const ref::Animal &A = e.animals[a];
        const int N = e.pn_tmp[a], M = e.ps_tmp[a];
        bool ok = e.pn_cnt[a] == N && e.ps_cnt[a] == M && e.pn_off[a] >= 0 && e.pn_off[a] <= e.ncap - N &&
                  e.ps_off[a] >= 0 && e.ps_off[a] <= e.ecap - M;
        ok = rank_list(e.pn_g + e.pn_off[a], ok ? N : 0, ok ? A.neuron_head : -1, e.nnext, e.ncap,
                       e.pn_list + e.pn_off[a], sm) && ok;
        ok = rank_list(e.ps_g + e.ps_off[a], ok ? M : 0, ok ? A.synapse_head : -1, e.snext, e.ecap,
                       e.ps_list + e.ps_off[a], sm) && ok;
        __syncthreads();
        if (!ok && threadIdx.x == 0) {
            atomicOr(e.status, ES_LIST);
            e.pn_cnt[a] = -1;                                 // not reproduced
        }
        __syncthreads();
    }
}

// ---- mutation on one thread (src/main.cu:1357-1660) --------------------------------
// The child's lists as arrays, tail first (list position i is entry len-1-i).
struct ChildLists {
    int *n, *s;
    int nn, ns;
};
__device__ int list_at(const int *l, int len, int ordinal) { return ordinal < len ? l[len - 1 - ordinal] : -1; }
__device__ void list_remove(int *l, int &len, int idx) {
    for (int i = idx; i + 1 < len; ++i) l[i] = l[i + 1];
    --len;
}
__device__ int random_hidden(const Eco &e, const ChildLists &c, const ref::Animal &b, unsigned long long &rng) {
    const int hidden = b.neuron_count - (kS + kM);
    if (hidden <= 0) return -1;
    int ordinal = randint(rng, hidden);
    for (int i = c.nn - 1; i >= 0; i -= 8) {                 // list order, eight loads before the tests
        int nb[8], pt[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) nb[j] = i - j >= 0 ? c.n[i - j] : -1;
#pragma unroll
        for (int j = 0; j < 8; ++j) pt[j] = nb[j] >= 0 ? e.nport[nb[j]] : 0;
        for (int j = 0; j < 8 && i - j >= 0; ++j)
            if (pt[j] < 0 && ordinal-- == 0) return nb[j];
    }
    return -1;
}
__device__ void remove_synapse_at(const Eco &e, ChildLists &c, ref::Animal &b, int target) {
    for (int i = c.ns - 1; i >= 0; --i) {
        if (c.s[i] != target) continue;
        const int next = e.snext[target];
        if (i == c.ns - 1) b.synapse_head = next;
        else e.snext[c.s[i + 1]] = next;
        --b.synapse_count;
        e.sowner[target] = -1;
        release_one(e.sused, target);
        list_remove(c.s, c.ns, i);
        return;
    }
}
__device__ void remove_hidden(const Eco &e, ChildLists &c, ref::Animal &b, int target, int *scratch) {
    if (target < 0 || e.nport[target] >= 0) return;
    int k = 0;                                                // synapses touching it, in list order
    for (int i = c.ns - 1; i >= 0; --i) {
        const ref::SynapseGene &g = e.sgene[c.s[i]];
        if (g.pre == target || g.post == target) scratch[k++] = c.s[i];
    }
    for (int j = 0; j < k; ++j) remove_synapse_at(e, c, b, scratch[j]);
    for (int i = c.nn - 1; i >= 0; --i) {
        if (c.n[i] != target) continue;
        const int next = e.nnext[target];
        if (i == c.nn - 1) b.neuron_head = next;
        else e.nnext[c.n[i + 1]] = next;
        --b.neuron_count;
        e.nowner[target] = -1;
        release_one(e.nused, target);
        list_remove(c.n, c.nn, i);
        return;
    }
}
__device__ void random_synapse(const Eco &e, const ChildLists &c, ref::SynapseGene &g, int child,
                               unsigned long long &rng) {
    const ref::Animal &body = e.animals[child];
    int active_sources = 0;
    float target_weight = 0;
    for (int i = c.nn - 1; i >= 0; i -= 8) {                 // list order, eight loads before the sums
        int act[8], pt[8];
        float aff[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int n = i - j >= 0 ? c.n[i - j] : -1;
            act[j] = n >= 0 ? e.ngene[n].active : 0;
            pt[j] = n >= 0 ? e.nport[n] : 0;
            aff[j] = n >= 0 ? e.ngene[n].affinity : 0.0f;
        }
        for (int j = 0; j < 8 && i - j >= 0; ++j) {
            if (!act[j]) continue;
            ++active_sources;
            if (pt[j] < 0 || pt[j] >= kS) target_weight += aff[j];
        }
    }
    g.pre = body.ports[0];
    int source_choice = randint(rng, active_sources);
    for (int i = c.nn - 1; i >= 0; --i)
        if (e.ngene[c.n[i]].active && source_choice-- == 0) { g.pre = c.n[i]; break; }
    g.post = body.ports[kS + randint(rng, kM)];
    float target_choice = uniform(rng) * target_weight;
    for (int i = c.nn - 1; i >= 0; --i) {
        const int n = c.n[i];
        const int port = e.nport[n];
        if (!e.ngene[n].active || (port >= 0 && port < kS)) continue;
        target_choice -= e.ngene[n].affinity;
        if (target_choice <= 0) { g.post = n; break; }
    }
    g.delay = (unsigned char)(1 + randint(rng, kD));
    g.branch = (unsigned char)randint(rng, 4);
    g.w0 = 0.5f + uniform(rng) * 3.5f;
    g.U = 0.55f;
    g.trec = 450.0f;
    g.tfac = 0;
    g.sites = 14;
    const bool pre_ok = (unsigned)g.pre < (unsigned)e.ncap, post_ok = (unsigned)g.post < (unsigned)e.ncap;
    if (!pre_ok || !post_ok) atomicOr(e.status, ES_SLOT);
    if (pre_ok && e.ngene[g.pre].type == 5) {
        g.w0 = 29.0f / (60.0f * 0.75f);
        g.U = 0.75f;
        g.trec = 50.0f;
        g.sites = 50;
        g.slow_rec = 7500.0f;
        g.slow_depl = 0.023f;
    }
    if (pre_ok && post_ok && e.ngene[g.pre].type == 0 && e.ngene[g.post].type == 1) {
        g.U = 0.1f;
        g.trec = 30.0f;
        g.tfac = 1700.0f;
    }
    const float draw = uniform(rng);
    g.plasticity = draw < 0.05f ? 5 : (draw < 0.10f ? 4 : (draw < 0.20f ? 3 : 2));
    g.receptors = g.plasticity == 3 ? (1 | 2) : (g.plasticity >= 4 ? 4 : 0);
    g.active = 1;
}
__device__ void prepend_neuron(const Eco &e, ChildLists &c, ref::Animal &b, int n, int child, const ref::NeuronGene &g,
                               unsigned long long &rng) {
    birth_neuron(e, n, child, -1, g, b.neuron_head, (uint32_t)random64(rng));
    b.neuron_head = n;
    ++b.neuron_count;
    c.n[c.nn++] = n;
}
__device__ void prepend_synapse(const Eco &e, ChildLists &c, ref::Animal &b, int s, int child,
                                const ref::SynapseGene &g, unsigned long long &rng) {
    birth_synapse(e, s, child, g, b.synapse_head, (uint32_t)random64(rng));
    b.synapse_head = s;
    ++b.synapse_count;
    c.s[c.ns++] = s;
}
__device__ void mutate(const Eco &e, ChildLists &c, int child, unsigned long long &rng, int *scratch) {
    ref::NeuronGene *NG = e.ngene;
    ref::SynapseGene *SG = e.sgene;
    const int mutations = 1 + randint(rng, 4);
    for (int m = 0; m < mutations; ++m) {
        const int choice = randint(rng, 12);
        ref::Animal body = e.animals[child];
        const int n = random_hidden(e, c, body, rng);
        const int syn = body.synapse_count ? list_at(c.s, c.ns, randint(rng, body.synapse_count)) : -1;
        if (choice == 0) {
            const float action = uniform(rng);
            if (action < 1.0f / 3.0f) {
                const int added = claim_one(e.nused, e.ncap, child * 131 + body.neuron_count);
                const int incoming = added >= 0 ? claim_one(e.sused, e.ecap, child * 257 + body.synapse_count) : -1;
                const int outgoing = incoming >= 0 ? claim_one(e.sused, e.ecap, child * 257 + body.synapse_count + 1) : -1;
                if (added >= 0 && incoming >= 0 && outgoing >= 0 && syn >= 0) {
                    int templ = syn;
                    for (int attempt = 0; attempt < 8; ++attempt) {
                        const int cand = list_at(c.s, c.ns, randint(rng, body.synapse_count));
                        const ref::SynapseGene &cg = SG[cand];
                        if ((unsigned)cg.pre >= (unsigned)e.ncap || (unsigned)cg.post >= (unsigned)e.ncap) {
                            atomicOr(e.status, ES_SLOT);
                            continue;
                        }
                        if (cg.active && NG[cg.pre].active && NG[cg.post].active) { templ = cand; break; }
                    }
                    const unsigned char type = (unsigned char)randint(rng, 7);
                    ref::NeuronGene g = e.profiles[type];
                    g.modulator = uniform(rng) < 0.12f ? (unsigned char)(1 + randint(rng, 3)) : 0;
                    prepend_neuron(e, c, body, added, child, g, rng);
                    ref::SynapseGene first = SG[templ], second = first;
                    first.post = added;
                    second.pre = added;
                    first.active = second.active = 1;
                    prepend_synapse(e, c, body, incoming, child, first, rng);
                    prepend_synapse(e, c, body, outgoing, child, second, rng);
                    e.animals[child] = body;
                } else {
                    if (outgoing >= 0) release_one(e.sused, outgoing);
                    if (incoming >= 0) release_one(e.sused, incoming);
                    if (added >= 0) release_one(e.nused, added);
                }
            } else if (action < 2.0f / 3.0f) {
                if (n >= 0) { remove_hidden(e, c, body, n, scratch); e.animals[child] = body; }
            } else if (n >= 0) {
                NG[n].active ^= 1;
            }
        } else if (choice == 1 && n >= 0) {
            const unsigned char active = NG[n].active;
            const unsigned char type = (unsigned char)randint(rng, 7);
            const unsigned char modulator = NG[n].modulator, inh = NG[n].inh_tx;
            const float affinity = NG[n].affinity;
            NG[n] = e.profiles[type];
            NG[n].active = active;
            NG[n].modulator = modulator;
            NG[n].inh_tx = inh;
            NG[n].affinity = affinity;
        } else if (choice == 2) {
            const int target = uniform(rng) < 0.2f ? body.ports[kS + randint(rng, kM)] : n;
            if (target < 0) continue;
            ref::NeuronGene &g = NG[target];
            if (g.type == 2) {
                float *scales = &g.lp.calcium;
                const int channel = randint(rng, 4);
                scales[channel] = clampf(scales[channel] * (0.9f + uniform(rng) * 0.2f), 0.2f, 3.0f);
            } else if (g.type == 3) {
                const int channel = randint(rng, 9);
                float &conductance = channel == 8 ? g.prinz_leak : g.prinz.g[channel];
                conductance = clampf((conductance + (channel >= 7 ? 2.0f : 0.0f)) * (0.9f + uniform(rng) * 0.2f), 0.0f,
                                     channel >= 7 ? 200.0f : 500000.0f);
            } else if (g.type == 5) {
                const int parameter = randint(rng, 4);
                if (parameter == 0) g.rec_base = clampf(g.rec_base + (uniform(rng) - 0.5f) * 2, 0, 30);
                if (parameter == 1) g.rec_gain = clampf(g.rec_gain + (uniform(rng) - 0.5f) * 10, 0, 300);
                if (parameter == 2) g.rec_event = clampf(g.rec_event * (0.9f + uniform(rng) * 0.2f), 0.5f, 6);
                if (parameter == 3) g.rec_decay = clampf(g.rec_decay * (0.9f + uniform(rng) * 0.2f), 1, 20);
            } else {
                g.vt = clampf(g.vt + (uniform(rng) - 0.5f) * 2, -60, -35);
            }
        } else if (choice == 3) {
            const float action = uniform(rng);
            if (action < 1.0f / 3.0f) {
                const int added = claim_one(e.sused, e.ecap, child * 257 + body.synapse_count);
                if (added >= 0) {
                    ref::SynapseGene g;
                    memset(&g, 0, sizeof g);
                    random_synapse(e, c, g, child, rng);
                    prepend_synapse(e, c, body, added, child, g, rng);
                    e.animals[child] = body;
                }
            } else if (action < 2.0f / 3.0f) {
                if (syn >= 0) { remove_synapse_at(e, c, body, syn); e.animals[child] = body; }
            } else if (syn >= 0) {
                SG[syn].active ^= 1;
            }
        } else if (choice == 4 && syn >= 0) {
            random_synapse(e, c, SG[syn], child, rng);
        } else if (choice == 5 && syn >= 0) {
            ref::SynapseGene &g = SG[syn];
            g.w0 = clampf(g.w0 + (uniform(rng) - 0.5f) * 0.5f, 0.1f, 8);
            g.sites = (unsigned char)clampf(g.sites + (uniform(rng) < 0.5f ? -1 : 1), 1, 64);
        } else if (choice == 6 && syn >= 0) {
            ref::SynapseGene &g = SG[syn];
            g.plasticity = (unsigned char)randint(rng, 6);
            g.receptors = g.plasticity == 3 ? (unsigned char)(1 + randint(rng, 3)) : (g.plasticity >= 4 ? 4 : 0);
            g.U = clampf(g.U + (uniform(rng) - 0.5f) * 0.1f, 0.02f, 0.8f);
            g.trec = clampf(g.trec + (uniform(rng) - 0.5f) * 50, 20, 1000);
            if (uniform(rng) < 0.15f) {
                g.slow_rec = g.slow_rec == 0 ? 7500.0f
                           : (uniform(rng) < 0.1f ? 0.0f : clampf(g.slow_rec + (uniform(rng) - 0.5f) * 500, 1000.0f, 20000.0f));
                g.slow_depl = g.slow_rec == 0 ? 0.0f : clampf(g.slow_depl + (uniform(rng) - 0.5f) * 0.01f, 0.0f, 0.1f);
            }
        } else if (choice == 7 && syn >= 0) {
            ref::SynapseGene &g = SG[syn];
            g.delay = (unsigned char)(1 + randint(rng, kD));
            g.tfac = g.tfac == 0 ? 500.0f + uniform(rng) * 3500.0f
                   : (uniform(rng) < 0.1f ? 0.0f : clampf(g.tfac + (uniform(rng) - 0.5f) * 200, 100, 4000));
            if (n >= 0) NG[n].b = clampf(NG[n].b + (uniform(rng) - 0.5f) * 5, 0, 150);
        } else if (choice == 8 && n >= 0) {
            ref::NeuronGene &g = NG[n];
            if (g.type == 0) {
                g.adp_b = clampf(g.adp_b + (uniform(rng) - 0.5f) * 20, 0, 200);
                g.adp_tau = clampf(g.adp_tau + (uniform(rng) - 0.5f) * 10, 10, 150);
            }
        } else if (choice == 9 && n >= 0) {
            if (NG[n].type != 5 && uniform(rng) < 0.5f) NG[n].modulator = (unsigned char)randint(rng, 4);
            else NG[n].inh_tx ^= 1;
        } else if (choice == 10) {
            const float action = uniform(rng);
            int afferent = -1;
            for (int attempt = 0; attempt < 12; ++attempt) {
                const int h = random_hidden(e, c, body, rng);
                if (h >= 0 && NG[h].sensory_channel >= 0) { afferent = h; break; }
            }
            if (action < 0.5f) {
                const int added = claim_one(e.nused, e.ncap, child * 131 + body.neuron_count);
                const int outgoing = added >= 0 ? claim_one(e.sused, e.ecap, child * 257 + body.synapse_count) : -1;
                if (added >= 0 && outgoing >= 0) {
                    int target = body.ports[kS + randint(rng, kM)];
                    for (int attempt = 0; attempt < 8; ++attempt) {
                        const int cand = list_at(c.n, c.nn, randint(rng, body.neuron_count));
                        if (cand >= 0 && (e.nport[cand] < 0 || e.nport[cand] >= kS)) { target = cand; break; }
                    }
                    const int source = afferent >= 0 && uniform(rng) < 0.5f ? afferent : body.ports[randint(rng, kS)];
                    if ((unsigned)source >= (unsigned)e.ncap) { atomicOr(e.status, ES_SLOT); continue; }
                    ref::NeuronGene g = NG[source];
                    g.modulator = 0;
                    g.active = 1;
                    prepend_neuron(e, c, body, added, child, g, rng);
                    ref::SynapseGene edge;
                    memset(&edge, 0, sizeof edge);
                    edge.pre = added;
                    edge.post = target;
                    edge.delay = (unsigned char)(1 + randint(rng, kD));
                    edge.branch = (unsigned char)randint(rng, 4);
                    edge.w0 = g.type == 5 ? 29.0f / (60.0f * 0.75f) : 1.0f;
                    edge.U = g.type == 5 ? 0.75f : 0.55f;
                    edge.trec = g.type == 5 ? 50.0f : 450.0f;
                    edge.sites = g.type == 5 ? 50 : 14;
                    edge.slow_rec = g.type == 5 ? 7500.0f : 0.0f;
                    edge.slow_depl = g.type == 5 ? 0.023f : 0.0f;
                    edge.active = 1;
                    prepend_synapse(e, c, body, outgoing, child, edge, rng);
                    e.animals[child] = body;
                } else {
                    if (outgoing >= 0) release_one(e.sused, outgoing);
                    if (added >= 0) release_one(e.nused, added);
                }
            } else if (action < 0.75f && afferent >= 0) {
                remove_hidden(e, c, body, afferent, scratch);
                e.animals[child] = body;
            } else if (afferent >= 0) {
                ref::NeuronGene &g = NG[afferent];
                const int channel = randint(rng, kS);
                const unsigned char active = g.active, inh = g.inh_tx;
                const float affinity = g.affinity;
                if (g.type == 5 && channel >= 6) g = e.profiles[0];
                else if (g.type != 5 && channel < 6) g = e.profiles[5];
                g.sensory_channel = (signed char)channel;
                g.active = active;
                g.inh_tx = inh;
                g.affinity = affinity;
            }
        } else if (choice == 11) {
            const int target = uniform(rng) < 0.3f ? body.ports[kS + randint(rng, kM)] : n;
            if (target >= 0)
                NG[target].affinity = clampf(NG[target].affinity * (uniform(rng) < 0.5f ? 0.5f : 2.0f), 0.125f, 256.0f);
        }
    }
}

// One CTA: the births of this step in ascending parent slot order (src/main.cu:1662-1737).
__global__ void __launch_bounds__(256) eco_births(Eco e) {
    __shared__ int s_child, s_n, s_s, s_start;
    __shared__ unsigned long long s_rng, s_final;
    __shared__ ref::Animal s_nb, s_parent;
    __shared__ unsigned long long s_jump[kJumpLevels * 64];
    const int t = threadIdx.x;
    const int np = parent_count(e);
    for (int i = t; i < kJumpLevels * 64; i += blockDim.x) s_jump[i] = e.jump[i];
    for (int q = 0; q < np; ++q) {
        const int a = e.parents[q];
        __syncthreads();
        if (e.pn_cnt[a] < 0) continue;                         // its lists failed the ranking
        if (t == 0) {
            s_parent = e.animals[a];
            unsigned long long r = s_parent.rng;
            s_start = randint(r, e.P);
            s_rng = r;
            s_child = INT_MAX;
        }
        __syncthreads();
        for (int base = 0; base < e.P; base += blockDim.x) {   // the first free animal slot from start
            const int j = base + t;
            const bool hit = j < e.P && e.animals[(s_start + j) % e.P].alive == 0;
            if (hit) atomicMin(&s_child, j);
            if (__syncthreads_or(hit)) break;                  // the same answer for every thread
        }
        if (s_child == INT_MAX) {
            if (t == 0) e.animals[a].rng = s_rng;
            continue;
        }
        const int child = (s_start + s_child) % e.P;
        if (t == 0) {
            e.animals[child].alive = -1;
            ref::Animal nb;
            memset(&nb, 0, sizeof nb);
            nb.neuron_head = nb.synapse_head = -1;
            for (int p = 0; p < kS + kM; ++p) nb.ports[p] = -1;
            unsigned long long r = s_rng;
            nb.x = clampf(s_parent.x + (uniform(r) - 0.5f) * 2, 0, (float)kW - 0.001f);
            nb.y = clampf(s_parent.y + (uniform(r) - 0.5f) * 2, 0, (float)kH - 0.001f);
            nb.heading = uniform(r) * 2 * 3.14159265358979323846f;
            nb.energy = 8;
            nb.health = 10;
            nb.generation = s_parent.generation + 1;
            s_rng = r;
            s_nb = nb;
        }
        __syncthreads();
        const int N = e.pn_tmp[a], M = e.ps_tmp[a];
        const int *pn = e.pn_list + e.pn_off[a], *ps = e.ps_list + e.ps_off[a];
        // neurons: claims, draws in order, copies
        // claims first (they draw nothing), then the birth's draws in the
        // reference's order: one per copied neuron, then one per copied synapse
        const int n_ok = claim_run(e.nused, e.ncap, child * 131, N, e.cn);
        const int s_ok = n_ok == N ? claim_run(e.sused, e.ecap, child * 257, M, e.cs) : 0;
        parallel_draws(s_jump, s_rng, n_ok, e.nseed, s_ok, e.sseed, &s_final);
        __syncthreads();
        if (t == 0) s_rng = s_final;
        __syncthreads();
        for (int k = t; k < n_ok; k += blockDim.x) {
            const int old = pn[k], n = e.cn[k];
            birth_neuron(e, n, child, e.nport[old], e.ngene[old], k ? e.cn[k - 1] : -1, e.nseed[k]);
            e.neuron_clone[old] = n;
        }
        __syncthreads();
        if (n_ok == N) {
            for (int k = t; k < s_ok; k += blockDim.x) {
                ref::SynapseGene g = e.sgene[ps[k]];
                if ((unsigned)g.pre >= (unsigned)e.ncap || (unsigned)g.post >= (unsigned)e.ncap) {
                    atomicOr(e.status, ES_SLOT);
                } else {
                    g.pre = e.neuron_clone[g.pre];
                    g.post = e.neuron_clone[g.post];
                }
                birth_synapse(e, e.cs[k], child, g, k ? e.cs[k - 1] : -1, e.sseed[k]);
            }
            __syncthreads();
        }
        if (n_ok < N || s_ok < M) {                            // pools full: the birth is undone
            for (int k = t; k < s_ok; k += blockDim.x) {
                e.sowner[e.cs[k]] = -1;
                atomicAnd(&e.sused[e.cs[k] >> 5], ~(1u << (e.cs[k] & 31)));
            }
            for (int k = t; k < n_ok; k += blockDim.x) {
                e.nowner[e.cn[k]] = -1;
                atomicAnd(&e.nused[e.cn[k] >> 5], ~(1u << (e.cn[k] & 31)));
            }
            __syncthreads();
            if (t == 0) {
                e.animals[child].alive = 0;
                e.animals[a].rng = s_rng;
            }
            continue;
        }
        if (t == 0) {
            ref::Animal nb = s_nb;
            for (int k = 0; k < n_ok; ++k) {
                const int port = e.nport[e.cn[k]];
                if (port >= 0 && port < kS + kM) nb.ports[port] = e.cn[k];
            }
            nb.neuron_head = n_ok ? e.cn[n_ok - 1] : -1;
            nb.neuron_count = n_ok;
            nb.synapse_head = s_ok ? e.cs[s_ok - 1] : -1;
            nb.synapse_count = s_ok;
            nb.id = atomicAdd(e.next_id, 1);
            nb.parent_id = s_parent.id;
            nb.alive = -1;
            e.animals[child] = nb;
            ChildLists c{e.cn, e.cs, n_ok, s_ok};
            unsigned long long r = s_rng;
            mutate(e, c, child, r, reinterpret_cast<int *>(e.sseed));   // sseed as scratch (reseeded below)
            s_n = c.nn;
            s_s = c.ns;
            s_rng = r;
        }
        __syncthreads();
        // new states: one draw per neuron, then per synapse, in list order
        parallel_draws(s_jump, s_rng, s_n, e.nseed, s_s, e.sseed, &s_final);
        __syncthreads();
        if (t == 0) s_rng = s_final;
        __syncthreads();
        for (int k = t; k < s_n; k += blockDim.x) birth_state(e, e.cn[s_n - 1 - k], e.nseed[k]);
        for (int k = t; k < s_s; k += blockDim.x) birth_synapse_state(e, e.cs[s_s - 1 - k], e.sseed[k]);
        for (int k = t; k < kS; k += blockDim.x) e.senses[(size_t)child * kS + k] = 0;
        for (int k = t; k < kM; k += blockDim.x) e.motors[(size_t)child * kM + k] = 0;
        __syncthreads();
        if (t == 0) {
            e.animals[child].rng = s_rng;
            ref::Animal p = s_parent;
            p.energy -= 10;
            ++p.behavior.offspring;
            p.rng = s_rng;
            e.animals[a] = p;
            __threadfence();
            e.animals[child].alive = 1;
            atomicAdd(e.births, 1);
        }
    }
}

template <class T> T *dev_zeros(std::vector<void *> &owned, size_t n) {
    void *p = nullptr;
    NSB_CHECK(cudaMalloc(&p, sizeof(T) * (n ? n : 1)));
    owned.push_back(p);
    NSB_CHECK(cudaMemset(p, 0, sizeof(T) * (n ? n : 1)));
    return static_cast<T *>(p);
}

class EcologyStage {
public:
    EcologyStage(const NsbWorldPools &p, const NsbWorldEcology &x) {
        if (!p.animals || !p.neurons || !p.synapses || !p.synapse_state || !p.neuron_owner || !p.synapse_owner ||
            !p.neuron_next || !p.synapse_next || !p.senses || !p.motors || p.animal_capacity <= 0 ||
            p.neuron_capacity <= 0 || p.synapse_capacity <= 0)
            throw std::runtime_error("Invalid world pools");
        if (!x.food || !x.kind || !x.cell_head || !x.cell_next || !x.bite_intent || !x.neuron_used ||
            !x.synapse_used || !x.founder_motor_steps || !x.founder_observed_steps || !x.deaths ||
            !x.predation_deaths || !x.bites || !x.life_count || !x.bite_event_count || x.life_capacity < 0 ||
            !x.neuron_clone || !x.births || !x.next_id || !p.neuron_state || !p.neuron_port || !p.pending_exc ||
            !p.pending_inh || !p.mod_event_tick || !p.spike_history)
            throw std::runtime_error("Invalid world ecology");
        x_.animals = static_cast<ref::Animal *>(const_cast<void *>(p.animals));
        x_.ngene = static_cast<ref::NeuronGene *>(const_cast<void *>(p.neurons));
        x_.sgene = static_cast<ref::SynapseGene *>(const_cast<void *>(p.synapses));
        x_.sstate = static_cast<ref::SynapseState *>(p.synapse_state);
        x_.nowner = const_cast<int *>(p.neuron_owner);
        x_.sowner = const_cast<int *>(p.synapse_owner);
        x_.nnext = const_cast<int *>(p.neuron_next);
        x_.snext = const_cast<int *>(p.synapse_next);
        x_.nstate = static_cast<ref::NeuronState *>(p.neuron_state);
        x_.nport = const_cast<int *>(p.neuron_port);
        x_.pexc = p.pending_exc;
        x_.pinh = p.pending_inh;
        x_.modtick = p.mod_event_tick;
        x_.hist = p.spike_history;
        x_.neuron_clone = x.neuron_clone;
        x_.births = x.births;
        x_.next_id = x.next_id;
        x_.senses = const_cast<float *>(p.senses);
        x_.motors = p.motors;
        x_.food = x.food; x_.kind = x.kind; x_.cell_head = x.cell_head; x_.cell_next = x.cell_next;
        x_.bite_intent = x.bite_intent;
        x_.nused = x.neuron_used; x_.sused = x.synapse_used;
        x_.f_motor = x.founder_motor_steps; x_.f_observed = x.founder_observed_steps;
        x_.deaths = x.deaths; x_.pred_deaths = x.predation_deaths; x_.bites = x.bites;
        x_.life = static_cast<ref::LifeRecord *>(x.life_records);
        x_.life_count = x.life_count;
        x_.bite_events = static_cast<ref::BiteEvent *>(x.bite_events);
        x_.bite_count = x.bite_event_count;
        x_.initial_count = x.initial_count;
        x_.instant_motors = x.instant_motors != 0;
        x_.life_capacity = x.life_records ? x.life_capacity : 0;
        x_.P = p.animal_capacity; x_.ncap = p.neuron_capacity; x_.ecap = p.synapse_capacity;
        const size_t P = (size_t)p.animal_capacity;
        x_.ecnt = dev_zeros<int>(owned_, kCells);
        x_.estart = dev_zeros<int>(owned_, kCells);
        x_.efill = dev_zeros<int>(owned_, kCells);
        x_.elist = dev_zeros<int>(owned_, P);
        x_.acnt = dev_zeros<int>(owned_, kCells);
        x_.astart = dev_zeros<int>(owned_, kCells);
        x_.afill = dev_zeros<int>(owned_, kCells);
        x_.alist = dev_zeros<int>(owned_, P);
        x_.asort = dev_zeros<int>(owned_, P);
        x_.flag = dev_zeros<unsigned char>(owned_, P);
        x_.prey = dev_zeros<int>(owned_, P);
        x_.rank = dev_zeros<int>(owned_, P);
        x_.base = dev_zeros<int>(owned_, 1);
        x_.active = dev_zeros<int>(owned_, P);
        x_.goff = dev_zeros<int>(owned_, P);
        x_.gcount = dev_zeros<int>(owned_, P);
        x_.gslot = dev_zeros<int>(owned_, (size_t)p.synapse_capacity);
        x_.dead = dev_zeros<int>(owned_, P);
        x_.stmp = dev_zeros<int>(owned_, P);
        x_.r_as = dev_zeros<int>(owned_, P);
        x_.r_ps = dev_zeros<int>(owned_, P);
        x_.r_an = dev_zeros<int>(owned_, P);
        x_.r_mn = dev_zeros<int>(owned_, P);
        x_.r_nc = dev_zeros<int>(owned_, P);
        x_.r_total = dev_zeros<float>(owned_, P);
        NSB_CHECK(cudaFuncSetAttribute(eco_rank_synapses, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
        NSB_CHECK(cudaFuncSetAttribute(eco_rank_parents, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
        const size_t NC = (size_t)p.neuron_capacity, EC = (size_t)p.synapse_capacity;
        x_.pflag = dev_zeros<unsigned char>(owned_, P);
        x_.prank = dev_zeros<int>(owned_, P);
        x_.parents = dev_zeros<int>(owned_, P);
        x_.pn_off = dev_zeros<int>(owned_, P);
        x_.ps_off = dev_zeros<int>(owned_, P);
        x_.pn_cnt = dev_zeros<int>(owned_, P);
        x_.ps_cnt = dev_zeros<int>(owned_, P);
        x_.pn_tmp = dev_zeros<int>(owned_, P);
        x_.ps_tmp = dev_zeros<int>(owned_, P);
        x_.pn_g = dev_zeros<int>(owned_, NC);
        x_.ps_g = dev_zeros<int>(owned_, EC);
        x_.pn_list = dev_zeros<int>(owned_, NC);
        x_.ps_list = dev_zeros<int>(owned_, EC);
        x_.cn = dev_zeros<int>(owned_, NC + kGrowth);
        x_.cs = dev_zeros<int>(owned_, EC + kGrowth);
        x_.nseed = dev_zeros<uint32_t>(owned_, NC + kGrowth);
        x_.sseed = dev_zeros<uint32_t>(owned_, EC + kGrowth);
        {   // columns of M^(2^j) for the xorshift64 step
            std::vector<unsigned long long> cols((size_t)kJumpLevels * 64);
            auto step = [](unsigned long long v) { v ^= v >> 12; v ^= v << 25; v ^= v >> 27; return v; };
            for (int b = 0; b < 64; ++b) cols[b] = step(1ull << b);
            for (int level = 1; level < kJumpLevels; ++level) {
                const unsigned long long *prev = &cols[(size_t)(level - 1) * 64];
                for (int b = 0; b < 64; ++b) {
                    unsigned long long v = prev[b], acc = 0;   // M^(2^(l-1)) applied to its own column
                    for (int k = 0; k < 64; ++k)
                        if ((v >> k) & 1ull) acc ^= prev[k];
                    cols[(size_t)level * 64 + b] = acc;
                }
            }
            auto *dj = dev_zeros<unsigned long long>(owned_, cols.size());
            NSB_CHECK(cudaMemcpy(dj, cols.data(), cols.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice));
            x_.jump = dj;
        }
        ref::NeuronGene prof[7];
        neuron_profiles(prof);
        auto *dprof = dev_zeros<ref::NeuronGene>(owned_, 7);
        NSB_CHECK(cudaMemcpy(dprof, prof, sizeof prof, cudaMemcpyHostToDevice));
        x_.profiles = dprof;
        x_.status = dev_zeros<int>(owned_, 1);
        NSB_CHECK(cudaMallocHost(&h_status_, sizeof(int)));
        int dev = 0;
        NSB_CHECK(cudaGetDevice(&dev));
        NSB_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
    }
    ~EcologyStage() {
        for (void *q : owned_) cudaFree(q);
        if (h_status_) cudaFreeHost(h_status_);
    }

    // body_step, spatial reset, index_animals, bite_animals, finish_predation.
    void body_step(int64_t step) {
        cudaStream_t st = 0;
        NSB_CHECK(cudaMemsetAsync(x_.ecnt, 0, sizeof(int) * kCells, st));
        eco_count_eaters<<<animal_grid(), 256, 0, st>>>(x_);
        eco_scan<int><<<1, 1024, 0, st>>>(x_.ecnt, kCells, x_.estart, nullptr, nullptr);
        NSB_CHECK(cudaMemsetAsync(x_.efill, 0, sizeof(int) * kCells, st));
        eco_place_eaters<<<animal_grid(), 256, 0, st>>>(x_);
        NSB_CHECK(cudaMemsetAsync(x_.active, 0, sizeof(int) * x_.P, st));
        eco_count_active<<<sms_ * 8, 256, 0, st>>>(x_);
        eco_body<<<(x_.P + 127) / 128, 128, 0, st>>>(x_);
        eco_commit_food<<<kCells / 256, 256, 0, st>>>(x_);
        index(st);
        NSB_CHECK(cudaMemsetAsync(x_.flag, 0, (size_t)x_.P, st));
        eco_bites<<<kCells / 128, 128, 0, st>>>(x_);
        // the event counter advances only when events are recorded (src/main.cu:1262-1268)
        eco_scan<unsigned char><<<1, 1024, 0, st>>>(x_.flag, x_.P, x_.rank, x_.bite_events ? x_.bite_count : nullptr,
                                                    x_.base);
        eco_bite_events<<<animal_grid(), 256, 0, st>>>(x_, step);
        eco_finish_predation<<<animal_grid(), 256, 0, st>>>(x_);
        finish(st);
    }

    void reclaim(int64_t step) {
        cudaStream_t st = 0;
        eco_reclaim_flags<<<animal_grid(), 256, 0, st>>>(x_);
        eco_scan<unsigned char><<<1, 1024, 0, st>>>(x_.flag, x_.P, x_.rank, x_.life_count, x_.base);
        eco_scan<int><<<1, 1024, 0, st>>>(x_.stmp, x_.P, x_.goff, nullptr, nullptr);
        eco_reclaim_list<<<animal_grid(), 256, 0, st>>>(x_);
        eco_gather_synapses<<<sms_ * 8, 256, 0, st>>>(x_);
        eco_release_neurons<<<sms_ * 8, 256, 0, st>>>(x_);
        eco_rank_synapses<<<sms_, 256, kRankSmem, st>>>(x_);
        eco_reclaim_finish<<<animal_grid(), 256, 0, st>>>(x_, step);
        finish(st);
    }

    // reproduce (src/main.cu:2765): parents in ascending slot order.
    void reproduce() {
        cudaStream_t st = 0;
        eco_parent_flags<<<animal_grid(), 256, 0, st>>>(x_);
        eco_scan<unsigned char><<<1, 1024, 0, st>>>(x_.pflag, x_.P, x_.prank, nullptr, nullptr);
        eco_scan<int><<<1, 1024, 0, st>>>(x_.pn_tmp, x_.P, x_.pn_off, nullptr, nullptr);
        eco_scan<int><<<1, 1024, 0, st>>>(x_.ps_tmp, x_.P, x_.ps_off, nullptr, nullptr);
        eco_parent_list<<<animal_grid(), 256, 0, st>>>(x_);
        eco_gather_parents<<<sms_ * 8, 256, 0, st>>>(x_);
        eco_rank_parents<<<sms_, 256, kRankSmem, st>>>(x_);
        eco_births<<<1, 256, 0, st>>>(x_);
        finish(st);
    }

    // regrow, spatial reset, index_animals, update_senses.
    void regrow_and_sense(int64_t step, unsigned long long seed, float renewal) {
        cudaStream_t st = 0;
        eco_regrow<<<kCells / 256, 256, 0, st>>>(x_, step, seed, renewal);
        index(st);
        eco_senses<<<(x_.P + 127) / 128, 128, 0, st>>>(x_);
        finish(st);
    }

private:
    int animal_grid() const { return std::min((x_.P + 255) / 256, sms_ * 8); }

    void index(cudaStream_t st) {
        NSB_CHECK(cudaMemsetAsync(x_.acnt, 0, sizeof(int) * kCells, st));
        eco_count_cells<<<animal_grid(), 256, 0, st>>>(x_);
        eco_scan<int><<<1, 1024, 0, st>>>(x_.acnt, kCells, x_.astart, nullptr, nullptr);
        NSB_CHECK(cudaMemsetAsync(x_.afill, 0, sizeof(int) * kCells, st));
        eco_place_cells<<<animal_grid(), 256, 0, st>>>(x_);
        eco_link_cells<<<kCells * 32 / 256, 256, 0, st>>>(x_);
    }

    void finish(cudaStream_t st) {
        NSB_CHECK(cudaGetLastError());
        NSB_CHECK(cudaMemcpyAsync(h_status_, x_.status, sizeof(int), cudaMemcpyDeviceToHost, st));
        NSB_CHECK(cudaStreamSynchronize(st));
        const int status = *h_status_;
        if (status) {
            NSB_CHECK(cudaMemset(x_.status, 0, sizeof(int)));
            if (status & ES_LIST) throw std::runtime_error("Animal neuron/synapse lists disagree with its counts");
            if (status & ES_SLOT) throw std::runtime_error("Pool slot outside the capacity");
            throw std::runtime_error("Food kind outside 0-2");
        }
    }

    Eco x_{};
    std::vector<void *> owned_;
    int *h_status_ = nullptr;
    int sms_ = 148;
};

template <class F> int guarded(void *h, F f) {
    try {
        if (!h) throw std::runtime_error("Invalid world ecology handle");
        f(*static_cast<EcologyStage *>(h));
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}

}  // namespace
}  // namespace nsb

extern "C" {

void *nsb_world_ecology_create(const NsbWorldPools *pools, const NsbWorldEcology *ecology) {
    try {
        if (!pools || !ecology) throw std::runtime_error("Missing world pools or ecology");
        return new nsb::EcologyStage(*pools, *ecology);
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return nullptr;
    }
}

void nsb_world_ecology_destroy(void *ecology) { delete static_cast<nsb::EcologyStage *>(ecology); }

int nsb_world_body_step(void *ecology, int64_t step) {
    return nsb::guarded(ecology, [&](nsb::EcologyStage &s) { s.body_step(step); });
}

int nsb_world_reclaim(void *ecology, int64_t step) {
    return nsb::guarded(ecology, [&](nsb::EcologyStage &s) { s.reclaim(step); });
}

int nsb_world_reproduce(void *ecology) {
    return nsb::guarded(ecology, [&](nsb::EcologyStage &s) { s.reproduce(); });
}

int nsb_world_regrow_and_sense(void *ecology, int64_t step, unsigned long long seed, float renewal_probability) {
    return nsb::guarded(ecology, [&](nsb::EcologyStage &s) { s.regrow_and_sense(step, seed, renewal_probability); });
}

}  // extern "C"
