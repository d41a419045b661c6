// Internal interfaces shared by the batch engine (ns_engine.cu) and the
// serving engine (ns_serve.cu): the device pool view the tick kernel reads,
// the unit planner, and launch helpers for kernels that live in ns_engine.cu
// (where the physiology constants are bound).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdexcept>
#include <string>
#include <vector>

#include "ns_engine.h"
#include "ns_layout.h"

namespace nsb {

#define NSB_CHECK(x)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kMetaCap = 6144;       // default synapse meta words staged in shared memory per unit
constexpr int kMaxUnitBrains = 128;  // brains packed into one small unit
constexpr int kMaxBrainNeurons = 16384;

// Device pools as the tick kernel sees them.
struct Pools {
    const float4 *ngene;     // N x 4
    const uint32_t *nflags;  // N
    const int *nsens;        // N
    const int *nxidx;        // N (index into heavy arrays, -1)
    const float *xgene;      // H x 16
    float *xstate;           // H x 16
    uint32_t *nstate;        // N x 16
    const int *inptr;        // N + 1
    const uint32_t *smeta;   // E
    const uint32_t *sgene;   // E x 8
    uint32_t *sstate;        // E x 16
    uint8_t *sarrived;       // E
    int16_t *slastp;         // E (-1 between calls)
    int64_t *btick;
    const int *bmotor;       // B x outputs, global neuron index
    const int4 *units;       // {n0, nn, e0, ne}
    const int2 *unitb;       // {first entry in ubrain, nb}
    const int *ubrain;       // unit brain lists (caller brain indices), pool order
    int channels, outputs, hw;
    unsigned long long *events;
    int pulse_period;        // > 0: a global modulator pulse at every tick divisible by it
    uint32_t pulse_mod;      // its modulator bits (1 NE, 2 5-HT, 4 DA)
    // Synapse meta words a CTA stages in shared memory (a unit with more
    // reads them from global memory); the launch's dynamic shared memory is
    // sized for it.
    int meta_cap = kMetaCap;
    // Heavy units: a warp with more LP and Prinz cells than this steps each on
    // its own lane, with fewer one after another on the whole warp; -1: the
    // build's default (kWarpCellsMax).
    int warp_cells = -1;
};

// Host plan of a set of brains: work units and every pool record, indexed
// from 0 (neurons, synapses, brains in caller order).
struct Plan {
    int n_neurons = 0, n_synapses = 0, n_units = 0, n_light_units = 0, n_big_units = 0, n_heavy = 0;
    int max_unit_neurons = 0, max_unit_brains = 0;
    // Light units stepped by thread-block clusters of 8, 4 and 2 CTAs (big
    // brains), first in queue order, then the light units of one CTA; the
    // largest unit of each group.
    int n_cluster[3] = {0, 0, 0};
    int max_small = 0, max_big = 0, max_heavy = 0;
    std::vector<int4> units;              // {n0, nn, e0, ne}, light units first, each by size descending
    std::vector<int2> unitb;              // {first entry in brain_order, nb}
    std::vector<int> brain_order;         // unit brain lists (caller indices)
    std::vector<float> ngene;             // N x 16
    std::vector<uint32_t> nflags, norig;
    std::vector<int> nsens, nbrain, nxidx;
    std::vector<float> xgene;             // heavy cells x 16
    std::vector<int> inptr;               // N + 1
    std::vector<uint32_t> smeta, sgene, sorig;
    std::vector<int> sbrain;
    std::vector<int> bmotor;              // B x outputs, pool neuron index
    std::vector<int> noff, soff;          // caller-order prefix offsets per brain
    std::vector<int> npos, spos;          // (brain, original index) -> pool index
    std::vector<int> bunit;               // brain -> unit
};

// Packs brains into units of at most unit_cap neurons (best-fit decreasing;
// a larger brain is a unit of its own; brains with LP/Prinz/LFS cells in
// separate, heavy units) and lays out their records. With heavy_target > 0
// the heavy units hold about 1/heavy_target of the heavy brains' neurons each
// (at most unit_cap), so that they spread over that many SMs. Throws
// std::runtime_error on invalid input with the reference's messages.
Plan make_plan(const std::vector<BrainSpec> &brains, int channels, int outputs, int max_delay, int unit_cap,
               bool cluster_big = false, int heavy_target = 0);
// Cluster sizes of the three big-brain groups, in queue order.
constexpr int kClusterSizes[3] = {8, 4, 2};

// Correctly rounded constant exponentials of the physiology (host side).
PhysConst make_constants();

// Spike-ring words per tick for units of up to max_unit_neurons neurons.
int spike_words(int max_unit_neurons, int block);
// Dynamic shared memory of the light tick kernel for hw ring words and
// meta_cap staged synapse meta words.
int tick_smem_bytes(int hw, int meta_cap = kMetaCap);
// Binds the physiology constants and the tick kernels' shared-memory limit on
// the current device (idempotent).
void prepare_tick_kernels(int smem);
// Dynamic shared memory of the serving loop's tick kernel (per-thread
// integration, warp-cooperative delivery).
int serve_smem_bytes(int hw, int meta_cap = kMetaCap);
// Resident CTAs per SM of the serving loop's tick kernel.
int tick_occupancy(int block, int smem);
// The serving loop's tick kernel over units [0, n_units) of P (queue reset on
// `stream`).
void launch_tick_light(const Pools &P, int n_units, int grid, int block, int smem, int *queue, const float *input,
                       const uint8_t *mask, float *output, int *status, int ticks, float gain, cudaStream_t stream);

}  // namespace nsb
