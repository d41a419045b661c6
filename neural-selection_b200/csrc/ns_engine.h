// B200 neural-tick engine: batched brains, one persistent fused kernel per
// call (all ticks of the call inside one launch).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <memory>
#include <string>
#include <vector>
#include "ns_layout.h"
#include "ns_refabi.h"

namespace nsb {

struct Pools;

// One brain in the reference's host representation (gym_adapter/native.cpp:23-38).
struct BrainSpec {
    const ref::NeuronGene *genes = nullptr;
    int count = 0;
    const ref::SynapseGene *conns = nullptr;
    int edges = 0;
    const int *motors = nullptr;        // outputs entries, brain-local
    const int *sensory = nullptr;       // count entries, ABI sensory index (-1 none)
    const uint32_t *orig_n = nullptr;   // optional original neuron indices (reset seeds)
    const uint32_t *orig_s = nullptr;   // optional original synapse indices
};

struct EngineConfig {
    int max_delay = 8;          // 8 = the reference ABI; up to 31
    int block = 256;            // threads per CTA = neurons per small work unit
    int ctas_per_sm = 0;        // 0: from occupancy
    // Small brains are packed into units of block * unit_slots neurons; 0:
    // 3, or 1 when units of 3 cannot fill the GPU (lower per-tick latency).
    int unit_slots = 0;
    bool count_events = true;   // count synaptic arrivals on the device
    // Brains above the unit size on thread-block clusters: 1 always, 0 never,
    // -1 when the batch has too few units to fill the GPU (a latency mode: a
    // big brain spread over up to 8 SMs; in full batches the one-CTA path
    // has the higher throughput).
    int cluster_big = -1;
    // LP and Prinz cells per warp up to which a heavy unit steps them one
    // after another on the whole warp instead of each on its own lane; -1: the
    // build's default (per lane). Both forms give the same bits.
    int warp_cells = -1;
};

struct Stats {
    int brains, units, big_units, neurons, synapses, heavy, max_unit_neurons;
    int grid, block, smem_bytes, ctas_per_sm;
};

// Launch configuration of one bucket of work units.
struct BucketConfig {
    int block = 256;         // threads per CTA: 128 or 256 (warps per unit: 4 or 8)
    int coop = 0;            // warp-cooperative delivery
    int cluster = 1;         // CTAs per unit: 1, or the bucket's cluster size (big units only)
    int meta_cap = 6144;     // synapse meta words staged in shared memory per CTA
    // One-CTA light units: 1 integrates from a per-tick list of the neurons
    // that need it (full warps), 0 lets each thread integrate its own neurons
    // (one barrier per tick).
    int list = 1;
};

// Work units of one size class, launched together with one configuration.
// Buckets, in order: units above 4, 2 and 1 times the unit size (one big
// brain each; stepped by clusters of 8, 4 and 2 CTAs when clustered), packed
// units of small brains, and units with LP, Prinz or LFS cells (heavy).
constexpr int kBuckets = 5;
constexpr int kBucketHeavy = 4, kBucketPacked = 3;
struct Bucket {
    int ub = 0, ue = 0;              // units [ub, ue) in queue order
    int max_neurons = 0, max_synapses = 0;
    int cluster_size = 1;            // the cluster a unit of this bucket would use (8, 4, 2), or 1
    bool heavy = false;
    BucketConfig cfg;
    int hw = 8, smem = 0, grid = 0;  // launch shape derived from cfg (grid: CTAs, or clusters)
    int units() const { return ue - ub; }
};

class Engine {
public:
    // Builds device pools for `brains`; throws std::runtime_error on invalid input.
    Engine(const std::vector<BrainSpec> &brains, int channels, int outputs, const EngineConfig &cfg);
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    int brains() const { return n_brains_; }
    int channels() const { return channels_; }
    int outputs() const { return outputs_; }
    Stats stats() const;

    // ns_gpu_reset semantics with host arrays; synchronous.
    void reset_host(const uint8_t *mask, const uint32_t *seeds);
    // ns_gpu_step semantics with host arrays (validated); synchronous.
    void step_host(const float *input, const uint8_t *mask, int ticks, float gain, float *output, int *status);
    // Device-resident step: all pointers device memory, asynchronous on `stream`.
    // No validation; ticks in [1, 10000], inputs in [0, 1].
    void step_device(const float *d_input, const uint8_t *d_mask, int ticks, float gain, float *d_output,
                     int *d_status, cudaStream_t stream);
    // step_device with the kernel's scratch memory in a static device array
    // instead of engine buffers: allocates nothing. At most 2,097,152 synapses;
    // calls that overlap on the GPU race on the shared array.
    void step_noalloc(const float *d_input, const uint8_t *d_mask, int ticks, float gain, float *d_output,
                      int *d_status, cudaStream_t stream);
    // Captures step_device on the engine's own buffers into a CUDA graph and
    // replays it (one graph per (ticks, gain)).
    void step_graph(int ticks, float gain, cudaStream_t stream);
    // Delivery mode of the light buckets: serial per neuron, or
    // warp-cooperative release (faster for dense, active brains). Both give
    // identical results. The default is chosen from the synapse density;
    // set_cooperative sets every light bucket.
    bool cooperative() const { return buckets_[kBucketPacked].cfg.coop != 0; }
    void set_cooperative(bool coop);
    // Per-bucket autotuner: two whole-batch switches (every light bucket on
    // per-thread integration; every big brain on one CTA), then coordinate
    // descent over the buckets of work units; each candidate configuration
    // of a bucket (threads per CTA,
    // delivery mode, meta staging depth, list or per-thread integration, one
    // CTA or a cluster for big brains) is timed in whole steps on the
    // engine's own buffers, from the same restored state (so the call has no
    // visible effect on the brains), and kept when it saves more than 1 %.
    // Returns the packed bucket's delivery mode.
    bool autotune(int ticks, float gain, cudaStream_t stream);
    // The buckets and their current configurations.
    const std::vector<Bucket> &buckets() const { return buckets_; }
    // Sets one bucket's configuration (validated against its units and the
    // device's shared memory); throws std::runtime_error when it cannot run.
    void set_bucket(int b, const BucketConfig &cfg);
    // A global modulator pulse: at every tick divisible by `period` (> 0)
    // every neuron's plasticity sees the modulator bits `mod` (1 NE, 2 5-HT,
    // 4 DA) as if a modulatory synapse had released onto it. 0 turns it off.
    void set_global_modulation(int period, uint32_t mod);
    // Engine-owned device buffers for step_device / step_graph.
    float *dev_input() { return d_input_; }
    uint8_t *dev_mask() { return d_mask_; }
    float *dev_output() { return d_output_; }
    int *dev_status() { return d_status_; }

    // Canonical state dump of one brain (oracle layout, original order).
    void dump(int brain, uint32_t *neuron_words, uint32_t *synapse_words, int64_t *tick);
    // Load one brain's state from reference records (checkpoint / host state).
    void load_state(int brain, const ref::NeuronState *neurons, const ref::SynapseState *synapses,
                    const unsigned char (*history)[9], int64_t tick);
    // Inverse of load_state: one brain's state as reference records, its
    // 9-slot spike history ring (index tick % 9) and tick.
    void export_state(int brain, ref::NeuronState *neurons, ref::SynapseState *synapses,
                      unsigned char (*history)[9], int64_t *tick);
    // Synaptic arrivals counted since the last call to take_events().
    unsigned long long take_events();
    int64_t host_tick(int brain) const { return h_tick_[brain]; }
    // Overwrite one brain's tick counter.
    void set_tick(int brain, int64_t tick);

private:
    void launch(const float *d_input, const uint8_t *d_mask, int ticks, float gain, float *d_output,
                int *d_status, cudaStream_t stream);
    void launch_groups(const Pools &P, int *queue, const float *d_input, const uint8_t *d_mask, int ticks, float gain,
                       float *d_output, int *d_status, cudaStream_t stream);
    // One bucket's launch on `stream` (its queue counter already zeroed).
    void launch_bucket(const Bucket &B, const Pools &P, int *queue, const float *d_input, const uint8_t *d_mask,
                       int ticks, float gain, float *d_output, int *d_status, cudaStream_t stream) const;
    // Derives hw, smem and grid from the bucket's configuration; false when
    // the configuration cannot run on this device.
    bool shape_bucket(Bucket &B) const;
    void drop_graphs();
    template <class T> T *alloc(size_t n);
    struct Pools pools(bool events) const;

    int n_brains_ = 0, channels_ = 0, outputs_ = 0, max_delay_ = 8;
    int n_neurons_ = 0, n_synapses_ = 0, n_heavy_ = 0, n_units_ = 0, n_big_units_ = 0;
    int max_unit_neurons_ = 0, hw_ = 0, meta_cap_ = 0, max_unit_brains_ = 0, unit_cap_ = 256;
    int block_ = 256, sms_ = 0, smem_optin_ = 0, ctas_cap_ = 0, n_light_units_ = 0;
    std::vector<Bucket> buckets_;
    cudaStream_t bstream_[kBuckets] = {};
    cudaEvent_t fork_ = nullptr, join_[kBuckets] = {};
    bool count_events_ = true;
    int warp_cells_ = -1;        // EngineConfig::warp_cells
    bool coop_ = false;
    int pulse_period_ = 0;
    uint32_t pulse_mod_ = 0;
    std::vector<void *> allocations_;
    // device pools
    float *d_ngene_ = nullptr; uint32_t *d_nflags_ = nullptr; int *d_nsens_ = nullptr; int *d_nxidx_ = nullptr;
    float *d_xgene_ = nullptr; float *d_xstate_ = nullptr; uint32_t *d_nstate_ = nullptr; int *d_inptr_ = nullptr;
    uint32_t *d_smeta_ = nullptr; uint32_t *d_sgene_ = nullptr; uint32_t *d_sstate_ = nullptr;
    uint8_t *d_sarrived_ = nullptr; int16_t *d_slastp_ = nullptr;
    int64_t *d_btick_ = nullptr; int *d_bmotor_ = nullptr; int *d_bunit_ = nullptr;
    int4 *d_units_ = nullptr; int2 *d_unitb_ = nullptr; int *d_ubrain_ = nullptr;
    int *d_nbrain_ = nullptr; uint32_t *d_norig_ = nullptr; int *d_sbrain_ = nullptr; uint32_t *d_sorig_ = nullptr;
    uint8_t *d_rmask_ = nullptr;
    int *d_queue_ = nullptr; unsigned long long *d_events_ = nullptr;
    float *d_input_ = nullptr; uint8_t *d_mask_ = nullptr; float *d_output_ = nullptr; int *d_status_ = nullptr;
    uint32_t *d_seeds_ = nullptr;
    // host mirrors for layout mapping
    std::vector<int> h_noff_, h_soff_;   // caller-order prefix offsets of neurons / synapses per brain
    std::vector<int> h_npos_, h_spos_;   // (brain, original index) -> pool index
    std::vector<int> h_bunit_;           // brain -> work unit
    std::vector<int4> h_units_;          // {n0, nn, e0, ne} per unit
    std::vector<int> h_nxidx_;
    std::vector<uint32_t> h_nflags_;
    std::vector<int64_t> h_tick_;
    std::vector<uint32_t> h_sinfo_;      // per pool synapse: sites | receptors << 8
    std::vector<float> h_w0_;
    struct Graph { int ticks; float gain; cudaGraphExec_t exec; };
    std::vector<Graph> graphs_;
    cudaStream_t stream_ = nullptr;
    PhysConst K_{};
    unsigned long long events_host_ = 0;
};

}  // namespace nsb
