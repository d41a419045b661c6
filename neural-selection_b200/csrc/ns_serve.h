// Serving loop for genome-evaluation episodes: continuous batching of
// episodes of different brain sizes and lengths into the persistent tick
// kernel, with the pole-on-cart environment, observation encoding and action
// decoding resident on the device.
//
// An episode is (registered genome, seed, number of steps). Requests are
// queued with their arrival time and admitted first come, first served, when
// (a) their bytes fit in the HBM budget, (b) the neurons in flight stay under
// the in-flight cap that bounds the step time, (c) an episode slot and pool
// ranges are free. Admitted brains of one round are packed into work units
// (best fit; larger brains alone) and written into free ranges of the device
// pools by one copy and one admission kernel. Every step then runs one
// tick-kernel launch over the active units and one environment kernel over
// the active slots; a finished episode masks its brain off on the device,
// reports through a host-mapped completion ring, and its unit's ranges
// return to the free lists once all of the unit's episodes have finished.
// Results depend only on the episode (genome, seed, steps), never on what
// else is in flight: each brain's arithmetic is independent of its unit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <string>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "ns_alloc.h"
#include "ns_engine.h"
#include "ns_internal.h"

namespace nsb {

struct ServeConfig {
    long long max_inflight_neurons = 4194304;   // admission cap on neurons in flight (bounds step time)
    double hbm_budget_bytes = 150e9;            // admission cap on bytes held by admitted episodes
    double synapses_per_neuron = 8.0;           // pool sizing
    double pool_headroom = 1.3;                 // pool capacity / in-flight cap (fragmentation room)
    int max_slots = 65536;                      // episodes in flight
    int max_brain_neurons = 4096;               // largest genome accepted
    int block = 256;
    int unit_slots = 3;                         // small brains packed into units of block*unit_slots neurons
    int ticks = 16;                             // neural ticks per environment step
    float gain = 230.0f;                        // input gain (ns_step input_gain)
    double smoothing = 0.4;                     // motor activity smoothing (SpikingPolicy smoothing)
    int max_delay = 8;
    long long staging_bytes = 64ll << 20;       // host staging per admission round
};

// One finished episode. Layout shared with nsb_serve_result (include/ns_b200.h).
struct ServeResult {
    uint64_t tag;
    int32_t genome, steps, reward, failures;    // steps run; steps without failure; pole falls
    uint32_t trace, seed;                       // FNV-1a over (action, motor counts) per step
    int32_t status, pad;                        // 0, or -1 when the neural state went non-finite
    double arrival_s, admit_s, done_s;          // server clock, seconds
};

struct ServeStats {
    long long steps, admitted, completed, queued, inflight, inflight_neurons, units;
    double neuron_ticks, busy_s, elapsed_s;
    unsigned long long events;
    long long pool_neurons, pool_synapses;
    double pool_bytes, inflight_bytes;
    double neuron_ticks_launched;   // neurons in flight x ticks, summed over launched steps
};

class Server {
public:
    explicit Server(const ServeConfig &cfg);
    ~Server();
    Server(const Server &) = delete;
    Server &operator=(const Server &) = delete;

    // Plans one genome (8 channels, 2 motors, cell types without LP/Prinz/LFS
    // models); returns its id. Throws std::runtime_error on invalid genomes.
    int register_genome(const BrainSpec &brain);
    // Queues episodes; arrival_s on the server clock (now() for "arrived now").
    void submit(int n, const int *genome, const uint32_t *seed, const int *steps, const uint64_t *tag,
                const double *arrival_s);
    // Background loop thread.
    void start();
    void stop();
    // Runs loop iterations on the calling thread until nothing is queued or in
    // flight (or max_iterations). Not while started.
    void run_until_idle(long long max_iterations);
    // Finished episodes (up to max), oldest first; returns the count.
    int poll(ServeResult *out, int max);
    double now() const;
    ServeStats stats();
    // Message of an error that stopped the background loop ("" if none).
    std::string error();
    int channels() const { return 8; }
    int outputs() const { return 2; }

private:
    struct Genome {
        int count = 0, edges = 0;
        std::vector<float> ngene;
        std::vector<uint32_t> nflags, norig, smeta, sgene, sorig;
        std::vector<int> nsens, inptr, motor;   // inptr: count + 1, from 0
        double bytes = 0;
    };
    struct Request {
        int genome;
        uint32_t seed;
        int steps;
        uint64_t tag;
        double arrival;
    };
    struct Unit {
        long long n0, nalloc, e0, ne;
        int nn;
        int remaining;
        std::vector<int> slots;
    };
    struct SlotInfo {
        int unit = -1;
        Request req{};
        double admit = 0;
        double bytes = 0;
        int neurons = 0;
    };

    void iteration();
    int admit_round();   // episodes admitted
    void retire(int slot);
    void upload_unit_table();
    void harvest(int ring);
    void drain();
    void loop();

    ServeConfig cfg_;
    int dev_ = 0, sms_ = 0, unit_cap_ = 768, hw_ = 0, smem_ = 0, grid_cap_ = 0;
    long long ncap_ = 0, ecap_ = 0;
    std::vector<Genome> genomes_;
    std::mutex genome_mu_;

    // queue and results (shared with the caller's thread)
    std::mutex mu_;
    std::deque<Request> queue_;
    std::deque<ServeResult> done_;
    std::atomic<bool> running_{false};
    std::thread thread_;
    std::string error_;

    // device pools
    std::vector<void *> allocations_;
    template <class T> T *alloc(size_t n);
    float *d_ngene_ = nullptr; uint32_t *d_nflags_ = nullptr; int *d_nsens_ = nullptr; int *d_nxidx_ = nullptr;
    uint32_t *d_nstate_ = nullptr; int *d_inptr_ = nullptr; float *d_xdummy_ = nullptr;
    uint32_t *d_smeta_ = nullptr; uint32_t *d_sgene_ = nullptr; uint32_t *d_sstate_ = nullptr;
    uint8_t *d_sarrived_ = nullptr; int16_t *d_slastp_ = nullptr;
    int64_t *d_btick_ = nullptr; int *d_bmotor_ = nullptr;
    int4 *d_units_ = nullptr; int2 *d_unitb_ = nullptr; int *d_ubrain_ = nullptr;
    int *d_queue_ = nullptr; unsigned long long *d_events_ = nullptr;
    float *d_input_ = nullptr; uint8_t *d_mask_ = nullptr; float *d_output_ = nullptr; int *d_status_ = nullptr;
    void *d_slot_ = nullptr;            // per-slot episode state (ns_serve.cu)
    unsigned char *d_stage_ = nullptr;  // device copy of an admission round
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    cudaEvent_t t0_[2] = {nullptr, nullptr};
    unsigned char *h_stage_[2] = {nullptr, nullptr};   // pinned staging, one per pipeline parity
    void *h_ring_[2] = {nullptr, nullptr};             // host-mapped completion rings
    void *d_ring_[2] = {nullptr, nullptr};

    // host bookkeeping (loop thread only)
    RangeAllocator nalloc_, ealloc_;
    std::vector<int> free_slots_, free_units_;
    std::vector<Unit> units_;            // by unit id
    std::vector<char> unit_live_;
    std::vector<SlotInfo> slots_;
    std::vector<int> active_units_;
    bool table_dirty_ = true;
    int n_table_ = 0;
    long long iter_ = 0;
    bool pending_[2] = {false, false};
    // counters written by the loop thread, read by stats()
    std::atomic<long long> inflight_neurons_{0}, inflight_{0}, admitted_{0}, completed_{0}, steps_run_{0},
        n_units_live_{0};
    std::atomic<double> inflight_bytes_{0}, neuron_ticks_{0}, busy_s_{0}, launched_ticks_{0};
    std::chrono::steady_clock::time_point epoch_;
    float keep_ = 0.6f, smooth_ = 0.4f;
};

}  // namespace nsb
