// Host-side record layouts that must match the reference byte for byte.
//
// The reference's Gym GPU entry point ns_gpu_create (gym_adapter/gpu.cu:66-109
// of mixic/neural-selection) receives opaque `Brain*` handles made by the host
// library's ns_create (gym_adapter/native.cpp:23-38) and reads their
// std::vector members directly. For this library's ns_gpu_create to accept
// those handles (and for its own ns_create handles to be accepted by the
// reference), the structs below reproduce that layout: same member types in
// the same order, so libstdc++ lays them out identically. Member names are
// this project's own. Sizes and offsets are checked by static_assert against
// the values of the reference built with g++ on x86-64 (NeuronGene 124 B,
// NeuronState 120 B, SynapseGene 40 B, SynapseState 80 B).
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace nsb {
namespace ref {

struct LpScale { float calcium, calcium_k, h, leak; };
struct PrinzG { float g[8]; };

struct NeuronGene {                     // src/physiology.cuh:29-45
    float cap, gl, el, vt, slope, a, tau_w, b, vr, adp_b, adp_tau;
    unsigned char type, active, modulator, inh_tx;
    LpScale lp;
    PrinzG prinz;
    float prinz_leak;
    signed char sensory_channel;
    float rec_base, rec_gain, rec_event, rec_decay, affinity;
};

struct NeuronState {                    // src/physiology.cuh:50-58
    float v, w, adp, inh, depol, log_ampa;
    float dend[4];
    float cell[16];                     // the LP / Prinz / LFS union (64 bytes)
    int total;
    unsigned char spike;
    float rec_ns;
    uint32_t rec_rng;
};

struct SynapseGene {                    // src/physiology.cuh:59-65
    float w0, U, trec, tfac;
    int pre, post;
    unsigned char delay, active, plasticity, branch, sites, receptors;
    float slow_rec, slow_depl;
};

struct SynapseState {                   // src/physiology.cuh:66-76
    float w, ru, pre_tr, post_tr, eltp, eltd, da_age, spine, st_age, pre_age, post_age;
    int64_t last;
    uint64_t ready;
    uint32_t rng;
    unsigned char arrived;
    float slow;
};

// gym_adapter/native.cpp:23-38
struct Brain {
    std::vector<NeuronGene> genes;
    std::vector<SynapseGene> connections;
    std::vector<NeuronState> neurons;
    std::vector<SynapseState> synapses;
    std::vector<int> motors;
    std::vector<std::array<unsigned char, 9>> history;
    std::vector<std::array<float, 4>> excitation;
    std::vector<float> inhibition;
    std::vector<unsigned char> modulation;
    std::vector<int> sensory;
    std::vector<uint32_t> original_neurons, original_synapses;
    int channels;
    int64_t tick = 0;
};

// World checkpoint records of the neural pools (src/main.cu:164-177): packed
// per occupied slot, ascending slot order (src/checkpoint_impl.cuh:190-211).
struct CheckpointNeuron {
    int slot, owner, next, port;
    NeuronGene gene;
    NeuronState state;
    float pending_exc[4], pending_inh;
    unsigned long long mod_event_tick[6];
    unsigned char spike_history[9];
};
struct CheckpointSynapse {
    int slot, owner, next;
    SynapseGene gene;
    SynapseState state;
};

// The 20 build constants the reference's checkpoint layout hash covers
// (src/checkpoint_impl.cuh:20-32): P, neuron and synapse capacities, S, M, W,
// H, DENDRITES, HISTORY, TICKS (src/main.cu:33-47, src/physiology.cuh:17),
// then the sizes of Animal, NeuronGene, NeuronState, SynapseGene,
// SynapseState, CheckpointNeuron, CheckpointSynapse, BehaviorTotals,
// LifeRecord and BiteEvent as the reference builds them with nvcc on x86-64.
constexpr uint64_t kLayoutValues[20] = {32768, 4194304, 8388608, 19, 5, 128, 128, 4, 9, 16,
                                        472, 124, 120, 40, 80, 344, 136, 528, 504, 24};
// FNV-1a over those values (the reference's checkpoint_layout()).
constexpr uint64_t layout_hash() {
    uint64_t h = 1469598103934665603ull;
    for (uint64_t v : kLayoutValues) {
        h ^= v;
        h *= 1099511628211ull;
    }
    return h;
}
static_assert(layout_hash() == 0x2b1cd1c766eebf82ull, "checkpoint layout hash");

// World simulator records (src/main.cu:66-104): the animal body with its
// observer-only behaviour counters, the plasticity cohort, and the records the
// world step appends (life records of reclaimed genomes, bite events).
struct Behavior {                        // src/main.cu:66-74; age bins 0-99, 100-299, 300+
    int opportunities[3][2][3];
    int accepted[3][2][3];
    int empty_steps[3][2], empty_eat[3][2];
    float approach_progress[3][3];
    float approach_travel[3][3];
    int first_b_age, offspring, death_cause;
};
static_assert(sizeof(Behavior) == 276, "Behavior layout");
struct Animal {
    float x, y, heading, energy, health, fullness, pain;
    float taste[4];
    float muscle[3];
    unsigned long long rng;
    int id, parent_id, generation, age, alive;
    int neuron_head, synapse_head, neuron_count, synapse_count;
    int ports[19 + 5];
    Behavior behavior;
};
struct LifeRecord {                      // src/main.cu:85-90
    Animal body;
    int64_t death_step;
    int active_neurons, active_synapses, modulatory_neurons, plastic_synapses;
    float mean_abs_weight_change;
};
struct BiteEvent {                       // src/main.cu:91-95
    int64_t step;
    int attacker_id, prey_id;
    float x, y;
};
static_assert(sizeof(LifeRecord) == 504 && offsetof(LifeRecord, death_step) == 472, "LifeRecord layout");
static_assert(sizeof(BiteEvent) == 24, "BiteEvent layout");
struct PlasticityCohort {                // src/main.cu:98-104
    int id, assigned, frozen, initial_age, initial_offspring;
    int final_age, final_offspring, alive, death_cause;
    int neurons, synapses, generation;
    float initial_energy, initial_health;
    int64_t start_step, observed_step, death_step;
};
static_assert(sizeof(Animal) == 472 && offsetof(Animal, id) == 64 && offsetof(Animal, age) == 76 &&
              offsetof(Animal, alive) == 80 && offsetof(Animal, neuron_head) == 84 &&
              offsetof(Animal, synapse_count) == 96, "Animal layout");
static_assert(sizeof(PlasticityCohort) == 80 && offsetof(PlasticityCohort, frozen) == 8 &&
              offsetof(PlasticityCohort, start_step) == 56, "PlasticityCohort layout");

static_assert(sizeof(NeuronGene) == 124, "NeuronGene layout");
static_assert(offsetof(NeuronGene, type) == 44 && offsetof(NeuronGene, lp) == 48, "NeuronGene layout");
static_assert(offsetof(NeuronGene, sensory_channel) == 100 && offsetof(NeuronGene, rec_base) == 104, "NeuronGene layout");
static_assert(sizeof(NeuronState) == 120 && offsetof(NeuronState, cell) == 40, "NeuronState layout");
static_assert(offsetof(NeuronState, spike) == 108 && offsetof(NeuronState, rec_ns) == 112, "NeuronState layout");
static_assert(sizeof(SynapseGene) == 40 && offsetof(SynapseGene, delay) == 24 && offsetof(SynapseGene, slow_rec) == 32,
              "SynapseGene layout");
static_assert(sizeof(SynapseState) == 80 && offsetof(SynapseState, last) == 48 && offsetof(SynapseState, rng) == 64 &&
              offsetof(SynapseState, slow) == 72, "SynapseState layout");
static_assert(sizeof(CheckpointNeuron) == 344 && offsetof(CheckpointNeuron, gene) == 16 &&
              offsetof(CheckpointNeuron, state) == 140 && offsetof(CheckpointNeuron, pending_exc) == 260 &&
              offsetof(CheckpointNeuron, pending_inh) == 276 && offsetof(CheckpointNeuron, mod_event_tick) == 280 &&
              offsetof(CheckpointNeuron, spike_history) == 328, "CheckpointNeuron layout");
static_assert(sizeof(CheckpointSynapse) == 136 && offsetof(CheckpointSynapse, gene) == 12 &&
              offsetof(CheckpointSynapse, state) == 56, "CheckpointSynapse layout");

}  // namespace ref

// initial_profile(0..6) of the reference (host; ns_abi.cu).
void neuron_profiles(ref::NeuronGene *out);
}  // namespace nsb
