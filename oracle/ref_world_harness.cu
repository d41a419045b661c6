// ORACLE — test/benchmark infrastructure only.
//
// Times the reference world simulator's own neural-tick kernels on a given
// population. src/main.cu is compiled from the reference tree with main()
// renamed (the pattern of the reference's tests/plasticity_ablation.cu:6-8);
// this file fills its Device pools (src/main.cu:105-140) with the population
// and replays the neural part of its step loop (src/main.cu:2634-2728 and
// 2751-2758): selection of occupied slots or block-brain tiers, then 16 ticks
// of synapse_delivery / synapse_plasticity_delivery / neuron_step /
// synapse_plasticity (global-slot form) or brain_block_step tiers, then
// homeostasis. Built with the world binary's own flags (--use_fast_math,
// CMakeLists.txt:8). Needs a stub png.h (no image is ever written).
#define main ecological_application_main
#include "main.cu"
#undef main

#include <algorithm>
#include <cstring>

namespace {
using namespace sim;

template <class T> T *dalloc(size_t n) {
    T *p = nullptr;
    if (cudaMalloc(reinterpret_cast<void **>(&p), sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, sizeof(T) * (n ? n : 1));
    return p;
}

struct World {
    Device d{};
    void *select_tmp = nullptr;
    size_t select_bytes = 0;
    int block_mode = 0;   // 0 fused global-slot, 1 block-brain tiers + global fallback
    int64_t step = 0;
};
}  // namespace

extern "C" {

// One animal per brain, genomes given as the Gym ABI rows (neuron rows of 10,
// synapse rows of 11 floats, brain-local pre/post), decoded into the
// reference's NeuronGene / SynapseGene with the rules of ns_create
// (gym_adapter/native.cpp:53-75) using the reference's own profiles. A
// sensory neuron reads world sense `channel` when channel < S. Returns NULL if
// the population exceeds the pools.
void *ref_world_create(int brains, const int64_t *noff, const int64_t *soff, const float *neuron_rows,
                       const float *synapse_rows, const int *motors, int outputs, uint32_t seed, int block_mode) {
    if (brains > P || noff[brains] > NEURON_CAPACITY || soff[brains] > SYNAPSE_CAPACITY) return nullptr;
    auto *w = new World;
    w->block_mode = block_mode;
    Device &d = w->d;
    d.trace_animal = -1;
    d.animals = dalloc<Animal>(P);
    d.neurons = dalloc<NeuronGene>(NEURON_CAPACITY);
    d.synapses = dalloc<SynapseGene>(SYNAPSE_CAPACITY);
    d.neuron_state = dalloc<NeuronState>(NEURON_CAPACITY);
    d.synapse_state = dalloc<SynapseState>(SYNAPSE_CAPACITY);
    d.neuron_owner = dalloc<int>(NEURON_CAPACITY);
    d.synapse_owner = dalloc<int>(SYNAPSE_CAPACITY);
    d.occupied_neurons = dalloc<int>(NEURON_CAPACITY);
    d.occupied_synapses = dalloc<int>(SYNAPSE_CAPACITY);
    d.occupied_neuron_count = dalloc<int>(1);
    d.occupied_synapse_count = dalloc<int>(1);
    d.block_animals = dalloc<int>(P);
    d.block_animal_count = dalloc<int>(1);
    d.medium_animals = dalloc<int>(P);
    d.medium_animal_count = dalloc<int>(1);
    d.neuron_next = dalloc<int>(NEURON_CAPACITY);
    d.synapse_next = dalloc<int>(SYNAPSE_CAPACITY);
    d.neuron_port = dalloc<int>(NEURON_CAPACITY);
    d.pending_exc = dalloc<float>((size_t)NEURON_CAPACITY * DENDRITES);
    d.pending_inh = dalloc<float>(NEURON_CAPACITY);
    d.mod_event_tick = dalloc<unsigned long long>((size_t)NEURON_CAPACITY * 6);
    d.spike_history = dalloc<unsigned char>((size_t)HISTORY * NEURON_CAPACITY);
    d.senses = dalloc<float>((size_t)P * S);
    d.motors = dalloc<int>((size_t)P * M);
    d.trace_exc_arrivals = dalloc<int>(M); d.trace_exc_releases = dalloc<int>(M);
    d.trace_inh_arrivals = dalloc<int>(M); d.trace_exc_ns = dalloc<float>(M);
    d.trace_inh_ns = dalloc<float>(M); d.trace_peak_mv = dalloc<float>(M);
    if (!d.animals || !d.neurons || !d.synapses || !d.neuron_state || !d.synapse_state || !d.spike_history) {
        delete w;
        return nullptr;
    }
    const int64_t N = noff[brains], E = soff[brains];
    std::vector<Animal> animals(P);
    std::vector<NeuronGene> ng(N);
    std::vector<SynapseGene> sg(E);
    std::vector<NeuronState> ns(N);
    std::vector<SynapseState> ss(E);
    std::vector<int> nowner(NEURON_CAPACITY, -1), sowner(SYNAPSE_CAPACITY, -1);
    std::vector<int> nnext(N, -1), snext(E, -1), port(N, -1);
    std::vector<float> senses((size_t)P * S, 0.0f);
    std::vector<int> sensory(N);
    for (int64_t i = 0; i < N; ++i) {
        const float *q = neuron_rows + i * 10;
        NeuronGene g = initial_profile(static_cast<unsigned char>(q[0]));
        sensory[i] = (int)q[1];
        g.active = q[2]; g.inhibitory_transmitter = q[3]; g.modulator = q[4];
        g.capacitance_pf *= q[5]; g.leak_ns *= q[6]; g.threshold_mv = q[7];
        g.receptor_baseline_hz = 0; g.receptor_gain_hz = q[8]; g.receptor_event_ns = q[9];
        ng[i] = g;
    }
    for (int64_t i = 0; i < E; ++i) {
        const float *q = synapse_rows + i * 11;
        SynapseGene g{};
        g.pre = q[0]; g.post = q[1]; g.initial_weight_ns = q[2]; g.active = q[3]; g.delay = q[4];
        g.branch = q[5]; g.utilization = q[6]; g.recovery_ms = q[7]; g.facilitation_ms = q[8];
        g.plasticity = q[9]; g.mod_receptors = q[10]; g.release_sites = 14;
        if (g.delay > D) g.delay = (unsigned char)((g.delay - 1) % D + 1);   // the world ring holds D = 8
        sg[i] = g;
    }
    for (int a = 0; a < P; ++a) {
        Animal &b = animals[a];
        std::memset(&b, 0, sizeof b);
        b.neuron_head = b.synapse_head = -1;
        for (int p = 0; p < S + M; ++p) b.ports[p] = -1;
        if (a >= brains) continue;
        b.alive = 1; b.id = a; b.age = 1;
        b.neuron_count = (int)(noff[a + 1] - noff[a]);
        b.synapse_count = (int)(soff[a + 1] - soff[a]);
        if (b.neuron_count) b.neuron_head = (int)noff[a];
        if (b.synapse_count) b.synapse_head = (int)soff[a];
        for (int64_t n = noff[a]; n < noff[a + 1]; ++n) {
            nowner[n] = a;
            nnext[n] = n + 1 < noff[a + 1] ? (int)(n + 1) : -1;
            NeuronGene &g = ng[n];
            const int ch = sensory[n];
            // world senses: channels < S read senses[a*S + channel]
            g.sensory_channel = ch >= 0 && ch < S ? (signed char)ch : (signed char)-1;
            if (ch >= 0 && ch < S) senses[(size_t)a * S + ch] = 1.0f;
            ns[n] = initial_neuron_state(g, seed + (uint32_t)n * 7919u);
        }
        for (int m = 0; m < outputs && m < M; ++m) {
            const int64_t n = noff[a] + motors[(size_t)a * outputs + m];
            port[n] = S + m;
        }
        for (int64_t e = soff[a]; e < soff[a + 1]; ++e) {
            sowner[e] = a;
            snext[e] = e + 1 < soff[a + 1] ? (int)(e + 1) : -1;
            sg[e].pre += (int)noff[a];
            sg[e].post += (int)noff[a];
            ss[e] = initial_synapse_state(sg[e], seed + (uint32_t)e * 104729u);
        }
    }
    cudaMemcpy(d.animals, animals.data(), sizeof(Animal) * P, cudaMemcpyHostToDevice);
    cudaMemcpy(d.neurons, ng.data(), sizeof(NeuronGene) * N, cudaMemcpyHostToDevice);
    cudaMemcpy(d.synapses, sg.data(), sizeof(SynapseGene) * E, cudaMemcpyHostToDevice);
    cudaMemcpy(d.neuron_state, ns.data(), sizeof(NeuronState) * N, cudaMemcpyHostToDevice);
    cudaMemcpy(d.synapse_state, ss.data(), sizeof(SynapseState) * E, cudaMemcpyHostToDevice);
    cudaMemcpy(d.neuron_owner, nowner.data(), sizeof(int) * NEURON_CAPACITY, cudaMemcpyHostToDevice);
    cudaMemcpy(d.synapse_owner, sowner.data(), sizeof(int) * SYNAPSE_CAPACITY, cudaMemcpyHostToDevice);
    cudaMemcpy(d.neuron_next, nnext.data(), sizeof(int) * N, cudaMemcpyHostToDevice);
    cudaMemcpy(d.synapse_next, snext.data(), sizeof(int) * E, cudaMemcpyHostToDevice);
    cudaMemcpy(d.neuron_port, port.data(), sizeof(int) * N, cudaMemcpyHostToDevice);
    cudaMemcpy(d.senses, senses.data(), sizeof(float) * P * S, cudaMemcpyHostToDevice);
    auto slots = thrust::make_counting_iterator<int>(0);
    size_t b1 = 0, b2 = 0, b3 = 0, b4 = 0, b5 = 0, b6 = 0;
    cub::DeviceSelect::If(nullptr, b1, slots, d.occupied_neurons, d.occupied_neuron_count, NEURON_CAPACITY, OwnedSlot{d.neuron_owner});
    cub::DeviceSelect::If(nullptr, b2, slots, d.occupied_synapses, d.occupied_synapse_count, SYNAPSE_CAPACITY, OwnedSlot{d.synapse_owner});
    cub::DeviceSelect::If(nullptr, b3, slots, d.block_animals, d.block_animal_count, P, BlockAnimal{d.animals});
    cub::DeviceSelect::If(nullptr, b4, slots, d.medium_animals, d.medium_animal_count, P, MediumAnimal{d.animals});
    cub::DeviceSelect::If(nullptr, b5, slots, d.occupied_neurons, d.occupied_neuron_count, NEURON_CAPACITY, FallbackOwnedSlot{d.neuron_owner, d.animals});
    cub::DeviceSelect::If(nullptr, b6, slots, d.occupied_synapses, d.occupied_synapse_count, SYNAPSE_CAPACITY, FallbackOwnedSlot{d.synapse_owner, d.animals});
    w->select_bytes = std::max({b1, b2, b3, b4, b5, b6});
    cudaMalloc(&w->select_tmp, w->select_bytes);
    cudaFuncSetAttribute(brain_block_step<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         sizeof(BlockBrain<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>));
    cudaFuncSetAttribute(brain_block_step<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         sizeof(BlockBrain<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>));
    if (cudaDeviceSynchronize() != cudaSuccess) { delete w; return nullptr; }
    return w;
}

}  // extern "C"

namespace {
// Selection buffers of a World whose pools are already set.
bool alloc_selection(World &w) {
    Device &d = w.d;
    d.occupied_neurons = dalloc<int>(NEURON_CAPACITY);
    d.occupied_synapses = dalloc<int>(SYNAPSE_CAPACITY);
    d.occupied_neuron_count = dalloc<int>(1);
    d.occupied_synapse_count = dalloc<int>(1);
    d.block_animals = dalloc<int>(P);
    d.block_animal_count = dalloc<int>(1);
    d.medium_animals = dalloc<int>(P);
    d.medium_animal_count = dalloc<int>(1);
    auto slots = thrust::make_counting_iterator<int>(0);
    size_t b[6] = {};
    cub::DeviceSelect::If(nullptr, b[0], slots, d.occupied_neurons, d.occupied_neuron_count, NEURON_CAPACITY, OwnedSlot{d.neuron_owner});
    cub::DeviceSelect::If(nullptr, b[1], slots, d.occupied_synapses, d.occupied_synapse_count, SYNAPSE_CAPACITY, OwnedSlot{d.synapse_owner});
    cub::DeviceSelect::If(nullptr, b[2], slots, d.block_animals, d.block_animal_count, P, BlockAnimal{d.animals});
    cub::DeviceSelect::If(nullptr, b[3], slots, d.medium_animals, d.medium_animal_count, P, MediumAnimal{d.animals});
    cub::DeviceSelect::If(nullptr, b[4], slots, d.occupied_neurons, d.occupied_neuron_count, NEURON_CAPACITY, FallbackOwnedSlot{d.neuron_owner, d.animals});
    cub::DeviceSelect::If(nullptr, b[5], slots, d.occupied_synapses, d.occupied_synapse_count, SYNAPSE_CAPACITY, FallbackOwnedSlot{d.synapse_owner, d.animals});
    w.select_bytes = *std::max_element(b, b + 6);
    cudaMalloc(&w.select_tmp, w.select_bytes);
    cudaFuncSetAttribute(brain_block_step<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         sizeof(BlockBrain<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>));
    cudaFuncSetAttribute(brain_block_step<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         sizeof(BlockBrain<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>));
    return d.occupied_neurons && d.occupied_synapses && w.select_tmp && cudaDeviceSynchronize() == cudaSuccess;
}

// The neural part of the world loop for `step` (src/main.cu:2634-2728):
// selection, the device-to-host count reads, 16 ticks.
int neural_stage(World &w, int64_t step, int &neuron_count, int &block_count, int &medium_count) {
    Device &d = w.d;
    auto slots = thrust::make_counting_iterator<int>(0);
    int synapse_count = 0;
    neuron_count = block_count = medium_count = 0;
    if (w.block_mode) {
        cub::DeviceSelect::If(w.select_tmp, w.select_bytes, slots, d.block_animals, d.block_animal_count, P, BlockAnimal{d.animals});
        cub::DeviceSelect::If(w.select_tmp, w.select_bytes, slots, d.medium_animals, d.medium_animal_count, P, MediumAnimal{d.animals});
        cub::DeviceSelect::If(w.select_tmp, w.select_bytes, slots, d.occupied_neurons, d.occupied_neuron_count, NEURON_CAPACITY, FallbackOwnedSlot{d.neuron_owner, d.animals});
        cub::DeviceSelect::If(w.select_tmp, w.select_bytes, slots, d.occupied_synapses, d.occupied_synapse_count, SYNAPSE_CAPACITY, FallbackOwnedSlot{d.synapse_owner, d.animals});
    } else {
        cub::DeviceSelect::If(w.select_tmp, w.select_bytes, slots, d.occupied_neurons, d.occupied_neuron_count, NEURON_CAPACITY, OwnedSlot{d.neuron_owner});
        cub::DeviceSelect::If(w.select_tmp, w.select_bytes, slots, d.occupied_synapses, d.occupied_synapse_count, SYNAPSE_CAPACITY, OwnedSlot{d.synapse_owner});
    }
    cudaMemcpy(&neuron_count, d.occupied_neuron_count, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(&synapse_count, d.occupied_synapse_count, sizeof(int), cudaMemcpyDeviceToHost);
    if (w.block_mode) {
        cudaMemcpy(&block_count, d.block_animal_count, sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemcpy(&medium_count, d.medium_animal_count, sizeof(int), cudaMemcpyDeviceToHost);
    }
    // A failed launch returns 100 x the CUDA error + the launch site
    // (1 selection, 2/3 block tiers, 4 delivery, 5 fused plasticity+delivery,
    // 6 neuron_step, 7 plasticity).
#define NS_SITE(k) do { const cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) return 100 * (int)e_ + (k); } while (0)
    NS_SITE(1);
    if (block_count)
        brain_block_step<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>
            <<<block_count, 128, sizeof(BlockBrain<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>)>>>(
                d, d.block_animals, block_count, (step - 1) * TICKS);
    NS_SITE(2);
    if (medium_count)
        brain_block_step<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>
            <<<medium_count, 128, sizeof(BlockBrain<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>)>>>(
                d, d.medium_animals, medium_count, (step - 1) * TICKS);
    NS_SITE(3);
    for (int t = 0; t < TICKS; ++t) {
        const int64_t tick = (step - 1) * TICKS + t;
        if (synapse_count) {
            if (t == 0) {
                synapse_delivery<<<(synapse_count + NEURAL_BLOCK - 1) / NEURAL_BLOCK, NEURAL_BLOCK>>>(d, tick, synapse_count);
                NS_SITE(4);
            } else {
                synapse_plasticity_delivery<<<(synapse_count + NEURAL_BLOCK - 1) / NEURAL_BLOCK, NEURAL_BLOCK>>>(
                    d, tick - 1, tick, synapse_count);
                NS_SITE(5);
            }
        }
        if (neuron_count)
            neuron_step<<<(neuron_count + NEURAL_BLOCK - 1) / NEURAL_BLOCK, NEURAL_BLOCK>>>(d, tick, neuron_count);
        NS_SITE(6);
        if (synapse_count && t == TICKS - 1)
            synapse_plasticity<<<(synapse_count + NEURAL_BLOCK - 1) / NEURAL_BLOCK, NEURAL_BLOCK>>>(d, tick, synapse_count);
        NS_SITE(7);
    }
#undef NS_SITE
    return (int)cudaGetLastError();
}

// Homeostasis launches of the world loop (src/main.cu:2751-2758).
void homeostasis_stage(World &w, int neuron_count, int block_count, int medium_count) {
    Device &d = w.d;
    if (neuron_count) homeostasis_step<<<(neuron_count + 255) / 256, 256>>>(d, neuron_count);
    if (block_count) homeostasis_block_animals<<<(block_count + 127) / 128, 128>>>(d, d.block_animals, block_count);
    if (medium_count) homeostasis_block_animals<<<(medium_count + 127) / 128, 128>>>(d, d.medium_animals, medium_count);
}

// Pool pointers in the layout of the library's NsbWorldPools.
struct PoolsArg {
    void *animals, *plasticity_cohort, *neurons, *synapses, *neuron_state, *synapse_state;
    float *pending_exc, *pending_inh, *senses;
    unsigned long long *mod_event_tick;
    unsigned char *spike_history;
    int *neuron_owner, *synapse_owner, *neuron_next, *synapse_next, *neuron_port, *motors;
    int *trace_exc_arrivals, *trace_exc_releases, *trace_inh_arrivals;
    float *trace_exc_ns, *trace_inh_ns, *trace_peak_mv;
    int trace_animal, silence_senses, silence_contact, animal_capacity, neuron_capacity, synapse_capacity;
};
struct PoolsWorld {
    World w;
    int counts[3] = {0, 0, 0};
};
}  // namespace

extern "C" {

// One world step of the neural stage and its homeostasis; returns 0 or a CUDA error code.
int ref_world_step(void *p) {
    World &w = *static_cast<World *>(p);
    int n = 0, b = 0, m = 0;
    const int rc = neural_stage(w, ++w.step, n, b, m);
    if (rc) return rc;
    homeostasis_stage(w, n, b, m);
    return (int)cudaGetLastError();
}

// The reference's neural kernels on caller-owned pools (device pointers in
// the library's NsbWorldPools layout, the build's full capacities). The
// selection buffers are the harness's own. block_mode 0: the default fused
// global-slot kernels; 1: the --block-brains tiers.
void *ref_world_pools_create(const void *pools, int block_mode) {
    const PoolsArg &p = *static_cast<const PoolsArg *>(pools);
    if (p.animal_capacity != P || p.neuron_capacity != NEURON_CAPACITY || p.synapse_capacity != SYNAPSE_CAPACITY)
        return nullptr;
    auto *h = new PoolsWorld;
    Device &d = h->w.d;
    h->w.block_mode = block_mode;
    d.trace_animal = p.trace_animal;
    d.silence_senses = p.silence_senses != 0;
    d.silence_contact = p.silence_contact != 0;
    d.animals = static_cast<Animal *>(p.animals);
    d.plasticity_cohort = static_cast<PlasticityCohort *>(p.plasticity_cohort);
    d.neurons = static_cast<NeuronGene *>(p.neurons);
    d.synapses = static_cast<SynapseGene *>(p.synapses);
    d.neuron_state = static_cast<NeuronState *>(p.neuron_state);
    d.synapse_state = static_cast<SynapseState *>(p.synapse_state);
    d.pending_exc = p.pending_exc; d.pending_inh = p.pending_inh; d.senses = p.senses;
    d.mod_event_tick = p.mod_event_tick; d.spike_history = p.spike_history;
    d.neuron_owner = p.neuron_owner; d.synapse_owner = p.synapse_owner;
    d.neuron_next = p.neuron_next; d.synapse_next = p.synapse_next; d.neuron_port = p.neuron_port;
    d.motors = p.motors;
    d.trace_exc_arrivals = p.trace_exc_arrivals; d.trace_exc_releases = p.trace_exc_releases;
    d.trace_inh_arrivals = p.trace_inh_arrivals; d.trace_exc_ns = p.trace_exc_ns; d.trace_inh_ns = p.trace_inh_ns;
    d.trace_peak_mv = p.trace_peak_mv;
    if (!alloc_selection(h->w)) {
        delete h;
        return nullptr;
    }
    return h;
}

int ref_world_pools_step(void *p, long long step) {
    auto *h = static_cast<PoolsWorld *>(p);
    const int rc = neural_stage(h->w, step, h->counts[0], h->counts[1], h->counts[2]);
    if (rc) return rc;
    return (int)cudaDeviceSynchronize();
}

int ref_world_pools_homeostasis(void *p) {
    auto *h = static_cast<PoolsWorld *>(p);
    homeostasis_stage(h->w, h->counts[0], h->counts[1], h->counts[2]);
    return (int)cudaDeviceSynchronize();
}

void ref_world_pools_destroy(void *p) {
    auto *h = static_cast<PoolsWorld *>(p);
    Device &d = h->w.d;
    void *ptrs[] = {d.occupied_neurons, d.occupied_synapses, d.occupied_neuron_count, d.occupied_synapse_count,
                    d.block_animals, d.block_animal_count, d.medium_animals, d.medium_animal_count, h->w.select_tmp};
    for (void *q : ptrs) cudaFree(q);
    delete h;
}

// Launch limits of the neural kernels as this build compiled them, 4 values
// each (registers per thread, maximum threads per CTA, local bytes per
// thread, static shared bytes): synapse_delivery, synapse_plasticity_delivery,
// neuron_step, synapse_plasticity, then the two brain_block_step tiers.
int ref_world_kernel_limits(int *out) {
    const void *k[6] = {(const void *)synapse_delivery, (const void *)synapse_plasticity_delivery,
                        (const void *)neuron_step, (const void *)synapse_plasticity,
                        (const void *)brain_block_step<BLOCK_BRAIN_NEURONS, BLOCK_BRAIN_SYNAPSES, false>,
                        (const void *)brain_block_step<MEDIUM_BRAIN_NEURONS, MEDIUM_BRAIN_SYNAPSES, false>};
    for (int i = 0; i < 6; ++i) {
        cudaFuncAttributes a{};
        const cudaError_t e = cudaFuncGetAttributes(&a, k[i]);
        if (e != cudaSuccess) return -(int)e;
        out[4 * i] = a.numRegs;
        out[4 * i + 1] = a.maxThreadsPerBlock;
        out[4 * i + 2] = (int)a.localSizeBytes;
        out[4 * i + 3] = (int)a.sharedSizeBytes;
    }
    return 6;
}

// Layout of the Animal and PlasticityCohort fields the neural stage reads, as
// the reference builds them: sizes, then offsets of Animal.id, .age, .alive,
// .neuron_head, .synapse_head, .neuron_count, .synapse_count and
// PlasticityCohort.frozen.
int ref_world_animal_layout(uint64_t *out) {
    const uint64_t v[10] = {sizeof(Animal), sizeof(PlasticityCohort), offsetof(Animal, id), offsetof(Animal, age),
                            offsetof(Animal, alive), offsetof(Animal, neuron_head), offsetof(Animal, synapse_head),
                            offsetof(Animal, neuron_count), offsetof(Animal, synapse_count),
                            offsetof(PlasticityCohort, frozen)};
    for (int i = 0; i < 10; ++i) out[i] = v[i];
    return 10;
}

int ref_world_sync() { return (int)cudaDeviceSynchronize(); }

// Sum of total_spikes over the first n neuron slots (activity check).
long long ref_world_total_spikes(void *p, int n) {
    World &w = *static_cast<World *>(p);
    std::vector<NeuronState> s(n);
    cudaMemcpy(s.data(), w.d.neuron_state, sizeof(NeuronState) * n, cudaMemcpyDeviceToHost);
    long long t = 0;
    for (auto &x : s) t += x.total_spikes;
    return t;
}

void ref_world_destroy(void *p) {
    World *w = static_cast<World *>(p);
    Device &d = w->d;
    void *ptrs[] = {d.animals, d.neurons, d.synapses, d.neuron_state, d.synapse_state, d.neuron_owner,
                    d.synapse_owner, d.occupied_neurons, d.occupied_synapses, d.occupied_neuron_count,
                    d.occupied_synapse_count, d.block_animals, d.block_animal_count, d.medium_animals,
                    d.medium_animal_count, d.neuron_next, d.synapse_next, d.neuron_port, d.pending_exc,
                    d.pending_inh, d.mod_event_tick, d.spike_history, d.senses, d.motors, d.trace_exc_arrivals,
                    d.trace_exc_releases, d.trace_inh_arrivals, d.trace_exc_ns, d.trace_inh_ns, d.trace_peak_mv,
                    w->select_tmp};
    for (void *q : ptrs) cudaFree(q);
    delete w;
}

// The reference's slot allocator (src/main.cu:364-385) replayed on one
// thread: claims for hints[0..count) in order on the device bitmap `used`.
__global__ void ref_claim_kernel(uint32_t *used, int capacity, const int *hints, int count, int *slots) {
    if (threadIdx.x || blockIdx.x) return;
    for (int i = 0; i < count; ++i) slots[i] = claim_slot(used, capacity, hints[i]);
}
int ref_world_claim_sequential(uint32_t *d_used, int capacity, const int *d_hints, int count, int *d_slots) {
    ref_claim_kernel<<<1, 1>>>(d_used, capacity, d_hints, count, d_slots);
    return (int)cudaDeviceSynchronize();
}

// Layout facts of the reference build: the 20 values its checkpoint layout
// hash covers (src/checkpoint_impl.cuh:20-32), the hash, and the offsets of
// the neural checkpoint records (src/main.cu:164-177).
int ref_world_layout(uint64_t *values, uint64_t *hash, uint64_t *offsets) {
    const uint64_t v[] = {P, NEURON_CAPACITY, SYNAPSE_CAPACITY, S, M, W, H, DENDRITES, HISTORY, TICKS,
                          sizeof(Animal), sizeof(NeuronGene), sizeof(NeuronState), sizeof(SynapseGene),
                          sizeof(SynapseState), sizeof(CheckpointNeuron), sizeof(CheckpointSynapse),
                          sizeof(BehaviorTotals), sizeof(LifeRecord), sizeof(BiteEvent)};
    for (int i = 0; i < 20; ++i) values[i] = v[i];
    *hash = checkpoint_layout();
    const uint64_t o[] = {offsetof(CheckpointNeuron, gene), offsetof(CheckpointNeuron, state),
                          offsetof(CheckpointNeuron, pending_exc), offsetof(CheckpointNeuron, pending_inh),
                          offsetof(CheckpointNeuron, mod_event_tick), offsetof(CheckpointNeuron, spike_history),
                          offsetof(CheckpointSynapse, gene), offsetof(CheckpointSynapse, state)};
    for (int i = 0; i < 8; ++i) offsets[i] = o[i];
    return 20;
}


// ---- the reference's world ecology kernels (src/main.cu:612-657, 1138-1338) ----
// On caller-owned pools (NsbWorldPools layout) and ecology state
// (NsbWorldEcology layout), the build's full capacities. sequential = 1
// replays every contended kernel one animal at a time in ascending slot order
// (body_step, index_animals, bite_animals, reclaim_dead_genomes): before each
// launch the other candidates are relabelled (alive 1 -> 1000 or 0 -> 1001, or
// their bite intent cleared), so the unmodified kernel acts for one animal,
// and the labels are restored after it. sequential = 0 launches the kernels
// as the host loop does (src/main.cu:2745-2770).
struct EcoArg {
    int *food, *kind, *cell_head, *cell_next;
    unsigned char *bite_intent;
    uint32_t *neuron_used, *synapse_used;
    int *founder_motor_steps, *founder_observed_steps, *deaths, *predation_deaths, *bites;
    void *life_records;
    int *life_count;
    void *bite_events;
    int *bite_event_count;
    int initial_count, instant_motors, life_capacity;
    int *neuron_clone, *births, *next_id;
};

__global__ void ref_relabel(Device d, int keep, int from, int to) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < P && a != keep && d.animals[a].alive == from) d.animals[a].alive = to;
}
__global__ void ref_keep_intent(Device d, const unsigned char *saved, int keep) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < P) d.bite_intent[a] = a == keep ? saved[a] : 0;
}

struct EcoWorld {
    Device d{};
    unsigned char *saved_intent = nullptr;
    std::vector<int> alive;
};

static void read_alive(EcoWorld &h) {
    h.alive.resize(P);
    cudaMemcpy2D(h.alive.data(), sizeof(int), &h.d.animals[0].alive, sizeof(Animal), sizeof(int), P,
                 cudaMemcpyDeviceToHost);
}
static void index_stage(EcoWorld &h, int sequential) {
    Device &d = h.d;
    cudaMemset(d.cell_head, 0xff, W * H * sizeof(int));
    if (!sequential) {
        index_animals<<<(P + 127) / 128, 128>>>(d);
        return;
    }
    read_alive(h);
    for (int a = 0; a < P; ++a) {
        if (h.alive[a] != 1) continue;
        ref_relabel<<<(P + 255) / 256, 256>>>(d, a, 1, 1000);
        index_animals<<<(P + 127) / 128, 128>>>(d);
        ref_relabel<<<(P + 255) / 256, 256>>>(d, -1, 1000, 1);
    }
}

void *ref_world_eco_create(const void *pools, const void *ecology) {
    const PoolsArg &p = *static_cast<const PoolsArg *>(pools);
    const EcoArg &x = *static_cast<const EcoArg *>(ecology);
    if (p.animal_capacity != P || p.neuron_capacity != NEURON_CAPACITY || p.synapse_capacity != SYNAPSE_CAPACITY)
        return nullptr;
    if (x.life_records && x.life_capacity != LIFE_RECORD_CAPACITY) return nullptr;
    auto *h = new EcoWorld;
    Device &d = h->d;
    d.initial_count = x.initial_count;
    d.instant_motors = x.instant_motors != 0;
    d.trace_animal = -1;
    d.animals = static_cast<Animal *>(p.animals);
    d.plasticity_cohort = static_cast<PlasticityCohort *>(p.plasticity_cohort);
    d.neurons = static_cast<NeuronGene *>(p.neurons);
    d.synapses = static_cast<SynapseGene *>(p.synapses);
    d.neuron_state = static_cast<NeuronState *>(p.neuron_state);
    d.synapse_state = static_cast<SynapseState *>(p.synapse_state);
    d.pending_exc = p.pending_exc; d.pending_inh = p.pending_inh; d.senses = p.senses;
    d.mod_event_tick = p.mod_event_tick; d.spike_history = p.spike_history;
    d.neuron_owner = p.neuron_owner; d.synapse_owner = p.synapse_owner;
    d.neuron_next = p.neuron_next; d.synapse_next = p.synapse_next; d.neuron_port = p.neuron_port;
    d.motors = p.motors;
    d.food = x.food; d.kind = x.kind; d.cell_head = x.cell_head; d.cell_next = x.cell_next;
    d.bite_intent = x.bite_intent;
    d.neuron_used = x.neuron_used; d.synapse_used = x.synapse_used;
    d.founder_motor_steps = x.founder_motor_steps; d.founder_observed_steps = x.founder_observed_steps;
    d.deaths = x.deaths; d.predation_deaths = x.predation_deaths; d.bites = x.bites;
    d.life_records = static_cast<LifeRecord *>(x.life_records);
    d.life_count = x.life_count;
    d.bite_events = static_cast<BiteEvent *>(x.bite_events);
    d.bite_event_count = x.bite_event_count;
    d.neuron_clone = x.neuron_clone;
    d.births = x.births;
    d.next_id = x.next_id;
    if (cudaMalloc(&h->saved_intent, P) != cudaSuccess) {
        delete h;
        return nullptr;
    }
    return h;
}

int ref_world_eco_body(void *p, long long step, int sequential) {
    EcoWorld &h = *static_cast<EcoWorld *>(p);
    Device &d = h.d;
    if (!sequential) {
        body_step<<<(P + 127) / 128, 128>>>(d);
    } else {
        read_alive(h);
        for (int a = 0; a < P; ++a) {
            if (h.alive[a] != 1) continue;
            ref_relabel<<<(P + 255) / 256, 256>>>(d, a, 1, 1000);
            body_step<<<(P + 127) / 128, 128>>>(d);
            ref_relabel<<<(P + 255) / 256, 256>>>(d, -1, 1000, 1);
        }
    }
    index_stage(h, sequential);
    if (!sequential) {
        bite_animals<<<(P + 127) / 128, 128>>>(d, step);
    } else {
        std::vector<unsigned char> intent(P);
        cudaMemcpy(h.saved_intent, d.bite_intent, P, cudaMemcpyDeviceToDevice);
        cudaMemcpy(intent.data(), d.bite_intent, P, cudaMemcpyDeviceToHost);
        for (int a = 0; a < P; ++a) {
            if (!intent[a]) continue;
            ref_keep_intent<<<(P + 255) / 256, 256>>>(d, h.saved_intent, a);
            bite_animals<<<(P + 127) / 128, 128>>>(d, step);
        }
        cudaMemcpy(d.bite_intent, h.saved_intent, P, cudaMemcpyDeviceToDevice);
    }
    finish_predation<<<(P + 127) / 128, 128>>>(d);
    return (int)cudaDeviceSynchronize();
}

int ref_world_eco_reclaim(void *p, long long step, int sequential) {
    EcoWorld &h = *static_cast<EcoWorld *>(p);
    Device &d = h.d;
    if (!sequential) {
        reclaim_dead_genomes<<<(P + 127) / 128, 128>>>(d, step);
        return (int)cudaDeviceSynchronize();
    }
    read_alive(h);
    for (int a = 0; a < P; ++a) {
        if (h.alive[a] != 0) continue;
        ref_relabel<<<(P + 255) / 256, 256>>>(d, a, 0, 1001);
        reclaim_dead_genomes<<<(P + 127) / 128, 128>>>(d, step);
        ref_relabel<<<(P + 255) / 256, 256>>>(d, -1, 1001, 0);
    }
    return (int)cudaDeviceSynchronize();
}

// reproduce (src/main.cu:1662-1737); sequential = 1: one parent at a time in
// ascending slot order (the parents of this step relabelled 1 -> 1000 but one).
int ref_world_eco_reproduce(void *p, int sequential) {
    EcoWorld &h = *static_cast<EcoWorld *>(p);
    Device &d = h.d;
    if (!sequential) {
        reproduce<<<(P + 127) / 128, 128>>>(d);
        return (int)cudaDeviceSynchronize();
    }
    std::vector<Animal> a(P);
    cudaMemcpy(a.data(), d.animals, sizeof(Animal) * P, cudaMemcpyDeviceToHost);
    std::vector<int> parents;
    for (int i = 0; i < P; ++i)
        if (a[i].alive == 1 && a[i].energy >= 22) parents.push_back(i);
    for (int q : parents) {
        ref_relabel<<<(P + 255) / 256, 256>>>(d, q, 1, 1000);
        reproduce<<<(P + 127) / 128, 128>>>(d);
        ref_relabel<<<(P + 255) / 256, 256>>>(d, -1, 1000, 1);
    }
    return (int)cudaDeviceSynchronize();
}

int ref_world_eco_regrow_and_sense(void *p, long long step, unsigned long long seed, float renewal,
                                   int sequential) {
    EcoWorld &h = *static_cast<EcoWorld *>(p);
    Device &d = h.d;
    regrow<<<(W * H + 255) / 256, 256>>>(d, step, seed, renewal);
    index_stage(h, sequential);
    update_senses<<<(P + 127) / 128, 128>>>(d);
    return (int)cudaDeviceSynchronize();
}

void ref_world_eco_destroy(void *p) {
    auto *h = static_cast<EcoWorld *>(p);
    cudaFree(h->saved_intent);
    delete h;
}

}  // extern "C"
