// C ABI of the B200 neural tick.
//
// The ns_* and ns_gpu_* entry points keep the reference's signatures, argument
// meaning, validation messages and return conventions
// (gym_adapter/native.cpp:45-108 and gym_adapter/gpu.cu:67-123 of
// mixic/neural-selection), so gym_adapter/adapter.py and gym_adapter/gpu.py can
// load this library in place of libgym_brain.so / libgym_brain_gpu.so. Brain
// handles share the reference's host layout (ns_refabi.h), so ns_gpu_create
// accepts handles made by either library. Every call runs the neural tick on
// the GPU; there is no CPU execution path. Exceptions never cross the ABI:
// failures return -1 or NULL and leave a thread-local message for ns_error.
//
// nsb_* entry points are this library's extensions (extended delay ring,
// bulk creation, device-resident stepping, CUDA-graph replay, state readback).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ns_engine.h"
#include "ns_refabi.h"
#include "ns_serve.h"

using namespace nsb;

namespace {

thread_local std::string g_error;

// Reference parameter profiles (src/physiology.cuh:82-176), host side.
ref::NeuronGene blank_gene() {
    ref::NeuronGene g;
    std::memset(&g, 0, sizeof g);
    g.sensory_channel = -1;
    g.rec_decay = 3.0f;
    g.affinity = 1.0f;
    return g;
}
ref::NeuronGene naud(bool inhibitory) {
    ref::NeuronGene g = blank_gene();
    if (inhibitory) {
        g.cap = 59; g.gl = 2.9f; g.el = -62; g.vt = -42; g.slope = 3.0f; g.a = 1.8f; g.tau_w = 16; g.b = 61;
        g.vr = -54; g.type = 1; g.active = 1; g.inh_tx = 1;
    } else {
        g.cap = 104; g.gl = 4.3f; g.el = -65; g.vt = -52; g.slope = 0.8f; g.a = -0.8f; g.tau_w = 88; g.b = 65;
        g.vr = -53; g.type = 0; g.active = 1;
    }
    return g;
}
ref::NeuronGene profile_for_type(unsigned char type) {
    ref::NeuronGene g;
    switch (type) {
    case 0: g = naud(false); g.vr = -68.0f; g.adp_b = 120.0f; g.adp_tau = 45.0f; break;
    case 1: g = naud(true); break;
    case 2: g = naud(true); g.type = 2; g.lp = {1, 1, 1, 1}; break;
    case 3:
        g = naud(true); g.type = 3;
        g.prinz = {{400 * 628.0f, 2.5f * 628, 6 * 628.0f, 50 * 628.0f, 10 * 628.0f, 100 * 628.0f, .01f * 628, 0}};
        break;
    case 4:
        g = naud(false); g.type = 4; g.cap = 8.7f; g.gl = 8.7f / 12.0f; g.el = -60.0f; g.vt = -40.0f;
        g.vr = -60.0f; g.a = 0; g.b = 0; break;
    case 5:
        g = naud(false); g.type = 5; g.cap = 10.0f; g.gl = 0.5f; g.el = -60.0f; g.vt = -40.0f; g.vr = -60.0f;
        g.a = 0; g.b = 0; g.rec_base = 7.0f; g.rec_gain = 43.0f; g.rec_event = 2.0f; g.rec_decay = 3.0f; break;
    default:
        g = naud(false); g.type = 6; g.cap = 1200.0f; g.gl = 1000.0f / 65.6f; g.el = -45.1f; g.vt = -51.8f; break;
    }
    return g;
}

}  // namespace

// initial_profile(0..6) (src/physiology.cuh:169-176), for device-side births.
void nsb::neuron_profiles(ref::NeuronGene *out) {
    for (int t = 0; t < 7; ++t) out[t] = profile_for_type(static_cast<unsigned char>(t));
}

namespace {

// A host brain handle: the reference layout first, this library's extras after.
struct HostBrain : ref::Brain {
    int max_delay = 8;
    std::unique_ptr<Engine> engine;   // single-brain engine for ns_step, built lazily
};

bool finite_row(const float *p, int n) {
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// ns_create row decoding and validation (gym_adapter/native.cpp:46-82).
// max_profile: 5 for the reference ABI; the extended creators also accept
// profile 6 (triplet STDP into a dopamine-gated eligibility trace).
HostBrain *make_brain(int count, int edges, int channels, int outputs, const float *ng, const float *sg,
                      const int *motors, int max_delay, int max_profile = 5) {
    if (count < 1 || edges < 0 || channels < 1 || channels > 65535 || outputs < 1)
        throw std::runtime_error("Invalid brain dimensions");
    if (max_delay < 1 || max_delay > kMaxDelay) throw std::runtime_error("Invalid delay ring");
    auto b = std::make_unique<HostBrain>();
    b->channels = channels;
    b->max_delay = max_delay;
    for (int i = 0; i < count; ++i) {
        const float *p = ng + (size_t)i * 10;
        if (!finite_row(p, 10) || p[0] < 0 || p[0] > 6 || p[1] < -1 || p[1] >= channels || p[2] < 0 || p[2] > 1 ||
            p[3] < 0 || p[3] > 1 || p[4] < 0 || p[4] > 3)
            throw std::runtime_error("Invalid neuron gene");
        ref::NeuronGene g = profile_for_type(static_cast<unsigned char>(p[0]));
        b->sensory.push_back(int(p[1]));
        g.sensory_channel = p[1] < 0 ? -1 : 0;
        g.active = (unsigned char)p[2];
        g.inh_tx = (unsigned char)p[3];
        g.modulator = (unsigned char)p[4];
        if (p[5] <= 0 || p[6] <= 0 || p[7] < -80 || p[7] > -20 || p[8] < 0 || p[9] < 0)
            throw std::runtime_error("Invalid membrane parameters");
        g.cap *= p[5]; g.gl *= p[6]; g.vt = p[7];
        g.rec_base = 0; g.rec_gain = p[8]; g.rec_event = p[9];
        b->genes.push_back(g);
    }
    for (int i = 0; i < edges; ++i) {
        const float *p = sg + (size_t)i * 11;
        if (!finite_row(p, 11) || p[0] < 0 || p[0] >= count || p[1] < 0 || p[1] >= count || p[2] < 0 || p[3] < 0 ||
            p[3] > 1 || p[4] < 1 || p[4] > max_delay || p[5] < 0 || p[5] >= 4 || p[6] <= 0 || p[6] > 1 ||
            p[7] <= 0 || p[8] < 0 || p[9] < 0 || p[9] > max_profile || p[10] < 0 || p[10] > 7)
            throw std::runtime_error("Invalid synapse gene");
        ref::SynapseGene g;
        std::memset(&g, 0, sizeof g);
        g.pre = (int)p[0]; g.post = (int)p[1]; g.w0 = p[2];
        g.active = (unsigned char)p[3]; g.delay = (unsigned char)p[4]; g.branch = (unsigned char)p[5];
        g.U = p[6]; g.trec = p[7]; g.tfac = p[8];
        g.plasticity = (unsigned char)p[9]; g.receptors = (unsigned char)p[10]; g.sites = 14;
        b->connections.push_back(g);
    }
    for (int i = 0; i < outputs; ++i) {
        if (motors[i] < 0 || motors[i] >= count) throw std::runtime_error("Invalid motor index");
        b->motors.push_back(motors[i]);
    }
    b->neurons.resize(count);
    b->synapses.resize(edges);
    b->history.resize(count);
    b->excitation.resize(count);
    b->inhibition.resize(count);
    b->modulation.resize(count);
    return b.release();
}

BrainSpec spec_of(const ref::Brain &b) {
    BrainSpec s;
    s.genes = b.genes.data(); s.count = (int)b.genes.size();
    s.conns = b.connections.data(); s.edges = (int)b.connections.size();
    s.motors = b.motors.data();
    s.sensory = b.sensory.data();
    s.orig_n = b.original_neurons.empty() ? nullptr : b.original_neurons.data();
    s.orig_s = b.original_synapses.empty() ? nullptr : b.original_synapses.data();
    return s;
}

int delay_ring_for(const std::vector<BrainSpec> &specs, int floor_delay) {
    int d = floor_delay;
    for (const auto &s : specs)
        for (int j = 0; j < s.edges; ++j) d = std::max<int>(d, s.conns[j].delay);
    return d;
}

Engine &brain_engine(HostBrain &b) {
    if (!b.engine) {
        std::vector<BrainSpec> specs{spec_of(b)};
        EngineConfig cfg;
        cfg.max_delay = b.max_delay;
        cfg.block = 128;
        if (const char *cl = std::getenv("NSB_CLUSTER")) cfg.cluster_big = std::atoi(cl);
        if (const char *wc = std::getenv("NSB_WARP_CELLS")) cfg.warp_cells = std::atoi(wc);
        b.engine = std::make_unique<Engine>(specs, b.channels, (int)b.motors.size(), cfg);
        // A brain stepped before any reset starts from its host records
        // (value-initialised by ns_create, as in the reference).
        b.engine->load_state(0, b.neurons.data(), b.synapses.data(),
                             reinterpret_cast<const unsigned char (*)[9]>(b.history.data()), b.tick);
    }
    return *b.engine;
}

struct GpuBatch {
    std::unique_ptr<Engine> engine;
    // Genes in the reference layout, kept for checkpoint records.
    std::vector<ref::NeuronGene> genes;
    std::vector<ref::SynapseGene> conns;
    std::vector<int> noff, soff, motors, sensory;
    int channels = 0, outputs = 0;
};

}  // namespace

namespace nsb {
void set_error(const char *message) { g_error = message; }
}  // namespace nsb

extern "C" {

const char *ns_error() { return g_error.c_str(); }

void *ns_create(int count, int edges, int channels, int outputs, const float *ng, const float *sg,
                const int *motors) {
    try {
        return make_brain(count, edges, channels, outputs, ng, sg, motors, 8);
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

void *nsb_create_ext(int count, int edges, int channels, int outputs, const float *ng, const float *sg,
                     const int *motors, int max_delay) {
    try {
        return make_brain(count, edges, channels, outputs, ng, sg, motors, max_delay, 6);
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

void ns_original_indices(void *p, const uint32_t *neurons, const uint32_t *synapses) {
    auto &b = *static_cast<HostBrain *>(p);
    b.original_neurons.assign(neurons, neurons + b.genes.size());
    if (!b.connections.empty()) b.original_synapses.assign(synapses, synapses + b.connections.size());
    b.engine.reset();   // reset seeds changed: rebuild on next use
}

void ns_destroy(void *p) { delete static_cast<HostBrain *>(p); }

void ns_reset(void *p, uint32_t seed) {
    try {
        auto &b = *static_cast<HostBrain *>(p);
        Engine &e = brain_engine(b);
        const uint8_t one = 1;
        e.reset_host(&one, &seed);
        b.tick = 0;
    } catch (const std::exception &e) {
        g_error = e.what();   // the reference's ns_reset has no failure channel
    }
}

int ns_step(void *p, const float *input, int ticks, float input_gain, float *output) {
    try {
        auto &b = *static_cast<HostBrain *>(p);
        if (ticks < 1 || ticks > 10000 || !std::isfinite(input_gain) || input_gain < 0)
            throw std::runtime_error("Invalid neural integration interval");
        for (int c = 0; c < b.channels; ++c)
            if (!std::isfinite(input[c]) || input[c] < 0 || input[c] > 1)
                throw std::runtime_error("Invalid encoded observation");
        Engine &e = brain_engine(b);
        const uint8_t one = 1;
        int status = 0;
        e.step_host(input, &one, ticks, input_gain, output, &status);
        if (status == -2) throw std::runtime_error("Tick counter exceeds the engine range");
        if (status != 0) {
            e.set_tick(0, b.tick);   // the reference keeps its tick on failure (native.cpp:101-102)
            throw std::runtime_error("Nonfinite neural state");
        }
        b.tick += ticks;
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_dump(void *p, uint32_t *neuron_words, uint32_t *synapse_words, int64_t *tick) {
    try {
        auto &b = *static_cast<HostBrain *>(p);
        brain_engine(b).dump(0, neuron_words, synapse_words, tick);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

static void *gpu_create(void **handles, int count, int max_delay_floor, int block) {
    if (count < 1) throw std::runtime_error("Empty GPU batch");
    if (const char *threads = std::getenv("GYM_CUDA_THREADS")) {
        int t = std::atoi(threads);
        if (t != 32 && t != 64 && t != 128 && t != 256) throw std::runtime_error("Invalid CUDA block size");
    }
    auto &first = *static_cast<ref::Brain *>(handles[0]);
    const int channels = first.channels, outputs = (int)first.motors.size();
    std::vector<BrainSpec> specs;
    specs.reserve(count);
    for (int i = 0; i < count; ++i) {
        auto &b = *static_cast<ref::Brain *>(handles[i]);
        if (b.channels != channels || (int)b.motors.size() != outputs) throw std::runtime_error("Batch ports differ");
        specs.push_back(spec_of(b));
    }
    EngineConfig cfg;
    cfg.max_delay = delay_ring_for(specs, max_delay_floor);
    if (block) cfg.block = block;
    if (const char *slots = std::getenv("NSB_UNIT_SLOTS")) cfg.unit_slots = std::max(1, std::atoi(slots));
    if (const char *cl = std::getenv("NSB_CLUSTER")) cfg.cluster_big = std::atoi(cl);
    if (const char *wc = std::getenv("NSB_WARP_CELLS")) cfg.warp_cells = std::atoi(wc);
    auto batch = std::make_unique<GpuBatch>();
    batch->engine = std::make_unique<Engine>(specs, channels, outputs, cfg);
    batch->channels = channels;
    batch->outputs = outputs;
    batch->noff.push_back(0);
    batch->soff.push_back(0);
    for (const auto &sp : specs) {
        batch->genes.insert(batch->genes.end(), sp.genes, sp.genes + sp.count);
        batch->conns.insert(batch->conns.end(), sp.conns, sp.conns + sp.edges);
        batch->motors.insert(batch->motors.end(), sp.motors, sp.motors + outputs);
        batch->sensory.insert(batch->sensory.end(), sp.sensory, sp.sensory + sp.count);
        batch->noff.push_back(batch->noff.back() + sp.count);
        batch->soff.push_back(batch->soff.back() + sp.edges);
    }
    return batch.release();
}

void *ns_gpu_create(void **handles, int count) {
    try {
        return gpu_create(handles, count, 8, 0);
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

void *nsb_gpu_create_ext(void **handles, int count, int max_delay, int block) {
    try {
        return gpu_create(handles, count, max_delay, block);
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

// Bulk creation from concatenated Gym-ABI rows: brain i owns neuron rows
// [neuron_offsets[i], neuron_offsets[i+1]) and synapse rows likewise; synapse
// pre/post are brain-local; motors is brains x outputs.
void *nsb_gpu_create_rows(int brains, const int64_t *neuron_offsets, const int64_t *synapse_offsets,
                          const float *ng, const float *sg, const int *motors, int channels, int outputs,
                          int max_delay, int block) {
    try {
        if (brains < 1) throw std::runtime_error("Empty GPU batch");
        std::vector<std::unique_ptr<HostBrain>> hosts;
        std::vector<void *> handles;
        hosts.reserve(brains);
        for (int i = 0; i < brains; ++i) {
            const int64_t n0 = neuron_offsets[i], n1 = neuron_offsets[i + 1];
            const int64_t e0 = synapse_offsets[i], e1 = synapse_offsets[i + 1];
            hosts.emplace_back(make_brain((int)(n1 - n0), (int)(e1 - e0), channels, outputs, ng + n0 * 10,
                                          sg + e0 * 11, motors + (size_t)i * outputs, max_delay, 6));
            handles.push_back(hosts.back().get());
        }
        return gpu_create(handles.data(), brains, max_delay, block);
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

void ns_gpu_destroy(void *p) { delete static_cast<GpuBatch *>(p); }

int ns_gpu_reset(void *p, const uint8_t *mask, const uint32_t *seeds) {
    try {
        static_cast<GpuBatch *>(p)->engine->reset_host(mask, seeds);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int ns_gpu_step(void *p, const float *input, const uint8_t *mask, int ticks, float gain, float *output,
                int *status) {
    try {
        static_cast<GpuBatch *>(p)->engine->step_host(input, mask, ticks, gain, output, status);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Device-resident step: every pointer is device memory; asynchronous on `stream`.
int nsb_gpu_step_device(void *p, const float *d_input, const uint8_t *d_mask, int ticks, float gain,
                        float *d_output, int *d_status, void *stream) {
    try {
        static_cast<GpuBatch *>(p)->engine->step_device(d_input, d_mask, ticks, gain, d_output, d_status,
                                                        static_cast<cudaStream_t>(stream));
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Allocation-free step (no counterpart in the reference): the same tick as
// nsb_gpu_step_device, for callers that may not allocate device memory when
// they step — processes whose device memory all belongs to another allocator
// (a host application's memory pool) or that forbid allocation once started.
// The kernel's scratch (work-queue counters, per-synapse plasticity
// bookkeeping) lives in a static device array of 4 MiB + 256 B that every GPU
// loading this library keeps until exit; batches above 2,097,152 synapses are
// rejected. The first call on a device looks up that array's address and
// should come before any stream capture. Calls that overlap on the GPU race
// on the shared array. Inputs and outputs are caller device buffers.
int nsb_gpu_step_noalloc(void *p, const float *d_input, const uint8_t *d_mask, int ticks, float gain,
                         float *d_output, int *d_status, void *stream) {
    try {
        static_cast<GpuBatch *>(p)->engine->step_noalloc(d_input, d_mask, ticks, gain, d_output, d_status,
                                                         static_cast<cudaStream_t>(stream));
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Replays the step on the batch's own device buffers from a captured CUDA graph.
int nsb_gpu_step_graph(void *p, int ticks, float gain, void *stream) {
    try {
        static_cast<GpuBatch *>(p)->engine->step_graph(ticks, gain, static_cast<cudaStream_t>(stream));
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Device pointers of the batch's own buffers: 0 input, 1 mask, 2 output, 3 status.
void *nsb_gpu_buffer(void *p, int which) {
    Engine &e = *static_cast<GpuBatch *>(p)->engine;
    switch (which) {
    case 0: return e.dev_input();
    case 1: return e.dev_mask();
    case 2: return e.dev_output();
    case 3: return e.dev_status();
    default: return nullptr;
    }
}

// Copy host observations and mask into the batch's own device buffers.
int nsb_gpu_upload(void *p, const float *input, const uint8_t *mask) {
    try {
        Engine &e = *static_cast<GpuBatch *>(p)->engine;
        if (input && cudaMemcpy(e.dev_input(), input, (size_t)e.brains() * e.channels() * sizeof(float),
                                cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("CUDA: input upload failed");
        if (mask && cudaMemcpy(e.dev_mask(), mask, (size_t)e.brains(), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("CUDA: mask upload failed");
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Copy the batch's device outputs and status to host memory (synchronises).
int nsb_gpu_download(void *p, float *output, int *status) {
    try {
        Engine &e = *static_cast<GpuBatch *>(p)->engine;
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("CUDA: step failed");
        if (output && cudaMemcpy(output, e.dev_output(), (size_t)e.brains() * e.outputs() * sizeof(float),
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("CUDA: output download failed");
        if (status && cudaMemcpy(status, e.dev_status(), (size_t)e.brains() * sizeof(int),
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("CUDA: status download failed");
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_gpu_dump(void *p, int brain, uint32_t *neuron_words, uint32_t *synapse_words, int64_t *tick) {
    try {
        static_cast<GpuBatch *>(p)->engine->dump(brain, neuron_words, synapse_words, tick);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Load brain `brain`'s state from a reference-layout handle's host records.
int nsb_gpu_load_state(void *p, int brain, void *handle) {
    try {
        auto &b = *static_cast<ref::Brain *>(handle);
        static_cast<GpuBatch *>(p)->engine->load_state(
            brain, b.neurons.data(), b.synapses.data(),
            reinterpret_cast<const unsigned char (*)[9]>(b.history.data()), b.tick);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// brains, units, big_units, neurons, synapses, heavy, max_unit_neurons, grid, block, smem_bytes, ctas_per_sm
int nsb_gpu_stats(void *p, int *out) {
    Stats s = static_cast<GpuBatch *>(p)->engine->stats();
    const int v[11] = {s.brains, s.units, s.big_units, s.neurons, s.synapses, s.heavy, s.max_unit_neurons,
                       s.grid, s.block, s.smem_bytes, s.ctas_per_sm};
    std::memcpy(out, v, sizeof v);
    return 11;
}

long long nsb_gpu_take_events(void *p) {
    try {
        return (long long)static_cast<GpuBatch *>(p)->engine->take_events();
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// The neural step of the reference's device maze batch
// (gym_adapter/maze_gpu.cu:85-90): the maze library (built from the
// reference sources) keeps the MiniGrid batch and its encoded observations on
// the device; this entry point steps this library's GpuBatch on those
// observations. Leading fields of the reference's MazeBatch, in its order.
struct RefMazeBatch {
    int count;
    int *grid;
    void *objects, *agents;
    unsigned char *observations;
    float *encoded, *lookup;
};
constexpr int kMazeChannels = 7 * 7 * 3 * 2;   // MS*MS*3*2 (gym_adapter/maze_gpu.cu:3)

int ns_maze_brain_step(void *maze, void *brain, const unsigned char *mask, int ticks, float gain, float *output,
                       int *status) {
    try {
        const RefMazeBatch &m = *static_cast<const RefMazeBatch *>(maze);
        GpuBatch &g = *static_cast<GpuBatch *>(brain);
        Engine &e = *g.engine;
        if (e.brains() != m.count || e.channels() != kMazeChannels)
            throw std::runtime_error("Maze/brain dimensions differ");
        if (ticks < 1 || ticks > 10000 || !std::isfinite(gain) || gain < 0)
            throw std::runtime_error("Invalid neural integration interval");
        if (cudaMemcpy(e.dev_mask(), mask, (size_t)e.brains(), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("CUDA: mask upload failed");
        e.step_device(m.encoded, e.dev_mask(), ticks, gain, e.dev_output(), e.dev_status(), nullptr);
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("CUDA: step failed");
        if (cudaMemcpy(output, e.dev_output(), (size_t)e.brains() * e.outputs() * sizeof(float),
                       cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(status, e.dev_status(), (size_t)e.brains() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("CUDA: output download failed");
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Global modulator pulse: every `period` ticks (0: off) all neurons' plasticity
// sees the modulator bits `mod` (1 NE, 2 5-HT, 4 DA).
int nsb_gpu_set_modulation(void *p, int period, int mod) {
    try {
        static_cast<GpuBatch *>(p)->engine->set_global_modulation(period, (uint32_t)mod);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Delivery mode of the light tick kernel: 1 warp-cooperative release, 0
// serial per neuron. Returns the previous mode, or -1.
int nsb_gpu_set_delivery(void *p, int cooperative) {
    try {
        Engine &e = *static_cast<GpuBatch *>(p)->engine;
        const int old = e.cooperative() ? 1 : 0;
        e.set_cooperative(cooperative != 0);
        return old;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Per-bucket autotuner on the batch's own buffers (state restored); returns
// the packed bucket's delivery mode (1 cooperative, 0 serial) or -1.
int nsb_gpu_autotune(void *p, int ticks, float gain, void *stream) {
    try {
        return static_cast<GpuBatch *>(p)->engine->autotune(ticks, gain, static_cast<cudaStream_t>(stream)) ? 1 : 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_gpu_buckets(void *p, int *out) {
    const auto &bs = static_cast<GpuBatch *>(p)->engine->buckets();
    int k = 0;
    for (const Bucket &B : bs) {
        const int v[11] = {B.ub, B.units(), B.max_neurons, B.max_synapses, B.cfg.block, B.cfg.coop, B.cfg.cluster,
                           B.cfg.meta_cap, B.cfg.list, B.smem, B.grid};
        std::memcpy(out + k, v, sizeof v);
        k += 11;
    }
    return k;
}

int nsb_gpu_set_bucket(void *p, int bucket, int block, int cooperative, int cluster, int meta_cap, int list) {
    try {
        static_cast<GpuBatch *>(p)->engine->set_bucket(bucket, BucketConfig{block, cooperative ? 1 : 0, cluster,
                                                                             meta_cap, list});
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

}  // extern "C"

// ---- checkpoint records (src/main.cu:164-264, src/checkpoint_impl.cuh) -----
namespace {

bool same_bits(float a, float b) { return std::memcmp(&a, &b, 4) == 0; }
bool gene_equal(const ref::NeuronGene &a, const ref::NeuronGene &b) {
    const float fa[] = {a.cap, a.gl, a.el, a.vt, a.slope, a.a, a.tau_w, a.b, a.vr, a.adp_b, a.adp_tau, a.lp.calcium,
                        a.lp.calcium_k, a.lp.h, a.lp.leak, a.prinz_leak, a.rec_base, a.rec_gain, a.rec_event,
                        a.rec_decay, a.affinity};
    const float fb[] = {b.cap, b.gl, b.el, b.vt, b.slope, b.a, b.tau_w, b.b, b.vr, b.adp_b, b.adp_tau, b.lp.calcium,
                        b.lp.calcium_k, b.lp.h, b.lp.leak, b.prinz_leak, b.rec_base, b.rec_gain, b.rec_event,
                        b.rec_decay, b.affinity};
    for (size_t i = 0; i < sizeof fa / sizeof fa[0]; ++i)
        if (!same_bits(fa[i], fb[i])) return false;
    for (int i = 0; i < 8; ++i)
        if (!same_bits(a.prinz.g[i], b.prinz.g[i])) return false;
    return a.type == b.type && a.active == b.active && a.modulator == b.modulator && a.inh_tx == b.inh_tx &&
           a.sensory_channel == b.sensory_channel;
}
bool conn_equal(const ref::SynapseGene &a, const ref::SynapseGene &b) {
    return same_bits(a.w0, b.w0) && same_bits(a.U, b.U) && same_bits(a.trec, b.trec) && same_bits(a.tfac, b.tfac) &&
           a.pre == b.pre && a.post == b.post && a.delay == b.delay && a.active == b.active &&
           a.plasticity == b.plasticity && a.branch == b.branch && a.sites == b.sites && a.receptors == b.receptors &&
           same_bits(a.slow_rec, b.slow_rec) && same_bits(a.slow_depl, b.slow_depl);
}
int port_of(const GpuBatch &g, int brain, int j) {
    const int sens = g.sensory[g.noff[brain] + j];
    if (sens >= 0) return sens;
    for (int k = 0; k < g.outputs; ++k)
        if (g.motors[(size_t)brain * g.outputs + k] == j) return g.channels + k;
    return -1;
}

}  // namespace

extern "C" {

// FNV-1a layout hash of the reference build's checkpoint (src/checkpoint_impl.cuh:20-32).
unsigned long long nsb_checkpoint_layout() { return ref::layout_hash(); }

// The state of every brain as the reference's checkpoint records: neuron
// records (sum of counts x 344 B) and synapse records (sum of edges x 136 B)
// in slot order, brain i's neurons at slots [sum of earlier counts, ...),
// owner = brain index, next = the brain's next slot (-1 last), port = sensory
// channel, or channels + motor index, or -1. Per-tick accumulators and the
// world's modulatory timestamps are zero between steps. ticks: one per brain.
int nsb_gpu_checkpoint_export(void *p, void *neuron_records, void *synapse_records, int64_t *ticks) {
    try {
        GpuBatch &g = *static_cast<GpuBatch *>(p);
        auto *nr = static_cast<ref::CheckpointNeuron *>(neuron_records);
        auto *sr = static_cast<ref::CheckpointSynapse *>(synapse_records);
        const int brains = (int)g.noff.size() - 1;
        for (int b = 0; b < brains; ++b) {
            const int n = g.noff[b + 1] - g.noff[b], m = g.soff[b + 1] - g.soff[b];
            std::vector<ref::NeuronState> ns(n);
            std::vector<ref::SynapseState> ss(std::max(m, 1));
            std::vector<std::array<unsigned char, 9>> hist(n);
            int64_t tick = 0;
            g.engine->export_state(b, ns.data(), ss.data(), reinterpret_cast<unsigned char (*)[9]>(hist.data()), &tick);
            for (int j = 0; j < n; ++j) {
                ref::CheckpointNeuron r;
                std::memset(&r, 0, sizeof r);
                r.slot = g.noff[b] + j;
                r.owner = b;
                r.next = j + 1 < n ? r.slot + 1 : -1;
                r.port = port_of(g, b, j);
                r.gene = g.genes[r.slot];
                r.state = ns[j];
                std::memcpy(r.spike_history, hist[j].data(), 9);
                nr[r.slot] = r;
            }
            for (int j = 0; j < m; ++j) {
                ref::CheckpointSynapse r;
                std::memset(&r, 0, sizeof r);
                r.slot = g.soff[b] + j;
                r.owner = b;
                r.next = j + 1 < m ? r.slot + 1 : -1;
                r.gene = g.conns[r.slot];
                r.state = ss[j];
                sr[r.slot] = r;
            }
            if (ticks) ticks[b] = tick;
        }
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// Loads every brain's state from checkpoint records laid out as the export
// writes them. The records' slots, owners and genes must describe this
// batch's brains; their states, spike histories and the ticks replace the
// batch's.
int nsb_gpu_checkpoint_import(void *p, const void *neuron_records, long long n_records, const void *synapse_records,
                              long long e_records, const int64_t *ticks) {
    try {
        GpuBatch &g = *static_cast<GpuBatch *>(p);
        const auto *nr = static_cast<const ref::CheckpointNeuron *>(neuron_records);
        const auto *sr = static_cast<const ref::CheckpointSynapse *>(synapse_records);
        const int brains = (int)g.noff.size() - 1;
        if (n_records != g.noff.back() || e_records != g.soff.back())
            throw std::runtime_error("Checkpoint record counts differ from the batch");
        for (int b = 0; b < brains; ++b) {
            const int n = g.noff[b + 1] - g.noff[b], m = g.soff[b + 1] - g.soff[b];
            std::vector<ref::NeuronState> ns(n);
            std::vector<ref::SynapseState> ss(std::max(m, 1));
            std::vector<std::array<unsigned char, 9>> hist(n);
            for (int j = 0; j < n; ++j) {
                const auto &r = nr[g.noff[b] + j];
                if (r.slot != g.noff[b] + j || r.owner != b) throw std::runtime_error("Invalid checkpoint neuron record");
                if (!gene_equal(r.gene, g.genes[r.slot])) throw std::runtime_error("Checkpoint genes differ from the batch");
                ns[j] = r.state;
                std::memcpy(hist[j].data(), r.spike_history, 9);
            }
            for (int j = 0; j < m; ++j) {
                const auto &r = sr[g.soff[b] + j];
                if (r.slot != g.soff[b] + j || r.owner != b) throw std::runtime_error("Invalid checkpoint synapse record");
                if (!conn_equal(r.gene, g.conns[r.slot])) throw std::runtime_error("Checkpoint genes differ from the batch");
                ss[j] = r.state;
            }
            g.engine->load_state(b, ns.data(), ss.data(), reinterpret_cast<const unsigned char (*)[9]>(hist.data()),
                                 ticks ? ticks[b] : 0);
        }
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

// ---- serving loop (no counterpart in the reference) ----------------------------
// Continuous batching of genome-evaluation episodes on a device-resident
// pole-on-cart environment; see neural-selection_b200/csrc/ns_serve.h.

static_assert(sizeof(ServeResult) == 64, "nsb_serve_result layout");

void *nsb_serve_create(long long max_inflight_neurons, double hbm_budget_bytes, double synapses_per_neuron,
                       int max_slots, int max_brain_neurons, int ticks, float gain, double smoothing) {
    try {
        ServeConfig cfg;
        cfg.max_inflight_neurons = max_inflight_neurons;
        cfg.hbm_budget_bytes = hbm_budget_bytes;
        cfg.synapses_per_neuron = synapses_per_neuron;
        cfg.max_slots = max_slots;
        cfg.max_brain_neurons = max_brain_neurons;
        cfg.ticks = ticks;
        cfg.gain = gain;
        cfg.smoothing = smoothing;
        return new Server(cfg);
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

void nsb_serve_destroy(void *p) { delete static_cast<Server *>(p); }

// Registers a genome in the Gym row format of ns_create (8 channels: the
// opponent-coded pole-on-cart observation; 2 motors: push left, push right).
int nsb_serve_register(void *p, int count, int edges, const float *neuron_rows, const float *synapse_rows,
                       const int *motors) {
    try {
        std::unique_ptr<HostBrain> b(make_brain(count, edges, 8, 2, neuron_rows, synapse_rows, motors, 8));
        return static_cast<Server *>(p)->register_genome(spec_of(*b));
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_serve_submit(void *p, int n, const int *genome, const uint32_t *seed, const int *steps, const uint64_t *tag,
                     const double *arrival_s) {
    try {
        static_cast<Server *>(p)->submit(n, genome, seed, steps, tag, arrival_s);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_serve_start(void *p) {
    try {
        static_cast<Server *>(p)->start();
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_serve_stop(void *p) {
    try {
        Server &s = *static_cast<Server *>(p);
        s.stop();
        const std::string err = s.error();
        if (!err.empty()) throw std::runtime_error(err);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_serve_run(void *p, long long max_iterations) {
    try {
        static_cast<Server *>(p)->run_until_idle(max_iterations);
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

int nsb_serve_poll(void *p, void *results, int max) {
    try {
        Server &s = *static_cast<Server *>(p);
        const std::string err = s.error();
        if (!err.empty()) throw std::runtime_error(err);
        return s.poll(static_cast<ServeResult *>(results), max);
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

double nsb_serve_now(void *p) { return static_cast<Server *>(p)->now(); }

// steps, admitted, completed, queued, inflight, inflight_neurons, units,
// neuron_ticks, busy_s, elapsed_s, events, pool_neurons, pool_synapses,
// pool_bytes, inflight_bytes, neuron_ticks_launched
int nsb_serve_stats(void *p, double *out) {
    try {
        const ServeStats s = static_cast<Server *>(p)->stats();
        const double v[16] = {(double)s.steps, (double)s.admitted, (double)s.completed, (double)s.queued,
                              (double)s.inflight, (double)s.inflight_neurons, (double)s.units, s.neuron_ticks,
                              s.busy_s, s.elapsed_s, (double)s.events, (double)s.pool_neurons,
                              (double)s.pool_synapses, s.pool_bytes, s.inflight_bytes, s.neuron_ticks_launched};
        std::memcpy(out, v, sizeof v);
        return 16;
    } catch (const std::exception &e) {
        g_error = e.what();
        return -1;
    }
}

}  // extern "C"
