/* C ABI of the B200 neural-tick library (libns_b200.so).
 *
 * Drop-in boundary. The first ten entry points keep the signatures, argument
 * meaning, validation messages and return conventions of the reference's Gym
 * bridge (mixic/neural-selection gym_adapter/native.cpp and gym_adapter/gpu.cu):
 * gym_adapter/adapter.py and gym_adapter/gpu.py bind them with ctypes
 * unchanged. All computation runs on the GPU (sm_100a). Exceptions never cross
 * the ABI: failures return -1 or NULL and ns_error() returns the thread-local
 * message. Brain handles share the reference's host layout, so ns_gpu_create
 * accepts handles made by either library's ns_create.
 *
 * Entry points prefixed nsb_ are this library's extensions.
 */
#ifndef NS_B200_H
#define NS_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces ns_error, gym_adapter/native.cpp:45 (thread-local message, :39). */
const char *ns_error(void);

/* Replaces ns_create, gym_adapter/native.cpp:46-82 (validation 49-76). ng: count x 10 rows
 * [profile 0-6, channel -1..channels-1, active, inhibitory, modulator 0-3,
 * capacitance x, leak x, threshold mV, receptor Hz gain, receptor event nS];
 * sg: edges x 11 rows [pre, post, weight nS, active, delay 1-8, branch 0-3,
 * U, recovery ms, facilitation ms, plasticity 0-5, receptor mask 0-7];
 * motors: outputs neuron indices. NULL on invalid input. */
void *ns_create(int count, int edges, int channels, int outputs, const float *ng, const float *sg,
                const int *motors);

/* Replaces ns_original_indices, gym_adapter/native.cpp:83-87 (reset seeds
 * use original indices after graph compilation). */
void ns_original_indices(void *brain, const uint32_t *neurons, const uint32_t *synapses);

/* Replaces ns_destroy, gym_adapter/native.cpp:88. */
void ns_destroy(void *brain);

/* Replaces ns_reset, gym_adapter/native.cpp:89-94: state seeded from
 * seed + index*7919 (neurons) and seed + index*104729 (synapses). */
void ns_reset(void *brain, uint32_t seed);

/* Replaces ns_step, gym_adapter/native.cpp:95-108: `ticks` 1 ms ticks (1..10000),
 * input[channels] in [0,1], output[outputs] = motor spikes during the call.
 * 0, or -1 ("Nonfinite neural state", invalid interval or observation). */
int ns_step(void *brain, const float *input, int ticks, float input_gain, float *output);

/* Replaces ns_gpu_create, gym_adapter/gpu.cu:67-109: a device batch built from
 * `count` brain handles with equal channels/outputs. Honours GYM_CUDA_THREADS
 * validation (32/64/128/256). */
void *ns_gpu_create(void **brains, int count);

/* Replaces ns_gpu_destroy, gym_adapter/gpu.cu:110. */
void ns_gpu_destroy(void *batch);

/* Replaces ns_gpu_reset, gym_adapter/gpu.cu:111-113: reset brains with mask[i]. */
int ns_gpu_reset(void *batch, const uint8_t *mask, const uint32_t *seeds);

/* Replaces ns_gpu_step, gym_adapter/gpu.cu:114-123: synchronous; input
 * count x channels, output count x outputs, status[i] = -1 on a non-finite
 * voltage (-2: tick counter past 2^31). */
int ns_gpu_step(void *batch, const float *input, const uint8_t *mask, int ticks, float gain, float *output,
                int *status);

/* gym_adapter/maze_gpu.cu:85-90. Steps the batch on the encoded observations
 * of a device maze batch made by the reference's maze library (ns_maze_create
 * in libgym_maze_gpu.so, whose MazeBatch starts {int count; int *grid; void
 * *objects, *agents; unsigned char *observations; float *encoded, *lookup;
 * ...}): mask host count, output host count x outputs, status host count.
 * The batch must have 294 channels (7 x 7 x 3 x 2). Synchronous. */
int ns_maze_brain_step(void *maze, void *batch, const unsigned char *mask, int ticks, float gain, float *output,
                       int *status);

/* ---- extensions (no reference counterpart) ---------------------------------- */

/* ns_create with a delay ring of max_delay ticks (1..31). The extended
 * creators (this one and nsb_gpu_create_rows) also accept plasticity profile
 * 6: triplet STDP written into a dopamine-gated eligibility trace. */
void *nsb_create_ext(int count, int edges, int channels, int outputs, const float *ng, const float *sg,
                     const int *motors, int max_delay);
/* ns_gpu_create with an explicit delay ring floor and CTA size (128 or 256; 0 = default). */
void *nsb_gpu_create_ext(void **brains, int count, int max_delay, int block);
/* Device batch straight from concatenated Gym-ABI rows: brain i owns neuron rows
 * [neuron_offsets[i], neuron_offsets[i+1]) and synapse rows likewise (pre/post
 * brain-local); motors is brains x outputs. */
void *nsb_gpu_create_rows(int brains, const int64_t *neuron_offsets, const int64_t *synapse_offsets,
                          const float *ng, const float *sg, const int *motors, int channels, int outputs,
                          int max_delay, int block);
/* Asynchronous step on device memory (cudaStream_t passed as void*). */
int nsb_gpu_step_device(void *batch, const float *d_input, const uint8_t *d_mask, int ticks, float gain,
                        float *d_output, int *d_status, void *stream);
/* No counterpart in the reference. Allocation-free step for callers that may
 * not allocate device memory when they step (their device memory belongs to
 * another allocator, or they forbid allocation once started): the same tick as
 * nsb_gpu_step_device, with the kernel's scratch memory in a static device
 * array (4 MiB + 256 B, held by every GPU that loads the library until exit)
 * instead of library-allocated buffers. Rejects batches above 2,097,152
 * synapses. The first call on a device sets up the array's address (make it
 * before any stream capture); the address is kept for the life of the
 * process, so the device's context must live as long (no cudaDeviceReset
 * between calls). Calls that overlap on the GPU race. Synaptic arrivals are
 * counted as in the other steps. */
int nsb_gpu_step_noalloc(void *batch, const float *d_input, const uint8_t *d_mask, int ticks, float gain,
                         float *d_output, int *d_status, void *stream);
/* Step on the batch's own device buffers, replayed from a captured CUDA graph. */
int nsb_gpu_step_graph(void *batch, int ticks, float gain, void *stream);
/* Copy host observations (count x channels) and/or mask (count) into the
 * batch's own device buffers; either pointer may be NULL. */
int nsb_gpu_upload(void *batch, const float *input, const uint8_t *mask);
/* Copy the batch's device outputs and status to host memory (synchronises). */
int nsb_gpu_download(void *batch, float *output, int *status);
/* Device pointer of the batch's buffer: 0 input, 1 mask, 2 output, 3 status. */
void *nsb_gpu_buffer(void *batch, int which);
/* Canonical state of one brain: 32 words per neuron, 20 per synapse, in the
 * brain's original order; tick after the last step. */
int nsb_gpu_dump(void *batch, int brain, uint32_t *neuron_words, uint32_t *synapse_words, int64_t *tick);
/* Same for a single ns_create brain. */
int nsb_dump(void *brain, uint32_t *neuron_words, uint32_t *synapse_words, int64_t *tick);
/* Load one batch brain's state from a brain handle's host records. */
int nsb_gpu_load_state(void *batch, int brain, void *brain_handle);
/* Layout facts: brains, units, big_units, neurons, synapses, heavy, max_unit_neurons,
 * grid, block, smem_bytes, ctas_per_sm. Returns the count written (11). */
int nsb_gpu_stats(void *batch, int *out);
/* Synaptic arrivals counted on the device since the previous call. */
long long nsb_gpu_take_events(void *batch);
/* No counterpart in the reference. A global modulator pulse: at every tick
 * divisible by `period` (0: off) the plasticity of every neuron sees the
 * modulator bits `mod` (1 NE, 2 5-HT, 4 DA) as if a modulatory synapse had
 * released onto it. Returns 0 or -1. */
int nsb_gpu_set_modulation(void *batch, int period, int mod);
/* Delivery mode of the tick kernel: 1 warp-cooperative stochastic release
 * (dense, active brains), 0 serial per neuron; results are identical.
 * Returns the previous mode, or -1. */
int nsb_gpu_set_delivery(void *batch, int cooperative);
/* No counterpart in the reference, which takes one block size for every
 * brain from GYM_CUDA_THREADS (gym_adapter/gpu.cu:71-72) and fixes its world
 * kernels' size tiers at compile time (src/main.cu:49-52). Per-bucket
 * autotuner: for each bucket of work units (see nsb_gpu_buckets) it times
 * candidate configurations (threads per CTA 128/256, serial or cooperative
 * delivery, shared-memory staging depth of the synapse meta words, list or
 * per-thread integration, one CTA or a thread-block cluster per big brain)
 * on the batch's own buffers, a few
 * launches each with the state restored afterwards, and keeps the fastest.
 * Results are identical under every configuration. Returns the packed
 * bucket's delivery mode (1 cooperative), or -1. */
int nsb_gpu_autotune(void *batch, int ticks, float gain, void *stream);
/* No counterpart in the reference. The batch's five work-unit buckets, in
 * order: units above 4, 2 and 1 times the unit size (one big brain each),
 * packed units of small brains, units with LP, Prinz or LFS cells. For each,
 * 11 ints: first unit, units, neurons and synapses of its largest unit,
 * threads per CTA, cooperative delivery, CTAs per unit (1, or the cluster
 * size 8, 4 or 2), staged synapse meta words, list integration (1: the
 * neurons that need integrating are gathered into a per-tick list and
 * integrated at full warp width; 0: each thread integrates its own),
 * dynamic shared memory bytes, grid (CTAs, or clusters). Returns the count
 * written (55). */
int nsb_gpu_buckets(void *batch, int *out);
/* No counterpart in the reference. Sets one bucket's configuration: block
 * 128 or 256, cooperative 0/1, cluster 1 or the bucket's cluster size,
 * meta_cap a multiple of 32, list 0/1 (one-CTA light units only; 1 for the
 * heavy bucket). Returns 0, or -1 when it cannot run (ns_error says why). */
int nsb_gpu_set_bucket(void *batch, int bucket, int block, int cooperative, int cluster, int meta_cap, int list);

/* Replaces compile_genome (gym_adapter/compile_graph.py:10-28), which the
 * reference's SpikingPolicy applies before ns_create (gym_adapter/adapter.py:197-210):
 * keeps the neurons with a causal path to a motor over active edges between
 * active neurons, in ascending original order, and the synapses among them in
 * original order with remapped endpoints. Outputs (any may be NULL except the
 * counts): rows (count x 10, edges x 11 at most), motors (outputs), original
 * indices for ns_original_indices. Host only; returns 0, or -1 on endpoints or
 * motors outside the genome. */
int nsb_compile_genome(int count, int edges, const float *neuron_rows, const float *synapse_rows, int outputs,
                       const int *motors, float *out_neuron_rows, float *out_synapse_rows, int *out_motors,
                       uint32_t *original_neurons, uint32_t *original_synapses, int *out_count, int *out_edges);

/* ---- World pool slots (src/main.cu:364-390). The reference claims neuron and
 * synapse slots with an atomic first-free-bit search from a hint word; these
 * replay the claims one after another, so the slots depend only on the
 * bitmap and the hints. d_used: device bitmap of `capacity` bits. */
/* slots[i] = the slot claimed for hints[i] (search from word hints[i] % words,
 * lowest free bit first), or -1. Host arrays; synchronous. */
int nsb_pool_claim(uint32_t *d_used, int capacity, const int *hints, int count, int *slots);
/* Clears the bits of slots[0..count) (negative entries ignored). */
int nsb_pool_release(uint32_t *d_used, const int *slots, int count);

/* ---- World neural stage. Replaces the neural part of the world simulator's
 * step loop (src/main.cu:2634-2728: slot selection, the 16 ticks of
 * synapse_delivery / synapse_plasticity_delivery / neuron_step /
 * synapse_plasticity, or the brain_block_step tiers) and its homeostasis
 * launches (src/main.cu:2751-2758), operating in place on the simulator's own
 * device pools (struct Device, src/main.cu:105-140) in the reference record
 * layouts: Animal 472 B, PlasticityCohort 80 B, NeuronGene 124 B,
 * NeuronState 120 B, SynapseGene 40 B, SynapseState 80 B. Pointers are device
 * pointers; capacities are the build's P, NEURON_CAPACITY and
 * SYNAPSE_CAPACITY (spike_history is indexed [tick % 9][neuron_capacity]).
 * World semantics (src/main.cu:659-801, 1122-1136, 1287-1300): only animals
 * with alive == 1 step; an edge delivers only when active, its endpoints
 * active and owned by the edge's animal; sensory neurons read
 * senses[animal][channel], through receptor events for type 5 on channels
 * below 6 and as channel level x 230 pA otherwise (silence flags zero them);
 * spikes of neurons with port 19..23 add to motors[animal][port - 19];
 * frozen plasticity cohorts skip plasticity and homeostasis; the traced
 * animal's motor neurons feed the trace counters. Per post-synaptic branch the
 * synaptic input is summed in the order of the animal's synapse list. */
typedef struct NsbWorldPools {
    const void *animals;            /* Animal[animal_capacity] */
    const void *plasticity_cohort;  /* PlasticityCohort[animal_capacity] or NULL */
    const void *neurons;            /* NeuronGene[neuron_capacity] */
    const void *synapses;           /* SynapseGene[synapse_capacity] */
    void *neuron_state;             /* NeuronState[neuron_capacity] */
    void *synapse_state;            /* SynapseState[synapse_capacity] */
    float *pending_exc;             /* [neuron_capacity][4] */
    float *pending_inh;             /* [neuron_capacity] */
    const float *senses;            /* [animal_capacity][19] */
    unsigned long long *mod_event_tick; /* [neuron_capacity][6] */
    unsigned char *spike_history;   /* [9][neuron_capacity] */
    const int *neuron_owner, *synapse_owner, *neuron_next, *synapse_next, *neuron_port;
    int *motors;                    /* [animal_capacity][5] */
    int *trace_exc_arrivals, *trace_exc_releases, *trace_inh_arrivals;  /* [5] each */
    float *trace_exc_ns, *trace_inh_ns, *trace_peak_mv;                 /* [5] each */
    int trace_animal;               /* animal slot, or -1 */
    int silence_senses, silence_contact;
    int animal_capacity, neuron_capacity, synapse_capacity;
} NsbWorldPools;
/* A world stage over the given pools (copied; the pools stay the caller's).
 * max_brain_neurons / max_brain_synapses bound one animal's brain (0: 4096 /
 * 65536). NULL on invalid arguments. */
void *nsb_world_create(const NsbWorldPools *pools, int max_brain_neurons, int max_brain_synapses);
void nsb_world_destroy(void *world);
/* The 16 ticks of world step `step` (ticks (step - 1) * 16 ... + 15) for
 * every living animal, on the legacy default stream; returns 0, or -1 when an
 * animal's lists disagree with its counts or exceed the maxima (ns_error()). */
int nsb_world_neural_step(void *world, int64_t step);
/* Homeostatic AMPA scaling after the world's body step: every active neuron
 * of a living, unfrozen animal, elapsed max(16, age x 16) ms. Launched on the
 * legacy default stream; returns without waiting for it. */
int nsb_world_homeostasis(void *world);
/* Work of the last neural step: out[0] animals stepped, [1] neurons,
 * [2] synapses, [3] synaptic events (arrivals). */
int nsb_world_stats(void *world, long long *out);
/* Layout facts the stage relies on: sizes of Animal, PlasticityCohort and the
 * offsets of Animal.id, .age, .alive, .neuron_head, .synapse_head,
 * .neuron_count, .synapse_count and PlasticityCohort.frozen (10 values). */
int nsb_world_layout(uint64_t *out);

/* ---- World ecology stage: the rest of the world step around the neural
 * stage (src/main.cu:612-657, 1138-1338; host loop order 2745-2770). The
 * state beside the neural pools in the simulator's struct Device
 * (src/main.cu:105-140). Grid 128 x 128 cells, row-major (y * 128 + x). */
typedef struct NsbWorldEcology {
    int *food, *kind;               /* [128 * 128]: food stock (0/1), kind 0-2 */
    int *cell_head;                 /* [128 * 128] spatial index heads */
    int *cell_next;                 /* [animal_capacity] */
    unsigned char *bite_intent;     /* [animal_capacity] */
    uint32_t *neuron_used, *synapse_used;   /* slot bitmaps, ceil(capacity / 32) words */
    int *founder_motor_steps;       /* [5] */
    int *founder_observed_steps, *deaths, *predation_deaths, *bites;
    void *life_records;             /* LifeRecord[life_capacity] (504 B), or NULL */
    int *life_count;
    void *bite_events;              /* BiteEvent[2 * animal_capacity] (24 B), or NULL */
    int *bite_event_count;
    int initial_count;              /* animals with id below it count as founders */
    int instant_motors;             /* motor force = spikes / 16 instead of the muscle model */
    int life_capacity;
    int *neuron_clone;              /* [neuron_capacity] reproduction scratch (parent slot -> child slot) */
    int *births, *next_id;          /* birth counter, next animal id */
} NsbWorldEcology;
/* Contended steps (food harvests, spatial index order, bites, record slots)
 * resolve as if the reference kernel's threads ran in ascending animal slot
 * order: one legal execution of the reference's atomics, the same every run.
 * All calls run on the legacy default stream and return after it finishes;
 * -1 with ns_error() on invalid handles, lists that disagree with their
 * counts, slots outside the capacities or a food kind outside 0-2. */
void *nsb_world_ecology_create(const NsbWorldPools *pools, const NsbWorldEcology *ecology);
void nsb_world_ecology_destroy(void *ecology);
/* body_step, spatial index, bite_animals, finish_predation (src/main.cu:2745-2749). */
int nsb_world_body_step(void *ecology, int64_t step);
/* reclaim_dead_genomes (src/main.cu:2763): life records, genome release. */
int nsb_world_reclaim(void *ecology, int64_t step);
/* reproduce with mutate (src/main.cu:2765): parents (alive, energy >= 22)
 * in ascending slot order, each birth complete before the next, slot claims
 * as claim_slot run alone. */
int nsb_world_reproduce(void *ecology);
/* regrow, spatial index, update_senses (src/main.cu:2767-2770). */
int nsb_world_regrow_and_sense(void *ecology, int64_t step, unsigned long long seed, float renewal_probability);

/* ---- Checkpoint records. The world simulator saves the neural pools as
 * CheckpointNeuron (344 B) and CheckpointSynapse (136 B) records, one per
 * occupied slot in ascending slot order (src/main.cu:164-264, packed by
 * pack_checkpoint_neurons/_synapses; stream order src/checkpoint_impl.cuh:190-211),
 * under a header whose layout hash covers the build's sizes
 * (src/checkpoint_impl.cuh:20-32). */
/* The reference build's checkpoint layout hash (0x2b1cd1c766eebf82). */
unsigned long long nsb_checkpoint_layout(void);
/* Every brain of the batch as checkpoint records (neuron_records: sum of
 * counts x 344 B, synapse_records: sum of edges x 136 B; brain i's neurons at
 * slots [sum of earlier counts, ...), owner = brain index, next = next slot of
 * the brain or -1, port = sensory channel, channels + motor index, or -1) and
 * one tick per brain. Returns 0 or -1. */
int nsb_gpu_checkpoint_export(void *batch, void *neuron_records, void *synapse_records, int64_t *ticks);
/* Loads states, spike histories and ticks from records laid out as the export
 * writes them; slots, owners and genes must describe this batch. */
int nsb_gpu_checkpoint_import(void *batch, const void *neuron_records, long long neuron_count,
                              const void *synapse_records, long long synapse_count, const int64_t *ticks);

/* ---- Serving loop. No counterpart in the reference: the reference evaluates
 * episodes with Gymnasium environments on the host (gym_adapter/gpu.py:57-83);
 * this server keeps episodes of different genomes and lengths on the device,
 * with a pole-on-cart environment, the adapter's opponent-coded observation
 * (gym_adapter/adapter.py:153-169) and its smoothed two-action decoding
 * (gym_adapter/gpu.py:66-83), and batches them continuously into the tick
 * kernel. */
typedef struct {
    uint64_t tag;
    int32_t genome, steps, reward, failures; /* steps run; steps without a fall; falls */
    uint32_t trace, seed;                    /* FNV-1a over (action, motor counts) of every step */
    int32_t status, pad;                     /* 0, or -1 when the neural state went non-finite */
    double arrival_s, admit_s, done_s;       /* server clock (seconds since creation) */
} nsb_serve_result;
/* Admission: first come first served while the neurons in flight stay within
 * max_inflight_neurons and the bytes of admitted episodes within
 * hbm_budget_bytes. Pools are sized for the in-flight cap. NULL on error. */
void *nsb_serve_create(long long max_inflight_neurons, double hbm_budget_bytes, double synapses_per_neuron,
                       int max_slots, int max_brain_neurons, int ticks, float gain, double smoothing);
void nsb_serve_destroy(void *server);
/* Genome in the ns_create row format with 8 channels and 2 motors; returns its id or -1. */
int nsb_serve_register(void *server, int count, int edges, const float *neuron_rows, const float *synapse_rows,
                       const int *motors);
/* Queue n episodes (genome id, seed, steps, caller tag, arrival time on the server clock). */
int nsb_serve_submit(void *server, int n, const int *genome, const uint32_t *seed, const int *steps,
                     const uint64_t *tag, const double *arrival_s);
/* Background loop thread. */
int nsb_serve_start(void *server);
int nsb_serve_stop(void *server);
/* Run the loop on the calling thread until nothing is queued or in flight. */
int nsb_serve_run(void *server, long long max_iterations);
/* Finished episodes, oldest first (nsb_serve_result[max]); returns the count or -1. */
int nsb_serve_poll(void *server, void *results, int max);
double nsb_serve_now(void *server);
/* steps, admitted, completed, queued, inflight, inflight_neurons, units,
 * neuron_ticks (of completed episodes), busy_s, elapsed_s, events,
 * pool_neurons, pool_synapses, pool_bytes, inflight_bytes,
 * neuron_ticks_launched (neurons in flight x ticks over launched steps).
 * Returns the count written (16). */
int nsb_serve_stats(void *server, double *out);

#ifdef __cplusplus
}
#endif
#endif
