/* ORACLE — test infrastructure only. Nothing in the product library includes,
 * links or calls this code; tests, the smoke check and the CPU-baseline leg of
 * bench.py use it as the checker.
 *
 * A plain-C restatement of the reference's neural tick:
 *   physiology  src/physiology.cuh:29-586, src/lp_cell.cuh:16-113,
 *               src/prinz_cell.cuh:17-121
 *   ordering    gym_adapter/core.cuh:25-75 (edge order per tick)
 *   ABI rules   gym_adapter/native.cpp:46-108
 * Parity pin: built in its libm mode (-DOR_LIBM) it reproduces the reference
 * host executor compiled from the reference's own sources (oracle/_ref) bit for
 * bit; in its default mode exp/log are correctly rounded (or_crmath.c), which
 * is the arithmetic the CUDA engine implements.
 */
#ifndef NS_ORACLE_H
#define NS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Canonical state dump layout shared by oracle, reference harness and the
 * CUDA engine's state readback (32-bit words). */
enum { OR_NEURON_WORDS = 32, OR_SYNAPSE_WORDS = 20 };

typedef struct or_brain or_brain;

/* ns_create semantics (gym_adapter/native.cpp:46-82); max_delay is 8 for
 * the reference ABI and up to 31 for the extended delay ring. Returns NULL and
 * fills err on invalid input. */
or_brain *or_create(int count, int edges, int channels, int outputs,
                    const float *ng, const float *sg, const int *motors,
                    int max_delay, char *err, int errlen);
void or_original_indices(or_brain *b, const uint32_t *neurons, const uint32_t *synapses);
void or_destroy(or_brain *b);
/* Global modulator pulse: at every tick divisible by `period` (0: off) all
 * neurons' plasticity sees the modulator bits `mod` (1 NE, 2 5-HT, 4 DA). */
void or_set_pulse(or_brain *b, int period, int mod);
void or_reset(or_brain *b, uint32_t seed);
/* ns_step semantics: 0, or -1 on a non-finite voltage. When stop_on_nonfinite
 * is 0 the step records the failure, keeps integrating (the CUDA batch
 * semantics of gym_adapter/gpu.cu:49) and returns -1 at the end.
 * raster (optional): ticks x count spike bytes. */
int or_step(or_brain *b, const float *input, int ticks, float gain, float *output,
            uint8_t *raster, int stop_on_nonfinite);
/* Canonical dump: neurons count x 32 words, synapses edges x 20 words. */
void or_dump(const or_brain *b, uint32_t *nw, uint32_t *sw, int64_t *tick);
int or_count(const or_brain *b);
int or_edges(const or_brain *b);
/* Number of synapses that arrived (delivered a spike) during the last or_step. */
int64_t or_last_events(const or_brain *b);

/* FP64 shadow: the same equations in binary64, stepped beside the binary32
 * state with the binary32 run's discrete outcomes (spikes and their substep,
 * receptor events, released sites, modulator bits), tracking after every tick
 * the maximum absolute and relative error of each binary32 state field
 * against it. or_shadow_enable returns -1 for brains with LP/Prinz cells. */
enum { OR_SHADOW_FIELDS = 15 };
int or_shadow_enable(or_brain *b);
/* Maxima over all ticks since enabling; returns the number of ticks tracked
 * (-1 without a shadow). Relative error = |x32 - x64| / max(|x64|, floor)
 * with floor 1 for mV/pA fields and 1e-3 otherwise. V_subthreshold_mV counts
 * only neurons whose FP64 voltage is below their threshold V_T, that is,
 * outside the exponential upswing where the AdEx equation amplifies any
 * rounding difference by up to ~200x per 0.25 ms substep. */
int64_t or_shadow_stats(const or_brain *b, double *maxabs, double *maxrel);
/* FP64 shadow voltages (count) and synaptic weights (edges), either may be NULL. */
void or_shadow_dump(const or_brain *b, double *v, double *syn_w);
const char *or_shadow_field(int i);

/* Correctly rounded binary32 exp/log (or_crmath.c). */
float or_cr_expf(float x);
float or_cr_logf(float x);
float or_cr_sinf(float x);
float or_cr_cosf(float x);
float or_cr_hypotf(float x, float y);
/* The exp/log this build binds the physiology to. */
float or_bound_expf(float x);
float or_bound_logf(float x);

/* One genome-evaluation episode (or_episode.c): reset with `seed`, then
 * `steps` environment steps of `ticks` neural ticks on the pole-on-cart
 * environment of the serving loop. out[5] = steps run, reward (steps without
 * a fall), falls, trace (FNV-1a of action and motor counts per step), status
 * (0, or -1 after a non-finite voltage). Returns 0, or -1 on bad arguments. */
int or_episode(or_brain *b, uint32_t seed, int steps, int ticks, float gain, double smoothing, int32_t *out);
/* The environment's binary64 elementary functions (or_episode.c). */
double or_env_exp(double x);
double or_env_tanh(double x);
void or_env_sincos(double x, double *s, double *c);
/* Fixed environment sequence for build comparisons (or_episode.c). */
void or_env_sequence(uint64_t *out);

/* World neural stage (src/main.cu:659-801 ordering; or_world_step follows the
 * reference's tick-major order over every living animal, with the per-branch
 * sums in each animal's synapse list order). Host pools in the reference
 * record layouts, fields as the library's NsbWorldPools. */
typedef struct or_world_pools {
    const void *animals, *plasticity_cohort, *neurons, *synapses;
    void *neuron_state, *synapse_state;
    float *pending_exc, *pending_inh;
    const float *senses;
    unsigned long long *mod_event_tick;
    unsigned char *spike_history;
    const int *neuron_owner, *synapse_owner, *neuron_next, *synapse_next, *neuron_port;
    int *motors;
    int *trace_exc_arrivals, *trace_exc_releases, *trace_inh_arrivals;
    float *trace_exc_ns, *trace_inh_ns, *trace_peak_mv;
    int trace_animal, silence_senses, silence_contact;
    int animal_capacity, neuron_capacity, synapse_capacity;
} or_world_pools;
/* One world step's 16 ticks; 0, or -1 on a live synapse gene the engine
 * rejects (delay outside 1-8, branch above 3). */
int or_world_step(const or_world_pools *w, int64_t step);
/* Homeostasis after the body step (src/main.cu:1287-1300). */
void or_world_homeostasis(const or_world_pools *w);
/* The brain's records in the reference layouts (NeuronGene, NeuronState,
 * SynapseGene, SynapseState); any pointer may be NULL. */
void or_records(const or_brain *b, void *neuron_genes, void *neuron_states, void *synapse_genes,
                void *synapse_states);
/* sizeof Animal, PlasticityCohort, NeuronGene, NeuronState, SynapseGene,
 * SynapseState, then offsets of Animal.id, .age, .alive, .neuron_head,
 * .synapse_head, .neuron_count, .synapse_count, PlasticityCohort.frozen. */
int or_world_layout(uint64_t *out);

/* World ecology (src/main.cu:612-657, 1138-1338), the reference kernels run
 * as loops in ascending animal slot order. Fields as the library's
 * NsbWorldEcology (host pointers). */
typedef struct or_world_eco {
    int *food, *kind, *cell_head, *cell_next;
    unsigned char *bite_intent;
    uint32_t *neuron_used, *synapse_used;
    int *founder_motor_steps;
    int *founder_observed_steps, *deaths, *predation_deaths, *bites;
    void *life_records;
    int *life_count;
    void *bite_events;
    int *bite_event_count;
    int initial_count, instant_motors, life_capacity;
    int *neuron_clone;           /* [neuron_capacity] scratch of reproduce */
    int *births, *next_id;
} or_world_eco;
/* body_step, spatial index, bite_animals, finish_predation. */
void or_world_body_step(const or_world_pools *w, const or_world_eco *x, int64_t step);
/* reclaim_dead_genomes with release_genome. */
void or_world_reclaim(const or_world_pools *w, const or_world_eco *x, int64_t step);
/* reproduce with mutate, parents in ascending slot order. */
void or_world_reproduce(const or_world_pools *w, const or_world_eco *x);
/* regrow, spatial index, update_senses. */
void or_world_regrow_and_sense(const or_world_pools *w, const or_world_eco *x, int64_t step,
                               unsigned long long seed, float renewal);

/* Reference protocol checks (tests/physiology.cpp, tests/event_synapses.cpp,
 * tests/cuda_relay_parity.cu restated); results written as floats. */
int or_protocols(float *out, int n);

#ifdef __cplusplus
}
#endif
#endif
