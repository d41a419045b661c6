// ORACLE — test infrastructure only.
//
// Builds the reference's own host executor, gym_adapter/native.cpp (with
// gym_adapter/core.cuh and src/physiology.cuh), in place from the reference
// source tree, and adds two read-only exports for parity checks:
//   ref_dump         canonical state dump (same layout as the oracle's or_dump)
//   ref_step_raster  ns_step that also records the per-tick spike raster
// The raster is captured through core.cuh's PHASE_END(2) hook (the point after
// every neuron has advanced, core.cuh:59); the reference code is unmodified.
// Built twice by oracle/build.py: against glibc expf/logf (the reference as
// shipped) and with -include ref_cr_shim.h (exp/log correctly rounded).
#include <cstdint>
#include <cstring>

static uint8_t *g_raster = nullptr;
static int g_raster_tick = 0;

#define PHASE_START
#define PHASE_END(i)                                                        \
    do {                                                                    \
        if ((i) == 2 && g_raster) {                                         \
            for (int q_ = 0; q_ < b.count; ++q_)                            \
                g_raster[(size_t)g_raster_tick * b.count + q_] = b.neurons[q_].spike; \
            ++g_raster_tick;                                                \
        }                                                                   \
    } while (0)
#include "core.cuh"
#undef PHASE_START
#undef PHASE_END
#include "native.cpp"

static uint32_t word_of(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

extern "C" void ref_dump(void *p, uint32_t *nw, uint32_t *sw, int64_t *tick) {
    auto &b = *static_cast<Brain *>(p);
    if (tick) *tick = b.tick;
    for (size_t i = 0; nw && i < b.neurons.size(); ++i) {
        const auto &s = b.neurons[i];
        uint32_t *o = nw + i * 32;
        std::memset(o, 0, 32 * 4);
        o[0] = word_of(s.voltage_mv); o[1] = word_of(s.adaptation_pa);
        o[2] = word_of(s.afterdepol_pa); o[3] = word_of(s.inh_ns);
        o[4] = word_of(s.recent_depol_mv); o[5] = word_of(s.log_ampa_scale);
        for (int k = 0; k < 4; ++k) o[6 + k] = word_of(s.dendrite_exc_ns[k]);
        std::memcpy(o + 10, &s.lp, 64);   // the union's 16 words
        o[26] = (uint32_t)s.total_spikes; o[27] = s.spike;
        o[28] = word_of(s.receptor_ns); o[29] = s.receptor_rng;
        uint32_t h = 0;
        for (int k = 0; k < 8; ++k) {
            int64_t t = b.tick - 1 - k;
            if (t < 0) break;
            if (b.history[i][t % 9]) h |= 1u << k;
        }
        o[30] = h;
    }
    for (size_t i = 0; sw && i < b.synapses.size(); ++i) {
        const auto &s = b.synapses[i];
        uint32_t *o = sw + i * 20;
        std::memset(o, 0, 20 * 4);
        o[0] = word_of(s.weight_ns); o[1] = word_of(s.running_utilization);
        o[2] = word_of(s.pre_trace); o[3] = word_of(s.post_trace);
        o[4] = word_of(s.eligible_ltp); o[5] = word_of(s.eligible_ltd);
        o[6] = word_of(s.da_age_ms); o[7] = word_of(s.spine_volume);
        o[8] = word_of(s.structural_age_ms); o[9] = word_of(s.pre_age_ms);
        o[10] = word_of(s.post_age_ms);
        o[11] = (uint32_t)(uint64_t)s.last_arrival_tick;
        o[12] = (uint32_t)((uint64_t)s.last_arrival_tick >> 32);
        o[13] = (uint32_t)s.ready_mask; o[14] = (uint32_t)(s.ready_mask >> 32);
        o[15] = s.rng_state; o[16] = s.arrived; o[17] = word_of(s.slow_resource);
    }
}

extern "C" int ref_step_raster(void *p, const float *input, int ticks, float gain,
                               float *output, uint8_t *raster) {
    g_raster = raster;
    g_raster_tick = 0;
    int rc = ns_step(p, input, ticks, gain, output);
    g_raster = nullptr;
    return rc;
}
