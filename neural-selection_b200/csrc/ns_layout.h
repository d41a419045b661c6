// Device record layouts of the engine (host and device).
//
// Neuron and synapse state live in 64-byte records (four float4) so a warp
// moves whole records with 16-byte vector loads; genes are precomputed into
// records of the same shape. Field meanings follow the reference structs
// (src/physiology.cuh:29-76 of mixic/neural-selection); the layout is this
// engine's own.
#pragma once
#include <stdint.h>

namespace nsb {

constexpr int kBranches = 4;
constexpr int kRing = 32;          // spike-history ring (ticks); delays 1..31
constexpr int kMaxDelay = kRing - 1;

// ---- neuron gene record (16 x f32) ------------------------------------------
enum NGene : int {
    G_CAP = 0, G_GL, G_EL, G_VT,
    G_SLOPE, G_A, G_TAUW, G_B,
    G_VR, G_ADPB, G_ADPDECAY, G_GLSLOPE,   // ADPDECAY = exp(-0.25/tau_adp); GLSLOPE = gl*slope
    G_RECBASE, G_RECGAIN, G_RECEVENT, G_RECDECAY,  // RECDECAY = exp(-1/tau_receptor)
    G_WORDS
};
// neuron flag word
enum : uint32_t {
    NF_TYPE_MASK = 0x7u,         // bits 0-2 profile type 0..6
    NF_ACTIVE = 1u << 3,
    NF_INH = 1u << 4,            // inhibitory transmitter
    NF_MOD_SHIFT = 5,            // bits 5-6 modulator 0..3
    NF_GENE_SENS = 1u << 7,      // gene sensory_channel >= 0 (receptor enabled)
    NF_ADP = 1u << 8,            // afterdepolarisation tau > 0
    NF_HAS_INPUT = 1u << 9,      // ABI sensory index >= 0
    NF_EXC_TYPE = 1u << 10,      // type in {0,4,5}
    NF_PLASTIC_IN = 1u << 11,    // at least one incoming synapse is plastic
    NF_SLOT_SHIFT = 16,          // bits 16-22: the neuron's brain slot within its work unit
    NF_SLOT_MASK = 0x7fu,
};
// extended gene record for LP (type 2) / Prinz (type 3): 16 x f32
//   LP: [0..3] calcium, calcium_k, h, leak scales
//   Prinz: [0..7] g, [8] ambient leak
// ---- neuron state record (16 x 32-bit) ----------------------------------------
enum NState : int {
    S_V = 0, S_W, S_ADP, S_INH,
    S_DEPOL, S_LOGAMPA, S_RECNS, S_RECRNG,   // RECRNG is u32
    S_D0, S_D1, S_D2, S_D3,
    S_TOTAL, S_SPIKE, S_HIST, S_PAD,          // TOTAL i32, SPIKE u32 0/1, HIST u32 ring bits (tick & 31)
    S_WORDS
};
// extended state (types 2, 3, 6): 16 x f32 (the reference union, physiology.cuh:53)

// ---- synapse gene record (8 x 32-bit) -----------------------------------------
enum SGene : int { Y_W0 = 0, Y_U, Y_TREC, Y_TFAC, Y_SLOWREC, Y_SLOWDEPL, Y_INFO, Y_PAD, Y_WORDS };
// Y_INFO: bits 0-7 release sites (1..64), bits 8-15 receptor mask
// ---- synapse meta word (hot, read every tick) ---------------------------------
enum : uint32_t {
    M_PRE_MASK = 0xffffu,        // bits 0-15: presynaptic neuron, unit-local
    M_DELAY_SHIFT = 16,          // bits 16-20: delay 1..31
    M_BRANCH_SHIFT = 21,         // bits 21-22
    M_KIND_SHIFT = 23,           // bits 23-24: 0 excitatory release, 1 inhibitory direct, 2 modulatory release
    M_MODID_SHIFT = 25,          // bits 25-26: modulator - 1
    M_LIVE = 1u << 27,           // active edge with active endpoints
    M_PLASTIC = 1u << 28,        // live, plasticity != 0 and excitatory pair
    M_PROF_SHIFT = 29,           // bits 29-31 plasticity profile
};
enum : uint32_t { KIND_EXC = 0, KIND_INH = 1, KIND_MOD = 2 };
// ---- synapse state record (16 x 32-bit) ---------------------------------------
enum SState : int {
    Z_W = 0, Z_RU, Z_PRETR, Z_POSTTR,
    Z_ELTP, Z_ELTD, Z_DAAGE, Z_SPINE,
    Z_STAGE, Z_PREAGE, Z_POSTAGE, Z_SLOW,
    Z_READYLO, Z_READYHI, Z_RNG, Z_LAST,     // LAST: i32 last arrival tick
    Z_WORDS
};

// Correctly rounded constant exponentials (filled by the host at init).
struct PhysConst {
    float exc_ms, inh_ms, exc_sub, inh_sub;      // exp(-1/3), exp(-1/10), exp(-.25/3), exp(-.25/10)
    float ltp, ltd, ne, sht;                     // exp(-1/17), exp(-1/34), exp(-1/7200), exp(-1/3600)
    float lfs_thr, lfs_open[3];                  // exp(-1/10), exp(-1/{10,40,750})
    float prinz_ca, dend_offset;                 // exp(-.025/200), 5/(1+exp(10))
    float log_up, log_down;                      // log(1.92), log(0.70)
    float tp, tm, ty, te;                        // exp(-1/16.8), exp(-1/33.7), exp(-1/114), exp(-1/200): profile 6
};

// Canonical dump layout (shared with the oracle's or_dump): 32 words per
// neuron, 20 per synapse.
constexpr int kDumpNeuronWords = 32;
constexpr int kDumpSynapseWords = 20;

}  // namespace nsb
