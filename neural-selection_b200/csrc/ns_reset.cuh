// Initial neuron and synapse state (src/physiology.cuh:179-202, 393-404 of
// mixic/neural-selection): seeds hashed per original index, xorshift32
// streams, and the reference's starting values.
#pragma once
#include <stdint.h>
#include "ns_layout.h"

namespace nsb {

__device__ __forceinline__ uint32_t seed_hash(uint32_t seed) {
    uint32_t x = seed ? seed : 1u;
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Neuron n of a pool: state record r (S_WORDS), heavy state xs (16 words, or
// nullptr), gene record g4 (4 x float4), flags, reset seed `seed + orig*7919`.
__device__ __forceinline__ void init_neuron(uint32_t *r, float *xs, const float4 *g4, uint32_t flags, uint32_t seed,
                                            uint32_t orig) {
    const uint32_t type = flags & NF_TYPE_MASK;
    const float el = g4[0].z;
    const uint32_t x = seed_hash(seed + orig * 7919u);
    for (int k = 0; k < S_WORDS; ++k) r[k] = 0u;
    float v = el;
    if (xs) {
        for (int k = 0; k < 16; ++k) xs[k] = 0.0f;
        if (type == 2) {
            const float init[16] = {-56, 0, .2f, 0, 1, 0, 0, 1, 0, 0, 1, 1, 0, .04f, .01f, -56};
            for (int k = 0; k < 16; ++k) xs[k] = init[k];
            v = xs[15] - 9.342518882f;
        } else if (type == 3) {
            xs[0] = -50.0f; xs[1] = .05f;
            for (int k = 0; k < 4; ++k) xs[9 + k] = 1.0f;
            v = xs[0];
        } else if (type == 6) {
            xs[0] = el;
            xs[1] = g4[0].w;   // threshold
        }
    }
    r[S_V] = __float_as_uint(v);
    r[S_RECRNG] = x ? x : 1u;
}

// Synapse e: state record z (Z_WORDS) from gene record y, seed `seed + orig*104729`.
__device__ __forceinline__ void init_synapse(uint32_t *z, const uint32_t *y, uint32_t seed, uint32_t orig) {
    uint32_t x = seed_hash(seed + orig * 104729u);
    if (!x) x = 1u;
    const int n = (int)(y[Y_INFO] & 0xffu);
    const uint64_t ready = n == 64 ? ~0ull : ((1ull << n) - 1ull);
    z[Z_W] = y[Y_W0];
    z[Z_RU] = 0u; z[Z_PRETR] = 0u; z[Z_POSTTR] = 0u; z[Z_ELTP] = 0u; z[Z_ELTD] = 0u;
    z[Z_DAAGE] = __float_as_uint(-1.0f); z[Z_SPINE] = __float_as_uint(1.0f); z[Z_STAGE] = __float_as_uint(-1.0f);
    z[Z_PREAGE] = __float_as_uint(1000000.0f); z[Z_POSTAGE] = __float_as_uint(1000000.0f);
    z[Z_SLOW] = __float_as_uint(1.0f);
    z[Z_READYLO] = (uint32_t)ready; z[Z_READYHI] = (uint32_t)(ready >> 32);
    z[Z_RNG] = x; z[Z_LAST] = (uint32_t)(-1000000);
}

}  // namespace nsb
