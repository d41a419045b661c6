// Genome compiler: removes the neurons and synapses of a Gym-ABI genome that
// have no causal path to a motor neuron (mixic/neural-selection
// gym_adapter/compile_graph.py:10-28, which the reference's SpikingPolicy
// applies before ns_create unless GYM_FULL_GRAPH=1, gym_adapter/adapter.py:197-210).
//
// Reachability runs backwards from the motors over every active edge whose
// endpoints are active, inhibitory and modulatory edges included. Kept
// neurons stay in ascending original order, kept synapses in original order,
// rows are copied unchanged except for the remapped endpoints, and the
// original indices are returned for ns_original_indices so that reset
// streams stay those of the full genome. Motor outputs of the compiled genome
// therefore equal the full genome's.
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "ns_b200.h"

namespace nsb {
void set_error(const char *message);   // ns_abi.cu
}

extern "C" int nsb_compile_genome(int count, int edges, const float *neuron_rows, const float *synapse_rows,
                                  int outputs, const int *motors, float *out_neuron_rows, float *out_synapse_rows,
                                  int *out_motors, uint32_t *original_neurons, uint32_t *original_synapses,
                                  int *out_count, int *out_edges) {
    try {
        if (count < 0 || edges < 0 || outputs < 0 || (count && !neuron_rows) || (edges && !synapse_rows) ||
            (outputs && !motors) || !out_count || !out_edges)
            throw std::runtime_error("Invalid genome dimensions");
        // the edge rule of compile_graph.py:13-15 (truthiness of active flags)
        std::vector<int> head((size_t)count, -1), next((size_t)edges, -1);
        std::vector<int> pre((size_t)edges), post((size_t)edges);
        std::vector<char> usable((size_t)edges, 0);
        for (int j = 0; j < edges; ++j) {
            const float *e = synapse_rows + (size_t)j * 11;
            const int a = (int)e[0], b = (int)e[1];
            if (a < 0 || a >= count || b < 0 || b >= count) throw std::runtime_error("Invalid synapse gene");
            pre[j] = a;
            post[j] = b;
            if (e[3] != 0.0f && neuron_rows[(size_t)a * 10 + 2] != 0.0f && neuron_rows[(size_t)b * 10 + 2] != 0.0f) {
                usable[j] = 1;
                next[j] = head[b];
                head[b] = j;
            }
        }
        std::vector<char> live((size_t)count, 0);
        std::vector<int> stack;
        for (int m = 0; m < outputs; ++m) {
            if (motors[m] < 0 || motors[m] >= count) throw std::runtime_error("Invalid motor neuron");
            if (!live[motors[m]]) { live[motors[m]] = 1; stack.push_back(motors[m]); }
        }
        while (!stack.empty()) {
            const int b = stack.back();
            stack.pop_back();
            for (int j = head[b]; j >= 0; j = next[j])
                if (!live[pre[j]]) { live[pre[j]] = 1; stack.push_back(pre[j]); }
        }
        std::vector<int> remap((size_t)count, -1);
        int n = 0;
        for (int i = 0; i < count; ++i)
            if (live[i]) {
                remap[i] = n;
                if (out_neuron_rows)
                    for (int k = 0; k < 10; ++k) out_neuron_rows[(size_t)n * 10 + k] = neuron_rows[(size_t)i * 10 + k];
                if (original_neurons) original_neurons[n] = (uint32_t)i;
                ++n;
            }
        int m = 0;
        for (int j = 0; j < edges; ++j) {
            if (!usable[j] || !live[pre[j]] || !live[post[j]]) continue;
            if (out_synapse_rows) {
                float *o = out_synapse_rows + (size_t)m * 11;
                for (int k = 0; k < 11; ++k) o[k] = synapse_rows[(size_t)j * 11 + k];
                o[0] = (float)remap[pre[j]];
                o[1] = (float)remap[post[j]];
            }
            if (original_synapses) original_synapses[m] = (uint32_t)j;
            ++m;
        }
        if (out_motors)
            for (int k = 0; k < outputs; ++k) out_motors[k] = remap[motors[k]];
        *out_count = n;
        *out_edges = m;
        return 0;
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return -1;
    }
}
