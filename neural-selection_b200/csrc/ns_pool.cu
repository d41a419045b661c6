// Deterministic slot allocation for the world simulator's neuron and synapse
// pools (src/main.cu:364-390 of mixic/neural-selection).
//
// The reference claims a slot with an atomic first-free-bit search starting
// at a hint word (claim_slot); under contention the slot a claim receives
// depends on thread timing. Run one claim after another in a given order, the
// result is a function of the bitmap and the hints alone, and that sequential
// replay is what "bit-exact pool allocation" means. This file performs it on
// the device: one thread walks the claims in order, with the reference's
// rules (search from word hint % words, wrapping; lowest free bit first; a
// free bit past the capacity ends the claim with -1).
#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace {

__device__ int claim_one(uint32_t *used, int capacity, int hint) {
    const int words = (capacity + 31) / 32;
    const int start = ((hint % words) + words) % words;
    for (int offset = 0; offset < words; ++offset) {
        const int word = (start + offset) % words;
        const uint32_t occupied = used[word];
        if (~occupied) {
            const int bit = __ffs(~occupied) - 1;
            const int slot = word * 32 + bit;
            if (slot >= capacity) return -1;
            used[word] = occupied | (1u << bit);
            return slot;
        }
    }
    return -1;
}

__global__ void claim_sequential(uint32_t *used, int capacity, const int *hints, int count, int *slots) {
    if (threadIdx.x || blockIdx.x) return;
    for (int i = 0; i < count; ++i) slots[i] = claim_one(used, capacity, hints[i]);
}

__global__ void release_slots(uint32_t *used, const int *slots, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int s = slots[i];
        if (s >= 0) atomicAnd(&used[s / 32], ~(1u << (s % 32)));
    }
}

struct DeviceInts {
    int *p = nullptr;
    explicit DeviceInts(int n) {
        if (cudaMalloc(reinterpret_cast<void **>(&p), sizeof(int) * (size_t)(n > 0 ? n : 1)) != cudaSuccess)
            throw std::runtime_error("CUDA: allocation failed");
    }
    ~DeviceInts() { cudaFree(p); }
};

void check(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
}

}  // namespace

namespace nsb {
void set_error(const char *message);
}

extern "C" {

// Claims `count` slots in order on the device bitmap `d_used` (capacity
// bits), each search starting at word hints[i] % words; slots[i] receives the
// slot or -1. Host arrays; synchronous.
int nsb_pool_claim(uint32_t *d_used, int capacity, const int *hints, int count, int *slots) {
    try {
        if (capacity < 1 || count < 0) throw std::runtime_error("Invalid pool claim");
        if (count == 0) return 0;
        DeviceInts h(count), s(count);
        check(cudaMemcpy(h.p, hints, sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
        claim_sequential<<<1, 1>>>(d_used, capacity, h.p, count, s.p);
        check(cudaGetLastError());
        check(cudaMemcpy(slots, s.p, sizeof(int) * (size_t)count, cudaMemcpyDeviceToHost));
        return 0;
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return -1;
    }
}

// Releases slots (negative entries ignored) on the device bitmap.
int nsb_pool_release(uint32_t *d_used, const int *slots, int count) {
    try {
        if (count < 0) throw std::runtime_error("Invalid pool release");
        if (count == 0) return 0;
        DeviceInts s(count);
        check(cudaMemcpy(s.p, slots, sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
        release_slots<<<(count + 255) / 256, 256>>>(d_used, s.p, count);
        check(cudaGetLastError());
        check(cudaDeviceSynchronize());
        return 0;
    } catch (const std::exception &e) {
        nsb::set_error(e.what());
        return -1;
    }
}

}  // extern "C"
