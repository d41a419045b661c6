// Serving loop: admission, device-resident episodes, completion harvest.
#include "ns_serve.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "ns_env.h"
#include "ns_reset.cuh"

namespace nsb {

namespace {

// Per-slot episode state on the device.
struct SlotState {
    double x, xd, th, thd;
    float a0, a1;
    int steps_done, steps_total, reward, failures;
    uint32_t seed, trace;
    int active, pad;
};

struct DoneRec {
    int slot, reward, failures, steps;
    uint32_t trace;
    int status, pad0, pad1;
};

struct Ring {
    int count, pad[3];
    DoneRec rec[1];   // max_slots entries
};

// One admission round as staged in memory (byte offsets from the start).
struct StageHeader {
    int n_units, n_brains, pad0, pad1;
    long long off_units, off_brains, off_inptr, off_ngene, off_nflags, off_nsens, off_norig;
    long long off_smeta, off_sorig, off_sslot, off_sgene;
};
struct UnitDesc {
    int dst_n0, nn, dst_e0, ne;
    int src_n, src_e, src_b, nb;
    int src_i, uid, pad0, pad1;
};
struct BrainRec {
    int slot, steps;
    uint32_t seed;
    int motor0, motor1, pad0, pad1, pad2;
};

constexpr uint32_t kFnvOffset = 2166136261u;

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

}  // namespace

// ---- kernels ------------------------------------------------------------------

// One CTA per admitted unit: copy the staged records into their pool ranges
// and initialise neuron, synapse and episode state (ns_gpu_reset semantics
// for the brain; environment reset from the episode seed).
__global__ void admit_kernel(const unsigned char *stage, Pools P, int *ubrain, uint8_t *mask, int *status,
                             float *input, SlotState *slots) {
    const StageHeader *H = reinterpret_cast<const StageHeader *>(stage);
    const UnitDesc U = reinterpret_cast<const UnitDesc *>(stage + H->off_units)[blockIdx.x];
    const BrainRec *brains = reinterpret_cast<const BrainRec *>(stage + H->off_brains) + U.src_b;
    const int *s_inptr = reinterpret_cast<const int *>(stage + H->off_inptr) + U.src_i;
    const float4 *s_ngene = reinterpret_cast<const float4 *>(stage + H->off_ngene) + (size_t)U.src_n * 4;
    const uint32_t *s_nflags = reinterpret_cast<const uint32_t *>(stage + H->off_nflags) + U.src_n;
    const int *s_nsens = reinterpret_cast<const int *>(stage + H->off_nsens) + U.src_n;
    const uint32_t *s_norig = reinterpret_cast<const uint32_t *>(stage + H->off_norig) + U.src_n;
    const uint32_t *s_smeta = reinterpret_cast<const uint32_t *>(stage + H->off_smeta) + U.src_e;
    const uint32_t *s_sorig = reinterpret_cast<const uint32_t *>(stage + H->off_sorig) + U.src_e;
    const int *s_sslot = reinterpret_cast<const int *>(stage + H->off_sslot) + U.src_e;
    const uint4 *s_sgene = reinterpret_cast<const uint4 *>(stage + H->off_sgene) + (size_t)U.src_e * 2;
    float4 *ngene = const_cast<float4 *>(P.ngene);
    for (int q = threadIdx.x; q < U.nn; q += blockDim.x) {
        const int n = U.dst_n0 + q;
        for (int k = 0; k < 4; ++k) ngene[(size_t)n * 4 + k] = s_ngene[(size_t)q * 4 + k];
        const uint32_t f = s_nflags[q];
        const_cast<uint32_t *>(P.nflags)[n] = f;
        const_cast<int *>(P.nsens)[n] = s_nsens[q];
        const_cast<int *>(P.nxidx)[n] = -1;
        const int bi = (int)((f >> NF_SLOT_SHIFT) & NF_SLOT_MASK);
        init_neuron(P.nstate + (size_t)n * S_WORDS, nullptr, s_ngene + (size_t)q * 4, f, brains[bi].seed, s_norig[q]);
    }
    for (int q = threadIdx.x; q <= U.nn; q += blockDim.x) const_cast<int *>(P.inptr)[U.dst_n0 + q] = s_inptr[q];
    for (int q = threadIdx.x; q < U.ne; q += blockDim.x) {
        const int e = U.dst_e0 + q;
        const_cast<uint32_t *>(P.smeta)[e] = s_smeta[q];
        uint4 *y = reinterpret_cast<uint4 *>(const_cast<uint32_t *>(P.sgene) + (size_t)e * Y_WORDS);
        y[0] = s_sgene[(size_t)q * 2];
        y[1] = s_sgene[(size_t)q * 2 + 1];
        init_synapse(P.sstate + (size_t)e * Z_WORDS, P.sgene + (size_t)e * Y_WORDS, brains[s_sslot[q]].seed,
                     s_sorig[q]);
        P.sarrived[e] = 0;
        P.slastp[e] = -1;
    }
    for (int i = threadIdx.x; i < U.nb; i += blockDim.x) {
        const BrainRec B = brains[i];
        const int slot = B.slot;
        ubrain[(size_t)U.uid * kMaxUnitBrains + i] = slot;
        P.btick[slot] = 0;
        int *bm = const_cast<int *>(P.bmotor) + (size_t)slot * 2;
        bm[0] = B.motor0;
        bm[1] = B.motor1;
        mask[slot] = 1;
        status[slot] = 0;
        const nse::Cart c = nse::cart_initial(B.seed, 0u);
        nse::cart_encode(c, input + (size_t)slot * 8);
        SlotState s;
        s.x = c.x; s.xd = c.xd; s.th = c.th; s.thd = c.thd;
        s.a0 = 0.0f; s.a1 = 0.0f;
        s.steps_done = 0; s.steps_total = B.steps; s.reward = 0; s.failures = 0;
        s.seed = B.seed; s.trace = kFnvOffset; s.active = 1; s.pad = 0;
        slots[slot] = s;
    }
}

// After each tick-kernel launch: decode motor counts into an action, step
// the cart, encode the next observation; finish episodes that reached their
// length (or whose neural state went non-finite).
__global__ void env_kernel(SlotState *slots, int n_slots, const float *output, float *input, uint8_t *mask,
                           const int *status, Ring *ring, float keep, float smoothing) {
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n_slots; slot += gridDim.x * blockDim.x) {
        SlotState s = slots[slot];
        if (!s.active) continue;
        const float s0 = output[(size_t)slot * 2], s1 = output[(size_t)slot * 2 + 1];
        const int st = status[slot];
        bool finish = st != 0;
        if (!finish) {
            const int action = nse::decode_action(s.a0, s.a1, s0, s1, keep, smoothing, s.seed, (uint32_t)s.steps_done);
            s.trace = nse::trace_step(s.trace, action, s0, s1);
            nse::Cart c{s.x, s.xd, s.th, s.thd};
            if (nse::cart_step(c, action)) {
                ++s.failures;
                c = nse::cart_initial(s.seed, (uint32_t)s.failures);
            } else {
                ++s.reward;
            }
            s.x = c.x; s.xd = c.xd; s.th = c.th; s.thd = c.thd;
            ++s.steps_done;
            finish = s.steps_done >= s.steps_total;
            if (!finish) nse::cart_encode(c, input + (size_t)slot * 8);
        }
        if (finish) {
            s.active = 0;
            mask[slot] = 0;
            const int idx = atomicAdd(&ring->count, 1);
            DoneRec r;
            r.slot = slot; r.reward = s.reward; r.failures = s.failures; r.steps = s.steps_done;
            r.trace = s.trace; r.status = st; r.pad0 = 0; r.pad1 = 0;
            ring->rec[idx] = r;
        }
        slots[slot] = s;
    }
}

// ---- host ------------------------------------------------------------------------

template <class T> T *Server::alloc(size_t n) {
    T *p = nullptr;
    if (n == 0) n = 1;
    NSB_CHECK(cudaMalloc(reinterpret_cast<void **>(&p), n * sizeof(T)));
    allocations_.push_back(p);
    return p;
}

static constexpr double kNeuronBytes = 64 + 64 + 4 + 4 + 4 + 4;   // gene, state, flags, sensory, heavy idx, inptr
static constexpr double kSynapseBytes = 4 + 32 + 64 + 1 + 2;      // meta, gene, state, arrived, lastp

Server::Server(const ServeConfig &cfg) : cfg_(cfg) {
    if (cfg.block != 128 && cfg.block != 256) throw std::runtime_error("Invalid CUDA block size");
    if (cfg.max_slots < 1 || cfg.max_slots > (1 << 22)) throw std::runtime_error("Invalid episode slot count");
    if (cfg.max_brain_neurons < 1 || cfg.max_brain_neurons > kMaxBrainNeurons)
        throw std::runtime_error("Invalid maximum brain size");
    if (cfg.max_delay < 1 || cfg.max_delay > kMaxDelay) throw std::runtime_error("Invalid delay ring");
    if (cfg.ticks < 1 || cfg.ticks > 10000 || !std::isfinite(cfg.gain) || cfg.gain < 0)
        throw std::runtime_error("Invalid neural integration interval");
    if (!(cfg.smoothing > 0 && cfg.smoothing <= 1)) throw std::runtime_error("Smoothing must be in (0, 1]");
    if (cfg.max_inflight_neurons < cfg.max_brain_neurons) throw std::runtime_error("In-flight cap below one brain");
    epoch_ = std::chrono::steady_clock::now();
    keep_ = (float)(1.0 - cfg.smoothing);
    smooth_ = (float)cfg.smoothing;
    unit_cap_ = cfg.block * std::max(1, cfg.unit_slots);
    NSB_CHECK(cudaGetDevice(&dev_));
    NSB_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_));
    hw_ = spike_words(std::max(cfg.max_brain_neurons, unit_cap_), cfg.block);
    smem_ = serve_smem_bytes(hw_);
    prepare_tick_kernels(smem_);
    grid_cap_ = sms_ * tick_occupancy(cfg.block, smem_);

    const int max_units = cfg.max_slots;
    ncap_ = (long long)std::ceil((double)cfg.max_inflight_neurons * cfg.pool_headroom) + max_units;
    ecap_ = (long long)std::ceil((double)cfg.max_inflight_neurons * cfg.pool_headroom * cfg.synapses_per_neuron);
    if (ncap_ >= (1ll << 31) || ecap_ >= (1ll << 31)) throw std::runtime_error("Pool exceeds 2^31 entries");
    const double pool_bytes = ncap_ * kNeuronBytes + ecap_ * kSynapseBytes;
    if (pool_bytes > cfg.hbm_budget_bytes) throw std::runtime_error("HBM budget is below the pools for the in-flight cap");

    NSB_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        NSB_CHECK(cudaEventCreate(&ev_[i]));
        NSB_CHECK(cudaEventCreate(&t0_[i]));
        NSB_CHECK(cudaHostAlloc(reinterpret_cast<void **>(&h_stage_[i]), (size_t)cfg.staging_bytes, cudaHostAllocDefault));
        const size_t ring_bytes = sizeof(Ring) + sizeof(DoneRec) * (size_t)cfg.max_slots;
        NSB_CHECK(cudaHostAlloc(&h_ring_[i], ring_bytes, cudaHostAllocMapped));
        std::memset(h_ring_[i], 0, ring_bytes);
        NSB_CHECK(cudaHostGetDevicePointer(&d_ring_[i], h_ring_[i], 0));
    }
    d_stage_ = alloc<unsigned char>((size_t)cfg.staging_bytes);
    d_ngene_ = alloc<float>((size_t)ncap_ * 16);
    d_nflags_ = alloc<uint32_t>(ncap_);
    d_nsens_ = alloc<int>(ncap_);
    d_nxidx_ = alloc<int>(ncap_);
    NSB_CHECK(cudaMemset(d_nxidx_, 0xff, (size_t)ncap_ * sizeof(int)));
    d_nstate_ = alloc<uint32_t>((size_t)ncap_ * S_WORDS);
    d_inptr_ = alloc<int>(ncap_ + 1);
    d_xdummy_ = alloc<float>(16);
    d_smeta_ = alloc<uint32_t>(ecap_);
    d_sgene_ = alloc<uint32_t>((size_t)ecap_ * Y_WORDS);
    d_sstate_ = alloc<uint32_t>((size_t)ecap_ * Z_WORDS);
    d_sarrived_ = alloc<uint8_t>(ecap_);
    d_slastp_ = alloc<int16_t>(ecap_);
    NSB_CHECK(cudaMemset(d_slastp_, 0xff, (size_t)ecap_ * sizeof(int16_t)));
    d_btick_ = alloc<int64_t>(cfg.max_slots);
    NSB_CHECK(cudaMemset(d_btick_, 0, (size_t)cfg.max_slots * 8));
    d_bmotor_ = alloc<int>((size_t)cfg.max_slots * 2);
    NSB_CHECK(cudaMemset(d_bmotor_, 0, (size_t)cfg.max_slots * 2 * 4));
    d_units_ = alloc<int4>(max_units);
    d_unitb_ = alloc<int2>(max_units);
    d_ubrain_ = alloc<int>((size_t)max_units * kMaxUnitBrains);
    d_queue_ = alloc<int>(1);
    d_events_ = alloc<unsigned long long>(1);
    NSB_CHECK(cudaMemset(d_events_, 0, 8));
    d_input_ = alloc<float>((size_t)cfg.max_slots * 8);
    NSB_CHECK(cudaMemset(d_input_, 0, (size_t)cfg.max_slots * 8 * 4));
    d_mask_ = alloc<uint8_t>(cfg.max_slots);
    NSB_CHECK(cudaMemset(d_mask_, 0, cfg.max_slots));
    d_output_ = alloc<float>((size_t)cfg.max_slots * 2);
    NSB_CHECK(cudaMemset(d_output_, 0, (size_t)cfg.max_slots * 2 * 4));
    d_status_ = alloc<int>(cfg.max_slots);
    NSB_CHECK(cudaMemset(d_status_, 0, (size_t)cfg.max_slots * 4));
    d_slot_ = alloc<SlotState>(cfg.max_slots);
    NSB_CHECK(cudaMemset(d_slot_, 0, (size_t)cfg.max_slots * sizeof(SlotState)));
    NSB_CHECK(cudaDeviceSynchronize());

    nalloc_.reset(ncap_);
    ealloc_.reset(ecap_);
    free_slots_.resize(cfg.max_slots);
    for (int i = 0; i < cfg.max_slots; ++i) free_slots_[i] = cfg.max_slots - 1 - i;
    free_units_.resize(max_units);
    for (int i = 0; i < max_units; ++i) free_units_[i] = max_units - 1 - i;
    units_.resize(max_units);
    unit_live_.assign(max_units, 0);
    slots_.resize(cfg.max_slots);
}

Server::~Server() {
    try { stop(); } catch (...) {}
    if (stream_) cudaStreamSynchronize(stream_);
    for (int i = 0; i < 2; ++i) {
        if (ev_[i]) cudaEventDestroy(ev_[i]);
        if (t0_[i]) cudaEventDestroy(t0_[i]);
        if (h_stage_[i]) cudaFreeHost(h_stage_[i]);
        if (h_ring_[i]) cudaFreeHost(h_ring_[i]);
    }
    for (void *p : allocations_) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
}

double Server::now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - epoch_).count();
}

int Server::register_genome(const BrainSpec &b) {
    if (b.count < 1 || b.count > cfg_.max_brain_neurons) throw std::runtime_error("Genome size outside the server's range");
    for (int j = 0; j < b.count; ++j) {
        const unsigned char t = b.genes[j].type;
        if (t == 2 || t == 3 || t == 6) throw std::runtime_error("Serving supports AdEx-family cells only (types 0, 1, 4, 5)");
    }
    // One unit holding the whole brain, neurons in the planner's order.
    Plan p = make_plan(std::vector<BrainSpec>{b}, 8, 2, cfg_.max_delay, 1 << 30);
    Genome g;
    g.count = p.n_neurons;
    g.edges = p.n_synapses;
    g.ngene = std::move(p.ngene);
    g.nflags = std::move(p.nflags);
    g.norig = std::move(p.norig);
    g.smeta = std::move(p.smeta);
    g.sgene = std::move(p.sgene);
    g.sorig = std::move(p.sorig);
    g.nsens = std::move(p.nsens);
    g.inptr = std::move(p.inptr);
    g.motor = {p.bmotor[0], p.bmotor[1]};
    g.bytes = g.count * kNeuronBytes + g.edges * kSynapseBytes + sizeof(SlotState);
    std::lock_guard<std::mutex> lk(genome_mu_);
    genomes_.push_back(std::move(g));
    return (int)genomes_.size() - 1;
}

void Server::submit(int n, const int *genome, const uint32_t *seed, const int *steps, const uint64_t *tag,
                    const double *arrival_s) {
    int ng;
    {
        std::lock_guard<std::mutex> lk(genome_mu_);
        ng = (int)genomes_.size();
    }
    for (int i = 0; i < n; ++i) {
        if (genome[i] < 0 || genome[i] >= ng) throw std::runtime_error("Unknown genome id");
        if (steps[i] < 1 || steps[i] > 1000000) throw std::runtime_error("Invalid episode length");
        if (!std::isfinite(arrival_s[i])) throw std::runtime_error("Invalid arrival time");
    }
    std::lock_guard<std::mutex> lk(mu_);
    for (int i = 0; i < n; ++i) {
        Request r{genome[i], seed[i], steps[i], tag[i], arrival_s[i]};
        // keep the queue ordered by arrival time (stable for equal times)
        auto it = queue_.end();
        while (it != queue_.begin() && std::prev(it)->arrival > r.arrival) --it;
        queue_.insert(it, r);
    }
}

int Server::admit_round() {
    const double t = now();
    const size_t stage_limit = (size_t)cfg_.staging_bytes * 3 / 4;   // the last quarter holds the unit table
    std::lock_guard<std::mutex> glk(genome_mu_);
    std::vector<Request> taken;
    {
        std::lock_guard<std::mutex> lk(mu_);
        long long neurons = inflight_neurons_.load();
        double bytes = inflight_bytes_.load();
        size_t slots = free_slots_.size();
        size_t stage = 4096;
        while (!queue_.empty() && queue_.front().arrival <= t && taken.size() < slots) {
            const Request &r = queue_.front();
            const Genome &g = genomes_[r.genome];
            const size_t sb = (size_t)g.count * 96 + (size_t)g.edges * 48 + 256;
            if (neurons + g.count > cfg_.max_inflight_neurons || bytes + g.bytes > cfg_.hbm_budget_bytes ||
                stage + sb > stage_limit)
                break;
            neurons += g.count;
            bytes += g.bytes;
            stage += sb;
            taken.push_back(r);
            queue_.pop_front();
        }
    }
    if (taken.empty()) return 0;
    // Pack: brains above the unit capacity alone, the rest best-fit decreasing.
    std::vector<int> order(taken.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return genomes_[taken[a].genome].count > genomes_[taken[b].genome].count; });
    std::vector<std::vector<int>> packs;
    std::vector<int> fill;
    std::multimap<int, int> open;
    for (int i : order) {
        const int n = genomes_[taken[i].genome].count;
        if (n > unit_cap_) { packs.push_back({i}); fill.push_back(n); continue; }
        auto it = open.lower_bound(n);
        if (it != open.end()) {
            const int u = it->second;
            open.erase(it);
            packs[u].push_back(i);
            fill[u] += n;
            const int rem = unit_cap_ - fill[u];
            if (rem > 0 && (int)packs[u].size() < kMaxUnitBrains) open.emplace(rem, u);
        } else {
            packs.push_back({i});
            fill.push_back(n);
            if (unit_cap_ - n > 0) open.emplace(unit_cap_ - n, (int)packs.size() - 1);
        }
    }
    // Allocate ranges; units that do not fit go back to the queue.
    struct Placed { int pack; long long n0, e0; int nn, ne; int uid; };
    std::vector<Placed> placed;
    std::vector<Request> back;
    for (int u = 0; u < (int)packs.size(); ++u) {
        int nn = 0, ne = 0;
        for (int i : packs[u]) { nn += genomes_[taken[i].genome].count; ne += genomes_[taken[i].genome].edges; }
        long long n0 = -1, e0 = -1;
        if (!free_units_.empty()) {
            n0 = nalloc_.allocate(nn + 1);
            if (n0 >= 0 && ne > 0) {
                e0 = ealloc_.allocate(ne);
                if (e0 < 0) { nalloc_.release(n0, nn + 1); n0 = -1; }
            } else if (n0 >= 0) {
                e0 = 0;
            }
        }
        if (n0 < 0) {
            for (int i : packs[u]) back.push_back(taken[i]);
            continue;
        }
        const int uid = free_units_.back();
        free_units_.pop_back();
        placed.push_back({u, n0, e0, nn, ne, uid});
    }
    if (!back.empty()) {
        std::stable_sort(back.begin(), back.end(), [](const Request &a, const Request &b) { return a.arrival < b.arrival; });
        std::lock_guard<std::mutex> lk(mu_);
        for (auto it = back.rbegin(); it != back.rend(); ++it) queue_.push_front(*it);
    }
    if (placed.empty()) return 0;

    // ---- stage records ----
    long long tot_n = 0, tot_e = 0, tot_b = 0, tot_i = 0;
    for (auto &p : placed) { tot_n += p.nn; tot_e += p.ne; tot_b += (long long)packs[p.pack].size(); tot_i += p.nn + 1; }
    const int par = (int)(iter_ & 1);
    unsigned char *S = h_stage_[par];
    StageHeader H{};
    size_t off = align16(sizeof(StageHeader));
    H.off_units = (long long)off; off = align16(off + sizeof(UnitDesc) * placed.size());
    H.off_brains = (long long)off; off = align16(off + sizeof(BrainRec) * (size_t)tot_b);
    H.off_inptr = (long long)off; off = align16(off + 4 * (size_t)tot_i);
    H.off_ngene = (long long)off; off = align16(off + 64 * (size_t)tot_n);
    H.off_nflags = (long long)off; off = align16(off + 4 * (size_t)tot_n);
    H.off_nsens = (long long)off; off = align16(off + 4 * (size_t)tot_n);
    H.off_norig = (long long)off; off = align16(off + 4 * (size_t)tot_n);
    H.off_smeta = (long long)off; off = align16(off + 4 * (size_t)tot_e);
    H.off_sorig = (long long)off; off = align16(off + 4 * (size_t)tot_e);
    H.off_sslot = (long long)off; off = align16(off + 4 * (size_t)tot_e);
    H.off_sgene = (long long)off; off = align16(off + 32 * (size_t)tot_e);
    if (off > stage_limit) throw std::runtime_error("admission round exceeds the staging buffer");
    H.n_units = (int)placed.size();
    H.n_brains = (int)tot_b;
    std::memcpy(S, &H, sizeof H);
    UnitDesc *ud = reinterpret_cast<UnitDesc *>(S + H.off_units);
    BrainRec *br = reinterpret_cast<BrainRec *>(S + H.off_brains);
    int *sinptr = reinterpret_cast<int *>(S + H.off_inptr);
    float *sngene = reinterpret_cast<float *>(S + H.off_ngene);
    uint32_t *snflags = reinterpret_cast<uint32_t *>(S + H.off_nflags);
    int *snsens = reinterpret_cast<int *>(S + H.off_nsens);
    uint32_t *snorig = reinterpret_cast<uint32_t *>(S + H.off_norig);
    uint32_t *ssmeta = reinterpret_cast<uint32_t *>(S + H.off_smeta);
    uint32_t *ssorig = reinterpret_cast<uint32_t *>(S + H.off_sorig);
    int *ssslot = reinterpret_cast<int *>(S + H.off_sslot);
    uint32_t *ssgene = reinterpret_cast<uint32_t *>(S + H.off_sgene);
    long long cn = 0, ce = 0, cb = 0, ci = 0;
    for (size_t k = 0; k < placed.size(); ++k) {
        const Placed &p = placed[k];
        const auto &members = packs[p.pack];
        UnitDesc d{};
        d.dst_n0 = (int)p.n0; d.nn = p.nn; d.dst_e0 = (int)p.e0; d.ne = p.ne;
        d.src_n = (int)cn; d.src_e = (int)ce; d.src_b = (int)cb; d.nb = (int)members.size();
        d.src_i = (int)ci; d.uid = p.uid;
        ud[k] = d;
        Unit &U = units_[p.uid];
        U.n0 = p.n0; U.nalloc = p.nn + 1; U.e0 = p.e0; U.ne = p.ne; U.nn = p.nn;
        U.remaining = (int)members.size();
        U.slots.clear();
        int no = 0, eo = 0;
        for (int bi = 0; bi < (int)members.size(); ++bi) {
            const Request &r = taken[members[bi]];
            const Genome &g = genomes_[r.genome];
            const int slot = free_slots_.back();
            free_slots_.pop_back();
            U.slots.push_back(slot);
            SlotInfo &si = slots_[slot];
            si.unit = p.uid; si.req = r; si.admit = t; si.bytes = g.bytes; si.neurons = g.count;
            inflight_neurons_ += g.count;
            inflight_bytes_.store(inflight_bytes_.load() + g.bytes);
            ++inflight_;
            ++admitted_;
            BrainRec b{};
            b.slot = slot; b.steps = r.steps; b.seed = r.seed;
            b.motor0 = (int)p.n0 + no + g.motor[0];
            b.motor1 = (int)p.n0 + no + g.motor[1];
            br[cb + bi] = b;
            for (int q = 0; q < g.count; ++q) {
                const long long s = cn + no + q;
                std::memcpy(sngene + s * 16, &g.ngene[(size_t)q * 16], 64);
                snflags[s] = (g.nflags[q] & ~((uint32_t)NF_SLOT_MASK << NF_SLOT_SHIFT)) | ((uint32_t)bi << NF_SLOT_SHIFT);
                snsens[s] = g.nsens[q];
                snorig[s] = g.norig[q];
                sinptr[ci + no + q] = (int)p.e0 + eo + g.inptr[q];
            }
            for (int q = 0; q < g.edges; ++q) {
                const long long s = ce + eo + q;
                const uint32_t m = g.smeta[q];
                const uint32_t pre = (m & M_PRE_MASK) + (uint32_t)no;
                if (pre > M_PRE_MASK) throw std::runtime_error("Unit exceeds 65536 neurons");
                ssmeta[s] = (m & ~M_PRE_MASK) | pre;
                ssorig[s] = g.sorig[q];
                ssslot[s] = bi;
                std::memcpy(ssgene + s * 8, &g.sgene[(size_t)q * 8], 32);
            }
            no += g.count;
            eo += g.edges;
        }
        sinptr[ci + p.nn] = (int)p.e0 + p.ne;
        cn += p.nn; ce += p.ne; cb += (long long)members.size(); ci += p.nn + 1;
        unit_live_[p.uid] = 1;
        active_units_.push_back(p.uid);
        ++n_units_live_;
    }
    NSB_CHECK(cudaMemcpyAsync(d_stage_, S, off, cudaMemcpyHostToDevice, stream_));
    Pools P{};
    P.ngene = reinterpret_cast<const float4 *>(d_ngene_); P.nflags = d_nflags_; P.nsens = d_nsens_; P.nxidx = d_nxidx_;
    P.xgene = d_xdummy_; P.xstate = d_xdummy_; P.nstate = d_nstate_; P.inptr = d_inptr_;
    P.smeta = d_smeta_; P.sgene = d_sgene_; P.sstate = d_sstate_; P.sarrived = d_sarrived_; P.slastp = d_slastp_;
    P.btick = d_btick_; P.bmotor = d_bmotor_; P.units = d_units_; P.unitb = d_unitb_; P.ubrain = d_ubrain_;
    P.channels = 8; P.outputs = 2; P.hw = hw_; P.events = d_events_;
    admit_kernel<<<(int)placed.size(), 256, 0, stream_>>>(d_stage_, P, d_ubrain_, d_mask_, d_status_, d_input_,
                                                         reinterpret_cast<SlotState *>(d_slot_));
    NSB_CHECK(cudaGetLastError());
    table_dirty_ = true;
    return (int)tot_b;
}

void Server::upload_unit_table() {
    // Largest units first (the persistent grid pulls from the front).
    std::stable_sort(active_units_.begin(), active_units_.end(),
                     [&](int a, int b) { return units_[a].nn > units_[b].nn; });
    n_table_ = (int)active_units_.size();
    if (n_table_ == 0) { table_dirty_ = false; return; }
    const int par = (int)(iter_ & 1);
    // The table goes at the end of this admission round's staging buffer.
    const size_t bytes = (size_t)n_table_ * (sizeof(int4) + sizeof(int2));
    if (bytes > (size_t)cfg_.staging_bytes / 4) throw std::runtime_error("unit table exceeds the staging buffer");
    unsigned char *base = h_stage_[par] + (size_t)cfg_.staging_bytes - align16(bytes);
    int4 *tu = reinterpret_cast<int4 *>(base);
    int2 *tb = reinterpret_cast<int2 *>(base + sizeof(int4) * (size_t)n_table_);
    for (int i = 0; i < n_table_; ++i) {
        const Unit &U = units_[active_units_[i]];
        tu[i] = make_int4((int)U.n0, U.nn, (int)U.e0, (int)U.ne);
        tb[i] = make_int2(active_units_[i] * kMaxUnitBrains, (int)U.slots.size());
    }
    NSB_CHECK(cudaMemcpyAsync(d_units_, tu, sizeof(int4) * (size_t)n_table_, cudaMemcpyHostToDevice, stream_));
    NSB_CHECK(cudaMemcpyAsync(d_unitb_, tb, sizeof(int2) * (size_t)n_table_, cudaMemcpyHostToDevice, stream_));
    table_dirty_ = false;
}

void Server::retire(int slot) {
    SlotInfo &si = slots_[slot];
    inflight_neurons_ -= si.neurons;
    inflight_bytes_.store(inflight_bytes_.load() - si.bytes);
    --inflight_;
    const int uid = si.unit;
    si.unit = -1;
    Unit &U = units_[uid];
    if (--U.remaining > 0) return;
    // Every episode of the unit has finished: free its ranges, slots and id.
    nalloc_.release(U.n0, U.nalloc);
    if (U.ne > 0) ealloc_.release(U.e0, U.ne);
    for (int s : U.slots) free_slots_.push_back(s);
    U.slots.clear();
    unit_live_[uid] = 0;
    free_units_.push_back(uid);
    active_units_.erase(std::find(active_units_.begin(), active_units_.end(), uid));
    --n_units_live_;
    table_dirty_ = true;
}

void Server::harvest(int ring) {
    Ring *R = reinterpret_cast<Ring *>(h_ring_[ring]);
    const int n = R->count;
    if (n == 0) return;
    const double t = now();
    std::vector<ServeResult> out;
    out.reserve(n);
    for (int i = 0; i < n; ++i) {
        const DoneRec r = R->rec[i];
        const SlotInfo &si = slots_[r.slot];
        ServeResult res;
        res.tag = si.req.tag;
        res.genome = si.req.genome;
        res.steps = r.steps;
        res.reward = r.reward;
        res.failures = r.failures;
        res.trace = r.trace;
        res.seed = si.req.seed;
        res.status = r.status;
        res.arrival_s = si.req.arrival;
        res.admit_s = si.admit;
        res.done_s = t;
        neuron_ticks_.store(neuron_ticks_.load() + (double)si.neurons * r.steps * cfg_.ticks);
        out.push_back(res);
        retire(r.slot);
        ++completed_;
    }
    R->count = 0;
    std::lock_guard<std::mutex> lk(mu_);
    for (auto &r : out) done_.push_back(r);
}

void Server::iteration() {
    const int par = (int)(iter_ & 1), prev = par ^ 1;
    if (admit_round() == 0 && inflight_ == 0 && !pending_[0] && !pending_[1]) {
        // Nothing in flight and the head of the queue has arrived but was not
        // admitted: it can never fit this server's pools or budget.
        std::lock_guard<std::mutex> lk(mu_);
        if (!queue_.empty() && queue_.front().arrival <= now())
            throw std::runtime_error("Queued episode does not fit the server's pools or HBM budget");
    }
    if (table_dirty_) upload_unit_table();
    bool stepped = false;
    if (n_table_ > 0) {
        Pools P{};
        P.ngene = reinterpret_cast<const float4 *>(d_ngene_); P.nflags = d_nflags_; P.nsens = d_nsens_;
        P.nxidx = d_nxidx_; P.xgene = d_xdummy_; P.xstate = d_xdummy_; P.nstate = d_nstate_; P.inptr = d_inptr_;
        P.smeta = d_smeta_; P.sgene = d_sgene_; P.sstate = d_sstate_; P.sarrived = d_sarrived_;
        P.slastp = d_slastp_; P.btick = d_btick_; P.bmotor = d_bmotor_; P.units = d_units_; P.unitb = d_unitb_;
        P.ubrain = d_ubrain_; P.channels = 8; P.outputs = 2; P.hw = hw_; P.events = d_events_;
        NSB_CHECK(cudaEventRecord(t0_[par], stream_));
        launch_tick_light(P, n_table_, std::min(n_table_, grid_cap_), cfg_.block, smem_, d_queue_, d_input_, d_mask_,
                          d_output_, d_status_, cfg_.ticks, cfg_.gain, stream_);
        env_kernel<<<std::max(1, std::min((cfg_.max_slots + 255) / 256, sms_ * 4)), 256, 0, stream_>>>(
            reinterpret_cast<SlotState *>(d_slot_), cfg_.max_slots, d_output_, d_input_, d_mask_, d_status_,
            reinterpret_cast<Ring *>(d_ring_[par]), keep_, smooth_);
        NSB_CHECK(cudaGetLastError());
        ++steps_run_;
        launched_ticks_.store(launched_ticks_.load() + (double)inflight_neurons_.load() * cfg_.ticks);
        stepped = true;
    }
    NSB_CHECK(cudaEventRecord(ev_[par], stream_));
    // The previous iteration's step has had this iteration's host work to run
    // behind; collect its completions.
    if (iter_ > 0) {
        NSB_CHECK(cudaEventSynchronize(ev_[prev]));
        if (pending_[prev]) {
            float ms = 0;
            NSB_CHECK(cudaEventElapsedTime(&ms, t0_[prev], ev_[prev]));
            busy_s_.store(busy_s_.load() + ms / 1e3);
            harvest(prev);
        }
    }
    pending_[par] = stepped;
    ++iter_;
}

void Server::run_until_idle(long long max_iterations) {
    if (running_) throw std::runtime_error("Server loop is running");
    NSB_CHECK(cudaSetDevice(dev_));
    for (long long i = 0; i < max_iterations; ++i) {
        bool queued;
        {
            std::lock_guard<std::mutex> lk(mu_);
            queued = !queue_.empty();
        }
        if (!queued && inflight_ == 0 && !pending_[0] && !pending_[1]) break;
        iteration();
    }
    drain();
}

void Server::drain() {
    NSB_CHECK(cudaStreamSynchronize(stream_));
    // the older of the two pending steps first
    const int newest = (int)((iter_ + 1) & 1);
    for (int k : {newest ^ 1, newest})
        if (pending_[k]) {
            float ms = 0;
            NSB_CHECK(cudaEventElapsedTime(&ms, t0_[k], ev_[k]));
            busy_s_.store(busy_s_.load() + ms / 1e3);
            harvest(k);
            pending_[k] = false;
        }
}

void Server::loop() {
    cudaSetDevice(dev_);
    while (running_) {
        bool idle;
        double next = -1;
        {
            std::lock_guard<std::mutex> lk(mu_);
            idle = inflight_ == 0 && !pending_[0] && !pending_[1];
            if (!queue_.empty()) next = queue_.front().arrival;
        }
        if (idle && (next < 0 || next > now())) {
            std::this_thread::sleep_for(std::chrono::microseconds(100));
            continue;
        }
        try {
            iteration();
        } catch (const std::exception &e) {
            std::lock_guard<std::mutex> lk(mu_);
            error_ = e.what();
            running_ = false;
            return;
        }
    }
    try {
        drain();
    } catch (const std::exception &e) {
        std::lock_guard<std::mutex> lk(mu_);
        error_ = e.what();
    }
}

std::string Server::error() {
    std::lock_guard<std::mutex> lk(mu_);
    return error_;
}

void Server::start() {
    if (running_) return;
    running_ = true;
    thread_ = std::thread([this] { loop(); });
}

void Server::stop() {
    if (!running_ && !thread_.joinable()) return;
    running_ = false;
    if (thread_.joinable()) thread_.join();
}

int Server::poll(ServeResult *out, int max) {
    std::lock_guard<std::mutex> lk(mu_);
    int n = 0;
    while (n < max && !done_.empty()) {
        out[n++] = done_.front();
        done_.pop_front();
    }
    return n;
}

ServeStats Server::stats() {
    ServeStats s{};
    {
        std::lock_guard<std::mutex> lk(mu_);
        s.queued = (long long)queue_.size();
    }
    s.steps = steps_run_;
    s.admitted = admitted_;
    s.completed = completed_;
    s.inflight = inflight_;
    s.inflight_neurons = inflight_neurons_;
    s.units = n_units_live_;
    s.neuron_ticks = neuron_ticks_;
    s.busy_s = busy_s_;
    s.elapsed_s = now();
    unsigned long long ev = 0;
    NSB_CHECK(cudaMemcpy(&ev, d_events_, 8, cudaMemcpyDeviceToHost));
    s.events = ev;
    s.pool_neurons = ncap_;
    s.pool_synapses = ecap_;
    s.pool_bytes = ncap_ * kNeuronBytes + ecap_ * kSynapseBytes;
    s.inflight_bytes = inflight_bytes_;
    s.neuron_ticks_launched = launched_ticks_;
    return s;
}

}  // namespace nsb
