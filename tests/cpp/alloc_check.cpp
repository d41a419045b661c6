// Randomised check of the serving loop's range allocator against a bitmap.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "ns_alloc.h"

int main(int argc, char **argv) {
    const long long cap = 10000;
    nsb::RangeAllocator a(cap);
    std::vector<char> used(cap, 0);
    std::vector<std::pair<long long, long long>> live;
    unsigned s = argc > 1 ? (unsigned)std::atoi(argv[1]) : 1u;
    auto rnd = [&]() { s = s * 1103515245u + 12345u; return (s >> 8) & 0xffffff; };
    for (int it = 0; it < 200000; ++it) {
        if (live.empty() || rnd() % 3 != 0) {
            const long long n = 1 + rnd() % 300;
            const long long p = a.allocate(n);
            if (p < 0) {
                // must really be full for n: no free run of length n
                long long run = 0, best = 0;
                for (long long i = 0; i < cap; ++i) { run = used[i] ? 0 : run + 1; if (run > best) best = run; }
                if (best >= n) { std::printf("FAIL: refused %lld with a free run of %lld\n", n, best); return 1; }
                continue;
            }
            for (long long i = p; i < p + n; ++i) {
                if (i >= cap || used[i]) { std::printf("FAIL: overlap at %lld\n", i); return 1; }
                used[i] = 1;
            }
            live.push_back({p, n});
        } else {
            const size_t k = rnd() % live.size();
            for (long long i = live[k].first; i < live[k].first + live[k].second; ++i) used[i] = 0;
            a.release(live[k].first, live[k].second);
            live[k] = live.back();
            live.pop_back();
        }
        long long u = 0;
        for (auto &l : live) u += l.second;
        if (u != a.used()) { std::printf("FAIL: used %lld != %lld\n", a.used(), u); return 1; }
    }
    for (auto &l : live) a.release(l.first, l.second);
    if (a.fragments() != 1 || a.largest() != cap) { std::printf("FAIL: not coalesced\n"); return 1; }
    std::printf("ok\n");
    return 0;
}
