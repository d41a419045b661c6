// ORACLE — test infrastructure only.
//
// Exhaustive check: the product's correctly rounded expf/logf
// (neural-selection_b200/csrc/ns_crmath.h) against the oracle's independent
// long-double/binary128 implementation (or_crmath.c), over every binary32
// input in [lo_bits, hi_bits) (both signs), split over threads. Also counts
// how often glibc's expf/logf differ from the correctly rounded value (the
// rate at which the reference's own host build departs from this engine).
//
// Usage: exhaustive_math <exp|log> <threads> [stride]
//   stride > 1 samples every stride-th bit pattern (for a quick run).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include "ns_crmath.h"

extern "C" float or_cr_expf(float);
extern "C" float or_cr_logf(float);

struct Tally { uint64_t checked = 0, bad = 0, glibc_diff = 0; uint32_t first_bad = 0; };

static bool same(float a, float b) {
    if (std::isnan(a) && std::isnan(b)) return true;
    uint32_t x, y; memcpy(&x, &a, 4); memcpy(&y, &b, 4); return x == y;
}

int main(int argc, char **argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s exp|log threads [stride]\n", argv[0]); return 2; }
    bool is_exp = strcmp(argv[1], "exp") == 0;
    int threads = atoi(argv[2]);
    uint64_t stride = argc > 3 ? strtoull(argv[3], nullptr, 10) : 1;
    std::vector<Tally> tally(threads);
    std::vector<std::thread> pool;
    const uint64_t total = 1ull << 32;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&, t] {
            Tally &my = tally[t];
            for (uint64_t u = (uint64_t)t * stride; u < total; u += (uint64_t)threads * stride) {
                uint32_t b = (uint32_t)u; float x; memcpy(&x, &b, 4);
                if (is_exp) {
                    if (!(x > -110.0f && x < 95.0f)) continue;   // outside: trivial 0/inf
                    float a = nsx::expf_cr(x), r = or_cr_expf(x);
                    ++my.checked;
                    if (!same(a, r)) { if (!my.bad) my.first_bad = b; ++my.bad; }
                    if (!same(expf(x), r)) ++my.glibc_diff;
                } else {
                    if (!(x >= 0.0f) || std::isinf(x)) continue;
                    float a = nsx::logf_cr(x), r = or_cr_logf(x);
                    ++my.checked;
                    if (!same(a, r)) { if (!my.bad) my.first_bad = b; ++my.bad; }
                    if (!same(logf(x), r)) ++my.glibc_diff;
                }
            }
        });
    }
    for (auto &th : pool) th.join();
    Tally sum;
    for (auto &x : tally) {
        sum.checked += x.checked; sum.bad += x.bad; sum.glibc_diff += x.glibc_diff;
        if (x.bad && !sum.first_bad) sum.first_bad = x.first_bad;
    }
    printf("{\"fn\": \"%s\", \"stride\": %llu, \"checked\": %llu, \"mismatches\": %llu, "
           "\"first_mismatch_bits\": %u, \"glibc_not_cr\": %llu}\n",
           argv[1], (unsigned long long)stride, (unsigned long long)sum.checked,
           (unsigned long long)sum.bad, sum.first_bad, (unsigned long long)sum.glibc_diff);
    return sum.bad ? 1 : 0;
}
