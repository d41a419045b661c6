// ORACLE — test infrastructure only.
//
// Exhaustive check: the product's correctly rounded expf/logf
// (neural-selection_b200/csrc/ns_crmath.h) against the oracle's independent
// long-double/binary128 implementation (or_crmath.c), over every binary32
// input in [lo_bits, hi_bits) (both signs), split over threads. Also counts
// how often glibc's expf/logf differ from the correctly rounded value (the
// rate at which the reference's own host build departs from this engine).
//
// Usage: exhaustive_math <exp|log|sin|cos|hypot> <threads> [stride]
//   stride > 1 samples every stride-th bit pattern (for a quick run).
//   hypot (two arguments) pairs each sampled x with a y drawn from a
//   per-input xorshift stream: within a few binades of x, a random pattern,
//   and x scaled by a Pythagorean ratio (3/4, 5/12, 8/15), where exact
//   midpoints and ties occur.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include "ns_crmath.h"

extern "C" float or_cr_expf(float);
extern "C" float or_cr_logf(float);
extern "C" float or_cr_sinf(float);
extern "C" float or_cr_cosf(float);
extern "C" float or_cr_hypotf(float, float);

struct Tally { uint64_t checked = 0, bad = 0, glibc_diff = 0; uint32_t first_bad = 0; };

static bool same(float a, float b) {
    if (std::isnan(a) && std::isnan(b)) return true;
    uint32_t x, y; memcpy(&x, &a, 4); memcpy(&y, &b, 4); return x == y;
}

int main(int argc, char **argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s exp|log threads [stride]\n", argv[0]); return 2; }
    const int fn = strcmp(argv[1], "exp") == 0 ? 0 : strcmp(argv[1], "log") == 0 ? 1 :
                   strcmp(argv[1], "sin") == 0 ? 2 : strcmp(argv[1], "cos") == 0 ? 3 :
                   strcmp(argv[1], "hypot") == 0 ? 4 : -1;
    if (fn < 0) { fprintf(stderr, "unknown function %s\n", argv[1]); return 2; }
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
                if (fn == 0) {
                    if (!(x > -110.0f && x < 95.0f)) continue;   // outside: trivial 0/inf
                    float a = nsx::expf_cr(x), r = or_cr_expf(x);
                    ++my.checked;
                    if (!same(a, r)) { if (!my.bad) my.first_bad = b; ++my.bad; }
                    if (!same(expf(x), r)) ++my.glibc_diff;
                } else if (fn == 1) {
                    if (!(x >= 0.0f) || std::isinf(x)) continue;
                    float a = nsx::logf_cr(x), r = or_cr_logf(x);
                    ++my.checked;
                    if (!same(a, r)) { if (!my.bad) my.first_bad = b; ++my.bad; }
                    if (!same(logf(x), r)) ++my.glibc_diff;
                } else if (fn == 2 || fn == 3) {
                    if (std::isnan(x) || std::isinf(x)) continue;
                    float a = fn == 2 ? nsx::sinf_cr(x) : nsx::cosf_cr(x);
                    float r = fn == 2 ? or_cr_sinf(x) : or_cr_cosf(x);
                    ++my.checked;
                    if (!same(a, r)) { if (!my.bad) my.first_bad = b; ++my.bad; }
                    if (!same(fn == 2 ? sinf(x) : cosf(x), r)) ++my.glibc_diff;
                } else {
                    if (std::isnan(x) || std::isinf(x)) continue;
                    uint32_t s = b * 2654435761u + 12345u;
                    for (int k = 0; k < 4; ++k) {
                        s ^= s << 13; s ^= s >> 17; s ^= s << 5;
                        float y;
                        if (k == 0) y = std::ldexp(x, (int)(s % 17) - 8) * (1.0f + (s >> 20) * 0x1p-13f);
                        else if (k == 1) { uint32_t yb = s; memcpy(&y, &yb, 4); if (std::isnan(y)) y = 1.0f; }
                        else if (k == 2) y = x * (s & 1 ? 0.75f : 2.4f);
                        else y = x * (s & 1 ? 1.875f : 0.5333333f);
                        float a = nsx::hypotf_cr(x, y), r = or_cr_hypotf(x, y);
                        ++my.checked;
                        if (!same(a, r)) { if (!my.bad) my.first_bad = b; ++my.bad; }
                        if (!same(hypotf(x, y), r)) ++my.glibc_diff;
                    }
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
