// Prints the library's environment functions (ns_env.h, host build) for the
// inputs read from stdin, one hex double per value, so the test can compare
// them bit for bit with the oracle's restatement.
#include <cstdio>
#include <cstdint>
#include <cstring>
#include "ns_env.h"

static unsigned long long bits(double d) { unsigned long long u; std::memcpy(&u, &d, 8); return u; }

int main() {
    double x;
    while (std::scanf("%lf", &x) == 1) {
        double s, c;
        nse::det_sincos(x, &s, &c);
        std::printf("%016llx %016llx %016llx %016llx\n", bits(nse::det_exp(x)), bits(nse::det_tanh(x)), bits(s),
                    bits(c));
    }
    // a short episode of the environment alone: fixed action pattern
    nse::Cart cart = nse::cart_initial(12345u, 0u);
    float enc[8];
    uint32_t h = 2166136261u;
    for (int t = 0; t < 500; ++t) {
        const int a = (t / 7) & 1;
        if (nse::cart_step(cart, a)) cart = nse::cart_initial(12345u, (uint32_t)t + 1);
        nse::cart_encode(cart, enc);
        for (int i = 0; i < 8; ++i) { uint32_t u; std::memcpy(&u, &enc[i], 4); h = (h ^ u) * 16777619u; }
    }
    float a0 = 0, a1 = 0;
    uint32_t acts = 0;
    for (int t = 0; t < 64; ++t)
        acts = acts * 3u + (uint32_t)nse::decode_action(a0, a1, (float)(t % 3), (float)(t % 2), 0.6f, 0.4f, 7u, (uint32_t)t);
    std::printf("episode %016llx %016llx %08x %08x\n", bits(cart.x), bits(cart.thd), h, acts);
    return 0;
}
