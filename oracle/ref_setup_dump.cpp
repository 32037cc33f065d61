// TEST INFRASTRUCTURE ONLY.  Driver that compiles the reference's own
// header-only basis setup (rns/host_setup.h:61-126, which needs only
// wide_host.h) and prints its constants, so the oracle's restatement of that
// setup can be checked value by value.  Built by oracle/Makefile into
// oracle/_ref/ when the reference sources are present; never shipped.
//
//   ref_setup_dump <n> <q as 28 hex u32 words, least significant first>
// prints one line per prime: p reciprocal psi bases_mod_q[29 words]
// and a final line: P mod q [29 words].
#include "rns/host_setup.h"
#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    if (argc != 2 + rns::AbiWords) {
        std::fprintf(stderr, "usage: %s n w0 .. w27 (hex)\n", argv[0]);
        return 2;
    }
    unsigned n = unsigned(std::strtoul(argv[1], nullptr, 10));
    rns::Words q(rns::AbiWords);
    for (unsigned i = 0; i < rns::AbiWords; ++i) q[i] = uint32_t(std::strtoul(argv[2 + i], nullptr, 16));
    auto s = rns::setup(n, q);
    for (unsigned i = 0; i < rns::PrimeCount; ++i) {
        std::printf("%u %llu %u", s.mods[i].p, (unsigned long long)s.mods[i].reciprocal,
                    s.forward[size_t(i) * n + (n > 1 ? 1 : 0)].value);
        for (unsigned k = 0; k < rns::AccumWords; ++k) std::printf(" %u", s.bases_mod_q[i * rns::AccumWords + k]);
        std::printf("\n");
    }
    for (unsigned k = 0; k < s.product_mod_q.size() && k < rns::AccumWords; ++k)
        std::printf("%s%u", k ? " " : "", s.product_mod_q[k]);
    std::printf("\n");
    return 0;
}
