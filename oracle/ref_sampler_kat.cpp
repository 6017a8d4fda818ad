// TEST INFRASTRUCTURE ONLY. Prints known-answer vectors of the reference's own PCG32 sampler
// (threedgptir_tracer/include/3dgptir/kernels/cuda/sampler.cuh, compiled for the host by
// oracle/Makefile). Output: one JSON object on stdout.
#include <cstdio>

#include <3dgptir/kernels/cuda/sampler.cuh>

int main() {
    const unsigned cases[][4] = {{0, 0, 0, 0}, {1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1},
                                 {127, 63, 3, 7}, {1023, 767, 127, 123456}, {4294967295u, 4294967295u, 4294967295u, 4294967295u}};
    std::printf("{\"cases\": [");
    const int nc = sizeof(cases) / sizeof(cases[0]);
    for (int c = 0; c < nc; ++c) {
        const unsigned* k = cases[c];
        Sampler s;
        s.initFromLaunch(k[0], k[1], k[2], k[3]);
        std::printf("%s{\"launch\": [%u, %u, %u, %u], \"seed\": %llu, \"u32\": [", c ? ", " : "", k[0], k[1], k[2], k[3],
                    Sampler::reproducibleLaunchSeed(k[0], k[1], k[2], k[3]));
        for (int i = 0; i < 16; ++i) std::printf("%s%u", i ? ", " : "", s.next_u32());
        std::printf("], \"next_1d\": [");
        Sampler t;
        t.initFromLaunch(k[0], k[1], k[2], k[3]);
        for (int i = 0; i < 8; ++i) std::printf("%s%.9g", i ? ", " : "", t.next_1d());
        std::printf("]}");
    }
    std::printf("]}\n");
    return 0;
}
