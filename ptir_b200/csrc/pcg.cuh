// Per-path random stream: PCG32 (O'Neill 2014, XSH-RR output, 64-bit LCG state) seeded from an
// FNV-1a-style mix of the launch index and frame number. Bit-compatible with the reference
// sampler (threedgptir_tracer/include/3dgptir/kernels/cuda/sampler.cuh:26-84), so that a path
// here and a path there consume identical sample sequences.
#pragma once

#include "vecmath.cuh"

struct Pcg32 {
    unsigned long long state;
    unsigned long long inc;

    static __device__ __forceinline__ unsigned long long launch_seed(unsigned x, unsigned y, unsigned z, unsigned frame) {
        constexpr unsigned long long kOffset = 1469598103934665603ull, kPrime = 1099511628211ull;
        unsigned long long s = kOffset;
        s ^= (unsigned long long)x + kPrime * s;
        s ^= (unsigned long long)y + kPrime * s;
        s ^= (unsigned long long)z + kPrime * s;
        s ^= (unsigned long long)frame + kPrime * s;
        return s ? s : 1ull;
    }
    __device__ __forceinline__ void seed(unsigned x, unsigned y, unsigned z, unsigned frame) {
        state = 0ull;
        inc = 1ull;  // stream 0
        step();
        state += launch_seed(x, y, z, frame);
        step();
    }
    __device__ __forceinline__ unsigned step() {
        const unsigned long long old = state;
        state = old * 6364136223846793005ull + inc;
        const unsigned xs = (unsigned)(((old >> 18) ^ old) >> 27);
        const unsigned rot = (unsigned)(old >> 59);
        return __funnelshift_r(xs, xs, rot);
    }
    // 24 random mantissa bits scaled to [0, 1)
    __device__ __forceinline__ float uniform() { return (float)(step() & 0x00FFFFFFu) * (1.0f / 16777216.0f); }
    // three draws, taken in the order the reference's 3-vector draw takes them (first component first)
    __device__ __forceinline__ float3 uniform3() {
        const float a = uniform();
        const float b = uniform();
        const float c = uniform();
        return make_float3(a, b, c);
    }
};
