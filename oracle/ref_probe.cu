// TEST INFRASTRUCTURE ONLY. Device-side probe of the evaluation order nvcc gives to the draws
// inside the reference's Sampler::next_3d() (threedgptir_tracer/include/3dgptir/kernels/cuda/
// sampler.cuh:80-82) and to a two-argument call whose arguments each draw once, the shape
// used by environment.cuh:245-250. Built by oracle/Makefile from the reference header.
#include <cuda_runtime.h>

#include <3dgptir/kernels/cuda/sampler.cuh>

__device__ __noinline__ float2 two_args(float a, float b) { return make_float2(a, b); }

__global__ void probe_kernel(float* out) {
    // out[0..2] next_3d; out[3..5] the 3 sequential next_1d of the same stream
    Sampler s;
    s.initFromLaunch(5u, 7u, 11u, 13u);
    const float3 v = s.next_3d();
    Sampler q;
    q.initFromLaunch(5u, 7u, 11u, 13u);
    const float a = q.next_1d();
    const float b = q.next_1d();
    const float c = q.next_1d();
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
    out[3] = a; out[4] = b; out[5] = c;
    // out[6..7] two_args((3 + next_1d()) / 8, (2 + next_1d()) / 4); out[8..9] two sequential draws
    Sampler r;
    r.initFromLaunch(5u, 7u, 11u, 13u);
    const float2 t = two_args((3.0f + r.next_1d()) / 8.0f, (2.0f + r.next_1d()) / 4.0f);
    Sampler w;
    w.initFromLaunch(5u, 7u, 11u, 13u);
    const float d0 = w.next_1d();
    const float d1 = w.next_1d();
    out[6] = t.x; out[7] = t.y; out[8] = (3.0f + d0) / 8.0f; out[9] = (2.0f + d1) / 4.0f;
}

extern "C" int ref_probe_draw_order(float* host_out /* 10 floats */) {
    float* d = nullptr;
    if (cudaMalloc(&d, 10 * sizeof(float)) != cudaSuccess) return 1;
    probe_kernel<<<1, 1>>>(d);
    cudaError_t e = cudaMemcpy(host_out, d, 10 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 2;
}
