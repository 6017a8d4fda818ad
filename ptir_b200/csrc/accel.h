// LBVH over the Gaussians' instance boxes (the replacement for the reference's OptiX IAS:
// threedgptir_tracer/src/optixTracer.cpp:633-907, particlePrimitives.cu:543-610).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "device_types.h"

namespace ptir {

struct AccelBuildOptions {
    float kernel_degree;     // generalized-Gaussian degree of the particle kernel
    float min_response;      // kernel support ends where the (clamped) response reaches this
    int density_clamping;    // adaptive support: the response threshold is divided by the density
    unsigned storage;        // attribute storage (storage.cuh): inputs are rounded to it first
    unsigned builder;        // kBuilderMorton: Karras hierarchy over the sorted keys; kBuilderPloc: PLOC
};

enum : unsigned { kBuilderMorton = 0, kBuilderPloc = 1 };

// Device buffers of one acceleration structure; grown on demand, never shrunk.
struct AccelState {
    int n = 0;                  // Gaussians in the current structure
    bool valid = false;
    float4* inst = nullptr;     // [n*4] unsorted leaf records
    float4* box = nullptr;      // [n*2] unsorted instance AABBs (lo.xyz kmax, hi.xyz -)
    unsigned long long* keys[2] = {nullptr, nullptr};  // Morton keys (sort in/out)
    unsigned* ids[2] = {nullptr, nullptr};             // Gaussian ids (sort in/out); ids[1] is the leaf order
    float4* leaves = nullptr;   // [n*4] Morton-ordered leaf records
    float4* nodes = nullptr;    // [(n-1)*4] internal nodes
    int* parent = nullptr;      // [2n-1] parent of internal node i / of leaf j at n-1+j
    unsigned* arrivals = nullptr;  // [n-1] refit arrival counters
    float4* partial = nullptr;  // [kReduceBlocks*2] per-block bounds
    float4* bounds = nullptr;   // [2] scene AABB
    int* wroot = nullptr;       // [n-1] binary node at the root of each 4-wide node
    int* wsrc = nullptr;        // [(n-1)*4] children of each 4-wide node as binary references (refits)
    int* wchild = nullptr;      // [(n-1)*4] the same children as 4-wide node indices or leaves
    unsigned* wcount = nullptr; // number of 4-wide nodes
    float4* nodes4 = nullptr;   // [(n-1)*8] 4-wide nodes traversed by the tracer
    void* sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    unsigned* ploc_host = nullptr;  // pinned [2]: cluster count and next node index read back by a PLOC build
    size_t capacity = 0;        // Gaussians the buffers can hold

    AccelView view() const { return AccelView{nodes4, leaves, bounds, valid ? n : 0, 0.0f}; }
};

// Build (rebuild != 0 or topology unusable) or refit the structure from per-Gaussian
// position [n,3], rotation [n,4] (wxyz), scale [n,3] and density [n,1] (device pointers).
// Returns a CUDA error code and a message in `err` on failure. A PLOC rebuild reads the cluster
// count back to the host between its iterations, so it synchronises the stream and cannot be
// captured in a CUDA graph (a refit can).
cudaError_t accel_build(AccelState& st, const AccelBuildOptions& opt, const float* pos, const float* rot,
                        const float* scl, const float* dns, int n, bool rebuild, cudaStream_t stream,
                        std::string& err);

void accel_free(AccelState& st);

}  // namespace ptir
