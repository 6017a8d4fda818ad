// Wavefront schedule of the tracer (wavefront.cu): buffers and launchers.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "device_types.h"

namespace ptir {

constexpr int kNumQueueCounts = 4;   // bounce, intersect, shadow, replay jobs
constexpr int kNumCursors = 256;     // one work cursor per stage launch of a chunk

// Per-path state and queues of one chunk of paths; grown on demand, never shrunk.
struct WavefrontBuffers {
    size_t slots = 0;        // paths per chunk the buffers hold
    void* seg = nullptr;     // Segment[slots]
    void* ps = nullptr;      // PathState[slots]
    void* rng = nullptr;     // u64[slots] PCG state
    void* q[3] = {nullptr, nullptr, nullptr};  // u32[slots] each
    void* jobs = nullptr;    // ReplayJob[2 * slots]
    void* counters = nullptr;  // u32[kNumQueueCounts + kNumCursors]
};

cudaError_t wavefront_reserve(WavefrontBuffers& b, size_t slots, cudaStream_t s);
void wavefront_free(WavefrontBuffers& b);

// chunk_tiles: 8x4 pixel tiles per chunk (32 paths each); kbuf: candidates per traversal (8, 16, 32)
cudaError_t launch_trace_fwd_wavefront(const TraceParams& p, const FwdOutputs& o, WavefrontBuffers& b,
                                       unsigned chunk_tiles, int kbuf, cudaStream_t s);
cudaError_t launch_trace_bwd_wavefront(const TraceParams& p, const BwdInputs& bi, WavefrontBuffers& b,
                                       unsigned chunk_tiles, int kbuf, cudaStream_t s);

}  // namespace ptir
