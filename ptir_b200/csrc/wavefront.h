// Wavefront schedule of the tracer (wavefront.cu): buffers and launchers.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "device_types.h"
#include "stages.h"

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
    void* sort_keys[2] = {nullptr, nullptr};  // u32[slots]: ray-order keys, unsorted and sorted
    void* sorted = nullptr;  // u32[slots]: the intersect queue in key order
    void* sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    void* parked = nullptr;  // f32, per resident thread of the intersection kernel (k_wf_trace)
    void* frontier = nullptr;  // uint2[2 * kFrontierCap] per thread of the intersection kernel
    size_t frontier_threads = 0;
};

// Entries of each of a lane's two frontier buffers (resumed trace calls, traverse.cuh). A call
// that sets more aside leaves its segment's next call to start from the root.
constexpr int kFrontierCap = 768;

cudaError_t frontier_reserve(WavefrontBuffers& b, size_t threads, cudaStream_t s);

cudaError_t wavefront_reserve(WavefrontBuffers& b, size_t slots, cudaStream_t s);
// device bytes the wavefront holds per path slot of a chunk (state, queues, replay jobs, sort)
size_t wavefront_bytes_per_slot();
void wavefront_free(WavefrontBuffers& b);

// Launch shape of the wavefront schedule. Only the k-buffer size can change a result: it moves
// the distance at which subtrees are culled, which decides which grazing candidate is kept.
struct WavefrontTuning {
    unsigned chunk_tiles = 131072;  // 8x4 pixel tiles per chunk (32 paths each)
    int kbuf = 16;                  // candidates per traversal: 8, 16 or 32
    int refill_lanes = 32;          // intersection: waiting lanes (1..32) before a warp refills
    int block = 128;                // threads per block: 64, 128 or 256
    bool sort_rays = true;          // intersect bounce rays in (octant, origin cell, direction cell) order
    int shadow_kbuf = 16;           // candidates per shadow-ray traversal: 8, 16 or 32
    bool resume_isect = false;      // intersection stage: rounds resumed from the previous round's frontier (K <= 16)
    bool resume_replay = true;      // backward replay: the same
    bool exact_candidates = false;  // the intersection kernel with the exact-candidate cull slack
};

cudaError_t launch_trace_fwd_wavefront(const TraceParams& p, const FwdOutputs& o, WavefrontBuffers& b,
                                       const WavefrontTuning& tune, const StageCtx& sc, cudaStream_t s);
cudaError_t launch_trace_bwd_wavefront(const TraceParams& p, const BwdInputs& bi, WavefrontBuffers& b,
                                       const WavefrontTuning& tune, const StageCtx& sc, cudaStream_t s);

}  // namespace ptir
