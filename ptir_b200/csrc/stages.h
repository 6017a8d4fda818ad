// Attribution of a trace's work to its kernels: per-stage device counters and, when enabled,
// CUDA events recorded around every launch on the launch stream.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device_types.h"

namespace ptir {

// The kernels of a trace, as the C ABI numbers them (PTIR_STAGE_* in include/ptir_b200.h).
enum Stage : int {
    kStageIntersect = 0,   // primary and bounce segments: traversal and compositing
    kStageShadow = 1,      // NEE shadow rays
    kStageReplay = 2,      // backward material-gradient re-traversals
    kStageShading = 3,     // camera rays, primary outputs, light gathering and BRDF sampling
    kStageMegakernel = 4,  // the whole-path kernels of the megakernel schedule
    kStageSort = 5,        // ray-order keys and their radix sort
    kNumStages = 6,
};

// Launch intervals of each stage, summed on demand. Event pairs are pooled and reused.
class StageTimer {
public:
    bool enabled = false;
    ~StageTimer();
    void begin(int stage, cudaStream_t s);
    void end(cudaStream_t s);
    // adds the recorded intervals of each stage to ms / launches and forgets them; waits for
    // their events
    cudaError_t collect(double* ms, unsigned long long* launches);

private:
    struct Interval {
        int stage;
        cudaEvent_t start, stop;
    };
    std::vector<Interval> pool_;
    size_t used_ = 0;
    bool open_ = false;
    cudaError_t error_ = cudaSuccess;
};

// What a launcher needs to attribute its launches.
struct StageCtx {
    unsigned long long* counters = nullptr;  // [kNumStages * kNumCounters], or null when not collected
    StageTimer* timer = nullptr;

    // kernel parameters whose counters point at the stage's block
    TraceParams at(const TraceParams& p, int stage) const {
        TraceParams q = p;
        q.counters = counters ? counters + (size_t)stage * kNumCounters : nullptr;
        return q;
    }
    // launch(params) between the stage's events
    template <class Launch>
    void run(int stage, const TraceParams& p, cudaStream_t s, Launch&& launch) const {
        const bool timed = timer && timer->enabled;
        if (timed) timer->begin(stage, s);
        launch(at(p, stage));
        if (timed) timer->end(s);
    }
};

}  // namespace ptir
