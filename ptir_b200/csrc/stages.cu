// StageTimer: CUDA event pairs around stage launches (host code).
#include "stages.h"

namespace ptir {

StageTimer::~StageTimer() {
    for (Interval& iv : pool_) {
        cudaEventDestroy(iv.start);
        cudaEventDestroy(iv.stop);
    }
}

void StageTimer::begin(int stage, cudaStream_t s) {
    if (error_ != cudaSuccess) return;
    if (used_ == pool_.size()) {
        Interval iv{stage, nullptr, nullptr};
        error_ = cudaEventCreate(&iv.start);
        if (error_ == cudaSuccess) error_ = cudaEventCreate(&iv.stop);
        if (error_ != cudaSuccess) return;
        pool_.push_back(iv);
    }
    Interval& iv = pool_[used_];
    iv.stage = stage;
    error_ = cudaEventRecord(iv.start, s);
    open_ = error_ == cudaSuccess;
}

void StageTimer::end(cudaStream_t s) {
    if (!open_) return;
    open_ = false;
    error_ = cudaEventRecord(pool_[used_].stop, s);
    if (error_ == cudaSuccess) ++used_;
}

cudaError_t StageTimer::collect(double* ms, unsigned long long* launches) {
    cudaError_t e = error_;
    for (size_t i = 0; e == cudaSuccess && i < used_; ++i) {
        float t = 0.0f;
        e = cudaEventSynchronize(pool_[i].stop);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, pool_[i].start, pool_[i].stop);
        if (e == cudaSuccess && pool_[i].stage >= 0 && pool_[i].stage < kNumStages) {
            ms[pool_[i].stage] += t;
            launches[pool_[i].stage] += 1;
        }
    }
    used_ = 0;
    open_ = false;
    error_ = cudaSuccess;
    return e;
}

}  // namespace ptir
