/* TEST INFRASTRUCTURE ONLY. Stand-in for the OptiX SDK header that the reference's device headers
 * include (the SDK is not vendored with the reference). The functions compiled from those headers
 * by oracle/ref_device_kat.cu call no OptiX API; PipelineParameters only names these two types in
 * its members, which the known-answer kernels never read. */
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#endif

typedef unsigned long long OptixTraversableHandle;
struct OptixAabb {
    float minX, minY, minZ, maxX, maxY, maxZ;
};
