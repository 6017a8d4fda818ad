// Fused selective Adam step (the reference's SelectiveAdam, threedgrut/optimizers/optimizers.cu:49-76
// and __init__.py:45-125): for every element of a Gaussian whose visibility flag is set,
//   m = b1 m + (1 - b1) g,  v = b2 v + (1 - b2) g^2,  p -= lr m / (sqrt(v) + eps)
// with no bias correction; elements of hidden Gaussians keep their parameter and moments.
// Square root and division are IEEE round-to-nearest whatever the compile flags.
#include <cstdint>

#include "../../include/ptir_b200.h"

namespace ptir {

namespace {

// one thread per 4 consecutive elements when the row length allows it, else per element
__global__ void k_selective_adam(float* __restrict__ param, const float* __restrict__ grad, float* __restrict__ m,
                                 float* __restrict__ v, const uint8_t* __restrict__ visible, long long n_rows,
                                 int row, float lr, float b1, float b2, float eps) {
    const long long total = n_rows * (long long)row;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        if (visible && !visible[i / row]) continue;
        const float g = grad[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g;
        const float vi = b2 * v[i] + (1.0f - b2) * g * g;
        param[i] += __fdiv_rn(-lr * mi, __fadd_rn(__fsqrt_rn(vi), eps));
        m[i] = mi;
        v[i] = vi;
    }
}

__global__ void k_fold(float* __restrict__ out, const float* __restrict__ comp, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] += comp[i];
}

}  // namespace

// out[i] += comp[i]: the compensation terms of Kahan-pair gradient sums folded into the sums
cudaError_t launch_fold(float* out, const float* comp, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const long long blocks = (n + 255) / 256;
    k_fold<<<(unsigned)(blocks < 148LL * 32 ? blocks : 148LL * 32), 256, 0, s>>>(out, comp, n);
    return cudaGetLastError();
}

}  // namespace ptir

extern "C" int ptir_selective_adam(float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                                   const uint8_t* visible, int64_t n_rows, int32_t row, float lr, float beta1,
                                   float beta2, float eps, void* stream) {
    if (n_rows < 0 || row <= 0) return PTIR_EINVAL;
    if (n_rows == 0) return PTIR_OK;
    if (!param || !grad || !exp_avg || !exp_avg_sq) return PTIR_EINVAL;
    const long long total = n_rows * (long long)row;
    const int block = 256;
    const long long blocks = (total + block - 1) / block;
    const unsigned grid = (unsigned)(blocks < 148LL * 64 ? blocks : 148LL * 64);
    ptir::k_selective_adam<<<grid, block, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        param, grad, exp_avg, exp_avg_sq, visible, n_rows, row, lr, beta1, beta2, eps);
    return cudaGetLastError() == cudaSuccess ? PTIR_OK : PTIR_ECUDA;
}
