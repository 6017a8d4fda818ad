// Packing of the caller's FP32 attribute tensors into 16-bit hot / cold records (storage.cuh).
#include "storage.cuh"

namespace ptir {

namespace {

// 16-bit values of v[0..count) (zero past it) into nwords words, two per word, low half first
__device__ void pack_words(unsigned storage, const float* v, int count, unsigned* words, int nwords) {
    for (int w = 0; w < nwords; ++w) {
        const unsigned lo = 2 * w < count ? to_bits(storage, v[2 * w]) : 0u;
        const unsigned hi = 2 * w + 1 < count ? to_bits(storage, v[2 * w + 1]) : 0u;
        words[w] = lo | (hi << 16);
    }
}

__global__ void k_pack_attributes(int n, const float* __restrict__ density, const float* __restrict__ material,
                                  const float* __restrict__ sph, int sph_stride, const float* __restrict__ snrm,
                                  unsigned storage, int cold_stride, uint4* __restrict__ hot, uint4* __restrict__ cold) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    float geo[11];  // pos.xyz dns quat.wxyz scale.xyz
    for (int k = 0; k < 11; ++k) geo[k] = __ldg(density + 12 * (size_t)g + k);
    unsigned hw[8];
    pack_words(storage, geo, 11, hw, 8);
    hot[2 * (size_t)g] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    hot[2 * (size_t)g + 1] = make_uint4(hw[4], hw[5], hw[6], hw[7]);
    float ms[8];  // material, then the shading normal
    for (int k = 0; k < 5; ++k) ms[k] = __ldg(material + 5 * (size_t)g + k);
    for (int k = 0; k < 3; ++k) ms[5 + k] = snrm ? __ldg(snrm + 3 * (size_t)g + k) : 0.0f;
    unsigned mw[4];
    pack_words(storage, ms, 8, mw, 4);
    uint4* c = cold + (size_t)cold_stride * g;
    c[0] = make_uint4(mw[0], mw[1], mw[2], mw[3]);
    const float* sr = sph + (size_t)sph_stride * g;
    for (int chunk = 0; chunk + 1 < cold_stride; ++chunk) {  // SH, 8 values per uint4
        float v[8];
        for (int k = 0; k < 8; ++k) {
            const int i = 8 * chunk + k;
            v[k] = i < sph_stride ? __ldg(sr + i) : 0.0f;
        }
        unsigned sw[4];
        pack_words(storage, v, 8, sw, 4);
        c[1 + chunk] = make_uint4(sw[0], sw[1], sw[2], sw[3]);
    }
}

}  // namespace

cudaError_t launch_pack_attributes(int n, const float* density, const float* material, const float* sph, int sph_stride,
                                   const float* snrm, unsigned storage, uint4* hot, uint4* cold, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int block = 256;
    k_pack_attributes<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(n, density, material, sph, sph_stride, snrm,
                                                                           storage, cold_stride_of(sph_stride), hot, cold);
    return cudaGetLastError();
}

}  // namespace ptir
