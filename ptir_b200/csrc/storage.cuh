// Reduced-precision attribute storage: the Gaussians' geometry, material, shading normal and
// SH coefficients held as BF16 or FP16 (round to nearest even) and widened to FP32 on load.
// All arithmetic stays FP32. In FP32 storage the kernels read the caller's tensors directly.
//
// Records (16-bit values, one Gaussian each):
//   hot  (2 x uint4 = 32 B):  pos.xyz dns | quat wxyz | scale.xyz | 0 0 0 0 0
//        read for every candidate (the reference's particle_density row, halved)
//   cold (cold_stride x uint4): material(albedo.rgb rough metal) snrm.xyz | SH coefficients
//        (coefficient-major, 8 per uint4) | zero padding to an even number of uint4
//        read for every composited hit
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "device_types.h"
#include "vecmath.cuh"

namespace ptir {

enum Storage : unsigned { kStoreF32 = 0u, kStoreBF16 = 1u, kStoreF16 = 2u };

// uint4 per cold record for `sph_stride` SH floats
inline int cold_stride_of(int sph_stride) {
    const int n = 1 + (sph_stride + 7) / 8;
    return (n + 1) & ~1;
}

// x rounded to the storage type (exact as a float)
PTIR_DEV float round_storage(unsigned storage, float x) {
    if (storage == kStoreBF16) return __bfloat162float(__float2bfloat16_rn(x));
    if (storage == kStoreF16) return __half2float(__float2half_rn(x));
    return x;
}

PTIR_DEV unsigned short to_bits(unsigned storage, float x) {
    if (storage == kStoreBF16) return __bfloat16_as_ushort(__float2bfloat16_rn(x));
    return __half_as_ushort(__float2half_rn(x));
}

// one 16-bit value widened
PTIR_DEV float widen(unsigned storage, unsigned short h) {
    return storage == kStoreBF16 ? __uint_as_float((unsigned)h << 16) : __half2float(__ushort_as_half(h));
}

// the two 16-bit values of a word, widened (low half first)
PTIR_DEV float2 widen2(unsigned storage, unsigned w) {
    return make_float2(widen(storage, (unsigned short)(w & 0xFFFFu)), widen(storage, (unsigned short)(w >> 16)));
}

struct Geom {
    float3 pos;
    float dns;
    float4 quat;  // wxyz
    float3 scl;
};

PTIR_DEV Geom load_geom(const ParticleView& V, unsigned id) {
    Geom g;
    if (V.storage == kStoreF32) {
        const float4* rec = V.density + 3 * (size_t)id;
        const float4 a = __ldg(rec + 0), q = __ldg(rec + 1), c = __ldg(rec + 2);
        g.pos = make_float3(a.x, a.y, a.z);
        g.dns = a.w;
        g.quat = q;
        g.scl = make_float3(c.x, c.y, c.z);
        return g;
    }
    const uint4* rec = V.hot + 2 * (size_t)id;
    const uint4 u = __ldg(rec), v = __ldg(rec + 1);
    const float2 p01 = widen2(V.storage, u.x), p2d = widen2(V.storage, u.y);
    const float2 q01 = widen2(V.storage, u.z), q23 = widen2(V.storage, u.w);
    const float2 s01 = widen2(V.storage, v.x), s2 = widen2(V.storage, v.y);
    g.pos = make_float3(p01.x, p01.y, p2d.x);
    g.dns = p2d.y;
    g.quat = make_float4(q01.x, q01.y, q23.x, q23.y);
    g.scl = make_float3(s01.x, s01.y, s2.x);
    return g;
}

PTIR_DEV void load_material(const ParticleView& V, unsigned id, float3& albedo, float& rough, float& metal) {
    if (V.storage == kStoreF32) {
        const float* m = V.material + 5 * (size_t)id;
        albedo = ld3(m);
        rough = __ldg(m + 3);
        metal = __ldg(m + 4);
        return;
    }
    const uint4 u = __ldg(V.cold + (size_t)V.cold_stride * id);
    const float2 a01 = widen2(V.storage, u.x), a2r = widen2(V.storage, u.y), mn = widen2(V.storage, u.z);
    albedo = make_float3(a01.x, a01.y, a2r.x);
    rough = a2r.y;
    metal = mn.x;
}

PTIR_DEV float3 load_snrm(const ParticleView& V, unsigned id) {
    if (V.storage == kStoreF32) return ld3(V.snrm + 3 * (size_t)id);
    const uint4 u = __ldg(V.cold + (size_t)V.cold_stride * id);
    const float2 mn = widen2(V.storage, u.z), n12 = widen2(V.storage, u.w);
    return make_float3(mn.y, n12.x, n12.y);
}

// Pack the caller's FP32 tensors (density [n,12], material [n,5], sph [n,sph_stride], snrm [n,3]
// or null) into hot [n,2] / cold [n,cold_stride] uint4 records (storage.cu).
cudaError_t launch_pack_attributes(int n, const float* density, const float* material, const float* sph, int sph_stride,
                                   const float* snrm, unsigned storage, uint4* hot, uint4* cold, cudaStream_t s);

}  // namespace ptir
