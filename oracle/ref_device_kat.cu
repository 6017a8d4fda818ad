// TEST INFRASTRUCTURE ONLY. Known-answer kernels compiled from the reference's own device headers
// (threedgptir_tracer/include/3dgptir/kernels/cuda/{gaussianParticles,material,environment,
// lightSampler,meshLight,sampler}.cuh) the way the reference compiles its device code: NVRTC with
// its options and JIT defines (cuoptixMacros.h:69-71: -use_fast_math, -default-device, -D__OPTIX__;
// optixTracer.cpp:240-272), against a stand-in optix.h (oracle/ref_stub). oracle/ref_kat.py compiles
// this file to a cubin (oracle/_ref/ref_device_kat.cubin) and launches its ref_* kernels; each
// evaluates one reference function for n cases, one thread per case (inputs [n, IN] floats,
// outputs [n, OUT] floats). tests/golden/make_device_golden.py runs them on a GPU and stores the
// inputs and outputs as fixtures, against which the oracle's restatement and the tracer's device
// functions are tested.
#include <3dgptir/pipelineParameters.h>
#include <3dgptir/kernels/cuda/sampler.cuh>

// The reference keeps its launch parameters in `__constant__ PipelineParameters params`
// (referenceOptix.cu:21), set from the host; here they are a device variable that ref_set_scene
// fills, so that no host code is compiled from the reference's headers.
__device__ PipelineParameters params;

#include <3dgptir/kernels/cuda/environment.cuh>

// environment.cuh declares the MIS power heuristic that pathTracer.cuh (which calls the OptiX API
// and is not compiled here) defines; its accumulateLightContribution, which no kernel here calls,
// refers to it. The same weight, a^2 / (a^2 + b^2):
static __device__ __forceinline__ float misWeight(float pdfA, float pdfB) {
    const float a2 = pdfA * pdfA;
    return a2 / fmaxf(a2 + pdfB * pdfB, 1e-6f);
}

#include <3dgptir/kernels/cuda/gaussianParticles.cuh>
#include <3dgptir/kernels/cuda/lightSampler.cuh>
#include <3dgptir/kernels/cuda/material.cuh>

namespace {

__device__ float3 in3(const float* p) { return make_float3(p[0], p[1], p[2]); }
__device__ void out3(float* p, float3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

// The reference builds its accessors on the host from torch tensors (its constructors exist only
// outside nvcc); here the members are filled through a struct of the same layout.
template <class T, int N>
struct AccessorBits {
    T* data;
    int32_t sizes[N];
    int32_t strides[N];
};

template <class T, int N>
PackedTensorAccessor32<T, N> accessor(T* data, const int (&sizes)[N]) {
    static_assert(sizeof(AccessorBits<T, N>) == sizeof(PackedTensorAccessor32<T, N>), "accessor layout");
    AccessorBits<T, N> b;
    b.data = data;
    int stride = 1;
    for (int k = N - 1; k >= 0; --k) {
        b.sizes[k] = sizes[k];
        b.strides[k] = stride;
        stride *= sizes[k];
    }
    PackedTensorAccessor32<T, N> a;
    memcpy(&a, &b, sizeof(a));
    return a;
}

template <class T>
PackedTensorAccessor32<T, 2> accessor2(T* data, int rows, int cols) {
    const int sizes[2] = {rows, cols};
    return accessor<T, 2>(data, sizes);
}

// processHit (gaussianParticles.cuh:343-440): in = ray o.xyz d.xyz, particle id (as float),
// transmittance before the hit; out = accepted, transmittance, radiance.xyz, depth, depth^2,
// material albedo.xyz roughness metallic, shading normal.xyz, normal.xyz (accumulated from 0)
__device__ void k_process_hit(int n, const float* in, float* out, const ParticleDensity* dens, const Material* mat,
                              const float* sph, const float* snrm, float min_response, float min_alpha, int sph_deg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 8 * i;
    float T = a[7];
    float3 rad = make_float3(0.0f), sn = make_float3(0.0f), nrm = make_float3(0.0f);
    float depth = 0.0f, depth2 = 0.0f;
    Material m;
    const bool acc = processHit<4, false>(in3(a), in3(a + 3), (int32_t)a[6], dens, mat, sph, min_response, min_alpha,
                                          sph_deg, snrm, &T, &rad, &depth, &depth2, &m, &sn, &nrm);
    float* o = out + 18 * i;
    o[0] = acc ? 1.0f : 0.0f;
    o[1] = T;
    out3(o + 2, rad);
    o[5] = depth;
    o[6] = depth2;
    out3(o + 7, m.albedo);
    o[10] = m.roughness;
    o[11] = m.metallic;
    out3(o + 12, sn);
    out3(o + 15, nrm);
}

// intersectInstanceParticle (gaussianParticles.cuh:484-500): in = object-space o.xyz d.xyz, tmin,
// tmax; out = hit, distance
__device__ void k_intersect(int n, const float* in, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 8 * i;
    float t = 0.0f;
    const bool hit = intersectInstanceParticle(in3(a), in3(a + 3), 0, a[6], a[7], 9.0f, t);
    out[2 * i] = hit ? 1.0f : 0.0f;
    out[2 * i + 1] = t;
}

// BRDF (material.cuh): in = wo.xyz, normal.xyz, albedo.xyz, metallic, roughness, rand.xyz or
// light direction.xyz
__device__ void k_brdf_sample(int n, const float* in, float* out) {  // sample_fast_brdf_throughput
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 16 * i;
    float3 next = make_float3(0.0f);
    float pdf = 0.0f;
    const float3 v = sample_fast_brdf_throughput(in3(a), in3(a + 3), in3(a + 6), a[9], a[10], in3(a + 11), next, pdf);
    float* o = out + 7 * i;
    out3(o, v);
    out3(o + 3, next);
    o[6] = pdf;
}

__device__ void k_brdf_eval(int n, const float* in, float* out) {  // eval_fast_brdf_light_sample
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 16 * i;
    float pdf = 0.0f;
    const float3 v = eval_fast_brdf_light_sample(in3(a), in3(a + 3), in3(a + 6), a[9], a[10], in3(a + 11), pdf);
    out3(out + 4 * i, v);
    out[4 * i + 3] = pdf;
}

__device__ void k_brdf_grads(int n, const float* in, float* out) {  // sample_fast_brdf_throughput_with_grads
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 16 * i;
    float3 next = make_float3(0.0f);
    float pdf = 0.0f;
    const FastBrdfValueGrad g =
        sample_fast_brdf_throughput_with_grads(in3(a), in3(a + 3), in3(a + 6), a[9], a[10], in3(a + 11), next, pdf);
    float* o = out + 19 * i;
    out3(o, g.value);
    out3(o + 3, g.dBrdf_dAlbedo);
    out3(o + 6, g.dBrdf_dMetallic);
    out3(o + 9, g.dBrdf_dRoughness);
    out3(o + 12, g.dNextDir_dRoughness);
    out3(o + 15, next);
    o[18] = pdf;
}

// environment (environment.cuh): lookups, the gradient scatter and alias sampling on params.environment
__device__ void k_env_lookup(int n, const float* in, float* out) {  // getBackgroundColor, environmentAliasPdf
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 d = in3(in + 3 * i);
    out3(out + 4 * i, getBackgroundColor(d));
    out[4 * i + 3] = params.environment.aliasTable.numCells > 0 ? environmentAliasPdf(d) : 0.0f;
}

__device__ void k_env_bwd(int n, const float* in, float* out, PipelineBackwardParameters& bp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 6 * i;
    float3 dir_grad = make_float3(0.0f);
    const float3 bg = getBackgroundColorBwd(in3(a), in3(a + 3), bp, &dir_grad);
    out3(out + 6 * i, bg);
    out3(out + 6 * i + 3, dir_grad);
}

// sampleEnvironmentAliasDirection from the launch stream (x, y, z, frame) = in[4] as floats
__device__ void k_env_sample(int n, const float* in, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 4 * i;
    Sampler s;
    s.initFromLaunch((unsigned)a[0], (unsigned)a[1], (unsigned)a[2], (unsigned)a[3]);
    float pdf = 0.0f;
    const float3 d = sampleEnvironmentAliasDirection(s, pdf);
    out3(out + 4 * i, d);
    out[4 * i + 3] = pdf;
}

// lightSampler.cuh: sampleLight from the launch stream (in = position.xyz, x, y, z, frame), and
// lightSamplerPdf (in = position.xyz, direction.xyz)
__device__ void k_light_sample(int n, const float* in, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 7 * i;
    Sampler s;
    s.initFromLaunch((unsigned)a[3], (unsigned)a[4], (unsigned)a[5], (unsigned)a[6]);
    const LightSample ls = sampleLight(in3(a), s);
    float* o = out + 10 * i;
    out3(o, ls.wi);
    out3(o + 3, ls.Li);
    o[6] = ls.pdf;
    o[7] = ls.dist;
    o[8] = (float)ls.lightType;
    o[9] = (float)ls.lightId;
}

__device__ void k_light_pdf(int n, const float* in, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 6 * i;
    out[i] = lightSamplerPdf(in3(a), in3(a + 3));
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// entry kernels (extern "C" names for the driver API)
extern "C" {

// The scene the environment and light kernels read: environment [eh, ew, 4] (equirect, or cube when
// eh == 6 ew), alias table [3, ah, aw], and the packed light tables (LightBuffers). One thread.
__global__ void ref_set_scene(const float* env, int eh, int ew, const float* alias, int ah, int aw,
                              const float* lights, int num_lights, const float* light_table, int entries,
                              const float* mesh_vertices, int num_vertices, const int* mesh_triangles,
                              int num_triangles, const float* mesh_lights, int num_mesh, const float* tri_table,
                              int tri_cols) {
    PipelineParameters& p = params;
    memset(&p, 0, sizeof(p));
    p.environment.data = reinterpret_cast<const float4*>(env);
    p.environment.width = ew;
    p.environment.height = eh;
    p.environment.type = (eh == 6 * ew) ? EnvironmentType_Cube : EnvironmentType_2D;
    p.environment.offset = make_float2(0.0f, 0.0f);
    p.environment.aliasTable.width = aw;
    p.environment.aliasTable.height = ah;
    p.environment.aliasTable.numCells = aw * ah;
    p.environment.aliasTable.prob = alias;
    p.environment.aliasTable.alias = alias ? alias + aw * ah : nullptr;
    p.environment.aliasTable.pdf = alias ? alias + 2 * aw * ah : nullptr;
    p.numLights = num_lights;
    p.lights = accessor2(const_cast<float*>(lights), num_lights, 9);
    p.numLightEntries = entries;
    p.lightAliasTable = accessor2(const_cast<float*>(light_table), 5, entries);
    p.numMeshLightVertices = num_vertices;
    p.meshLightVertices = accessor2(const_cast<float*>(mesh_vertices), num_vertices, 3);
    p.numMeshLightTriangles = num_triangles;
    p.meshLightTriangles = accessor2(const_cast<int*>(mesh_triangles), num_triangles, 3);
    p.numMeshLights = num_mesh;
    p.meshLights = accessor2(const_cast<float*>(mesh_lights), num_mesh, 8);
    p.meshLightTriangleAliasTable = accessor2(const_cast<float*>(tri_table), 3, tri_cols);
    p.hitMinGaussianResponse = 0.0113f;
    p.alphaMinThreshold = 1.0f / 255.0f;
}

__global__ void ref_process_hit(int n, const float* in, float* out, const float* dens, const float* mat,
                                const float* sph, const float* snrm, float min_response, float min_alpha,
                                int sph_deg) {
    k_process_hit(n, in, out, reinterpret_cast<const ParticleDensity*>(dens), reinterpret_cast<const Material*>(mat),
                  sph, snrm, min_response, min_alpha, sph_deg);
}
__global__ void ref_intersect(int n, const float* in, float* out) { k_intersect(n, in, out); }
__global__ void ref_brdf_sample(int n, const float* in, float* out) { k_brdf_sample(n, in, out); }
__global__ void ref_brdf_eval(int n, const float* in, float* out) { k_brdf_eval(n, in, out); }
__global__ void ref_brdf_grads(int n, const float* in, float* out) { k_brdf_grads(n, in, out); }
__global__ void ref_env_lookup(int n, const float* in, float* out) { k_env_lookup(n, in, out); }
__global__ void ref_env_sample(int n, const float* in, float* out) { k_env_sample(n, in, out); }
__global__ void ref_light_sample(int n, const float* in, float* out) { k_light_sample(n, in, out); }
__global__ void ref_light_pdf(int n, const float* in, float* out) { k_light_pdf(n, in, out); }

// env_grad: [eh, ew, 4] floats, accumulated into (atomics, as the reference scatters)
__global__ void ref_env_bwd(int n, const float* in, float* out, float* env_grad, int eh, int ew) {
    PipelineBackwardParameters bp;
    memset(&bp, 0, sizeof(bp));
    const int sizes[3] = {eh, ew, 4};
    bp.environmentGrad = accessor<float, 3>(env_grad, sizes);
    k_env_bwd(n, in, out, bp);
}

}  // extern "C"
