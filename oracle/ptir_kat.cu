// TEST INFRASTRUCTURE ONLY. The tracer's own device functions (ptir_b200/csrc) behind the same
// known-answer entry points as the reference's kernels of oracle/ref_device_kat.cu: one thread per
// case, inputs [n, IN] and outputs [n, OUT] floats in the same layouts, so that
// tests/test_gpu_device_kat.py can run both on the cases of tests/golden/device_kat.npz. Also the
// tracer's radix sort on device buffers (tests/test_gpu_sort.py). Built by `make -C oracle` with
// the library's own nvcc flags.
#include <cmath>
#include <cstring>

#include "../ptir_b200/csrc/path.cuh"
#include "../ptir_b200/csrc/radix_sort.cuh"

namespace {

using namespace ptir;

__device__ float3 in3(const float* p) { return make_float3(p[0], p[1], p[2]); }
__device__ void out3(float* p, float3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

TraceParams g_params;  // the scene of the environment and light kernels (set by ptirkat_set_scene)

// processHit: composite_one on a fresh accumulator with the given transmittance
__global__ void k_process_hit(int n, const float* in, float* out, TraceParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 8 * i;
    Composite c;
    c.o = in3(a);
    c.d = in3(a + 3);
    c.radiance = c.normal = c.albedo = c.snrm = f3(0.0f);
    c.transmittance = a[7];
    c.depth = c.hit2 = c.distortion = c.hits_count = c.rough = c.metal = 0.0f;
    c.last_hit = 0.0f;
    c.clip_end = 1e30f;
    c.hit = false;
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    composite_one<false>(P, ctr, c, 1.0f, (unsigned)a[6], nullptr);
    float* o = out + 18 * i;
    o[0] = c.hits_count;
    o[1] = c.transmittance;
    out3(o + 2, c.radiance);
    o[5] = c.depth;
    o[6] = c.hit2;
    out3(o + 7, c.albedo);
    o[10] = c.rough;
    o[11] = c.metal;
    out3(o + 12, c.snrm);
    out3(o + 15, c.normal);
}

__global__ void k_intersect(int n, const float* in, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 8 * i;
    float t = 0.0f;
    const bool hit = instance_hit(in3(a), in3(a + 3), a[6], a[7], t);
    out[2 * i] = hit ? 1.0f : 0.0f;
    out[2 * i + 1] = t;
}

__global__ void k_brdf(int n, const float* in, float* out, int which) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 16 * i;
    const float3 wo = in3(a), nrm = in3(a + 3), alb = in3(a + 6), r3 = in3(a + 11);
    float3 next = f3(0.0f);
    if (which == 0) {  // sample
        const BrdfSample s = sample_brdf<false>(wo, nrm, alb, a[9], a[10], r3, false, next);
        float* o = out + 7 * i;
        out3(o, s.value);
        out3(o + 3, next);
        o[6] = s.pdf;
    } else if (which == 1) {  // eval
        float pdf = 0.0f;
        const BrdfTerms t = eval_brdf<false>(wo, nrm, alb, a[9], a[10], r3, false, pdf);
        out3(out + 4 * i, t.value);
        out[4 * i + 3] = pdf;
    } else {  // sample with gradients
        const BrdfSample s = sample_brdf<true>(wo, nrm, alb, a[9], a[10], r3, false, next);
        float* o = out + 19 * i;
        out3(o, s.value);
        out3(o + 3, s.d_albedo);
        out3(o + 6, s.d_metallic);
        out3(o + 9, s.d_rough);
        out3(o + 12, s.d_next_dir);
        out3(o + 15, next);
        o[18] = s.pdf;
    }
}

__global__ void k_env_lookup(int n, const float* in, float* out, TraceParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 d = in3(in + 3 * i);
    unsigned lookups = 0;
    out3(out + 4 * i, env_radiance(P.env, d, lookups));
    out[4 * i + 3] = P.env.cells > 0 ? env_pdf(P.env, d) : 0.0f;
}

__global__ void k_env_bwd(int n, const float* in, float* out, TraceParams P, float* env_grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 6 * i;
    StackEntry stack[1];
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    CtxT<16> C{P, stack, ctr};
    BwdInputs B{};
    B.environment_grad = env_grad;
    float3 dir_grad = f3(0.0f);
    out3(out + 6 * i, env_radiance_bwd(C, B, in3(a), in3(a + 3), dir_grad));
    out3(out + 6 * i + 3, dir_grad);
}

__global__ void k_env_sample(int n, const float* in, float* out, TraceParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 4 * i;
    Pcg32 rng;
    rng.seed((unsigned)a[0], (unsigned)a[1], (unsigned)a[2], (unsigned)a[3]);
    float pdf = 0.0f;
    out3(out + 4 * i, sample_env_direction(P.env, rng, pdf));
    out[4 * i + 3] = pdf;
}

__global__ void k_light_sample(int n, const float* in, float* out, TraceParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 7 * i;
    Pcg32 rng;
    rng.seed((unsigned)a[3], (unsigned)a[4], (unsigned)a[5], (unsigned)a[6]);
    unsigned lookups = 0;
    const LightSample ls = sample_light(P, in3(a), rng, lookups);
    float* o = out + 9 * i;
    out3(o, ls.wi);
    out3(o + 3, ls.Li);
    o[6] = ls.pdf;
    o[7] = ls.dist;
    o[8] = (float)ls.type;
}

__global__ void k_light_pdf(int n, const float* in, float* out, TraceParams P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 6 * i;
    out[i] = light_sampler_pdf(P, in3(a), in3(a + 3));
}

int finish() { return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1; }
unsigned blocks(int n) { return (unsigned)((n + 127) / 128); }

}  // namespace

extern "C" {

// the scene of the environment and light entries: device pointers as in ptir_trace_args
int ptirkat_set_scene(const float* env, int eh, int ew, const float* alias, int ah, int aw, const float* lights,
                      int num_lights, const float* light_table, int entries, const float* mesh_vertices,
                      int num_vertices, const int* mesh_triangles, int num_triangles, const float* mesh_lights,
                      int num_mesh, const float* tri_table, int tri_cols) {
    TraceParams& p = g_params;
    std::memset(&p, 0, sizeof(p));
    p.env.data = reinterpret_cast<const float4*>(env);
    p.env.w = ew;
    p.env.h = eh;
    p.env.cube = eh == 6 * ew;
    if (alias && ah > 0 && aw > 0) {
        p.env.aw = aw;
        p.env.ah = ah;
        p.env.cells = aw * ah;
        p.env.prob = alias;
        p.env.alias = alias + p.env.cells;
        p.env.pdf = alias + 2 * p.env.cells;
    }
    // the tracer's environment offset (ptir_b200/csrc/api.cu)
    p.env.offset_x = 0.0f;
    p.env.offset_y = 0.0f;
    p.lights.lights = num_lights > 0 ? lights : nullptr;
    p.lights.num_lights = num_lights;
    p.lights.table = entries > 0 ? light_table : nullptr;
    p.lights.entries = entries;
    p.lights.vertices = num_vertices > 0 ? mesh_vertices : nullptr;
    p.lights.num_vertices = num_vertices;
    p.lights.triangles = num_triangles > 0 ? mesh_triangles : nullptr;
    p.lights.num_triangles = num_triangles;
    p.lights.mesh = num_mesh > 0 ? mesh_lights : nullptr;
    p.lights.num_mesh = num_mesh;
    p.lights.tri_table = tri_cols > 0 ? tri_table : nullptr;
    p.lights.tri_cols = tri_cols;
    p.flags = kMis | kNormals;
    return 0;
}

int ptirkat_process_hit(int n, const float* in, float* out, const float* dens, const float* mat, const float* sph,
                        const float* snrm, float min_response, float min_alpha, int sph_deg) {
    TraceParams P;
    std::memset(&P, 0, sizeof(P));
    P.part.density = reinterpret_cast<const float4*>(dens);
    P.part.material = mat;
    P.part.sph = sph;
    P.part.snrm = snrm;
    P.part.sph_stride = 48;
    P.part.sph_degree = sph_deg;
    P.part.storage = 0;  // FP32
    P.flags = kNormals;
    P.kernel_degree = 4;
    P.min_response = min_response;
    P.alpha_min = min_alpha;
    P.min_transmittance = 0.0f;
    k_process_hit<<<blocks(n), 128>>>(n, in, out, P);
    return finish();
}
int ptirkat_intersect(int n, const float* in, float* out) { k_intersect<<<blocks(n), 128>>>(n, in, out); return finish(); }
int ptirkat_brdf_sample(int n, const float* in, float* out) { k_brdf<<<blocks(n), 128>>>(n, in, out, 0); return finish(); }
int ptirkat_brdf_eval(int n, const float* in, float* out) { k_brdf<<<blocks(n), 128>>>(n, in, out, 1); return finish(); }
int ptirkat_brdf_grads(int n, const float* in, float* out) { k_brdf<<<blocks(n), 128>>>(n, in, out, 2); return finish(); }
int ptirkat_env_lookup(int n, const float* in, float* out) {
    k_env_lookup<<<blocks(n), 128>>>(n, in, out, g_params);
    return finish();
}
int ptirkat_env_bwd(int n, const float* in, float* out, float* env_grad, int eh, int ew) {
    (void)eh;
    (void)ew;
    k_env_bwd<<<blocks(n), 128>>>(n, in, out, g_params, env_grad);
    return finish();
}
int ptirkat_env_sample(int n, const float* in, float* out) {
    k_env_sample<<<blocks(n), 128>>>(n, in, out, g_params);
    return finish();
}
int ptirkat_light_sample(int n, const float* in, float* out) {
    k_light_sample<<<blocks(n), 128>>>(n, in, out, g_params);
    return finish();
}
int ptirkat_light_pdf(int n, const float* in, float* out) {
    k_light_pdf<<<blocks(n), 128>>>(n, in, out, g_params);
    return finish();
}

// the tracer's radix sort of device buffers (keys of 32 or 64 bits, 32-bit values) by bits
// [begin_bit, end_bit); 0 on success
int ptirkat_radix_sort(int key_bytes, const void* keys_in, void* keys_out, const unsigned* vals_in, unsigned* vals_out,
                       long long n, int begin_bit, int end_bit) {
    const size_t bytes = key_bytes == 8 ? radix_sort_temp_bytes<unsigned long long>(n) : radix_sort_temp_bytes<unsigned>(n);
    void* temp = nullptr;
    if (bytes && cudaMalloc(&temp, bytes) != cudaSuccess) return 1;
    cudaError_t e = key_bytes == 8
                        ? radix_sort_pairs<unsigned long long>(temp, bytes, static_cast<const unsigned long long*>(keys_in),
                                                               static_cast<unsigned long long*>(keys_out), vals_in, vals_out, n,
                                                               begin_bit, end_bit, 0)
                        : radix_sort_pairs<unsigned>(temp, bytes, static_cast<const unsigned*>(keys_in),
                                                     static_cast<unsigned*>(keys_out), vals_in, vals_out, n, begin_bit,
                                                     end_bit, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (temp) cudaFree(temp);
    return e == cudaSuccess ? 0 : 1;
}

}  // extern "C"
