// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A scalar CPU restatement of PTIR's differentiable Gaussian-field path tracer (the
// `threedgptir_tracer` forward `trace` and backward `trace_bwd`, reference pipeline
// `reference`/`referenceBwd`, primitive `instances`). It is templated on the scalar type:
// the double instantiation is the FP64 oracle used by the parity tests, the float
// instantiation is the timed CPU baseline of bench.py. Nothing in the shipped library links
// or calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU legs do.
//
// Every function cites the reference file:line whose behaviour it restates (paths are
// relative to the reference project root). The candidate set of a `trace` call (which the
// reference delegates to OptiX) is stated here in its order-independent form:
//   a Gaussian is a candidate of trace(ray, tmin, tend) iff the object-space ray hits the
//   unit instance box [-1,1]^3 for some t in [tmin, tend] (optixTracer.cpp:560-610, the
//   1-primitive GAS) AND intersectInstanceParticle accepts it
//   (gaussianParticles.cuh:484-500: tmin < t* < tend and perp^2/|d'|^2 < 9);
//   the call returns the 16 candidates with the smallest t*, ascending
//   (referenceOptix.cu:95-133 any-hit insertion into 16 sorted payload slots).
// A CPU BVH over the instance world AABBs only prunes; every surviving Gaussian is tested
// exactly, so the result equals brute force.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------------------
// vector helpers
template <class T>
struct V3 {
    T x, y, z;
};
template <class T> inline V3<T> v3(T a) { return {a, a, a}; }
template <class T> inline V3<T> v3(T a, T b, T c) { return {a, b, c}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T>& operator+=(V3<T>& a, V3<T> b) { a = a + b; return a; }
template <class T> inline V3<T>& operator-=(V3<T>& a, V3<T> b) { a = a - b; return a; }
template <class T> inline V3<T>& operator*=(V3<T>& a, V3<T> b) { a = a * b; return a; }
template <class T> inline V3<T>& operator*=(V3<T>& a, T s) { a = a * s; return a; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline bool is_zero(V3<T> a) { return a.x == T(0) && a.y == T(0) && a.z == T(0); }
template <class T> inline T vmax(V3<T> a) { return std::fmax(a.x, std::fmax(a.y, a.z)); }
// mathUtils.h:390-393: v / |v| when |v|^2 > 0, else v unchanged.
template <class T> inline V3<T> safe_normalize(V3<T> v) {
    const T l = dot(v, v);
    return l > T(0) ? v * (T(1) / std::sqrt(l)) : v;
}
template <class T> struct M33 {
    V3<T> r[3];  // rows
};
// the reference's `p * m` (mathUtils.h:457-459): (dot(m0,p), dot(m1,p), dot(m2,p))
template <class T> inline V3<T> rowmul(const M33<T>& m, V3<T> p) {
    return {dot(m.r[0], p), dot(m.r[1], p), dot(m.r[2], p)};
}
// the reference's `m * p` (mathUtils.h:450-455): sum_i m_i * p_i
template <class T> inline V3<T> colmul(const M33<T>& m, V3<T> p) {
    return m.r[0] * p.x + m.r[1] * p.y + m.r[2] * p.z;
}
// gaussianParticles.cuh:26-46 — rows of R^T for the wxyz quaternion q (not normalised).
template <class T> inline M33<T> quat_to_rt(T r, T x, T y, T z) {
    M33<T> m;
    m.r[0] = {T(1) - T(2) * (y * y + z * z), T(2) * (x * y + r * z), T(2) * (x * z - r * y)};
    m.r[1] = {T(2) * (x * y - r * z), T(1) - T(2) * (x * x + z * z), T(2) * (y * z + r * x)};
    m.r[2] = {T(2) * (x * z + r * y), T(2) * (y * z - r * x), T(1) - T(2) * (x * x + y * y)};
    return m;
}
// mathUtils.h:535-545 — rows of R.
template <class T> inline M33<T> quat_to_r(T r, T x, T y, T z) {
    M33<T> m;
    m.r[0] = {T(1) - T(2) * (y * y + z * z), T(2) * (x * y - r * z), T(2) * (x * z + r * y)};
    m.r[1] = {T(2) * (x * y + r * z), T(1) - T(2) * (x * x + z * z), T(2) * (y * z - r * x)};
    m.r[2] = {T(2) * (x * z - r * y), T(2) * (y * z + r * x), T(1) - T(2) * (x * x + y * y)};
    return m;
}
// mathUtils.h:442-448 (Pixar's branchless orthonormal basis).
template <class T> inline void branchless_onb(V3<T> n, V3<T>& b1, V3<T>& b2) {
    const T sign = std::copysign(T(1), n.z);
    const T a = T(-1) / (sign + n.z);
    const T b = n.x * n.y * a;
    b1 = {T(1) + sign * n.x * n.x * a, sign * b, -sign * n.x};
    b2 = {b, sign + n.y * n.y * a, -n.y};
}

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------
// sampler.cuh:26-84 — PCG32 seeded by a hash of the launch index and frame.
// The order in which the three draws of a 3-vector (sampler.cuh:80-82) and the two uv jitter
// draws of the alias sampler (environment.cuh:245-250) are taken is fixed by `kDrawOrder`
// below; 0 = first argument first. It is pinned against nvcc by tests/golden.
struct Sampler {
    uint64_t state = 0, inc = 1;
    static uint64_t seed_of(uint32_t x, uint32_t y, uint32_t z, uint32_t frame) {
        uint64_t s = 1469598103934665603ull;
        s ^= uint64_t(x) + 1099511628211ull * s;
        s ^= uint64_t(y) + 1099511628211ull * s;
        s ^= uint64_t(z) + 1099511628211ull * s;
        s ^= uint64_t(frame) + 1099511628211ull * s;
        return s ? s : 1ull;
    }
    void init_launch(uint32_t x, uint32_t y, uint32_t z, uint32_t frame) { init(seed_of(x, y, z, frame), 0); }
    void init(uint64_t seed, uint64_t seq) {
        state = 0;
        inc = (seq << 1u) | 1ull;
        next_u32();
        state += seed;
        next_u32();
    }
    uint32_t next_u32() {
        const uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((-int(rot)) & 31));
    }
    // exact float value (u & 0xFFFFFF) / 2^24, representable in any T
    float next_1d() { return float(next_u32() & 0x00FFFFFFu) * (1.0f / 16777216.0f); }
};
extern int kDrawOrder;  // 0: left-to-right, 1: right-to-left
template <class T> inline V3<T> next_3d(Sampler& s) {
    if (kDrawOrder == 0) {
        const T a = s.next_1d(); const T b = s.next_1d(); const T c = s.next_1d();
        return {a, b, c};
    }
    const T c = s.next_1d(); const T b = s.next_1d(); const T a = s.next_1d();
    return {a, b, c};
}
inline void next_2(Sampler& s, float& first_arg, float& second_arg) {
    if (kDrawOrder == 0) { first_arg = s.next_1d(); second_arg = s.next_1d(); }
    else { second_arg = s.next_1d(); first_arg = s.next_1d(); }
}

// ---------------------------------------------------------------------------------------
// configuration and inputs
struct Config {
    int kernel_degree = 4;            // render.particle_kernel_degree
    float min_response = 0.0113f;     // render.particle_kernel_min_response
    int density_clamping = 1;         // render.particle_kernel_density_clamping
    int sph_max_coeffs = 16;          // (render.particle_radiance_sph_degree + 1)^2
    int enable_normals = 1, enable_hitcounts = 1, enable_mis = 1, enable_metallic = 0, visualize_lights = 0;
};

struct Inputs {
    int n = 0;
    // geometry the acceleration structure was built from (Tracer.build_acc)
    const float *bpos = nullptr, *brot = nullptr, *bscl = nullptr, *bdns = nullptr;
    // trace-time particle tensors (tracer.py:163-166 layouts)
    const float* density = nullptr;   // [n,12] pos3 dns1 rot4(wxyz) scl3 pad1
    const float* material = nullptr;  // [n,5] albedo3 roughness1 metallic1
    const float* sph = nullptr;       // [n, sph_max_coeffs*3], coefficient-major
    const float* snrm = nullptr;      // [n,3]
    const float* env = nullptr;       // [eh, ew, 4]
    int eh = 0, ew = 0;
    const float* alias = nullptr;     // [3, ah, aw]: prob, alias (as float), pdf
    int ah = 0, aw = 0;
    float ray_to_world[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    const float *ray_ori = nullptr, *ray_dir = nullptr;  // [nz, h, w, 3]
    int nz = 0, h = 0, w = 0;
    uint32_t frame = 0;
    int sph_degree = 3;
    float min_transmittance = 0.001f;
    uint32_t max_bounces = 3;
    uint32_t render_opts = 0;
    // punctual and area lights (threedgptir_tracer/tracer.py:40-119 LightBuffers), row-major
    const float* lights = nullptr;          // [num_lights, 9]: type, position xyz, radius, radiance rgb, two_sided
    const float* light_table = nullptr;     // [5, light_entries]: prob, alias, type, index, selection pdf
    const float* mesh_vertices = nullptr;   // [num_mesh_vertices, 3]
    const int* mesh_triangles = nullptr;    // [num_mesh_triangles, 3]
    const float* mesh_lights = nullptr;     // [num_mesh_lights, 8]: tri offset, tri count, vtx offset, vtx count,
                                            //   radiance rgb, two_sided
    const float* mesh_tri_table = nullptr;  // [3, mesh_tri_cols]: prob, local alias, area pdf
    int num_lights = 0, light_entries = 0, num_mesh_vertices = 0, num_mesh_triangles = 0, num_mesh_lights = 0,
        mesh_tri_cols = 0;
};

// per-sample forward outputs (optixTracer.cpp:931-944 shapes), all [nz,h,w,C] float
struct FwdOut {
    float *radiance = nullptr, *density = nullptr, *hit = nullptr, *hit2 = nullptr, *distortion = nullptr,
          *normal = nullptr, *snormal = nullptr, *material = nullptr, *hits_count = nullptr, *pbr = nullptr,
          *light = nullptr, *components = nullptr;  // components [nz,h,w,2,3]
    float* visibility = nullptr;                    // [n] (1.0 where any accepted hit)
    uint32_t* path_sig = nullptr;                   // [nz,h,w] decision signature of each path
};

// backward inputs (the saved forward outputs plus their gradients) and outputs
struct BwdIn {
    const float *pbr = nullptr, *light = nullptr;          // [nz,h,w,3]
    const float *pbr_grad = nullptr, *light_grad = nullptr, *material_grad = nullptr;  // [..,3],[..,3],[..,5]
};
struct BwdOut {
    double* material_grad = nullptr;  // [n,5]
    double* env_grad = nullptr;       // [eh,ew,4]
};

struct Stats {
    uint64_t segments = 0;      // primary + shadow + bounce rays traced (forward semantics)
    uint64_t trace_calls = 0;   // k-buffer rounds
    uint64_t candidates = 0;    // candidates returned by trace calls
    uint64_t accepted = 0;      // hits accepted by processHit
    uint64_t env_lookups = 0;   // bilinear environment lookups
    uint64_t replay_segments = 0;  // re-traversals of the backward
};

// ---------------------------------------------------------------------------------------
// particlePrimitives.cu:27-51 — kernel support radius in units of the particle scale.
template <class T> inline T kernel_scale(T density, T min_response, bool clamping, int degree) {
    const T modulation = clamping ? density : T(1);
    const T min_resp = std::fmin(min_response / modulation, T(0.97));
    if (degree < 0) {
        const T k = std::fabs(T(degree));
        const T s = T(1) / std::pow(T(3), k);
        return std::pow((T(1) / (std::log(min_resp) - T(1)) + T(1)) / s, T(1) / k);
    }
    if (degree == 0) return ((T(1) - min_resp) / T(3)) / T(-0.329630334487);
    const T b = T(degree);
    const T a = T(-4.5) / std::pow(T(3), b);
    return std::pow(std::log(min_resp) / a, T(1) / b);
}

// gaussianParticles.cuh:260-301 — generalized Gaussian response of squared distance d2.
template <class T> inline T particle_response(int degree, T d2) {
    switch (degree) {
    case 8: { const T q = d2 * d2; return std::exp(T(-0.000685871056241) * q * q); }
    case 5: return std::exp(T(-0.0185185185185) * d2 * d2 * std::sqrt(d2));
    case 4: return std::exp(T(-0.0555555555556) * d2 * d2);
    case 3: return std::exp(T(-0.166666666667) * d2 * std::sqrt(d2));
    case 1: return std::exp(T(-1.5) * std::sqrt(d2));
    case 0: return std::fmax(T(1) + T(-0.329630334487) * std::sqrt(d2), T(0));
    default: return std::exp(T(-0.5) * d2);
    }
}

// Acceleration structure: per-Gaussian object-space transform (the inverse of the instance
// transform of particlePrimitives.cu:595-606) and world AABB of the instance box.
template <class T> struct Instances {
    int n = 0;
    std::vector<M33<T>> inv;   // diag(1/kscl) R^T
    std::vector<V3<T>> center;
    std::vector<V3<T>> lo, hi; // world AABB of the transformed [-1,1]^3
    V3<T> scene_lo{}, scene_hi{};
    bool empty = true;
    // CPU BVH (prune only)
    struct Node { V3<T> lo, hi; int left, right, first, count; };
    std::vector<Node> nodes;
    std::vector<int> order;
};

template <class T> void build_instances(const Config& cfg, const Inputs& in, Instances<T>& I);

// ---------------------------------------------------------------------------------------
// environment helpers (environment.cuh)
template <class T> struct EnvView {
    const float* data = nullptr;
    int w = 0, h = 0;
    bool cube = false;
    const float *prob = nullptr, *alias = nullptr, *pdf = nullptr;
    int aw = 0, ah = 0, cells = 0;
    bool has_env() const { return data != nullptr && w > 0 && h > 0; }
    bool has_light() const { return has_env() && cells > 0; }
};

struct Footprint { int x0, x1, y0, y1; double w00, w10, w01, w11; };

}  // namespace oracle
