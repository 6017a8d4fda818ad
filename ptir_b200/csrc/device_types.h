// Plain-old-data views handed from the C-ABI layer to the kernels (by value, as kernel
// parameters). Every pointer is device memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ptir {

// Acceleration structure over the Gaussians' instance boxes. The LBVH is built binary and
// traversed 4-wide: every binary node at even depth becomes a 4-wide node holding the boxes of
// its (up to four) grandchildren, so one 128-byte fetch tests four boxes.
//   node4 = 8 x float4: lo.x[4] lo.y[4] lo.z[4] hi.x[4] hi.y[4] hi.z[4] child[4] kmax[4]
//           (kmax: the largest kernel support radius of any Gaussian under the child);
//           a child c >= 0 is a 4-wide node, kNoChild an empty slot, any other c < 0 leaf ~c.
//   leaf  = 4 x float4: rows of the world->instance affine map [A | b] (A = diag(1/k) R^T,
//           b = -A mu, k = kernel support scale per axis), then (gaussian id, kmax, 0, 0).
// (The binary nodes, 4 x float4 each: (L.lo.xyz, L.hi.x) (L.hi.yz, R.lo.xy) (R.lo.z, R.hi.xyz)
//  (left, right, -, -), are kept for refits.)
constexpr int kNoChild = (int)0x80000000;

struct AccelView {
    const float4* nodes;  // 4-wide nodes
    const float4* leaves;
    const float4* bounds;  // [2]: scene AABB lo.xyz, hi.xyz (union of the instance AABBs)
    int n;                 // number of Gaussians (leaves)
    // Subtree culling against the K-th distance t_K. 0: a subtree is culled when the ray enters its
    // box after t_K, as the reference's traversal culls (order dependent for grazing candidates).
    // > 0: culled only when no Gaussian under it can have its closest approach t* before t_K,
    // using t* >= box entry - kCullSlack * kmax / |d| (exact K-nearest candidates).
    float cull_slack;
};

// A ray that hits a Gaussian's instance box [-1,1]^3 and misses the inscribed unit sphere has
// its closest approach (in instance units) at distance p in [1, sqrt(3)] from the centre, and the
// box entry lies at most sqrt(3 - p^2) <= sqrt(2) instance units past it along the ray; one
// instance unit is at most kmax / |d| of the ray parameter. (A ray through the sphere has t* in
// the box.) With a margin for rounding:
constexpr float kCullSlack = 1.4143f;

struct EnvView {
    const float4* data;  // [h, w] RGBA texels, null when absent
    int w, h;
    int cube;            // 1 when h == 6 w
    const float* prob;   // alias table [3, ah, aw]: prob, alias index (as float), pdf
    const float* alias;
    const float* pdf;
    int aw, ah, cells;
    float offset_x, offset_y;  // environment offset (fixed at (0, 0)), turned into the rotation per lookup
};

enum Flags : unsigned {
    kNormals = 1u,
    kHitCounts = 2u,
    kMis = 4u,
    kMetallic = 8u,
    kVisualizeLights = 16u,
    kExactReplay = 32u,  // backward re-traversals include the segment's last composited Gaussian
    kWarpAggregate = 64u,  // gradient rows shared by lanes of a warp are summed before the atomics
    kPathSig = 128u,       // keep a per-path signature of the path's discrete decisions (FwdOutputs::path_sig)
};

// Punctual and area lights: the reference's LightBuffers (threedgptir_tracer/tracer.py:40-119),
// read as the packed float tables lightSampler.cuh and meshLight.cuh index. Counts of 0 leave
// the environment as the only light.
struct LightView {
    const float* lights;     // [num_lights, 9]: type, position / center xyz, radius, radiance rgb, two_sided
    const float* table;      // [5, entries]: alias prob, alias entry, light type, light index, selection pdf
    const float* vertices;   // [num_vertices, 3] mesh-light vertices
    const int* triangles;    // [num_triangles, 3] global vertex indices
    const float* mesh;       // [num_mesh, 8]: triangle offset, triangle count, vertex offset, vertex count,
                             //   radiance rgb, two_sided
    const float* tri_table;  // [3, tri_cols]: alias prob, alias (local to the mesh), area pdf
    int num_lights, entries, num_vertices, num_triangles, num_mesh, tri_cols;
};

struct ParticleView {
    const float4* density;   // [n, 3] float4 = pos.xyz dns | quat wxyz | scale.xyz pad
    const float* material;   // [n, 5]
    const float* sph;        // [n, sph_stride]
    const float* snrm;       // [n, 3] or null (also the "normals present" flag in 16-bit storage)
    int sph_stride;          // floats per particle (3 * max coefficients)
    int sph_degree;          // evaluation degree (<= max)
    unsigned storage;        // Storage (storage.cuh): FP32 reads the four arrays above, else hot / cold
    const uint4* hot;        // [n, 2] 16-bit geometry records
    const uint4* cold;       // [n, cold_stride] 16-bit material / normal / SH records
    int cold_stride;         // uint4 per cold record
};

// One launch of a batch (a camera view with its own extent and sample count). Launch indices
// of a view run over (z, y, x) row-major from `offset` in the batch's flat ray and output arrays;
// its 8x4 pixel tiles run from `tile0` in the batch's tile order. Paths are seeded from the
// view's own (x, y, z) and frame, so a batch traces exactly what separate launches would.
struct ViewDesc {
    long long offset;
    long long tile0;
    const float* to_world;  // [4, 4] row-major (only the first matrix of a launch applies)
    int w, h, z;
    unsigned frame;
};

constexpr int kMaxViews = 64;  // views of one batch (passed by value with the kernel parameters)

// Element strides of a per-sample array (PackedTensorAccessor32 semantics): element (z, y, x, c)
// of a [Z,H,W,C] launch array at z*sz + y*sy + x*sx + c*sc; in a batch of views the arrays are
// flat [T,C] and sample t (the flat launch index) lies at t*sx + c*sc.
struct SampleLayout {
    long long sz, sy, sx, sc;
};

// offset of channel 0 of a sample: (z, y, x) within its launch, li its flat index in the batch
__device__ __forceinline__ long long sample_offset(const SampleLayout& L, bool flat, unsigned z, unsigned y,
                                                   unsigned x, size_t li) {
    return flat ? (long long)li * L.sx : (long long)z * L.sz + (long long)y * L.sy + (long long)x * L.sx;
}

struct TraceParams {
    AccelView accel;
    ParticleView part;
    EnvView env;
    LightView lights;
    const float* ray_ori;        // [z, h, w, 3], strided (ray_ori_layout)
    const float* ray_dir;
    SampleLayout ray_ori_layout, ray_dir_layout;
    int flat_samples;            // 1: per-sample arrays are flat [T,C] over the batch of views
    ViewDesc views[kMaxViews];   // the launches of this trace (one for the reference's single launch)
    int nviews;
    long long tiles;             // 8x4 pixel tiles of all views
    unsigned flags;
    int kernel_degree;
    float min_response;          // hitMinGaussianResponse
    float alpha_min;             // 1/255
    float min_transmittance;
    unsigned max_bounces;
    unsigned render_opts;
    unsigned* error_word;        // set on a bounded-loop violation (stack overflow, runaway loop)
    unsigned long long* counters;  // [kNumCounters] indexed by Counter

};

struct FwdOutputs {
    float* radiance;    // [z,h,w,3]
    float* density;     // [z,h,w,1]
    float* hit;         // [z,h,w,2]
    float* hit2;        // [z,h,w,1]
    float* distortion;  // [z,h,w,1]
    float* normal;      // [z,h,w,3]
    float* snormal;     // [z,h,w,3]
    float* material;    // [z,h,w,5]
    float* hits_count;  // [z,h,w,1]
    float* pbr;         // [z,h,w,3]
    float* light;       // [z,h,w,3]
    float* components;  // [z,h,w,2,3]
    float* visibility;  // [n] float32 tensor holding int32 1 where an accepted hit occurred
    unsigned* path_sig; // [z,h,w] decision signature of each path (kPathSig), or null
};

struct BwdInputs {
    const float* pbr;            // [z,h,w,3], strided (pbr_layout)
    const float* light;          // [z,h,w,3]
    const float* pbr_grad;       // [z,h,w,3]
    const float* light_grad;     // [z,h,w,3]
    const float* material_grad;  // [z,h,w,5]
    SampleLayout pbr_layout, light_layout, pbr_grad_layout, light_grad_layout, material_grad_layout;
    float* particle_material_grad;  // [n,5]
    float* environment_grad;        // [eh,ew,4]
    float* particle_material_comp;  // [n,5] compensation terms of the material gradient sums, or null
    float* environment_comp;        // [eh,ew,4] compensation terms of the environment sums, or null
};

enum Counter : int {
    kCtrSegments = 0,
    kCtrTraceCalls = 1,
    kCtrCandidates = 2,
    kCtrAccepted = 3,
    kCtrEnvLookups = 4,
    kCtrReplay = 5,
    kCtrReplayAccepted = 6,
    kCtrNodes = 7,
    kCtrLeaves = 8,
    kNumCounters = 10,
};

enum ErrorBits : unsigned {
    kErrStackOverflow = 1u,
    kErrLoopBound = 2u,
};

// megakernel schedule (tracer.cu): one thread per path
struct StageCtx;
cudaError_t launch_trace_fwd(const TraceParams& p, const FwdOutputs& o, const StageCtx& sc, cudaStream_t s);
cudaError_t launch_trace_bwd(const TraceParams& p, const BwdInputs& b, const StageCtx& sc, cudaStream_t s);

}  // namespace ptir
