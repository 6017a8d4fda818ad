/*
 * ptir_b200 — C ABI of the B200-native Gaussian-field path tracer.
 *
 * Drop-in boundary for the native half of PTIR's `threedgptir_tracer` extension. Each entry
 * point replaces one method of the reference's pybind11 class `OptixTracer`
 * (threedgptir_tracer/bindings.cpp:32-38, include/3dgptir/optixTracer.h:130-217):
 *
 *   ptir_create      <- OptixTracer::OptixTracer   (optixTracer.h:130-144, optixTracer.cpp:274-343)
 *   ptir_destroy     <- OptixTracer::~OptixTracer  (optixTracer.h:146, optixTracer.cpp:345-371)
 *   ptir_build_bvh   <- OptixTracer::buildBVH      (optixTracer.h:212-217, optixTracer.cpp:633-907)
 *   ptir_trace       <- OptixTracer::trace         (optixTracer.h:148-168, optixTracer.cpp:909-1013)
 *   ptir_trace_bwd   <- OptixTracer::traceBwd      (optixTracer.h:170-210, optixTracer.cpp:1015-1145)
 *   ptir_last_error  <- (new) the reference logs CUDA/OptiX errors without raising
 *                       (cuoptixMacros.h:22-44); here every entry returns a status and the
 *                       message is kept on the handle.
 *
 * Conventions
 *   - Every pointer named in an args struct is DEVICE memory, float32, in the reference's tensor
 *     layout; the caller owns all of it (inputs and outputs), as torch does for the reference
 *     (optixTracer.cpp:931-944, 1057-1063). Particle, environment and light tables and every
 *     output are C-contiguous (the reference passes them through getPtr, a contiguous copy,
 *     tensorBuffering.h:30-39). The per-sample inputs (ray origins and directions, and the
 *     backward's saved outputs and incoming gradients) may be strided, as the reference reads
 *     them through PackedTensorAccessor32 (tensorBuffering.h:41-45, optixTracer.cpp:963-964,
 *     1082-1113): with `use_strides` set in the args struct, each has a `*_strides[4]` field,
 *     the element strides of its [Z,H,W,C] index (z, y, x, c), 0 for a broadcast dimension; with
 *     `use_strides` 0 they are C-contiguous and the stride fields are ignored. In the batched
 *     entry points (ptir_trace_views) the per-sample arrays are flat [T,C]: element (t, c) lies
 *     at t * strides[2] + c * strides[3], strides[0] and [1] are unused. Output
 *     buffers need no initialisation: every element is written (the reference's zero-filled
 *     outputs are written as zeros).
 *   - The library owns its acceleration structure and scratch; buffers grow, never shrink.
 *   - All work is enqueued on `stream` (a cudaStream_t); no entry point synchronises the host
 *     with the device, so a trace can be captured in a CUDA graph once the structure exists. The
 *     one exception is a rebuild by ptir_build_bvh with the PLOC builder (the default), which
 *     reads a count back between its iterations; a refit does not.
 *   - Return value: PTIR_OK (0) or a PTIR_E* code; ptir_last_error() describes the last failure.
 *   - A handle is not thread-safe (nor is the reference's object).
 */
#ifndef PTIR_B200_H
#define PTIR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PTIR_ABI_VERSION 6

enum {
    PTIR_OK = 0,
    PTIR_EINVAL = 1,   /* bad argument: shape, null pointer, unsupported option */
    PTIR_ECUDA = 2,    /* a CUDA call failed */
    PTIR_ESTATE = 3,   /* trace before build_bvh, or particle count differs from the structure */
    PTIR_EDEVICE = 4,  /* a kernel hit one of its loop bounds (reported by ptir_device_status) */
};

typedef struct ptir_tracer ptir_tracer;

/* Construction options: the arguments of OptixTracer(...) that change the traced result
 * (optixTracer.h:130-144; the JIT defines of optixTracer.cpp:240-272). The pipeline and
 * primitive names of the reference select its OptiX programs; only the configured
 * `reference` pipeline with `instances` primitives exists here. */
typedef struct ptir_config {
    float kernel_degree;          /* render.particle_kernel_degree (default 4) */
    float kernel_min_response;    /* render.particle_kernel_min_response (0.0113) */
    int32_t density_clamping;     /* render.particle_kernel_density_clamping */
    int32_t sph_degree;           /* render.particle_radiance_sph_degree: rows hold (d+1)^2*3 floats */
    int32_t enable_normals;       /* render.enable_normals */
    int32_t enable_hitcounts;     /* render.enable_hitcounts */
    int32_t enable_mis;           /* render.enable_mis */
    int32_t enable_metallic;      /* render.enable_metallic */
    int32_t visualize_lights;     /* render.visualize_lights */
    int32_t collect_counters;     /* keep per-launch segment/candidate counters (cheap) */
    /* B200 schedule (render.b200.*; no counterpart in the reference, results are identical): */
    int32_t schedule;             /* PTIR_SCHEDULE_WAVEFRONT (default) or PTIR_SCHEDULE_MEGAKERNEL */
    int32_t chunk_tiles;          /* wavefront: 8x4 pixel tiles per chunk of paths (0 = sized at the tracer's
                                     first trace to a third of the free device memory, at least 32768) */
    int32_t kbuffer;              /* wavefront: candidates gathered per traversal, 8, 16 or 32 (0 = 16).
                                     Segments are composited in the reference's rounds of 16 candidates
                                     with 16 and 32: a 32-entry traversal stands for two rounds when its
                                     second half is exactly the next round's candidates, else the next
                                     round is traced. 8 composites in rounds of 8, which changes a small
                                     share of the samples (a round's candidates must have their box
                                     crossed within the round's interval). */
    int32_t refill_lanes;         /* wavefront intersection: waiting lanes, 1..32, before a warp refills (0 = 32) */
    int32_t block_size;           /* wavefront: threads per block, 64, 128 or 256 (0 = 128) */
    int32_t collect_timings;      /* record CUDA events around every kernel launch (ptir_get_stage_times) */
    int32_t ray_order;            /* wavefront bounce rays: 0 = intersected in (octant, origin cell, direction cell)
                                     order (default), 1 = in queue order; results are the same */
    int32_t exact_replay;         /* 0 = the reference's adjoint: backward re-traversals end where its float
                                     epsilon leaves out each segment's last composited Gaussian, and the
                                     NEE albedo term is weighted by the environment's radiance whatever
                                     light was sampled; 1 = re-traversals include that Gaussian and the
                                     NEE term uses the sampled light's radiance, which makes the adjoint
                                     the exact derivative of the same-sample estimator for albedo and
                                     the environment (no counterpart in the reference) */
    int32_t grad_sums;            /* gradient scatter: 0 = compensated (Kahan-pair) float atomics (default),
                                     1 = plain float atomics as the reference */
    int32_t storage;              /* attribute storage: PTIR_STORAGE_FP32 (the caller's tensors are read as
                                     they are), _BF16 or _FP16 (geometry, material, shading normal and SH
                                     rounded to nearest even once per call and by build_bvh; arithmetic
                                     stays FP32) */
    int32_t grad_aggregate;       /* gradient scatter: 0 = lanes of a warp that add to the same Gaussian or
                                     texel sum their terms first and one of them issues the atomics
                                     (default), 1 = one atomic per lane and term as the reference */
    int32_t shadow_kbuffer;       /* wavefront: candidates per NEE shadow-ray traversal, 8, 16 or 32 (0 = 16);
                                     a shadow walk visits hits in distance order whatever the size */
    int32_t exact_candidates;     /* 0 = subtrees culled at the K-th distance by their box entry, as the
                                     reference's traversal culls: a Gaussian whose closest approach lies
                                     before its box entry (a ray grazing a box corner) is kept or not
                                     depending on the traversal order; 1 = every traversal returns exactly
                                     the K nearest candidates (its subtrees culled only when no closest
                                     approach under them can lie before the K-th distance), so the results
                                     depend on neither the order nor the k-buffer size (no counterpart in
                                     the reference) */
    int32_t resume_rounds;        /* wavefront, k-buffer 8 or 16: which traversals start a segment's
                                     next k-buffer round from the subtrees, leaves and candidates its
                                     previous round set aside against the K-th distance, instead of
                                     from the root (fewer node visits; the same candidates up to the
                                     grazing case above): 0 = the backward replay's (default), 1 =
                                     none, 2 = the replay's and the intersection stage's */
    int32_t bvh_builder;          /* hierarchy of a rebuild: 0 = default (PTIR_BVH_PLOC), PTIR_BVH_MORTON =
                                     the Karras hierarchy over the sorted keys, PTIR_BVH_PLOC = agglomerative
                                     clustering by surface area over the same sorted leaves (a better tree, a
                                     slower build that synchronises its stream: a rebuild then cannot be
                                     captured in a CUDA graph, a refit can). The traced results are the same
                                     up to the order-dependent grazing case of exact_candidates */
} ptir_config;

enum { PTIR_BVH_DEFAULT = 0, PTIR_BVH_MORTON = 1, PTIR_BVH_PLOC = 2 };

enum { PTIR_STORAGE_FP32 = 0, PTIR_STORAGE_BF16 = 1, PTIR_STORAGE_FP16 = 2 };

enum { PTIR_SCHEDULE_WAVEFRONT = 0, PTIR_SCHEDULE_MEGAKERNEL = 1 };

/* Inputs of one trace, shared by the forward and the backward
 * (the arguments of OptixTracer::trace, optixTracer.h:148-168). */
typedef struct ptir_trace_args {
    uint32_t frame;                 /* frameNumber: seeds the per-path random streams */
    const float* ray_to_world;      /* [B,4,4]; only the first matrix is applied (optixTracer.cpp:962) */
    const float* ray_origin;        /* [Z,H,W,3] */
    const float* ray_direction;     /* [Z,H,W,3] */
    int32_t z, h, w;                /* launch extent: Z = spp * B */
    const float* particle_density;  /* [N,12]: pos3 density1 rot4(wxyz) scale3 pad1 */
    const float* particle_material; /* [N,5]: albedo3 roughness1 metallic1 */
    const float* particle_radiance; /* [N,(sph_degree+1)^2*3] SH coefficients, coefficient-major */
    const float* particle_shading_normal; /* [N,3] */
    int32_t n;                      /* N; must equal the count of the last ptir_build_bvh */
    const float* environment;       /* [EH,EW,4] or NULL; cube map when EH == 6*EW */
    int32_t env_h, env_w;
    const float* environment_alias; /* [3,AH,AW] prob/alias/pdf or NULL */
    int32_t alias_h, alias_w;
    /* Punctual and area lights: the LightBuffers tensors (tracer.py:40-119), float32 / int32,
     * row-major, as the reference's light sampler reads them (lightSampler.cuh, meshLight.cuh).
     * With num_light_entries == 0 the environment is the only light, as in the reference. */
    const float* lights;              /* [num_lights, 9]: type (1 point, 2 sphere), position xyz, radius,
                                         radiance rgb, two_sided */
    const float* light_alias;         /* [5, num_light_entries]: alias prob, alias entry, light type
                                         (0 environment, 1 point, 2 sphere, 3 mesh), light index,
                                         selection pdf */
    const float* mesh_light_vertices; /* [num_mesh_light_vertices, 3] */
    const int32_t* mesh_light_triangles; /* [num_mesh_light_triangles, 3] vertex indices */
    const float* mesh_lights;         /* [num_mesh_lights, 8]: triangle offset, triangle count, vertex
                                         offset, vertex count, radiance rgb, two_sided */
    const float* mesh_light_alias;    /* [3, mesh_light_alias_cols]: alias prob, alias (local to the
                                         mesh), area pdf per triangle */
    int32_t num_lights, num_light_entries, num_mesh_lights;
    int32_t num_mesh_light_vertices, num_mesh_light_triangles, mesh_light_alias_cols;
    uint32_t sh_indirect;           /* RenderOpts: 0 = NONE, 1 = INDIRECT */
    int32_t sph_eval_degree;        /* SH degree evaluated (<= sph_degree) */
    float min_transmittance;        /* render.min_transmittance */
    uint32_t max_bounces;           /* render.max_bounces */
    int32_t use_strides;              /* 1: ray_origin / ray_direction are read with the strides below, 0: they
                                         are C-contiguous (see Conventions) */
    int64_t ray_origin_strides[4];    /* element strides of ray_origin */
    int64_t ray_direction_strides[4]; /* element strides of ray_direction */
} ptir_trace_args;

/* Forward outputs, [Z,H,W,C] (optixTracer.cpp:931-944). */
typedef struct ptir_trace_outputs {
    float* radiance;                   /* C=3 */
    float* density;                    /* C=1 (opacity) */
    float* hit_distance;               /* C=2 (integrated depth, last hit distance) */
    float* hit_distance_second_moment; /* C=1 */
    float* depth_distortion;           /* C=1 */
    float* normal;                     /* C=3 */
    float* shading_normal;             /* C=3 */
    float* material;                   /* C=5 */
    float* hits_count;                 /* C=1 */
    float* pbr;                        /* C=3 */
    float* light;                      /* C=3 */
    float* pbr_components;             /* [Z,H,W,2,3] direct / indirect */
    float* visibility;                 /* [N,1]: int32 1 stored in the float32 element per visible Gaussian;
                                          cleared by the call */
    uint32_t* path_signature;          /* [Z,H,W] or NULL (no counterpart in the reference): per path an FNV-1a
                                          hash of its discrete decisions in path order (each segment's
                                          accepted-hit count, interaction and escape flags; NEE shadow ray
                                          cast and occluded; continuation after each BRDF sample). Two
                                          evaluations of a path with equal signatures took the same branches;
                                          the oracle computes the same hash. */
} ptir_trace_outputs;

/* Backward inputs: the saved forward outputs and the gradients flowing into them
 * (OptixTracer::traceBwd, optixTracer.h:170-210). Gradients may be NULL (treated as zero). */
typedef struct ptir_bwd_args {
    const float* pbr;             /* [Z,H,W,3] forward rayPbr */
    const float* light;           /* [Z,H,W,3] forward rayLight */
    const float* pbr_grad;        /* [Z,H,W,3] */
    const float* light_grad;      /* [Z,H,W,3] */
    const float* material_grad;   /* [Z,H,W,5] */
    /* 1: the five arrays above are read with these element strides, 0: they are C-contiguous (see
     * Conventions) */
    int32_t use_strides;
    int64_t pbr_strides[4], light_strides[4], pbr_grad_strides[4], light_grad_strides[4], material_grad_strides[4];
} ptir_bwd_args;

/* Backward outputs. The reference's backward fills only the material and environment
 * gradients; its density / SH / shading-normal gradients are zero tensors
 * (optixTracer.cpp:1057-1063) and are left to the caller here. Both buffers are cleared by
 * the call. */
typedef struct ptir_bwd_outputs {
    float* particle_material_grad; /* [N,5] */
    float* environment_grad;       /* [EH,EW,4] or NULL */
} ptir_bwd_outputs;

/* Device counters of the most recent trace / trace_bwd (collect_counters = 1). */
typedef struct ptir_counters {
    uint64_t segments;        /* rays traced through the field: primary, shadow and bounce rays
                                 (the backward counts its replay of the forward path the same way) */
    uint64_t trace_calls;     /* k-buffer traversals */
    uint64_t candidates;      /* candidates returned by the traversals */
    uint64_t accepted;        /* hits composited by primary / bounce segments */
    uint64_t env_lookups;     /* bilinear environment lookups */
    uint64_t replay;          /* backward re-traversals of a segment that scatter material gradients */
    uint64_t replay_accepted; /* hits that received a material gradient */
    uint64_t node_visits;     /* internal BVH nodes fetched (implementation overhead) */
    uint64_t leaf_tests;      /* exact instance tests */
} ptir_counters;

/* The kernels of a trace, for ptir_get_stage_counters / ptir_get_stage_times. */
enum {
    PTIR_STAGE_INTERSECT = 0,  /* wavefront: primary and bounce segments (traversal + compositing) */
    PTIR_STAGE_SHADOW = 1,     /* wavefront: NEE shadow rays */
    PTIR_STAGE_REPLAY = 2,     /* wavefront backward: material-gradient re-traversals */
    PTIR_STAGE_SHADING = 3,    /* wavefront: camera rays, primary outputs, light gathering, BRDF sampling */
    PTIR_STAGE_MEGAKERNEL = 4, /* megakernel schedule: the whole-path kernel */
    PTIR_STAGE_SORT = 5,       /* wavefront: ray-order keys and their radix sort */
    PTIR_NUM_STAGES = 6
};

/* Device time of each stage's launches since the previous read (collect_timings = 1). */
typedef struct ptir_stage_times {
    double ms[PTIR_NUM_STAGES];          /* summed launch intervals, CUDA events on the launch stream */
    uint64_t launches[PTIR_NUM_STAGES];  /* launches timed */
} ptir_stage_times;

int ptir_abi_version(void);

/* OptixTracer(path, cuda_path, pipeline, backwardPipeline, primitive, ...) */
int ptir_create(const ptir_config* config, ptir_tracer** out);
void ptir_destroy(ptir_tracer* tracer);

/* buildBVH(mogPos[N,3], mogRot[N,4], mogScl[N,3], mogDns[N,1], rebuild, allow_update):
 * a refit keeps the tree topology when rebuild == 0, allow_update != 0 and N is unchanged,
 * like the reference's OPTIX_BUILD_OPERATION_UPDATE; otherwise the tree is rebuilt. */
int ptir_build_bvh(ptir_tracer* tracer, const float* pos, const float* rot, const float* scl, const float* dns,
                   int32_t n, int32_t rebuild, int32_t allow_update, void* stream);

/* trace(...) -> 13 outputs */
int ptir_trace(ptir_tracer* tracer, const ptir_trace_args* args, const ptir_trace_outputs* out, void* stream);

/* trace_bwd(...) -> (densityGrad, materialGrad, radianceGrad, shadingNormalGrad, environmentGrad) */
int ptir_trace_bwd(ptir_tracer* tracer, const ptir_trace_args* args, const ptir_bwd_args* bwd,
                   const ptir_bwd_outputs* out, void* stream);

/* One camera view of a batched trace. No counterpart in the reference, whose launches share one
 * extent: a batch traces views of different resolutions and sample counts in one launch
 * sequence, each exactly as its own ptir_trace would (same per-path seeds, same outputs). */
typedef struct ptir_view {
    int32_t z, h, w;             /* launch extent of the view (Z = spp x cameras) */
    uint32_t frame;              /* frameNumber of the view */
    const float* ray_to_world;   /* [>=1,4,4] of the view; only the first matrix applies */
} ptir_view;

#define PTIR_MAX_VIEWS 64

/* trace / trace_bwd over `nviews` (1..PTIR_MAX_VIEWS) views: ray_origin, ray_direction and every
 * per-sample input and output are the views' [Z,H,W,C] arrays concatenated in view order (flat,
 * sum of Z*H*W rows); the args' own z, h, w, frame and ray_to_world are ignored. */
int ptir_trace_views(ptir_tracer* tracer, const ptir_trace_args* args, const ptir_view* views, int32_t nviews,
                     const ptir_trace_outputs* out, void* stream);
int ptir_trace_bwd_views(ptir_tracer* tracer, const ptir_trace_args* args, const ptir_view* views, int32_t nviews,
                         const ptir_bwd_args* bwd, const ptir_bwd_outputs* out, void* stream);

/* Counters of the last launch; synchronises `stream`. */
int ptir_get_counters(ptir_tracer* tracer, ptir_counters* out, void* stream);

/* Counters of one stage (PTIR_STAGE_*) of the last launch; synchronises `stream`. */
int ptir_get_stage_counters(ptir_tracer* tracer, int32_t stage, ptir_counters* out, void* stream);

/* Stage times recorded since the previous call, then cleared; waits for the recorded events. */
int ptir_get_stage_times(ptir_tracer* tracer, ptir_stage_times* out);

/* Turn the launch timing of collect_timings on or off (off while a CUDA graph is captured). */
int ptir_set_collect_timings(ptir_tracer* tracer, int32_t on);

/* Bounded-loop status word of the last launches (0 = clean); synchronises `stream` and clears it. */
int ptir_device_status(ptir_tracer* tracer, uint32_t* status_word, void* stream);

/* Scene AABB of the current structure as 6 floats (lo.xyz, hi.xyz); synchronises `stream`. */
int ptir_scene_bounds(ptir_tracer* tracer, float* out6, void* stream);

/* Copies of the acceleration structure for tests: nodes [max(N-1,1)*16] floats,
 * leaves [N*16] floats (see ptir_b200/csrc/device_types.h for the record layouts); synchronises. */
int ptir_debug_accel(ptir_tracer* tracer, float* nodes_host, float* leaves_host, void* stream);

/* Fused selective Adam step of the training iteration (SelectiveAdam.step,
 * threedgrut/optimizers/__init__.py:89-125 and optimizers.cu:49-76): param, grad, exp_avg and
 * exp_avg_sq are [n_rows, row] float32 device arrays; rows whose visible[r] is 0 are skipped
 * (visible may be null: every row). No bias correction, as in the reference. Asynchronous on
 * `stream`; needs no tracer. */
int ptir_selective_adam(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, const uint8_t* visible,
                        int64_t n_rows, int32_t row, float lr, float beta1, float beta2, float eps, void* stream);

/* Environment importance table (the tracer's environment_alias input) built on the device:
 * build_environment_alias_table (threedgrut/model/aliastable.py:244-297) with its Vose alias
 * construction (aliastable.py:49-116), which the reference runs on the host every few training
 * steps. environment: [env_h, env_w, channels >= 3] float32; an equirect map is area-averaged to
 * table_h x table_w (the reference's 64 x 128), a cube map (env_h == 6 env_w) is used at its
 * own size. table_out: [3, h, w] float32 = probability, alias index (as float), pdf per
 * steradian. scratch: device memory of ptir_env_table_scratch_bytes(h * w) bytes, reused per
 * call. Asynchronous on `stream`; needs no tracer. */
size_t ptir_env_table_scratch_bytes(int32_t cells);
int ptir_build_env_table(const float* environment, int32_t env_h, int32_t env_w, int32_t channels, int32_t table_h,
                         int32_t table_w, float* table_out, void* scratch, size_t scratch_bytes, void* stream);

const char* ptir_last_error(const ptir_tracer* tracer);

/* Allocation-free scene bounds. This entry point has no counterpart in the reference.
 * It is for callers that cannot allocate device memory once running, e.g. a process that
 * reserves all device memory for its own pool at start-up, or a plugin whose host forbids
 * device allocation after initialisation. For them a cudaMalloc fails or stalls the device.
 * It writes the scene AABB of the Gaussians' instance boxes (the bounds every trace clips
 * its rays to, identical to ptir_scene_bounds after ptir_build_bvh of a tracer with the same
 * options) into bounds_out: 8 floats, lo.xyz 0 hi.xyz 0, device memory, 16-byte aligned. Inputs
 * are device pointers as in ptir_build_bvh; kernel_degree / kernel_min_response /
 * density_clamping / storage are the ptir_config fields (with BF16 / FP16 storage the
 * attributes are rounded as ptir_build_bvh rounds them). No handle is needed and nothing is
 * allocated: the only scratch is a fixed 128 KiB device array in the library.
 * Limit: N <= 8,388,608; larger N returns PTIR_EINVAL. N = 0 writes the empty box, lo = +3e38
 * and hi = -3e38 on every axis (ptir_scene_bounds has no structure to read then and returns
 * PTIR_ESTATE). The first call on a device resolves the array's device address, so make that
 * first call before any stream capture; the address is kept, so do not use the library across a
 * cudaDeviceReset. Calls share the array: calls that overlap on the GPU (unordered streams)
 * race. Errors are also described in err[err_len] when err is not NULL. */
int ptir_instance_bounds_noalloc(float kernel_degree, float kernel_min_response, int32_t density_clamping,
                                 int32_t storage, const float* pos, const float* rot, const float* scl,
                                 const float* dns, int32_t n, float* bounds_out, void* stream, char* err,
                                 int32_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* PTIR_B200_H */
