// C ABI of the tracer (include/ptir_b200.h): argument checks, state, launches.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/ptir_b200.h"
#include "accel.h"
#include "device_types.h"
#include "stages.h"
#include "storage.cuh"
#include "wavefront.h"

namespace ptir {
cudaError_t launch_fold(float* out, const float* comp, long long n, cudaStream_t s);  // optim.cu
}

static_assert(PTIR_MAX_VIEWS == ptir::kMaxViews, "view table size of the C ABI");
static_assert(sizeof(ptir::TraceParams) <= 4000, "kernel parameters must stay within 4 KB");
static_assert((int)PTIR_STAGE_INTERSECT == (int)ptir::kStageIntersect &&
                  (int)PTIR_STAGE_SHADOW == (int)ptir::kStageShadow &&
                  (int)PTIR_STAGE_REPLAY == (int)ptir::kStageReplay &&
                  (int)PTIR_STAGE_SHADING == (int)ptir::kStageShading &&
                  (int)PTIR_STAGE_MEGAKERNEL == (int)ptir::kStageMegakernel &&
                  (int)PTIR_STAGE_SORT == (int)ptir::kStageSort && (int)PTIR_NUM_STAGES == (int)ptir::kNumStages,
              "stage numbering of the C ABI");

struct ptir_tracer {
    ptir_config cfg;
    ptir::AccelState accel;
    ptir::WavefrontBuffers wave;
    ptir::StageTimer timer;
    uint4* hot = nullptr;     // 16-bit attribute records (storage != FP32)
    uint4* cold = nullptr;
    size_t attr_capacity = 0;  // Gaussians the record buffers hold
    float* comp = nullptr;     // compensation terms of the gradient sums
    size_t comp_capacity = 0;  // floats
    unsigned* error_word = nullptr;
    unsigned long long* counters = nullptr;  // [kNumStages][kNumCounters]
    unsigned auto_chunk_tiles = 0;           // wavefront chunk chosen at the first trace (chunk_tiles = 0)
    std::string last_error;
};

namespace {

int fail(ptir_tracer* t, int code, const std::string& msg) {
    if (t) t->last_error = msg;
    return code;
}

int cuda_fail(ptir_tracer* t, cudaError_t e, const char* what) {
    return fail(t, PTIR_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

ptir::WavefrontTuning tuning_of(const ptir_config& c) {
    ptir::WavefrontTuning w;
    if (c.chunk_tiles > 0) w.chunk_tiles = (unsigned)c.chunk_tiles;
    if (c.kbuffer > 0) w.kbuf = c.kbuffer;
    if (c.shadow_kbuffer > 0) w.shadow_kbuf = c.shadow_kbuffer;
    if (c.refill_lanes > 0) w.refill_lanes = c.refill_lanes;
    if (c.block_size > 0) w.block = c.block_size;
    w.sort_rays = c.ray_order == 0;
    w.resume_isect = c.resume_rounds == 2;
    w.resume_replay = c.resume_rounds != 1;
    w.exact_candidates = c.exact_candidates != 0;
    return w;
}

// The launch shape of a trace. With chunk_tiles = 0 the chunk is sized once per tracer, at its
// first trace: as many 8x4 tiles as a third of the device memory then free holds (at least
// 32768 tiles), since larger chunks sort more rays together and leave fewer tails (the whole
// 8-view, 100M-path frame in one chunk measured 8 % faster than 131072-tile chunks). It then
// stays fixed, so later calls and CUDA-graph captures use the same buffers.
ptir::WavefrontTuning tuning_for(ptir_tracer* t) {
    ptir::WavefrontTuning w = tuning_of(t->cfg);
    if (t->cfg.chunk_tiles > 0) return w;
    if (t->auto_chunk_tiles == 0) {
        size_t free_b = 0, total_b = 0;
        unsigned tiles = 32768;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const size_t per_tile = 32 * ptir::wavefront_bytes_per_slot();
            const size_t fit = (free_b / 3) / per_tile;
            tiles = (unsigned)std::max<size_t>(32768, std::min<size_t>(fit, (size_t)1 << 26));
        }
        t->auto_chunk_tiles = tiles;
    }
    w.chunk_tiles = t->auto_chunk_tiles;
    return w;
}

constexpr size_t kCounterBytes = sizeof(unsigned long long) * ptir::kNumStages * ptir::kNumCounters;

ptir::StageCtx stage_ctx(ptir_tracer* t) {
    ptir::StageCtx sc;
    sc.counters = t->cfg.collect_counters ? t->counters : nullptr;
    sc.timer = &t->timer;
    return sc;
}

unsigned flags_of(const ptir_config& c) {
    unsigned f = 0;
    if (c.enable_normals) f |= ptir::kNormals;
    if (c.enable_hitcounts) f |= ptir::kHitCounts;
    if (c.enable_mis) f |= ptir::kMis;
    if (c.enable_metallic) f |= ptir::kMetallic;
    if (c.visualize_lights) f |= ptir::kVisualizeLights;
    if (c.exact_replay) f |= ptir::kExactReplay;
    if (c.grad_aggregate == 0) f |= ptir::kWarpAggregate;
    return f;
}

// Element strides of a per-sample array: the caller's when `strided`, else C-contiguous with
// `channels` channels; false for a negative stride. `flat`: the batched [T,C] form, where only the
// sample stride (strides[2]) and the channel stride (strides[3]) apply.
bool sample_layout(bool strided, const int64_t* s, int channels, int h, int w, bool flat, ptir::SampleLayout& L) {
    if (!strided) {
        L.sc = 1;
        L.sx = channels;
        L.sy = flat ? 0 : (long long)channels * w;
        L.sz = flat ? 0 : (long long)channels * w * h;
        return true;
    }
    if (s[0] < 0 || s[1] < 0 || s[2] < 0 || s[3] < 0) return false;
    L.sz = flat ? 0 : s[0];
    L.sy = flat ? 0 : s[1];
    L.sx = s[2];
    L.sc = s[3];
    return true;
}

// checks shared by every trace entry point; fills the kernel parameters and the launch count.
// `views` null: the single launch of the reference (args' extent, frame and ray_to_world).
int prepare(ptir_tracer* t, const ptir_trace_args* a, const ptir_view* views, int nviews, ptir::TraceParams& p,
            long long& launches) {
    if (!a) return fail(t, PTIR_EINVAL, "null trace arguments");
    const bool flat = views != nullptr;
    ptir_view single;
    if (!views) {
        single.z = a->z;
        single.h = a->h;
        single.w = a->w;
        single.frame = a->frame;
        single.ray_to_world = a->ray_to_world;
        views = &single;
        nviews = 1;
    }
    if (nviews < 1 || nviews > PTIR_MAX_VIEWS)
        return fail(t, PTIR_EINVAL, "view count must lie in [1, " + std::to_string(PTIR_MAX_VIEWS) + "]");
    launches = 0;
    long long tiles = 0;
    for (int v = 0; v < nviews; ++v) {
        const ptir_view& V = views[v];
        if (V.z < 0 || V.h < 0 || V.w < 0) return fail(t, PTIR_EINVAL, "negative launch extent");
        const long long n = (long long)V.z * V.h * V.w;
        if (n > 0 && !V.ray_to_world) return fail(t, PTIR_EINVAL, "ray_to_world is required");
        launches += n;
        tiles += (long long)((V.w + 7) / 8) * ((V.h + 3) / 4) * V.z;
        if (launches > (1ll << 31) - 1) return fail(t, PTIR_EINVAL, "launch extent exceeds 2^31 - 1 paths");
    }
    if (launches > 0 && (!a->ray_origin || !a->ray_direction))
        return fail(t, PTIR_EINVAL, "ray_origin and ray_direction are required");
    if (a->max_bounces > 64) return fail(t, PTIR_EINVAL, "max_bounces above 64");
    if (!t->accel.valid) return fail(t, PTIR_ESTATE, "trace called before build_bvh");
    if (a->n != t->accel.n)
        return fail(t, PTIR_ESTATE, "particle count " + std::to_string(a->n) + " differs from the acceleration structure (" +
                                        std::to_string(t->accel.n) + ")");
    if (a->n > 0 && (!a->particle_density || !a->particle_material || !a->particle_radiance))
        return fail(t, PTIR_EINVAL, "particle density, material and radiance are required");
    if (t->cfg.enable_normals && a->n > 0 && !a->particle_shading_normal)
        return fail(t, PTIR_EINVAL, "particle_shading_normal is required when normals are enabled");
    if (a->sph_eval_degree < 0 || a->sph_eval_degree > t->cfg.sph_degree || a->sph_eval_degree > 3)
        return fail(t, PTIR_EINVAL, "sph_eval_degree must lie in [0, min(3, sph_degree)]");
    if (a->num_lights < 0 || a->num_light_entries < 0 || a->num_mesh_lights < 0 || a->num_mesh_light_vertices < 0 ||
        a->num_mesh_light_triangles < 0 || a->mesh_light_alias_cols < 0)
        return fail(t, PTIR_EINVAL, "negative light table size");
    if ((a->num_lights > 0 && !a->lights) || (a->num_light_entries > 0 && !a->light_alias) ||
        (a->num_mesh_lights > 0 && !a->mesh_lights) || (a->num_mesh_light_vertices > 0 && !a->mesh_light_vertices) ||
        (a->num_mesh_light_triangles > 0 && !a->mesh_light_triangles) ||
        (a->mesh_light_alias_cols > 0 && !a->mesh_light_alias))
        return fail(t, PTIR_EINVAL, "a light table with a non-zero size has no data");
    if ((reinterpret_cast<uintptr_t>(a->particle_density) & 15u) != 0)
        return fail(t, PTIR_EINVAL, "particle_density must be 16-byte aligned");
    const bool env = a->environment != nullptr && a->env_h > 0 && a->env_w > 0;
    if (env && (reinterpret_cast<uintptr_t>(a->environment) & 15u) != 0)
        return fail(t, PTIR_EINVAL, "environment must be 16-byte aligned");
    const bool alias = a->environment_alias != nullptr && a->alias_h > 0 && a->alias_w > 0;

    std::memset(&p, 0, sizeof(p));
    p.accel = t->accel.view();
    p.accel.cull_slack = t->cfg.exact_candidates ? ptir::kCullSlack : 0.0f;
    p.part.density = reinterpret_cast<const float4*>(a->particle_density);
    p.part.material = a->particle_material;
    p.part.sph = a->particle_radiance;
    p.part.snrm = a->particle_shading_normal;
    p.part.sph_stride = (t->cfg.sph_degree + 1) * (t->cfg.sph_degree + 1) * 3;
    p.part.sph_degree = a->sph_eval_degree;
    p.env.data = env ? reinterpret_cast<const float4*>(a->environment) : nullptr;
    p.env.w = env ? a->env_w : 0;
    p.env.h = env ? a->env_h : 0;
    p.env.cube = env && a->env_h == 6 * a->env_w;
    if (alias) {
        p.env.aw = a->alias_w;
        p.env.ah = a->alias_h;
        p.env.cells = a->alias_w * a->alias_h;
        p.env.prob = a->environment_alias;
        p.env.alias = a->environment_alias + p.env.cells;
        p.env.pdf = a->environment_alias + 2 * p.env.cells;
    }
    // environment offset, fixed at (0, 0) as in the reference
    p.env.offset_x = 0.0f;
    p.env.offset_y = 0.0f;
    p.lights.lights = a->num_lights > 0 ? a->lights : nullptr;
    p.lights.num_lights = a->num_lights;
    p.lights.table = a->num_light_entries > 0 ? a->light_alias : nullptr;
    p.lights.entries = a->num_light_entries;
    p.lights.vertices = a->num_mesh_light_vertices > 0 ? a->mesh_light_vertices : nullptr;
    p.lights.num_vertices = a->num_mesh_light_vertices;
    p.lights.triangles = a->num_mesh_light_triangles > 0 ? a->mesh_light_triangles : nullptr;
    p.lights.num_triangles = a->num_mesh_light_triangles;
    p.lights.mesh = a->num_mesh_lights > 0 ? a->mesh_lights : nullptr;
    p.lights.num_mesh = a->num_mesh_lights;
    p.lights.tri_table = a->mesh_light_alias_cols > 0 ? a->mesh_light_alias : nullptr;
    p.lights.tri_cols = a->mesh_light_alias_cols;
    p.ray_ori = a->ray_origin;
    p.ray_dir = a->ray_direction;
    p.flat_samples = flat ? 1 : 0;
    const bool rs = a->use_strides != 0;
    if (!sample_layout(rs, a->ray_origin_strides, 3, a->h, a->w, flat, p.ray_ori_layout) ||
        !sample_layout(rs, a->ray_direction_strides, 3, a->h, a->w, flat, p.ray_dir_layout))
        return fail(t, PTIR_EINVAL, "negative ray stride");
    long long offset = 0, tile0 = 0;
    for (int v = 0; v < nviews; ++v) {
        const ptir_view& V = views[v];
        ptir::ViewDesc& D = p.views[v];
        D.offset = offset;
        D.tile0 = tile0;
        D.to_world = V.ray_to_world;
        D.w = V.w;
        D.h = V.h;
        D.z = V.z;
        D.frame = V.frame;
        offset += (long long)V.z * V.h * V.w;
        tile0 += (long long)((V.w + 7) / 8) * ((V.h + 3) / 4) * V.z;
    }
    p.nviews = nviews;
    p.tiles = tiles;
    p.flags = flags_of(t->cfg);
    p.kernel_degree = (int)t->cfg.kernel_degree;
    p.min_response = t->cfg.kernel_min_response;
    p.alpha_min = 1.0f / 255.0f;
    p.min_transmittance = a->min_transmittance;
    p.max_bounces = a->max_bounces;
    p.render_opts = a->sh_indirect ? 1u : 0u;
    p.error_word = t->error_word;
    p.counters = nullptr;  // per stage, set by the launchers (StageCtx)
    return PTIR_OK;
}

// 16-bit storage: round and pack this call's attribute tensors into the tracer's records
int pack_attributes(ptir_tracer* t, const ptir_trace_args* a, ptir::TraceParams& p, cudaStream_t s) {
    if (t->cfg.storage == PTIR_STORAGE_FP32 || a->n <= 0) return PTIR_OK;
    const int cold_stride = ptir::cold_stride_of(p.part.sph_stride);
    if ((size_t)a->n > t->attr_capacity) {
        cudaError_t e = cudaSuccess;
        if (t->hot) e = cudaFreeAsync(t->hot, s);
        if (e == cudaSuccess && t->cold) e = cudaFreeAsync(t->cold, s);
        t->hot = t->cold = nullptr;
        t->attr_capacity = 0;
        if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&t->hot), sizeof(uint4) * 2 * (size_t)a->n, s);
        if (e == cudaSuccess)
            e = cudaMallocAsync(reinterpret_cast<void**>(&t->cold), sizeof(uint4) * cold_stride * (size_t)a->n, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "allocate attribute records");
        t->attr_capacity = (size_t)a->n;
    }
    const cudaError_t e = ptir::launch_pack_attributes(a->n, a->particle_density, a->particle_material,
                                                       a->particle_radiance, p.part.sph_stride,
                                                       a->particle_shading_normal, (unsigned)t->cfg.storage, t->hot,
                                                       t->cold, s);
    if (e != cudaSuccess) return cuda_fail(t, e, "pack attributes");
    p.part.storage = (unsigned)t->cfg.storage;
    p.part.hot = t->hot;
    p.part.cold = t->cold;
    p.part.cold_stride = cold_stride;
    return PTIR_OK;
}

int read_counters(ptir_tracer* t, int first, int last, ptir_counters* out, void* stream) {
    unsigned long long h[ptir::kNumStages * ptir::kNumCounters];
    cudaError_t e = cudaMemcpyAsync(h, t->counters, kCounterBytes, cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(t, e, "read counters");
    unsigned long long v[ptir::kNumCounters] = {};
    for (int st = first; st < last; ++st)
        for (int k = 0; k < ptir::kNumCounters; ++k) v[k] += h[st * ptir::kNumCounters + k];
    out->segments = v[ptir::kCtrSegments];
    out->trace_calls = v[ptir::kCtrTraceCalls];
    out->candidates = v[ptir::kCtrCandidates];
    out->accepted = v[ptir::kCtrAccepted];
    out->env_lookups = v[ptir::kCtrEnvLookups];
    out->replay = v[ptir::kCtrReplay];
    out->replay_accepted = v[ptir::kCtrReplayAccepted];
    out->node_visits = v[ptir::kCtrNodes];
    out->leaf_tests = v[ptir::kCtrLeaves];
    return PTIR_OK;
}

}  // namespace

extern "C" {

int ptir_abi_version(void) { return PTIR_ABI_VERSION; }

int ptir_create(const ptir_config* config, ptir_tracer** out) {
    if (!config || !out) return PTIR_EINVAL;
    *out = nullptr;
    if (config->sph_degree < 0 || config->sph_degree > 3) return PTIR_EINVAL;
    const float deg = config->kernel_degree;
    const int ideg = (int)deg;
    if (!(ideg == 0 || ideg == 1 || ideg == 2 || ideg == 3 || ideg == 4 || ideg == 5 || ideg == 8)) return PTIR_EINVAL;
    if (!(config->kernel_min_response > 0.0f && config->kernel_min_response < 1.0f)) return PTIR_EINVAL;
    if (config->schedule != PTIR_SCHEDULE_WAVEFRONT && config->schedule != PTIR_SCHEDULE_MEGAKERNEL) return PTIR_EINVAL;
    if (config->chunk_tiles < 0) return PTIR_EINVAL;
    if (!(config->kbuffer == 0 || config->kbuffer == 8 || config->kbuffer == 16 || config->kbuffer == 32)) return PTIR_EINVAL;
    if (!(config->shadow_kbuffer == 0 || config->shadow_kbuffer == 8 || config->shadow_kbuffer == 16 ||
          config->shadow_kbuffer == 32))
        return PTIR_EINVAL;
    if (config->refill_lanes < 0 || config->refill_lanes > 32) return PTIR_EINVAL;
    if (!(config->block_size == 0 || config->block_size == 64 || config->block_size == 128 || config->block_size == 256))
        return PTIR_EINVAL;
    if (config->ray_order != 0 && config->ray_order != 1) return PTIR_EINVAL;
    if (config->grad_sums != 0 && config->grad_sums != 1) return PTIR_EINVAL;
    if (config->grad_aggregate != 0 && config->grad_aggregate != 1) return PTIR_EINVAL;
    if (config->exact_candidates != 0 && config->exact_candidates != 1) return PTIR_EINVAL;
    if (config->resume_rounds < 0 || config->resume_rounds > 2) return PTIR_EINVAL;
    if (config->bvh_builder != PTIR_BVH_DEFAULT && config->bvh_builder != PTIR_BVH_MORTON &&
        config->bvh_builder != PTIR_BVH_PLOC)
        return PTIR_EINVAL;
    if (config->storage != PTIR_STORAGE_FP32 && config->storage != PTIR_STORAGE_BF16 &&
        config->storage != PTIR_STORAGE_FP16)
        return PTIR_EINVAL;
    ptir_tracer* t = new ptir_tracer();
    t->cfg = *config;
    t->timer.enabled = config->collect_timings != 0;
    if (cudaMalloc(&t->error_word, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&t->counters, kCounterBytes) != cudaSuccess) {
        cudaFree(t->error_word);
        cudaFree(t->counters);
        delete t;
        return PTIR_ECUDA;
    }
    cudaMemset(t->error_word, 0, sizeof(unsigned));
    cudaMemset(t->counters, 0, kCounterBytes);
    *out = t;
    return PTIR_OK;
}

void ptir_destroy(ptir_tracer* t) {
    if (!t) return;
    cudaDeviceSynchronize();
    ptir::accel_free(t->accel);
    ptir::wavefront_free(t->wave);
    cudaFree(t->error_word);
    cudaFree(t->counters);
    cudaFree(t->hot);
    cudaFree(t->cold);
    cudaFree(t->comp);
    delete t;
}

int ptir_build_bvh(ptir_tracer* t, const float* pos, const float* rot, const float* scl, const float* dns, int32_t n,
                   int32_t rebuild, int32_t allow_update, void* stream) {
    if (!t) return PTIR_EINVAL;
    if (n < 0) return fail(t, PTIR_EINVAL, "negative particle count");
    if (n > 0 && (!pos || !rot || !scl || !dns)) return fail(t, PTIR_EINVAL, "null particle pointer");
    ptir::AccelBuildOptions opt{t->cfg.kernel_degree, t->cfg.kernel_min_response, t->cfg.density_clamping,
                                (unsigned)t->cfg.storage,
                                t->cfg.bvh_builder == PTIR_BVH_MORTON ? ptir::kBuilderMorton : ptir::kBuilderPloc};
    // the reference refits only when asked and allowed and the count is unchanged (optixTracer.cpp:646-649, 819-822)
    const bool do_rebuild = rebuild != 0 || allow_update == 0 || n != t->accel.n;
    std::string err;
    const cudaError_t e = ptir::accel_build(t->accel, opt, pos, rot, scl, dns, n, do_rebuild, as_stream(stream), err);
    if (e != cudaSuccess) return fail(t, PTIR_ECUDA, "build_bvh: " + err);
    return PTIR_OK;
}

}  // extern "C"

namespace {

int trace_impl(ptir_tracer* t, const ptir_trace_args* a, const ptir_view* views, int nviews,
               const ptir_trace_outputs* o, void* stream) {
    if (!t) return PTIR_EINVAL;
    ptir::TraceParams p;
    long long launches = 0;
    const int rc = prepare(t, a, views, nviews, p, launches);
    if (rc != PTIR_OK) return rc;
    if (!o) return fail(t, PTIR_EINVAL, "null outputs");
    if (launches > 0 && (!o->radiance || !o->density || !o->hit_distance || !o->hit_distance_second_moment ||
                         !o->depth_distortion || !o->normal || !o->shading_normal || !o->material || !o->hits_count ||
                         !o->pbr || !o->light || !o->pbr_components))
        return fail(t, PTIR_EINVAL, "every per-sample output buffer is required");
    cudaStream_t s = as_stream(stream);
    if (pack_attributes(t, a, p, s) != PTIR_OK) return PTIR_ECUDA;
    cudaError_t e;
    if (o->visibility && a->n > 0) {
        e = cudaMemsetAsync(o->visibility, 0, sizeof(float) * (size_t)a->n, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "clear visibility");
    }
    if (t->cfg.collect_counters) {
        e = cudaMemsetAsync(t->counters, 0, kCounterBytes, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "clear counters");
    }
    ptir::FwdOutputs fo;
    fo.radiance = o->radiance;
    fo.density = o->density;
    fo.hit = o->hit_distance;
    fo.hit2 = o->hit_distance_second_moment;
    fo.distortion = o->depth_distortion;
    fo.normal = o->normal;
    fo.snormal = o->shading_normal;
    fo.material = o->material;
    fo.hits_count = o->hits_count;
    fo.pbr = o->pbr;
    fo.light = o->light;
    fo.components = o->pbr_components;
    fo.visibility = o->visibility;
    fo.path_sig = o->path_signature;
    if (o->path_signature) p.flags |= ptir::kPathSig;
    const ptir::StageCtx sc = stage_ctx(t);
    e = t->cfg.schedule == PTIR_SCHEDULE_MEGAKERNEL
            ? ptir::launch_trace_fwd(p, fo, sc, s)
            : ptir::launch_trace_fwd_wavefront(p, fo, t->wave, tuning_for(t), sc, s);
    if (e != cudaSuccess) return cuda_fail(t, e, "trace launch");
    return PTIR_OK;
}

int trace_bwd_impl(ptir_tracer* t, const ptir_trace_args* a, const ptir_view* views, int nviews,
                   const ptir_bwd_args* b, const ptir_bwd_outputs* o, void* stream) {
    if (!t) return PTIR_EINVAL;
    ptir::TraceParams p;
    long long launches = 0;
    const int rc = prepare(t, a, views, nviews, p, launches);
    if (rc != PTIR_OK) return rc;
    if (!b || !o) return fail(t, PTIR_EINVAL, "null backward arguments");
    if (launches > 0 && (!b->pbr || !b->light)) return fail(t, PTIR_EINVAL, "forward pbr and light are required");
    if (a->n > 0 && !o->particle_material_grad) return fail(t, PTIR_EINVAL, "particle_material_grad is required");
    cudaStream_t s = as_stream(stream);
    if (pack_attributes(t, a, p, s) != PTIR_OK) return PTIR_ECUDA;
    cudaError_t e;
    if (a->n > 0) {
        e = cudaMemsetAsync(o->particle_material_grad, 0, sizeof(float) * 5 * (size_t)a->n, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "clear material grad");
    }
    const bool env = p.env.data != nullptr;
    if (env && o->environment_grad) {
        e = cudaMemsetAsync(o->environment_grad, 0, sizeof(float) * 4 * (size_t)p.env.w * p.env.h, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "clear environment grad");
    }
    if (t->cfg.collect_counters) {
        e = cudaMemsetAsync(t->counters, 0, kCounterBytes, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "clear counters");
    }
    ptir::BwdInputs bi{};
    bi.pbr = b->pbr;
    bi.light = b->light;
    bi.pbr_grad = b->pbr_grad;
    bi.light_grad = b->light_grad;
    bi.material_grad = b->material_grad;
    const bool flat = views != nullptr;
    const bool bs = b->use_strides != 0;
    if (!sample_layout(bs, b->pbr_strides, 3, a->h, a->w, flat, bi.pbr_layout) ||
        !sample_layout(bs, b->light_strides, 3, a->h, a->w, flat, bi.light_layout) ||
        !sample_layout(bs, b->pbr_grad_strides, 3, a->h, a->w, flat, bi.pbr_grad_layout) ||
        !sample_layout(bs, b->light_grad_strides, 3, a->h, a->w, flat, bi.light_grad_layout) ||
        !sample_layout(bs, b->material_grad_strides, 5, a->h, a->w, flat, bi.material_grad_layout))
        return fail(t, PTIR_EINVAL, "negative stride of a backward input");
    bi.particle_material_grad = o->particle_material_grad;
    bi.environment_grad = env ? o->environment_grad : nullptr;
    // compensation buffers of the Kahan-pair gradient sums: [n,5] then [eh,ew,4], zeroed per call
    const size_t n_mat = a->n > 0 ? 5 * (size_t)a->n : 0;
    const size_t n_env = bi.environment_grad ? 4 * (size_t)p.env.w * p.env.h : 0;
    const bool comp = t->cfg.grad_sums == 0 && n_mat + n_env > 0;
    if (comp) {
        if (n_mat + n_env > t->comp_capacity) {
            if (t->comp) e = cudaFreeAsync(t->comp, s);
            t->comp = nullptr;
            t->comp_capacity = 0;
            e = cudaMallocAsync(reinterpret_cast<void**>(&t->comp), sizeof(float) * (n_mat + n_env), s);
            if (e != cudaSuccess) return cuda_fail(t, e, "allocate gradient compensation");
            t->comp_capacity = n_mat + n_env;
        }
        e = cudaMemsetAsync(t->comp, 0, sizeof(float) * (n_mat + n_env), s);
        if (e != cudaSuccess) return cuda_fail(t, e, "clear gradient compensation");
        bi.particle_material_comp = n_mat ? t->comp : nullptr;
        bi.environment_comp = n_env ? t->comp + n_mat : nullptr;
    }
    const ptir::StageCtx sc = stage_ctx(t);
    e = t->cfg.schedule == PTIR_SCHEDULE_MEGAKERNEL
            ? ptir::launch_trace_bwd(p, bi, sc, s)
            : ptir::launch_trace_bwd_wavefront(p, bi, t->wave, tuning_for(t), sc, s);
    if (e != cudaSuccess) return cuda_fail(t, e, "trace_bwd launch");
    if (comp) {
        if (n_mat) e = ptir::launch_fold(bi.particle_material_grad, bi.particle_material_comp, (long long)n_mat, s);
        if (e == cudaSuccess && n_env) e = ptir::launch_fold(bi.environment_grad, bi.environment_comp, (long long)n_env, s);
        if (e != cudaSuccess) return cuda_fail(t, e, "fold gradient compensation");
    }
    return PTIR_OK;
}

}  // namespace

extern "C" {

int ptir_trace(ptir_tracer* t, const ptir_trace_args* a, const ptir_trace_outputs* o, void* stream) {
    return trace_impl(t, a, nullptr, 0, o, stream);
}

int ptir_trace_bwd(ptir_tracer* t, const ptir_trace_args* a, const ptir_bwd_args* b, const ptir_bwd_outputs* o,
                   void* stream) {
    return trace_bwd_impl(t, a, nullptr, 0, b, o, stream);
}

int ptir_trace_views(ptir_tracer* t, const ptir_trace_args* a, const ptir_view* views, int32_t nviews,
                     const ptir_trace_outputs* o, void* stream) {
    if (!views) return fail(t, PTIR_EINVAL, "null view table");
    return trace_impl(t, a, views, nviews, o, stream);
}

int ptir_trace_bwd_views(ptir_tracer* t, const ptir_trace_args* a, const ptir_view* views, int32_t nviews,
                         const ptir_bwd_args* b, const ptir_bwd_outputs* o, void* stream) {
    if (!views) return fail(t, PTIR_EINVAL, "null view table");
    return trace_bwd_impl(t, a, views, nviews, b, o, stream);
}

int ptir_get_counters(ptir_tracer* t, ptir_counters* out, void* stream) {
    if (!t || !out) return PTIR_EINVAL;
    return read_counters(t, 0, ptir::kNumStages, out, stream);
}

int ptir_get_stage_counters(ptir_tracer* t, int32_t stage, ptir_counters* out, void* stream) {
    if (!t || !out || stage < 0 || stage >= ptir::kNumStages) return PTIR_EINVAL;
    return read_counters(t, stage, stage + 1, out, stream);
}

int ptir_set_collect_timings(ptir_tracer* t, int32_t on) {
    if (!t) return PTIR_EINVAL;
    t->timer.enabled = on != 0;
    return PTIR_OK;
}

int ptir_get_stage_times(ptir_tracer* t, ptir_stage_times* out) {
    if (!t || !out) return PTIR_EINVAL;
    double ms[ptir::kNumStages] = {};
    unsigned long long n[ptir::kNumStages] = {};
    const cudaError_t e = t->timer.collect(ms, n);
    if (e != cudaSuccess) return cuda_fail(t, e, "read stage times");
    for (int k = 0; k < ptir::kNumStages; ++k) {
        out->ms[k] = ms[k];
        out->launches[k] = n[k];
    }
    return PTIR_OK;
}

int ptir_device_status(ptir_tracer* t, uint32_t* status_word, void* stream) {
    if (!t || !status_word) return PTIR_EINVAL;
    unsigned h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, t->error_word, sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess) e = cudaMemsetAsync(t->error_word, 0, sizeof(unsigned), as_stream(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(t, e, "read device status");
    *status_word = h;
    return h ? fail(t, PTIR_EDEVICE, "a kernel exceeded a loop bound (status " + std::to_string(h) + ")") : PTIR_OK;
}

int ptir_scene_bounds(ptir_tracer* t, float* out6, void* stream) {
    if (!t || !out6) return PTIR_EINVAL;
    if (!t->accel.valid || t->accel.n == 0) return fail(t, PTIR_ESTATE, "no acceleration structure");
    float4 h[2];
    cudaError_t e = cudaMemcpyAsync(h, t->accel.bounds, sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(t, e, "read bounds");
    out6[0] = h[0].x; out6[1] = h[0].y; out6[2] = h[0].z;
    out6[3] = h[1].x; out6[4] = h[1].y; out6[5] = h[1].z;
    return PTIR_OK;
}

int ptir_debug_accel(ptir_tracer* t, float* nodes_host, float* leaves_host, void* stream) {
    if (!t) return PTIR_EINVAL;
    if (!t->accel.valid) return fail(t, PTIR_ESTATE, "no acceleration structure");
    const int n = t->accel.n;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaSuccess;
    if (nodes_host && n > 1)
        e = cudaMemcpyAsync(nodes_host, t->accel.nodes, sizeof(float4) * 4 * (size_t)(n - 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && leaves_host && n > 0)
        e = cudaMemcpyAsync(leaves_host, t->accel.leaves, sizeof(float4) * 4 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(t, e, "copy acceleration structure");
    return PTIR_OK;
}

const char* ptir_last_error(const ptir_tracer* t) { return t ? t->last_error.c_str() : "null tracer"; }

}  // extern "C"
