// Wavefront path tracer and adjoint: each path stage is its own kernel over a compacted queue.
//
// Paths are processed in chunks of whole 8x4 pixel tiles (slot q of a chunk = lane q % 32 of
// tile q / 32, so the primary rays of a warp stay coherent). Per chunk, the forward runs
//   primary  : primary segment, primary outputs, NEE light sample     -> shadow queue | bounce queue
//   shadow   : stochastic shadow ray of the NEE sample                -> bounce queue
//   bounce d : light gathering, path termination, BRDF sample          -> intersect queue
//   intersect: next segment                                            -> bounce queue
// and the backward the same with the adjoint stages, whose re-traversals (the reference's
// rayIntersectBwd) go to a replay queue drained after every bounce stage. Path state lives in
// HBM between stages; queues are appended with one atomic per warp (ballot + popc). The per-path
// order of random draws is the megakernel's, so both schedules produce the same paths.
#include <algorithm>

#include "path.cuh"
#include "wavefront.h"

namespace ptir {

namespace {

constexpr int kThreads = 128;

struct WfView {
    Segment* seg;
    PathState* ps;
    unsigned long long* rng;
    unsigned* q[3];          // bounce, intersect, shadow
    unsigned* count;         // [kNumQueueCounts]
    unsigned* cursor;        // [kNumCursors]
    ReplayJob* jobs;
    unsigned tile0;          // first tile of the chunk
    unsigned slots;          // paths in the chunk (32 per tile)
};

enum : int { kQBounce = 0, kQIsect = 1, kQShadow = 2, kQJobs = 3 };

PTIR_DEV unsigned lane() { return threadIdx.x & 31u; }

// the next 32 items of a queue for this warp (uniform across the warp)
PTIR_DEV unsigned fetch32(unsigned* cursor) {
    unsigned base = 0;
    if (lane() == 0) base = atomicAdd(cursor, 32u);
    return __shfl_sync(0xFFFFFFFFu, base, 0);
}

// append `value` for the lanes with `pred` (called by the whole warp)
PTIR_DEV void push(unsigned* items, unsigned* count, unsigned value, bool pred) {
    const unsigned mask = __ballot_sync(0xFFFFFFFFu, pred);
    if (!mask) return;
    const unsigned leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane() == leader) base = atomicAdd(count, __popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (pred) items[base + __popc(mask & ((1u << lane()) - 1u))] = value;
}

PTIR_DEV void push_job(ReplayJob* jobs, unsigned* count, const ReplayJob& j, bool pred) {
    const unsigned mask = __ballot_sync(0xFFFFFFFFu, pred);
    if (!mask) return;
    const unsigned leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane() == leader) base = atomicAdd(count, __popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (pred) jobs[base + __popc(mask & ((1u << lane()) - 1u))] = j;
}

// slot q of the chunk -> launch index (x, y, z); false for slots outside the image
PTIR_DEV bool slot_index(const TraceParams& P, const WfView& W, unsigned q, unsigned& x, unsigned& y, unsigned& z) {
    const unsigned tile = W.tile0 + (q >> 5), ln = q & 31u;
    const unsigned tiles_x = (unsigned)(P.w + 7) >> 3, tiles_y = (unsigned)(P.h + 3) >> 2;
    const unsigned per_z = tiles_x * tiles_y;
    z = tile / per_z;
    const unsigned t = tile - z * per_z;
    const unsigned ty = t / tiles_x, tx = t - ty * tiles_x;
    x = (tx << 3) + (ln & 7u);
    y = (ty << 2) + (ln >> 3);
    return z < (unsigned)P.nz && x < (unsigned)P.w && y < (unsigned)P.h;
}

PTIR_DEV size_t launch_of(const TraceParams& P, unsigned x, unsigned y, unsigned z) {
    return ((size_t)z * P.h + y) * P.w + x;
}

PTIR_DEV void store_rng(const WfView& W, unsigned q, const Pcg32& r) { W.rng[q] = r.state; }
PTIR_DEV Pcg32 load_rng(const WfView& W, unsigned q) {
    Pcg32 r;
    r.state = W.rng[q];
    r.inc = 1ull;
    return r;
}

PTIR_DEV void write_pbr(const FwdOutputs& O, size_t li, const PathState& ps) {
    float* pb = O.pbr + 3 * li;
    pb[0] = ps.acc.x; pb[1] = ps.acc.y; pb[2] = ps.acc.z;
    float* lg = O.light + 3 * li;
    lg[0] = ps.acc_light.x; lg[1] = ps.acc_light.y; lg[2] = ps.acc_light.z;
    float* cp = O.components + 6 * li;
    cp[0] = ps.acc_direct.x; cp[1] = ps.acc_direct.y; cp[2] = ps.acc_direct.z;
    cp[3] = ps.acc_indirect.x; cp[4] = ps.acc_indirect.y; cp[5] = ps.acc_indirect.z;
}

#define PTIR_STAGE_PROLOGUE                         \
    int stack[kStackDepth];                         \
    float stack_t[kStackDepth];                     \
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0}; \
    CtxT<K> C{P, stack, stack_t, ctr};

// ---------------------------------------------------------------------------------------
// forward
template <int K>
__global__ void __launch_bounds__(kThreads) k_wf_fwd_primary(TraceParams P, FwdOutputs O, WfView W) {
    PTIR_STAGE_PROLOGUE
    const bool mis = (P.flags & kMis) != 0;
    while (true) {
        const unsigned base = fetch32(W.cursor + 0);
        if (base >= W.slots) break;
        const unsigned q = base + lane();
        unsigned x = 0, y = 0, z = 0;
        const bool valid = q < W.slots && slot_index(P, W, q, x, y, z);
        bool cont = false, shadow = false;
        if (valid) {
            const size_t li = launch_of(P, x, y, z);
            Pcg32 rng;
            rng.seed(x, y, z, P.frame);
            PathState ps;
            path_init(ps, effective_bounces(P));
            Segment s;
            float3 o, d;
            world_ray(P, li, o, d);
            segment_reset(s, o, d, 0.0f);
            ++ctr.segments;
            intersect_mark<false>(C, s, rng, O.visibility);
            float* r = O.radiance + 3 * li;
            r[0] = s.radiance.x; r[1] = s.radiance.y; r[2] = s.radiance.z;
            O.density[li] = 1.0f - s.transmittance;
            O.hit[2 * li] = s.depth;
            O.hit[2 * li + 1] = s.last_hit;
            O.hit2[li] = s.hit2;
            O.distortion[li] = s.distortion;
            const bool nrm = (P.flags & kNormals) != 0;
            float* n = O.normal + 3 * li;
            n[0] = nrm ? s.normal.x : 0.0f; n[1] = nrm ? s.normal.y : 0.0f; n[2] = nrm ? s.normal.z : 0.0f;
            float* sn = O.snormal + 3 * li;
            sn[0] = nrm ? s.snrm.x : 0.0f; sn[1] = nrm ? s.snrm.y : 0.0f; sn[2] = nrm ? s.snrm.z : 0.0f;
            float* m = O.material + 5 * li;
            m[0] = s.albedo.x; m[1] = s.albedo.y; m[2] = s.albedo.z; m[3] = s.rough; m[4] = s.metal;
            O.hits_count[li] = (P.flags & kHitCounts) ? s.hits_count : 0.0f;
            write_pbr(O, li, ps);  // zeros; rewritten when the path ends
            cont = (P.flags & kVisualizeLights) || s.ivalid;
            if (cont) {
                if (mis) shadow = nee_prepare(C, ps, s, rng);
                W.seg[q] = s;
                W.ps[q] = ps;
                store_rng(W, q, rng);
            }
        }
        push(W.q[kQShadow], W.count + kQShadow, q, cont && shadow);
        push(W.q[kQBounce], W.count + kQBounce, q, cont && !shadow);
    }
    flush_counters(P, ctr);
}

template <int K>
__global__ void __launch_bounds__(kThreads) k_wf_shadow(TraceParams P, WfView W) {
    PTIR_STAGE_PROLOGUE
    const unsigned count = W.count[kQShadow];
    while (true) {
        const unsigned base = fetch32(W.cursor + 1);
        if (base >= count) break;
        const unsigned i = base + lane();
        const bool valid = i < count;
        const unsigned q = valid ? W.q[kQShadow][i] : 0u;
        if (valid) {
            const Segment& s = W.seg[q];
            PathState ps = W.ps[q];
            Pcg32 rng = load_rng(W, q);
            nee_shadow(C, ps, s, rng);
            W.ps[q].em = ps.em;
            store_rng(W, q, rng);
        }
        push(W.q[kQBounce], W.count + kQBounce, q, valid);
    }
    flush_counters(P, ctr);
}

template <int K>
__global__ void __launch_bounds__(kThreads) k_wf_fwd_bounce(TraceParams P, FwdOutputs O, WfView W, unsigned depth,
                                                            unsigned cursor) {
    PTIR_STAGE_PROLOGUE
    const unsigned count = W.count[kQBounce];
    while (true) {
        const unsigned base = fetch32(W.cursor + cursor);
        if (base >= count) break;
        const unsigned i = base + lane();
        const bool valid = i < count;
        const unsigned q = valid ? W.q[kQBounce][i] : 0u;
        bool cont = false;
        if (valid) {
            Segment s = W.seg[q];
            PathState ps = W.ps[q];
            Pcg32 rng = load_rng(W, q);
            accumulate_light(C, ps, s);
            ps.active &= (unsigned)((depth + 1u < ps.max_bounces) && s.ivalid);
            if (ps.active) {
                ps.bounces = depth + 1u;
                sample_next(C, ps, s, rng);
                cont = ps.active && !(max3(ps.throughput) < 1e-4f);
            }
            if (cont) {
                W.seg[q] = s;
                W.ps[q] = ps;
                store_rng(W, q, rng);
            } else {
                unsigned x, y, z;
                slot_index(P, W, q, x, y, z);
                write_pbr(O, launch_of(P, x, y, z), ps);
            }
        }
        push(W.q[kQIsect], W.count + kQIsect, q, cont);
    }
    flush_counters(P, ctr);
}

template <int K, bool kMark>
__global__ void __launch_bounds__(kThreads) k_wf_isect(TraceParams P, float* vis, WfView W, unsigned cursor) {
    PTIR_STAGE_PROLOGUE
    const unsigned count = W.count[kQIsect];
    while (true) {
        const unsigned base = fetch32(W.cursor + cursor);
        if (base >= count) break;
        const unsigned i = base + lane();
        const bool valid = i < count;
        const unsigned q = valid ? W.q[kQIsect][i] : 0u;
        if (valid) {
            Segment s = W.seg[q];
            Pcg32 rng = load_rng(W, q);
            ++ctr.segments;
            intersect_mark<true>(C, s, rng, kMark ? vis : nullptr);
            W.seg[q] = s;
            store_rng(W, q, rng);
        }
        push(W.q[kQBounce], W.count + kQBounce, q, valid);
    }
    flush_counters(P, ctr);
}

// ---------------------------------------------------------------------------------------
// backward
template <int K>
__global__ void __launch_bounds__(kThreads) k_wb_primary(TraceParams P, BwdInputs B, WfView W) {
    PTIR_STAGE_PROLOGUE
    const bool mis = (P.flags & kMis) != 0;
    while (true) {
        const unsigned base = fetch32(W.cursor + 0);
        if (base >= W.slots) break;
        const unsigned q = base + lane();
        unsigned x = 0, y = 0, z = 0;
        const bool valid = q < W.slots && slot_index(P, W, q, x, y, z);
        bool cont = false, shadow = false;
        if (valid) {
            const size_t li = launch_of(P, x, y, z);
            Pcg32 rng;
            rng.seed(x, y, z, P.frame);
            PathState ps;
            path_init(ps, effective_bounces(P));
            ps.acc = ld3(B.pbr + 3 * li);
            ps.acc_grad = B.pbr_grad ? ld3(B.pbr_grad + 3 * li) : f3(0.0f);
            ps.acc_light = ld3(B.light + 3 * li);
            ps.acc_light_grad = B.light_grad ? ld3(B.light_grad + 3 * li) : f3(0.0f);
            Segment s;
            float3 o, d;
            world_ray(P, li, o, d);
            segment_reset(s, o, d, 0.0f);
            ++ctr.segments;
            intersect_mark<false>(C, s, rng, nullptr);
            if (s.ivalid && B.material_grad) {
                const float* mg = B.material_grad + 5 * li;
                s.d_albedo += ld3(mg);
                s.d_rough += __ldg(mg + 3);
                if (P.flags & kMetallic) s.d_metal += __ldg(mg + 4);
            }
            cont = (P.flags & kVisualizeLights) || s.ivalid;
            if (cont) {
                if (mis) shadow = nee_prepare(C, ps, s, rng);
                W.seg[q] = s;
                W.ps[q] = ps;
                store_rng(W, q, rng);
            }
        }
        push(W.q[kQShadow], W.count + kQShadow, q, cont && shadow);
        push(W.q[kQBounce], W.count + kQBounce, q, cont && !shadow);
    }
    flush_counters(P, ctr);
}

template <int K>
__global__ void __launch_bounds__(kThreads) k_wb_bounce(TraceParams P, BwdInputs B, WfView W, unsigned depth,
                                                        unsigned cursor) {
    PTIR_STAGE_PROLOGUE
    const unsigned count = W.count[kQBounce];
    while (true) {
        const unsigned base = fetch32(W.cursor + cursor);
        if (base >= count) break;
        const unsigned i = base + lane();
        const bool valid = i < count;
        const unsigned q = valid ? W.q[kQBounce][i] : 0u;
        bool cont = false;
        ReplayJob job[2];
        bool has[2] = {false, false};
        if (valid) {
            Segment s = W.seg[q];
            PathState ps = W.ps[q];
            Pcg32 rng = load_rng(W, q);
            accumulate_light_bwd(C, B, ps, s);
            pending_bwd(ps, s, [&](const ReplayJob& j) {
                job[0] = j;
                has[0] = true;
            });
            ps.active &= (unsigned)((depth + 1u < ps.max_bounces) && s.ivalid);
            if (ps.active) {
                ps.bounces = depth + 1u;
                sample_next_bwd(C, ps, s, rng, [&](const ReplayJob& j) {
                    job[1] = j;
                    has[1] = true;
                });
                cont = ps.active && !(max3(ps.throughput) < 1e-4f);
            }
            if (cont) {
                W.seg[q] = s;
                W.ps[q] = ps;
                store_rng(W, q, rng);
            }
        }
        push_job(W.jobs, W.count + kQJobs, job[0], has[0]);
        push_job(W.jobs, W.count + kQJobs, job[1], has[1]);
        push(W.q[kQIsect], W.count + kQIsect, q, cont);
    }
    flush_counters(P, ctr);
}

template <int K>
__global__ void __launch_bounds__(kThreads) k_wb_replay(TraceParams P, BwdInputs B, WfView W, unsigned cursor) {
    PTIR_STAGE_PROLOGUE
    const unsigned count = W.count[kQJobs];
    while (true) {
        const unsigned base = fetch32(W.cursor + cursor);
        if (base >= count) break;
        const unsigned i = base + lane();
        if (i < count) {
            const ReplayJob j = W.jobs[i];
            replay_material_grad(C, B, j);
        }
    }
    flush_counters(P, ctr);
}

int grid_for(const void* fn) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 4;
    return sms * per_sm;
}

}  // namespace

// ---------------------------------------------------------------------------------------
cudaError_t wavefront_reserve(WavefrontBuffers& b, size_t slots, cudaStream_t s) {
    if (slots <= b.slots && b.seg) return cudaSuccess;
    auto rel = [&](void* p) {
        if (p) cudaFreeAsync(p, s);
    };
    rel(b.seg); rel(b.ps); rel(b.rng); rel(b.q[0]); rel(b.q[1]); rel(b.q[2]); rel(b.jobs);
    void* counters = b.counters;
    b = WavefrontBuffers{};
    b.counters = counters;
    cudaError_t e = cudaSuccess;
    auto get = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMallocAsync(p, bytes, s);
    };
    get(&b.seg, sizeof(Segment) * slots);
    get(&b.ps, sizeof(PathState) * slots);
    get(&b.rng, sizeof(unsigned long long) * slots);
    for (int k = 0; k < 3; ++k) get(&b.q[k], sizeof(unsigned) * slots);
    get(&b.jobs, sizeof(ReplayJob) * 2 * slots);
    if (!b.counters) get(&b.counters, sizeof(unsigned) * (kNumQueueCounts + kNumCursors));
    if (e == cudaSuccess) b.slots = slots;
    return e;
}

void wavefront_free(WavefrontBuffers& b) {
    for (void* p : {b.seg, b.ps, b.rng, b.q[0], b.q[1], b.q[2], b.jobs, b.counters})
        if (p) cudaFree(p);
    b = WavefrontBuffers{};
}

static WfView view_of(const WavefrontBuffers& b, unsigned tile0, unsigned slots) {
    WfView W;
    W.seg = static_cast<Segment*>(b.seg);
    W.ps = static_cast<PathState*>(b.ps);
    W.rng = static_cast<unsigned long long*>(b.rng);
    for (int k = 0; k < 3; ++k) W.q[k] = static_cast<unsigned*>(b.q[k]);
    W.count = static_cast<unsigned*>(b.counters);
    W.cursor = W.count + kNumQueueCounts;
    W.jobs = static_cast<ReplayJob*>(b.jobs);
    W.tile0 = tile0;
    W.slots = slots;
    return W;
}

static unsigned long long total_tiles(const TraceParams& p) {
    return (unsigned long long)((p.w + 7) / 8) * ((p.h + 3) / 4) * (unsigned long long)p.nz;
}

template <int K>
static cudaError_t run_fwd(const TraceParams& p, const FwdOutputs& o, WavefrontBuffers& b, unsigned chunk_tiles,
                           cudaStream_t s) {
    const unsigned long long tiles = total_tiles(p);
    if (tiles == 0) return cudaSuccess;
    chunk_tiles = (unsigned)std::min<unsigned long long>(chunk_tiles, tiles);
    cudaError_t e = wavefront_reserve(b, (size_t)chunk_tiles * 32, s);
    if (e != cudaSuccess) return e;
    static int g_primary = 0, g_shadow = 0, g_bounce = 0, g_isect = 0;
    if (!g_primary) {
        g_primary = grid_for((const void*)k_wf_fwd_primary<K>);
        g_shadow = grid_for((const void*)k_wf_shadow<K>);
        g_bounce = grid_for((const void*)k_wf_fwd_bounce<K>);
        g_isect = grid_for((const void*)k_wf_isect<K, true>);
    }
    const unsigned mb = p.render_opts ? std::min(p.max_bounces, 2u) : p.max_bounces;
    if (2u + 3u * mb > (unsigned)kNumCursors) return cudaErrorInvalidValue;
    for (unsigned long long t0 = 0; t0 < tiles; t0 += chunk_tiles) {
        const unsigned nt = (unsigned)std::min<unsigned long long>(chunk_tiles, tiles - t0);
        const WfView W = view_of(b, (unsigned)t0, nt * 32u);
        e = cudaMemsetAsync(b.counters, 0, sizeof(unsigned) * (kNumQueueCounts + kNumCursors), s);
        if (e != cudaSuccess) return e;
        const int gp = std::min<long long>(g_primary, ((long long)nt * 32 + kThreads - 1) / kThreads);
        k_wf_fwd_primary<K><<<gp, kThreads, 0, s>>>(p, o, W);
        if (p.flags & kMis) k_wf_shadow<K><<<g_shadow, kThreads, 0, s>>>(p, W);
        unsigned cursor = 2;
        for (unsigned depth = 0; depth < mb; ++depth) {
            cudaMemsetAsync(W.count + kQIsect, 0, sizeof(unsigned), s);
            k_wf_fwd_bounce<K><<<g_bounce, kThreads, 0, s>>>(p, o, W, depth, cursor++);
            if (depth + 1 >= mb) break;
            cudaMemsetAsync(W.count + kQBounce, 0, sizeof(unsigned), s);
            k_wf_isect<K, true><<<g_isect, kThreads, 0, s>>>(p, o.visibility, W, cursor++);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int K>
static cudaError_t run_bwd(const TraceParams& p, const BwdInputs& bi, WavefrontBuffers& b, unsigned chunk_tiles,
                           cudaStream_t s) {
    const unsigned long long tiles = total_tiles(p);
    if (tiles == 0) return cudaSuccess;
    chunk_tiles = (unsigned)std::min<unsigned long long>(chunk_tiles, tiles);
    cudaError_t e = wavefront_reserve(b, (size_t)chunk_tiles * 32, s);
    if (e != cudaSuccess) return e;
    static int g_primary = 0, g_shadow = 0, g_bounce = 0, g_isect = 0, g_replay = 0;
    if (!g_primary) {
        g_primary = grid_for((const void*)k_wb_primary<K>);
        g_shadow = grid_for((const void*)k_wf_shadow<K>);
        g_bounce = grid_for((const void*)k_wb_bounce<K>);
        g_isect = grid_for((const void*)k_wf_isect<K, false>);
        g_replay = grid_for((const void*)k_wb_replay<K>);
    }
    const unsigned mb = p.render_opts ? std::min(p.max_bounces, 2u) : p.max_bounces;
    if (2u + 3u * mb > (unsigned)kNumCursors) return cudaErrorInvalidValue;
    for (unsigned long long t0 = 0; t0 < tiles; t0 += chunk_tiles) {
        const unsigned nt = (unsigned)std::min<unsigned long long>(chunk_tiles, tiles - t0);
        const WfView W = view_of(b, (unsigned)t0, nt * 32u);
        e = cudaMemsetAsync(b.counters, 0, sizeof(unsigned) * (kNumQueueCounts + kNumCursors), s);
        if (e != cudaSuccess) return e;
        const int gp = std::min<long long>(g_primary, ((long long)nt * 32 + kThreads - 1) / kThreads);
        k_wb_primary<K><<<gp, kThreads, 0, s>>>(p, bi, W);
        if (p.flags & kMis) k_wf_shadow<K><<<g_shadow, kThreads, 0, s>>>(p, W);
        unsigned cursor = 2;
        for (unsigned depth = 0; depth < mb; ++depth) {
            cudaMemsetAsync(W.count + kQIsect, 0, sizeof(unsigned), s);
            cudaMemsetAsync(W.count + kQJobs, 0, sizeof(unsigned), s);
            k_wb_bounce<K><<<g_bounce, kThreads, 0, s>>>(p, bi, W, depth, cursor++);
            k_wb_replay<K><<<g_replay, kThreads, 0, s>>>(p, bi, W, cursor++);
            if (depth + 1 >= mb) break;
            cudaMemsetAsync(W.count + kQBounce, 0, sizeof(unsigned), s);
            k_wf_isect<K, false><<<g_isect, kThreads, 0, s>>>(p, nullptr, W, cursor++);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_trace_fwd_wavefront(const TraceParams& p, const FwdOutputs& o, WavefrontBuffers& b,
                                       unsigned chunk_tiles, int kbuf, cudaStream_t s) {
    switch (kbuf) {
    case 8: return run_fwd<8>(p, o, b, chunk_tiles, s);
    case 32: return run_fwd<32>(p, o, b, chunk_tiles, s);
    default: return run_fwd<16>(p, o, b, chunk_tiles, s);
    }
}

cudaError_t launch_trace_bwd_wavefront(const TraceParams& p, const BwdInputs& bi, WavefrontBuffers& b,
                                       unsigned chunk_tiles, int kbuf, cudaStream_t s) {
    switch (kbuf) {
    case 8: return run_bwd<8>(p, bi, b, chunk_tiles, s);
    case 32: return run_bwd<32>(p, bi, b, chunk_tiles, s);
    default: return run_bwd<16>(p, bi, b, chunk_tiles, s);
    }
}

}  // namespace ptir
