// Wavefront path tracer and adjoint: each path stage is its own kernel over a compacted queue.
//
// Paths are processed in chunks of whole 8x4 pixel tiles (slot q of a chunk = lane q % 32 of
// tile q / 32, so the primary rays of a warp stay coherent). Per chunk, the forward runs
//   camera   : sampler seed and primary ray of every slot              -> intersect queue
//   intersect: primary segment                                        (all slots)
//   primary  : primary outputs, NEE light sample                       -> shadow queue | bounce queue
//   shadow   : stochastic shadow ray of the NEE sample                -> bounce queue
//   bounce d : light gathering, path termination, BRDF sample          -> intersect queue
//   sort     : the intersect queue in (octant, origin cell, direction cell) order
//   intersect: next segment                                            -> bounce queue
// and the backward the same with the adjoint stages, whose re-traversals (the reference's
// rayIntersectBwd) go to a replay queue drained after every bounce stage. Path state lives in
// HBM between stages; queues are appended with one atomic per warp (ballot + popc). The
// intersect stage refills lanes one by one (k_wf_trace). The per-path order of random draws is
// the megakernel's, so both schedules produce the same paths.

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include "radix_sort.cuh"
#include "path.cuh"
#include "wavefront.h"

namespace ptir {

namespace {

constexpr int kMaxThreads = 256;  // largest block size; the kernels use warps only, no block barriers

struct WfView {
    Segment* seg;
    PathState* ps;
    unsigned long long* rng;
    unsigned* q[3];          // bounce, intersect, shadow
    unsigned* count;         // [kNumQueueCounts]
    unsigned* cursor;        // [kNumCursors]
    ReplayJob* jobs;
    float* parked;           // intersection: parked accumulators and k-buffer batches, per thread
    uint2* frontier;         // intersection: two frontier buffers of frontier_cap entries per thread
    int frontier_cap;
    unsigned long long tile0;  // first tile of the chunk
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

// slot q of the chunk -> view, launch index (x, y, z) and flat launch index li; false for slots
// outside every image
PTIR_DEV bool slot_index(const TraceParams& P, const WfView& W, unsigned q, int& view, unsigned& x, unsigned& y,
                         unsigned& z, size_t& li) {
    return tile_launch(P, (long long)W.tile0 + (q >> 5), q & 31u, view, x, y, z, li);
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
    if (O.path_sig) O.path_sig[li] = ps.sig;
}

#define PTIR_STAGE_PROLOGUE                         \
    StackEntry stack[kStackDepth];                     \
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0}; \
    CtxT<K> C{P, stack, ctr};

// ---------------------------------------------------------------------------------------
// ray order

// Sort key of a ray: direction octant (3 bits), then the Morton code of its origin's cell (4 bits
// per axis of the scene bounds), then the Morton code of its direction's cell within the octant
// (4 bits per axis of the normalised |d|): 27 bits. Coarse origin cells with fine direction cells keep
// the rays of a warp on similar traversals; against octant + 8-bit origin cells alone this cut
// the intersection stage by 7 % on the 1M-Gaussian scene. Queue entries past the count get
// kSortPad, above all.
constexpr int kSortKeyBits = 28;
constexpr unsigned kSortPad = 1u << 27;

PTIR_DEV unsigned spread3_8(unsigned v) {
    v &= 0xFFu;
    v = (v | (v << 8)) & 0x0000F00Fu;
    v = (v | (v << 4)) & 0x000C30C3u;
    v = (v | (v << 2)) & 0x00249249u;
    return v;
}

// Keys of queue in_q: the intersect queue's segment rays, or the shadow queue's rays toward their
// light samples.
__global__ void __launch_bounds__(kMaxThreads) k_wf_sort_keys(TraceParams P, WfView W, int in_q, unsigned* keys) {
    const unsigned count = W.count[in_q];
    float3 lo = f3(0.0f), scale = f3(0.0f);
    if (P.accel.n > 0) {
        const float4 a = __ldg(P.accel.bounds), b = __ldg(P.accel.bounds + 1);
        lo = make_float3(a.x, a.y, a.z);
        scale = make_float3(255.0f / fmaxf(b.x - a.x, 1e-30f), 255.0f / fmaxf(b.y - a.y, 1e-30f),
                            255.0f / fmaxf(b.z - a.z, 1e-30f));
    }
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < W.slots; i += gridDim.x * blockDim.x) {
        unsigned key = kSortPad;
        if (i < count) {
            const unsigned q = W.q[in_q][i];
            float3 o = W.seg[q].o, d = W.seg[q].d;
            if (in_q == kQShadow) {
                d = W.ps[q].em.dir;
                o = W.seg[q].pos + d * 2e-2f;
            }
            const unsigned oct = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
            const float3 c = (o - lo) * scale * (1.0f / 16.0f);
            const unsigned cx = (unsigned)fminf(fmaxf(c.x, 0.0f), 15.0f);
            const unsigned cy = (unsigned)fminf(fmaxf(c.y, 0.0f), 15.0f);
            const unsigned cz = (unsigned)fminf(fmaxf(c.z, 0.0f), 15.0f);
            const float dn = rsqrtf(fmaxf(dot(d, d), 1e-30f));
            const unsigned dx = (unsigned)fminf(fabsf(d.x) * dn * 16.0f, 15.0f);
            const unsigned dy = (unsigned)fminf(fabsf(d.y) * dn * 16.0f, 15.0f);
            const unsigned dz = (unsigned)fminf(fabsf(d.z) * dn * 16.0f, 15.0f);
            const unsigned ocell = (spread3_8(cx) << 2) | (spread3_8(cy) << 1) | spread3_8(cz);
            const unsigned dcell = (spread3_8(dx) << 2) | (spread3_8(dy) << 1) | spread3_8(dz);
            key = (oct << 24) | (ocell << 12) | dcell;
        }
        keys[i] = key;
    }
}

// ---------------------------------------------------------------------------------------
// intersection with per-lane refill

PTIR_DEV unsigned lanes_below() { return (1u << lane()) - 1u; }

// The compositing accumulators of a lane's segment, parked in global memory while its warp
// traverses (they are only touched between trace calls, about three times per segment, and stay
// in L2), so that they hold no registers during the traversal and no shared memory: L1 keeps
// all of its capacity for node and leaf records. One float per field and thread, field-major
// with the grid's thread count as stride (coalesced).
constexpr int kParkedFields = 22;

struct Parked {
    float* base;  // this thread's first field
    int stride;   // threads of the grid
    __device__ __forceinline__ float& f(int k) const { return base[k * stride]; }
    __device__ __forceinline__ void save(const Composite& c) const {
        f(0) = c.radiance.x; f(1) = c.radiance.y; f(2) = c.radiance.z;
        f(3) = c.normal.x; f(4) = c.normal.y; f(5) = c.normal.z;
        f(6) = c.albedo.x; f(7) = c.albedo.y; f(8) = c.albedo.z;
        f(9) = c.snrm.x; f(10) = c.snrm.y; f(11) = c.snrm.z;
        f(12) = c.transmittance; f(13) = c.depth; f(14) = c.hit2; f(15) = c.distortion;
        f(16) = c.hits_count; f(17) = c.rough; f(18) = c.metal; f(19) = c.last_hit; f(20) = c.clip_end;
        f(21) = c.hit ? 1.0f : 0.0f;
    }
    __device__ __forceinline__ void load(Composite& c, float3 o, float3 d) const {
        c.o = o;
        c.d = d;
        c.radiance = make_float3(f(0), f(1), f(2));
        c.normal = make_float3(f(3), f(4), f(5));
        c.albedo = make_float3(f(6), f(7), f(8));
        c.snrm = make_float3(f(9), f(10), f(11));
        c.transmittance = f(12); c.depth = f(13); c.hit2 = f(14); c.distortion = f(15);
        c.hits_count = f(16); c.rough = f(17); c.metal = f(18); c.last_hit = f(19); c.clip_end = f(20);
        c.hit = f(21) != 0.0f;
    }
};

// Intersection stage: each lane carries one segment of queue `in_q` (read from `items`, the
// queue in queue or sorted order) through as many trace calls as it needs (composite_begin /
// trace / composite_hits / composite_end). A lane whose call has finished composites its batch
// and starts the next call, or writes its segment, hands it to queue `out_q` (when >= 0) and
// takes the next one from the queue, so that no lane waits for the slowest segment of its warp.
// The warp leaves its traversal loop once `refill` lanes wait (a finished call, or idle while
// the queue still holds segments). W.parked holds, per thread of the grid, the parked
// accumulators and, while a batch is composited, its k-buffer (kParkedFields + 2K floats).
// Registers per thread of k_wf_trace (and of the shadow kernel of the same k-buffer size). The
// kernels use no shared memory, so registers alone set the resident warps. K <= 16: 96, five
// 128-thread blocks per SM, 5 % faster than the compiler's own 127 (four blocks) despite a few
// spills; 80 (six blocks) was 11 % slower. K = 32: 128, four blocks, 6 % faster for the step
// than 168 (three blocks); 96 (five blocks) was 23 % slower.
constexpr int trace_regs(int K) { return K > 16 ? 128 : 96; }

// Seed of the k-buffer rounds in the intersection stage: the cut starts at the round's tmin plus
// this multiple of a span, the previous round's (its K-th less its first distance) for a segment's
// later rounds. On 2 views of 512x384x4 (1M Gaussians) 17 % of those rounds were continued past
// the seed at 2, and the step took 150.9 ms, against 163.8 ms unseeded, 154.6 ms at 1.5 and 154.1
// ms at 3. Seeding the first rounds as well (from the lane's last segment) took it to 142.0 ms (5.6 %
// of them continued), against 145.5 ms at 1.5 and 143.2 ms at 3.
constexpr float kSeedSpan = 2.0f;

//
// With K = 32 a traversal stands for two of the reference's 16-candidate rounds (the rounds of
// pathTracer.cuh:216-311): its first 16 candidates are the first round, and its last 16 are the
// second when each of them is a candidate of the second round's own call, i.e. lies past the
// first round's last hit and has its instance box crossed within the second round's interval;
// otherwise the second round is traced. The results are those of 16-candidate rounds (a 32-entry
// traversal culls at a farther distance, so it keeps grazing candidates that a 16-entry one can
// cull, as an exact nearest-16 selection would), with about a third fewer node visits per segment.
//
// With kResume (K <= 16) a segment's calls after its first resume from the frontier its previous
// call set aside (traverse.cuh), in a lane's part of W.frontier. kSlack builds the kernel that
// applies the exact-candidate cull slack (only tracers with exact_candidates launch it).
template <int K, bool kMark, bool kSelfOcc, bool kResume, bool kSlack>
__global__ void __maxnreg__(trace_regs(K)) k_wf_trace(TraceParams P, float* vis, WfView W, int in_q,
                                                      const unsigned* items, int out_q, unsigned cursor, int refill) {
    constexpr bool kPair = K == 32;  // traversals gather two 16-candidate rounds (leaf-index k-buffer)
    static_assert(!(kPair && kResume), "resumed calls take the 16-candidate rounds one by one");
    static_assert(!(kSlack && kResume), "the exact-candidate slack is applied by the rounds from the root");
    constexpr bool kIdx = kPair || kResume;  // the k-buffer holds leaf record indices
    const int nthreads = (int)(gridDim.x * blockDim.x);
    const Frontier F{kResume ? W.frontier + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2 * W.frontier_cap
                             : nullptr,
                     W.frontier_cap};
    float* const base = W.parked + blockIdx.x * blockDim.x + threadIdx.x;
    const Parked pk{base, nthreads};
    float* const batch_t = base + kParkedFields * nthreads;
    unsigned* const batch_id = reinterpret_cast<unsigned*>(batch_t + K * nthreads);
    StackEntry stack[kStackDepth];
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    constexpr unsigned kFull = 0xFFFFFFFFu;
    enum : int { kIdle = 0, kTracing = 1, kReady = 2 };
    const unsigned count = W.count[in_q];
    int phase = kIdle;
    unsigned q = 0;
    int rounds = 0;
    bool drained = false;
    float3 ro = f3(0.0f), rd = f3(0.0f);  // the lane's segment ray
    TraceState t;
    bool seeded = false;  // the lane's call started with a cut estimated from its previous round
    float first_span = 0.0f;  // K-th distance less tmin of the first round of the lane's last segment
    float kt[K];  // a call found nothing when kt[0] == kFarT
    unsigned kid[K];
    // next trace call of this lane's segment, or ready with nothing found when it is complete. The
    // rounds of the reference's k-buffer of 16 (from the root) are seeded (traverse.cuh: a call that
    // does not fill its k-buffer below its seed is continued past it): a segment's later round with
    // the cut tmin + kSeedSpan x the previous round's span of distances, its first round with tmin +
    // kSeedSpan x the first-round span (K-th distance less tmin) of the lane's last segment, a
    // neighbouring ray in the queue's order. Rounds of 8 are not seeded: their spans are short, and
    // a seed that close culls more grazing Gaussians (0.17 % of the paths changed on a scene of
    // Gaussians up to 0.3 in size).
    auto next_call = [&](const Composite& c) {
        if (!composite_open(P, c)) {
            kt[0] = kFarT;
            phase = kReady;
            return;
        }
        if (++rounds > kMaxRounds + 1) {
            atomicOr(P.error_word, kErrLoopBound);
            kt[0] = kFarT;
            phase = kReady;
            return;
        }
        float cap = kFarT;
        seeded = false;
        if constexpr (!kIdx && K == 16) {
            // kt still holds the previous round (a full k-buffer) when there is one
            const float span = rounds > 1 ? kt[K - 1] - kt[0] : first_span;
            if (span > 0.0f) {
                cap = composite_tmin(c) + kSeedSpan * span;
                seeded = cap < composite_tend(c);
                if (!seeded) cap = kFarT;
            }
        }
        phase = trace_start<K, kIdx, kResume>(P.accel, ro, rd, composite_tmin(c), composite_tend(c), kt, kid, t, ctr,
                                              &F, rounds > 1, cap)
                    ? kTracing
                    : kReady;
    };
    // the segment is complete: no call remains
    auto no_call = [&]() {
        kt[0] = kFarT;
        phase = kReady;
    };
    while (true) {
        // refill the idle lanes
        const unsigned idle = __ballot_sync(kFull, phase == kIdle);
        if (!drained && idle) {
            const unsigned n_idle = __popc(idle);
            unsigned base = 0;
            if (lane() == 0) base = atomicAdd(W.cursor + cursor, n_idle);
            base = __shfl_sync(kFull, base, 0);
            drained = base + n_idle >= count;
            if (phase == kIdle) {
                const unsigned i = base + __popc(idle & lanes_below());
                if (i < count) {
                    q = items[i];
                    Composite c;
                    composite_begin(P, c, W.seg[q].o, W.seg[q].d);
                    ro = c.o;
                    rd = c.d;
                    ++ctr.segments;
                    rounds = 0;
                    next_call(c);
                    pk.save(c);
                }
            }
        }
        const unsigned busy = __ballot_sync(kFull, phase != kIdle);
        if (!busy) {
            if (drained) break;
            continue;
        }
        // traverse until enough lanes wait
        const unsigned eligible = drained ? busy : kFull;
        while (true) {
            const unsigned tracing = __ballot_sync(kFull, phase == kTracing);
            if (!tracing || __popc(eligible & ~tracing) >= refill) break;
            if (phase == kTracing &&
                !trace_step<K, kIdx, kResume, kSlack>(P.accel, ro, rd, t, kt, kid, stack, P.error_word, ctr,
                                                      &F)) {
                if (seeded && kid[K - 1] == kNoHit) {
                    seeded = false;
                    trace_continue(t, kt, ctr);
                } else {
                    phase = kReady;
                }
            }
        }
        // composite the finished calls; hand on the finished segments
        bool done = false;
        if (phase == kReady) {
            Composite c;
            pk.load(c, ro, rd);
            if (kt[0] < kFarT) {
                // the batch goes to the parked buffer, so compositing holds no k-buffer registers
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    batch_t[i * nthreads] = kt[i];
                    batch_id[i * nthreads] = kid[i];
                }
                float* const mark = kMark ? vis : nullptr;
                if constexpr (kPair) {
                    composite_leaf_batch<kSelfOcc>(P, ctr, c, batch_t, batch_id, nthreads, 0, 16, mark);
                    bool call = composite_open(P, c) && batch_id[16 * nthreads] != kNoHit;
                    if (call) {
                        const float tmin2 = composite_tmin(c), tend2 = composite_tend(c);
                        bool second = true;
#pragma unroll 1
                        for (int i = 16; i < 32 && second; ++i) {
                            const unsigned p = batch_id[i * nthreads];
                            if (p == kNoHit) break;
                            second = batch_t[i * nthreads] > tmin2 && leaf_box_hit(P.accel, p, ro, rd, tmin2, tend2);
                        }
                        if (second) {
                            composite_leaf_batch<kSelfOcc>(P, ctr, c, batch_t, batch_id, nthreads, 16, 32, mark);
                            call = composite_open(P, c) && batch_id[31 * nthreads] != kNoHit;
                        }
                    }
                    if (call) next_call(c);
                    else no_call();
                } else {
                    if constexpr (kIdx)
                        composite_leaf_batch<kSelfOcc>(P, ctr, c, batch_t, batch_id, nthreads, 0, K, mark);
                    else
                        composite_hits_strided<kSelfOcc, K>(P, ctr, c, batch_t, batch_id, nthreads, mark);
                    // a k-buffer that is not full held every candidate of the call: a later call finds none
                    if (rounds == 1 && kid[K - 1] != kNoHit) first_span = kt[K - 1] - t.tmin;
                    if (kid[K - 1] != kNoHit) next_call(c);
                    else no_call();
                }
            }
            // nothing found, segment closed, or loop bound: the segment is complete
            if (phase == kReady && kt[0] >= kFarT) {
                Segment s;
                Pcg32 rng = load_rng(W, q);
                composite_end(P, c, W.seg[q].scatter_pdf, W.seg[q].light_pdf, s, rng);
                W.seg[q] = s;
                store_rng(W, q, rng);
                phase = kIdle;
                done = true;
            } else {
                pk.save(c);
            }
        }
        if (out_q >= 0) push(W.q[out_q], W.count + out_q, q, done);
    }
    flush_counters(P, ctr);
}

// ---------------------------------------------------------------------------------------
// forward

// Camera segments of the chunk: the sampler seed and the primary ray of every slot inside the
// image, queued for intersection.
__global__ void __launch_bounds__(kMaxThreads) k_wf_camera(TraceParams P, WfView W) {
    while (true) {
        const unsigned base = fetch32(W.cursor + 0);
        if (base >= W.slots) break;
        const unsigned q = base + lane();
        unsigned x = 0, y = 0, z = 0;
        int view = 0;
        size_t li = 0;
        const bool valid = q < W.slots && slot_index(P, W, q, view, x, y, z, li);
        if (valid) {
            Pcg32 rng;
            rng.seed(x, y, z, P.views[view].frame);
            Segment s;
            float3 o, d;
            world_ray(P, view, x, y, z, li, o, d);
            segment_reset(s, o, d, 0.0f);
            W.seg[q] = s;
            store_rng(W, q, rng);
        }
        push(W.q[kQIsect], W.count + kQIsect, q, valid);
    }
}

// primary outputs and the first NEE sample of every camera segment
template <int K>
__global__ void __launch_bounds__(kMaxThreads) k_wf_fwd_primary(TraceParams P, FwdOutputs O, WfView W) {
    PTIR_STAGE_PROLOGUE
    const bool mis = (P.flags & kMis) != 0;
    while (true) {
        const unsigned base = fetch32(W.cursor + 2);
        if (base >= W.slots) break;
        const unsigned q = base + lane();
        unsigned x = 0, y = 0, z = 0;
        int view = 0;
        size_t li = 0;
        const bool valid = q < W.slots && slot_index(P, W, q, view, x, y, z, li);
        bool cont = false, shadow = false;
        if (valid) {
            Pcg32 rng = load_rng(W, q);
            PathState ps;
            path_init(ps, effective_bounces(P));
            Segment s = W.seg[q];
            sig_event(P, ps, sig_segment(s));
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

// NEE shadow rays (the stochastic occlusion walk of pathTracer.cuh:161-214, as shadow_occluded in
// path.cuh) with per-lane refill, as in k_wf_trace: a lane whose ray is decided hands its slot
// to the bounce queue and takes the next shadow ray, so that no lane waits for the longest walk
// of its warp. The warp leaves its traversal loop once `refill` lanes wait. The random draws of
// a ray are those of shadow_occluded, in the same order. Against one ray per lane for the whole
// walk this cut the stage by 15 % on the 1M-Gaussian scene, and the register cap of the
// intersection kernel (more resident warps) by 6 % more.
template <int K>
__global__ void __maxnreg__(trace_regs(K)) k_wf_shadow(TraceParams P, WfView W, int refill, const unsigned* items) {
    StackEntry stack[kStackDepth];
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    constexpr unsigned kFull = 0xFFFFFFFFu;
    enum : int { kIdle = 0, kTracing = 1, kReady = 2 };
    const unsigned count = W.count[kQShadow];
    int phase = kIdle;
    unsigned q = 0;
    int rounds = 0;
    bool drained = false;
    float3 ro = f3(0.0f), rd = f3(0.0f);
    float start = 0.0f, end = 0.0f;
    Pcg32 rng;
    TraceState t;
    bool seeded = false;      // the lane's call started with a cut estimated from a span, as in k_wf_trace
    float first_span = 0.0f;  // K-th distance less tmin of the first round of the lane's last shadow ray
    float kt[K];
    unsigned kid[K];
    // next trace call of the lane's ray over (start, end), or the ray is decided (unoccluded). Rounds
    // of 16 are seeded as in k_wf_trace: a later round from the previous round's span, a first round
    // from the first-round span of the lane's last shadow ray (a neighbour in the sorted queue).
    auto next_call = [&]() -> bool {
        if (!(start < end)) return false;
        if (++rounds > (1 << 16) + 1) {
            atomicOr(P.error_word, kErrLoopBound);
            return false;
        }
        float cap = kFarT;
        seeded = false;
        if constexpr (K == 16) {
            // kt still holds the previous round (a full k-buffer) when there is one
            const float span = rounds > 1 ? kt[K - 1] - kt[0] : first_span;
            if (span > 0.0f) {
                cap = start + 1e-9f + kSeedSpan * span;
                seeded = cap < end;
                if (!seeded) cap = kFarT;
            }
        }
        phase = trace_start(P.accel, ro, rd, start + 1e-9f, end, kt, kid, t, ctr, nullptr, false, cap) ? kTracing
                                                                                                       : kReady;
        return true;
    };
    while (true) {
        bool done = false, occluded = false;
        const unsigned idle = __ballot_sync(kFull, phase == kIdle);
        if (!drained && idle) {
            const unsigned n_idle = __popc(idle);
            unsigned base = 0;
            if (lane() == 0) base = atomicAdd(W.cursor + 3, n_idle);
            base = __shfl_sync(kFull, base, 0);
            drained = base + n_idle >= count;
            if (phase == kIdle) {
                const unsigned i = base + __popc(idle & lanes_below());
                if (i < count) {
                    q = items[i];
                    const float3 wi = W.ps[q].em.dir;
                    ro = W.seg[q].pos + wi * 2e-2f;
                    rd = wi;
                    rng = load_rng(W, q);
                    ++ctr.segments;
                    rounds = 0;
                    const float2 clip = clip_scene(P, ro, rd);
                    start = fmaxf(0.0f, clip.x - 1e-9f);
                    end = fminf(W.ps[q].em.tmax, clip.y) + 1e-9f;
                    phase = kTracing;
                    if (!next_call()) done = true;  // nothing in front of the light
                }
            }
        }
        const unsigned busy = __ballot_sync(kFull, phase != kIdle && !done);
        if (!busy && !__any_sync(kFull, done)) {
            if (drained) break;
            continue;
        }
        // traverse until enough lanes wait
        const unsigned eligible = drained ? busy : kFull;
        while (true) {
            const unsigned tracing = __ballot_sync(kFull, phase == kTracing && !done);
            if (!tracing || __popc(eligible & ~tracing) >= refill) break;
            if (phase == kTracing && !done &&
                !trace_step(P.accel, ro, rd, t, kt, kid, stack, P.error_word, ctr)) {
                if (seeded && kid[K - 1] == kNoHit) {
                    seeded = false;
                    trace_continue(t, kt, ctr);
                } else {
                    phase = kReady;
                }
            }
        }
        // walk the finished batches: the first hit that occludes decides the ray
        if (phase == kReady && !done) {
            if (rounds == 1 && kid[K - 1] != kNoHit) first_span = kt[K - 1] - t.tmin;
            if (kid[0] == kNoHit) {
                done = true;
            } else {
                float batch_end = start;
                bool stop = false;
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    if (stop || occluded) continue;
                    const unsigned id = kid[i];
                    if (id == kNoHit || kt[i] > end) {
                        stop = true;
                        continue;
                    }
                    batch_end = fmaxf(batch_end, kt[i]);
                    if (self_occluded(P, kt[i], id, rd)) continue;
                    float dns;
                    const Response r = respond(P, id, ro, rd, dns);
                    const float alpha = (r.gres > P.min_response && r.alpha > P.alpha_min) ? r.alpha : 0.0f;
                    if (alpha > 0.0f && rng.uniform() < alpha) occluded = true;
                }
                if (occluded || batch_end <= start || kid[K - 1] == kNoHit) {
                    done = true;  // decided, or no candidate left (the k-buffer was not full)
                } else {
                    start = batch_end;
                    if (!next_call()) done = true;
                }
            }
        }
        if (done) {
            if (occluded) {
                Emitter em = W.ps[q].em;
                emitter_clear(em);
                W.ps[q].em = em;
            }
            if (P.flags & kPathSig) W.ps[q].sig = sig_mix(W.ps[q].sig, kSigShadow | (occluded ? 1u : 0u));
            store_rng(W, q, rng);
            phase = kIdle;
        }
        push(W.q[kQBounce], W.count + kQBounce, q, done);
    }
    flush_counters(P, ctr);
}

template <int K>
__global__ void __launch_bounds__(kMaxThreads) k_wf_fwd_bounce(TraceParams P, FwdOutputs O, WfView W, unsigned depth,
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
            if (depth > 0) sig_event(P, ps, sig_segment(s));
            accumulate_light(C, ps, s);
            ps.active &= (unsigned)((depth + 1u < ps.max_bounces) && s.ivalid);
            if (ps.active) {
                ps.bounces = depth + 1u;
                sample_next(C, ps, s, rng);
                cont = path_continues(ps);
                sig_event(P, ps, kSigCont | (cont ? 1u : 0u));
            }
            if (cont) {
                W.seg[q] = s;
                W.ps[q] = ps;
                store_rng(W, q, rng);
            } else {
                unsigned x, y, z;
                int view;
                size_t li;
                slot_index(P, W, q, view, x, y, z, li);
                write_pbr(O, li, ps);
            }
        }
        push(W.q[kQIsect], W.count + kQIsect, q, cont);
    }
    flush_counters(P, ctr);
}

// ---------------------------------------------------------------------------------------
// backward

// adjoint state and the first NEE sample of every camera segment
template <int K>
__global__ void __launch_bounds__(kMaxThreads) k_wb_primary(TraceParams P, BwdInputs B, WfView W) {
    PTIR_STAGE_PROLOGUE
    const bool mis = (P.flags & kMis) != 0;
    while (true) {
        const unsigned base = fetch32(W.cursor + 2);
        if (base >= W.slots) break;
        const unsigned q = base + lane();
        unsigned x = 0, y = 0, z = 0;
        int view = 0;
        size_t li = 0;
        const bool valid = q < W.slots && slot_index(P, W, q, view, x, y, z, li);
        bool cont = false, shadow = false;
        if (valid) {
            Pcg32 rng = load_rng(W, q);
            PathState ps;
            path_init(ps, effective_bounces(P));
            load_adjoint_inputs(P, B, x, y, z, li, ps);
            Segment s = W.seg[q];
            add_material_output_grad(P, B, x, y, z, li, s);
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
__global__ void __launch_bounds__(kMaxThreads) k_wb_bounce(TraceParams P, BwdInputs B, WfView W, unsigned depth,
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
__global__ void __launch_bounds__(kMaxThreads) k_wb_replay(TraceParams P, BwdInputs B, WfView W, unsigned cursor,
                                                           bool resume) {
    PTIR_STAGE_PROLOGUE
    const unsigned count = W.count[kQJobs];
    // with `resume` a replay's rounds after its first resume from the previous round's frontier
    const Frontier F{resume ? W.frontier + (size_t)(blockIdx.x * blockDim.x + threadIdx.x) * 2 * W.frontier_cap
                            : nullptr,
                     W.frontier_cap};
    while (true) {
        const unsigned base = fetch32(W.cursor + cursor);
        if (base >= count) break;
        const unsigned i = base + lane();
        if (i < count) {
            const ReplayJob j = W.jobs[i];
            replay_material_grad(C, B, j, F.buf ? &F : nullptr);
        }
    }
    flush_counters(P, ctr);
}

// persistent grid: resident blocks per SM x SMs (defined below)
int grid_cached(const void* fn, int block, size_t smem);

// The shadow stage with its own k-buffer size. A shadow walk visits the hits in distance order
// until one occludes, whatever the batch size, so its size is free of the intersection's: a
// walk usually ends in its first batch, which a smaller buffer gathers with less traversal.
static void launch_shadow(int ks, const TraceParams& q, const WfView& W, int B, int R, const unsigned* items,
                          cudaStream_t s) {
    switch (ks) {
    case 8: k_wf_shadow<8><<<grid_cached((const void*)k_wf_shadow<8>, B, 0), B, 0, s>>>(q, W, R, items); break;
    case 32: k_wf_shadow<32><<<grid_cached((const void*)k_wf_shadow<32>, B, 0), B, 0, s>>>(q, W, R, items); break;
    default: k_wf_shadow<16><<<grid_cached((const void*)k_wf_shadow<16>, B, 0), B, 0, s>>>(q, W, R, items); break;
    }
}

// persistent grid: resident blocks per SM x SMs
int grid_for(const void* fn, int block, size_t smem) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    return sms * per_sm;
}

// floats of W.parked for every thread the device can hold resident (k-buffer up to 32)
size_t parked_floats() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    if (sms <= 0) sms = 148;
    if (per_sm <= 0) per_sm = 2048;
    return (size_t)(kParkedFields + 2 * 32) * (size_t)sms * (size_t)per_sm;
}

// grid of a kernel at a block size, computed once per (kernel, block size)
int grid_cached(const void* fn, int block, size_t smem = 0) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({fn, block});
    if (it != cache.end()) return it->second;
    // more than the default 48 KB of dynamic shared memory needs the kernel's opt-in
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int g = grid_for(fn, block, smem);
    cache[{fn, block}] = g;
    return g;
}

}  // namespace

// ---------------------------------------------------------------------------------------
cudaError_t wavefront_reserve(WavefrontBuffers& b, size_t slots, cudaStream_t s) {
    if (slots <= b.slots && b.seg) return cudaSuccess;
    auto rel = [&](void* p) {
        if (p) cudaFreeAsync(p, s);
    };
    rel(b.seg); rel(b.ps); rel(b.rng); rel(b.q[0]); rel(b.q[1]); rel(b.q[2]); rel(b.jobs);
    rel(b.sort_keys[0]); rel(b.sort_keys[1]); rel(b.sorted); rel(b.sort_temp); rel(b.parked);
    void* counters = b.counters;
    void* frontier = b.frontier;
    const size_t frontier_threads = b.frontier_threads;
    b = WavefrontBuffers{};
    b.counters = counters;
    b.frontier = frontier;  // sized by the intersection grid, not by the chunk
    b.frontier_threads = frontier_threads;
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
    get(&b.sort_keys[0], sizeof(unsigned) * slots);
    get(&b.sort_keys[1], sizeof(unsigned) * slots);
    get(&b.sorted, sizeof(unsigned) * slots);
    get(&b.parked, sizeof(float) * parked_floats());
    if (e == cudaSuccess) {
        b.sort_temp_bytes = radix_sort_temp_bytes<unsigned>((long long)slots);
        get(&b.sort_temp, b.sort_temp_bytes);
    }
    if (e == cudaSuccess) b.slots = slots;
    return e;
}

size_t wavefront_bytes_per_slot() {
    // path state, RNG, three queues, two replay jobs, two sort keys + the sorted queue, and the
    // radix sort's scratch (a key / value pair per slot and its digit counts, rounded up)
    return sizeof(Segment) + sizeof(PathState) + sizeof(unsigned long long) + 3 * sizeof(unsigned) +
           2 * sizeof(ReplayJob) + 3 * sizeof(unsigned) + 4 * sizeof(unsigned);
}

void wavefront_free(WavefrontBuffers& b) {
    for (void* p : {b.seg, b.ps, b.rng, b.q[0], b.q[1], b.q[2], b.jobs, b.counters, b.sort_keys[0], b.sort_keys[1],
                    b.sorted, b.sort_temp, b.parked, b.frontier})
        if (p) cudaFree(p);
    b = WavefrontBuffers{};
}

// frontier buffers for `threads` threads of the intersection kernel (grown on demand)
cudaError_t frontier_reserve(WavefrontBuffers& b, size_t threads, cudaStream_t s) {
    if (threads <= b.frontier_threads && b.frontier) return cudaSuccess;
    if (b.frontier) cudaFreeAsync(b.frontier, s);
    b.frontier = nullptr;
    b.frontier_threads = 0;
    const cudaError_t e = cudaMallocAsync(&b.frontier, sizeof(uint2) * 2 * (size_t)kFrontierCap * threads, s);
    if (e == cudaSuccess) b.frontier_threads = threads;
    return e;
}

static WfView view_of(const WavefrontBuffers& b, unsigned long long tile0, unsigned slots, bool resume) {
    WfView W;
    W.seg = static_cast<Segment*>(b.seg);
    W.ps = static_cast<PathState*>(b.ps);
    W.rng = static_cast<unsigned long long*>(b.rng);
    for (int k = 0; k < 3; ++k) W.q[k] = static_cast<unsigned*>(b.q[k]);
    W.count = static_cast<unsigned*>(b.counters);
    W.cursor = W.count + kNumQueueCounts;
    W.jobs = static_cast<ReplayJob*>(b.jobs);
    W.parked = static_cast<float*>(b.parked);
    W.frontier = resume ? static_cast<uint2*>(b.frontier) : nullptr;
    W.frontier_cap = resume ? kFrontierCap : 0;
    W.tile0 = tile0;
    W.slots = slots;
    return W;
}

static unsigned long long total_tiles(const TraceParams& p) { return (unsigned long long)p.tiles; }

// The intersect queue in ray order (or as queued when sorting is off): keys, then a key/slot
// radix sort of the whole chunk capacity (the count stays on the device).
static const unsigned* sort_queue(const TraceParams& p, const WavefrontBuffers& b, const WfView& W,
                                  const WavefrontTuning& tune, const StageCtx& sc, cudaStream_t s, int in_q = kQIsect) {
    if (!tune.sort_rays) return W.q[in_q];
    unsigned* keys_in = static_cast<unsigned*>(b.sort_keys[0]);
    unsigned* keys_out = static_cast<unsigned*>(b.sort_keys[1]);
    unsigned* sorted = static_cast<unsigned*>(b.sorted);
    const int grid = grid_cached((const void*)k_wf_sort_keys, tune.block);
    sc.run(kStageSort, p, s, [&](const TraceParams& q) {
        k_wf_sort_keys<<<grid, tune.block, 0, s>>>(q, W, in_q, keys_in);
        radix_sort_pairs<unsigned>(b.sort_temp, b.sort_temp_bytes, keys_in, keys_out, W.q[in_q], sorted,
                                   (long long)W.slots, 0, kSortKeyBits, s);
    });
    return sorted;
}

// Cursor of each stage launch within a chunk: camera 0, primary intersection 1, primary outputs
// 2, shadow 3, then per bounce depth the bounce stage, (the adjoint's replay,) and intersection.
constexpr unsigned kFirstBounceCursor = 4;

// intersection kernels with resumed rounds (K <= 16)
template <int K>
static bool use_resume(const WavefrontTuning& tune) {
    return K <= 16 && tune.resume_isect && !tune.exact_candidates;
}

// the intersection kernel of a launch: resumed rounds, the exact-candidate slack, or neither
template <int K, bool kMark, bool kSelfOcc>
static const void* trace_kernel(bool resume, bool slack) {
    if constexpr (K <= 16) {
        if (resume) return (const void*)k_wf_trace<K, kMark, kSelfOcc, true, false>;
    }
    if (slack) return (const void*)k_wf_trace<K, kMark, kSelfOcc, false, true>;
    return (const void*)k_wf_trace<K, kMark, kSelfOcc, false, false>;
}

template <int K, bool kMark, bool kSelfOcc>
static int trace_grid(bool resume, bool slack, int B) {
    return grid_cached(trace_kernel<K, kMark, kSelfOcc>(resume, slack), B);
}

template <int K, bool kMark, bool kSelfOcc>
static void launch_trace(bool resume, bool slack, int grid, int B, cudaStream_t s, const TraceParams& q, float* vis,
                         const WfView& W, int in_q, const unsigned* items, int out_q, unsigned cursor, int R) {
    if constexpr (K <= 16) {
        if (resume) {
            k_wf_trace<K, kMark, kSelfOcc, true, false><<<grid, B, 0, s>>>(q, vis, W, in_q, items, out_q, cursor, R);
            return;
        }
    }
    if (slack)
        k_wf_trace<K, kMark, kSelfOcc, false, true><<<grid, B, 0, s>>>(q, vis, W, in_q, items, out_q, cursor, R);
    else
        k_wf_trace<K, kMark, kSelfOcc, false, false><<<grid, B, 0, s>>>(q, vis, W, in_q, items, out_q, cursor, R);
}

template <int K>
static cudaError_t run_fwd(const TraceParams& p, const FwdOutputs& o, WavefrontBuffers& b, const WavefrontTuning& tune,
                           const StageCtx& sc, cudaStream_t s) {
    const unsigned long long tiles = total_tiles(p);
    if (tiles == 0) return cudaSuccess;
    const unsigned chunk_tiles = (unsigned)std::min<unsigned long long>(tune.chunk_tiles, tiles);
    cudaError_t e = wavefront_reserve(b, (size_t)chunk_tiles * 32, s);
    if (e != cudaSuccess) return e;
    const int B = tune.block, R = tune.refill_lanes;
    const int g_camera = grid_cached((const void*)k_wf_camera, B);
    const int g_primary = grid_cached((const void*)k_wf_fwd_primary<K>, B);
    const int g_bounce = grid_cached((const void*)k_wf_fwd_bounce<K>, B);
    const bool resume = use_resume<K>(tune), slack = tune.exact_candidates;
    const int g_trace0 = trace_grid<K, true, false>(resume, slack, B);
    const int g_trace = trace_grid<K, true, true>(resume, slack, B);
    if (resume && (e = frontier_reserve(b, std::max(g_trace0, g_trace) * B, s)) != cudaSuccess) return e;
    const unsigned mb = p.render_opts ? std::min(p.max_bounces, 2u) : p.max_bounces;
    if (kFirstBounceCursor + 2u * mb > (unsigned)kNumCursors) return cudaErrorInvalidValue;
    for (unsigned long long t0 = 0; t0 < tiles; t0 += chunk_tiles) {
        const unsigned nt = (unsigned)std::min<unsigned long long>(chunk_tiles, tiles - t0);
        const WfView W = view_of(b, t0, nt * 32u, resume);
        e = cudaMemsetAsync(b.counters, 0, sizeof(unsigned) * (kNumQueueCounts + kNumCursors), s);
        if (e != cudaSuccess) return e;
        const int cap = (int)std::min<long long>(INT32_MAX, ((long long)nt * 32 + B - 1) / B);
        sc.run(kStageShading, p, s, [&](const TraceParams& q) {
            k_wf_camera<<<std::min(g_camera, cap), B, 0, s>>>(q, W);
        });
        sc.run(kStageIntersect, p, s, [&](const TraceParams& q) {
            launch_trace<K, true, false>(resume, slack, std::min(g_trace0, cap), B, s, q, o.visibility, W, kQIsect,
                                         W.q[kQIsect], -1, 1, R);
        });
        sc.run(kStageShading, p, s, [&](const TraceParams& q) {
            k_wf_fwd_primary<K><<<std::min(g_primary, cap), B, 0, s>>>(q, o, W);
        });
        if (p.flags & kMis) {
            const unsigned* shadow_items = sort_queue(p, b, W, tune, sc, s, kQShadow);
            sc.run(kStageShadow, p, s,
                   [&](const TraceParams& q) { launch_shadow(tune.shadow_kbuf, q, W, B, R, shadow_items, s); });
        }
        unsigned cursor = kFirstBounceCursor;
        for (unsigned depth = 0; depth < mb; ++depth) {
            cudaMemsetAsync(W.count + kQIsect, 0, sizeof(unsigned), s);
            sc.run(kStageShading, p, s, [&](const TraceParams& q) {
                k_wf_fwd_bounce<K><<<g_bounce, B, 0, s>>>(q, o, W, depth, cursor);
            });
            ++cursor;
            if (depth + 1 >= mb) break;
            cudaMemsetAsync(W.count + kQBounce, 0, sizeof(unsigned), s);
            const unsigned* items = sort_queue(p, b, W, tune, sc, s);
            sc.run(kStageIntersect, p, s, [&](const TraceParams& q) {
                launch_trace<K, true, true>(resume, slack, g_trace, B, s, q, o.visibility, W, kQIsect, items, kQBounce,
                                            cursor, R);
            });
            ++cursor;
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int K>
static cudaError_t run_bwd(const TraceParams& p, const BwdInputs& bi, WavefrontBuffers& b, const WavefrontTuning& tune,
                           const StageCtx& sc, cudaStream_t s) {
    const unsigned long long tiles = total_tiles(p);
    if (tiles == 0) return cudaSuccess;
    const unsigned chunk_tiles = (unsigned)std::min<unsigned long long>(tune.chunk_tiles, tiles);
    cudaError_t e = wavefront_reserve(b, (size_t)chunk_tiles * 32, s);
    if (e != cudaSuccess) return e;
    const int B = tune.block, R = tune.refill_lanes;
    const int g_camera = grid_cached((const void*)k_wf_camera, B);
    const int g_primary = grid_cached((const void*)k_wb_primary<K>, B);
    const int g_bounce = grid_cached((const void*)k_wb_bounce<K>, B);
    const bool resume = use_resume<K>(tune), slack = tune.exact_candidates;
    const bool resume_replay = K <= 16 && tune.resume_replay;
    const int g_trace0 = trace_grid<K, false, false>(resume, slack, B);
    const int g_trace = trace_grid<K, false, true>(resume, slack, B);
    const int g_replay = grid_cached((const void*)k_wb_replay<K>, B);
    const int g_front = std::max(resume ? std::max(g_trace0, g_trace) : 0, resume_replay ? g_replay : 0);
    if (g_front > 0 && (e = frontier_reserve(b, (size_t)g_front * B, s)) != cudaSuccess) return e;
    const unsigned mb = p.render_opts ? std::min(p.max_bounces, 2u) : p.max_bounces;
    if (kFirstBounceCursor + 3u * mb > (unsigned)kNumCursors) return cudaErrorInvalidValue;
    for (unsigned long long t0 = 0; t0 < tiles; t0 += chunk_tiles) {
        const unsigned nt = (unsigned)std::min<unsigned long long>(chunk_tiles, tiles - t0);
        const WfView W = view_of(b, t0, nt * 32u, g_front > 0);
        e = cudaMemsetAsync(b.counters, 0, sizeof(unsigned) * (kNumQueueCounts + kNumCursors), s);
        if (e != cudaSuccess) return e;
        const int cap = (int)std::min<long long>(INT32_MAX, ((long long)nt * 32 + B - 1) / B);
        sc.run(kStageShading, p, s, [&](const TraceParams& q) {
            k_wf_camera<<<std::min(g_camera, cap), B, 0, s>>>(q, W);
        });
        sc.run(kStageIntersect, p, s, [&](const TraceParams& q) {
            launch_trace<K, false, false>(resume, slack, std::min(g_trace0, cap), B, s, q, nullptr, W, kQIsect,
                                          W.q[kQIsect], -1, 1, R);
        });
        sc.run(kStageShading, p, s, [&](const TraceParams& q) {
            k_wb_primary<K><<<std::min(g_primary, cap), B, 0, s>>>(q, bi, W);
        });
        if (p.flags & kMis) {
            const unsigned* shadow_items = sort_queue(p, b, W, tune, sc, s, kQShadow);
            sc.run(kStageShadow, p, s,
                   [&](const TraceParams& q) { launch_shadow(tune.shadow_kbuf, q, W, B, R, shadow_items, s); });
        }
        unsigned cursor = kFirstBounceCursor;
        for (unsigned depth = 0; depth < mb; ++depth) {
            cudaMemsetAsync(W.count + kQIsect, 0, sizeof(unsigned), s);
            cudaMemsetAsync(W.count + kQJobs, 0, sizeof(unsigned), s);
            sc.run(kStageShading, p, s, [&](const TraceParams& q) {
                k_wb_bounce<K><<<g_bounce, B, 0, s>>>(q, bi, W, depth, cursor);
            });
            ++cursor;
            sc.run(kStageReplay, p, s, [&](const TraceParams& q) {
                k_wb_replay<K><<<g_replay, B, 0, s>>>(q, bi, W, cursor, resume_replay);
            });
            ++cursor;
            if (depth + 1 >= mb) break;
            cudaMemsetAsync(W.count + kQBounce, 0, sizeof(unsigned), s);
            const unsigned* items = sort_queue(p, b, W, tune, sc, s);
            sc.run(kStageIntersect, p, s, [&](const TraceParams& q) {
                launch_trace<K, false, true>(resume, slack, g_trace, B, s, q, nullptr, W, kQIsect, items, kQBounce,
                                             cursor, R);
            });
            ++cursor;
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_trace_fwd_wavefront(const TraceParams& p, const FwdOutputs& o, WavefrontBuffers& b,
                                       const WavefrontTuning& tune, const StageCtx& sc, cudaStream_t s) {
    switch (tune.kbuf) {
    case 8: return run_fwd<8>(p, o, b, tune, sc, s);
    case 32: return run_fwd<32>(p, o, b, tune, sc, s);
    default: return run_fwd<16>(p, o, b, tune, sc, s);
    }
}

cudaError_t launch_trace_bwd_wavefront(const TraceParams& p, const BwdInputs& bi, WavefrontBuffers& b,
                                       const WavefrontTuning& tune, const StageCtx& sc, cudaStream_t s) {
    switch (tune.kbuf) {
    case 8: return run_bwd<8>(p, bi, b, tune, sc, s);
    case 32: return run_bwd<32>(p, bi, b, tune, sc, s);
    default: return run_bwd<16>(p, bi, b, tune, sc, s);
    }
}

}  // namespace ptir
