// Software LBVH traversal with a register k-buffer: the replacement for OptiX's
// optixTrace + __intersection__is + __anyhit__ah of the reference
// (threedgptir_tracer/include/3dgptir/kernels/cuda/pathTracer.cuh:58-113,
//  src/kernels/cuda/referenceOptix.cu:73-133, gaussianParticles.cuh:484-500).
//
// One call returns the K candidates with the smallest closest-approach parameter t* in
// (tmin, tend), ascending. A Gaussian is a candidate when its object-space ray hits the unit
// instance box [-1,1]^3 within [tmin, tend] and passes the perpendicular-distance test.
//
// Culling (AccelView::cull_slack = 0) follows the reference's traversal: subtrees are culled by
// their instance-box AABBs against [tmin, t_K], where t_K is the K-th distance found so far (the
// reference's any-hit program shrinks the ray's tmax to the 16th distance). This returns the K
// nearest candidates except for a Gaussian whose closest approach lies before its own box entry
// (a ray grazing a box corner): like the reference, it is then kept only if reached before t_K
// drops below its box entry, which depends on the traversal order. Its response can pass the
// acceptance threshold, so K (which sets t_K) and the order can change the image. With
// cull_slack > 0 a subtree is culled only when its box entry, less kCullSlack times the largest
// kernel support radius under it over |d|, lies past t_K: a lower bound of every t* under it, so
// a call returns exactly the K nearest candidates, whatever the order or K.
//
// Resumed calls (kResume): a segment's calls after its first start from a frontier instead of
// the root. A call keeps, as (code, lower bound) pairs, everything it set aside against its K-th
// distance: the subtrees and untested leaves culled by their box entry, the leaves whose t* lay
// past the K-th distance when tested, and the candidates evicted from the k-buffer. Every
// candidate of the next call (interval starting past the last composited hit, so later than
// this call's) lies in one of those, since what a call rejects for any other reason (t* before
// tmin or past tend, the box missed within the interval, the perpendicular distance) stays
// rejected under a later tmin. The next call processes the frontier's entries in order, those
// still past its own K-th distance going to its own frontier. The candidates are those of a call
// from the root (up to the order-dependent grazing case above), with about half the node visits.
//
// Seeded calls (TraceState::cap): a caller that can estimate where the call's K-th candidate lies
// (the wavefront kernel does for a segment's later rounds, from the previous round's span) starts
// the call with that distance as its cut, so that subtrees past it are culled before the k-buffer
// is full. A call that fills its k-buffer below the seed has its K nearest candidates. One that
// does not (fewer than K candidates before the seed) holds every candidate before the seed and is
// continued past it (TraceState::floor = the seed, no cap): subtrees whose clipped box ends before
// the floor are culled and leaves need t* >= floor. Both passes keep the reference's candidate
// test; only the grazing case above (a closest approach outside the Gaussian's own box interval)
// can be culled by one order and kept by another.
#pragma once

#include "device_types.h"
#include "vecmath.cuh"

namespace ptir {

constexpr int kKBuf = 16;            // reference MaxNumHitPerTrace; the kernels also build K = 8 and 32
constexpr int kStackDepth = 64;      // traversal stack entries

// traversal stack entry: x = node index, y = its entry distance (float bits)
using StackEntry = int2;
constexpr unsigned kNoHit = 0xFFFFFFFFu;
constexpr float kFarT = 1e20f;

struct TraceCounters {
    unsigned segments, calls, candidates, accepted, env, replay, replay_accepted, nodes, leaves;
};

template <int K>
PTIR_DEV void kbuf_clear(float (&kt)[K], unsigned (&kid)[K]) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
        kt[j] = kFarT;
        kid[j] = kNoHit;
    }
}

// number of filled slots (a filled slot has a distance below kFarT)
template <int K>
PTIR_DEV unsigned kbuf_count(const float (&kt)[K]) {
    unsigned c = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) c += kt[j] < kFarT ? 1u : 0u;
    return c;
}

// sorted insertion; an entry equal to an existing distance goes behind it (a NaN goes nowhere).
// Measured against a version that finds the slot by K independent compares and a tree sum and
// moves every slot from it: the step chain here was 4 % faster in the intersection stage.
template <int K>
PTIR_DEV void kbuf_insert(float (&kt)[K], unsigned (&kid)[K], float t, unsigned id) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const bool lt = t < kt[j];
        const float tt = kt[j];
        const unsigned ii = kid[j];
        kt[j] = lt ? t : tt;
        kid[j] = lt ? id : ii;
        t = lt ? tt : t;
        id = lt ? ii : id;
    }
}

// sorted insertion that returns the entry pushed out of a full buffer (id kNoHit when none; the
// entry itself when it goes nowhere)
template <int K>
PTIR_DEV void kbuf_insert_evict(float (&kt)[K], unsigned (&kid)[K], float t, unsigned id, float& et, unsigned& eid) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const bool lt = t < kt[j];
        const float tt = kt[j];
        const unsigned ii = kid[j];
        kt[j] = lt ? t : tt;
        kid[j] = lt ? id : ii;
        t = lt ? tt : t;
        id = lt ? ii : id;
    }
    et = t;
    eid = id;
}

// ray vs AABB slab interval (inverse direction precomputed; NaNs from 0*inf are ignored by fmin/fmax)
PTIR_DEV void slab(float3 lo, float3 hi, float3 o, float3 inv, float& t0, float& t1) {
    const float ax = (lo.x - o.x) * inv.x, bx = (hi.x - o.x) * inv.x;
    const float ay = (lo.y - o.y) * inv.y, by = (hi.y - o.y) * inv.y;
    const float az = (lo.z - o.z) * inv.z, bz = (hi.z - o.z) * inv.z;
    t0 = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
    t1 = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
}

// three-input minimum / maximum (one instruction on sm_100a); a NaN input is ignored
PTIR_DEV float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
PTIR_DEV float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// The instance intersection of the reference (intersectInstanceParticle,
// gaussianParticles.cuh:484-500) for the object-space ray (od, dd): the closest approach to the
// centre t* = -(od . dd) / |dd|^2 within (tmin, tmax), at a squared distance (over |dd|^2) below 9.
PTIR_DEV bool instance_hit(float3 od, float3 dd, float tmin, float tmax, float& ts) {
    const float den = 1.0f / dot(dd, dd);
    ts = -dot(od, dd) * den;
    if (!(ts > tmin && ts < tmax)) return false;
    const float3 c = cross(normalize_or_keep(dd), od);
    return dot(c, c) * den < 9.0f;
}

// Exact instance test of leaf record p against ray (o, d) over (tmin, min(tend, cut)): true with
// the candidate's distance and Gaussian id when it is one. The reference's any-hit traversal
// invokes its intersection program only for instances whose unit box the ray crosses within the
// current interval, so the box test is part of the candidate test.
PTIR_DEV bool leaf_candidate(const AccelView& A, int p, float3 o, float3 d, float tmin, float tend, float cut,
                             float& ts_out, unsigned& id_out, float floor = -kFarT) {
    const float4* rec = A.leaves + 4 * (size_t)p;
    const float4 r0 = __ldg(rec + 0), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
    const float3 od = make_float3(r0.x * o.x + r0.y * o.y + r0.z * o.z + r0.w,
                                  r1.x * o.x + r1.y * o.y + r1.z * o.z + r1.w,
                                  r2.x * o.x + r2.y * o.y + r2.z * o.z + r2.w);
    const float3 dd = make_float3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z,
                                  r2.x * d.x + r2.y * d.y + r2.z * d.z);
    // the three conditions of a candidate, cheapest rejection first: the closest approach's
    // interval, the object-space unit box within [tmin, tend] (which rejects most of the rest), then
    // the perpendicular distance of instance_hit (almost never the deciding one)
    const float den = 1.0f / dot(dd, dd);
    const float ts = -dot(od, dd) * den;
    if (!(ts > tmin && ts >= floor && ts < fminf(tend, cut))) return false;
    const float3 inv = make_float3(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    float b0, b1;
    slab(f3(-1.0f), f3(1.0f), od, inv, b0, b1);
    if (fmaxf(b0, tmin) > fminf(b1, tend)) return false;
    const float3 c = cross(normalize_or_keep(dd), od);
    if (!(dot(c, c) * den < 9.0f)) return false;
    ts_out = ts;
    id_out = __float_as_uint(__ldg(&rec[3].x));
    return true;
}

// exact instance test of leaf record p, inserted into the k-buffer when it is a candidate: as its
// Gaussian id, or with kLeafIndex as the leaf record's index (leaf_gaussian maps it to the id).
// A seeded call passes its cap, a continued one its floor.
template <int K, bool kLeafIndex = false, class Ids>
PTIR_DEV void test_leaf(const AccelView& A, int p, float3 o, float3 d, float tmin, float tend, float (&kt)[K],
                        Ids& kid, float cap = kFarT, float floor = -kFarT) {
    float ts;
    unsigned gid;
    if (leaf_candidate(A, p, o, d, tmin, tend, fminf(kt[K - 1], cap), ts, gid, floor))
        kbuf_insert(kt, kid, ts, kLeafIndex ? (unsigned)p : gid);
}

// Gaussian id of leaf record p
PTIR_DEV unsigned leaf_gaussian(const AccelView& A, unsigned p) { return __float_as_uint(__ldg(&A.leaves[4 * (size_t)p + 3].x)); }

// Whether the ray crosses the unit instance box of leaf record p within [tmin, tend]: the part of the
// candidate test that depends on the call's interval (a candidate of an earlier call that passes it
// with a later tmin is a candidate of that later call too)
PTIR_DEV bool leaf_box_hit(const AccelView& A, unsigned p, float3 o, float3 d, float tmin, float tend) {
    const float4* rec = A.leaves + 4 * (size_t)p;
    const float4 r0 = __ldg(rec + 0), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
    const float3 od = make_float3(r0.x * o.x + r0.y * o.y + r0.z * o.z + r0.w,
                                  r1.x * o.x + r1.y * o.y + r1.z * o.z + r1.w,
                                  r2.x * o.x + r2.y * o.y + r2.z * o.z + r2.w);
    const float3 dd = make_float3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z,
                                  r2.x * d.x + r2.y * d.y + r2.z * d.z);
    const float3 inv = make_float3(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    float b0, b1;
    slab(f3(-1.0f), f3(1.0f), od, inv, b0, b1);
    return fmaxf(b0, tmin) <= fminf(b1, tend);
}

// A trace call in progress: the next node to visit and the stack depth (the stack itself is
// the caller's: kStackDepth StackEntry, each a node index and its entry distance, so that a push
// or a pop is one 8-byte local store or load; measured 1 % faster in the intersection stage than
// separate index and distance arrays).
struct TraceState {
    float3 inv;
    float tmin, tend;
    float slack;  // cull_slack / |d|: a child's cull distance is its box entry less slack * its kmax
    float cap;    // seeded calls: the cut until the k-buffer is full (kFarT: none)
    float floor;  // continued calls: candidates have t* >= floor, subtrees ending before it are culled
    int node, sp;
    // resumed calls: which of the lane's two frontier buffers is read, its entries, the next one to
    // read, and the entries set aside so far for the next call (more than the capacity: overflowed)
    int fr_cur, fr_n, fr_pos, fr_next;
};

// A lane's two frontier buffers of `cap` (code, lower bound) entries each: code >= 0 a 4-wide
// node, else the leaf record ~code.
struct Frontier {
    uint2* buf;
    int cap;
};

// set a subtree or leaf aside for the segment's next call
PTIR_DEV void defer(const Frontier& F, TraceState& t, int code, float lower) {
    if (t.fr_next < F.cap) F.buf[(1 - t.fr_cur) * F.cap + t.fr_next] = make_uint2((unsigned)code, __float_as_uint(lower));
    ++t.fr_next;
}

// the next frontier entry that can still hold a candidate nearer than the K-th distance (the
// others go to the next frontier); false when the frontier is exhausted
template <int K>
PTIR_DEV bool pull(const Frontier& F, TraceState& t, const float (&kt)[K], int& code) {
    while (t.fr_pos < t.fr_n) {
        const uint2 e = F.buf[t.fr_cur * F.cap + t.fr_pos];
        ++t.fr_pos;
        const float lower = __uint_as_float(e.y);
        if (lower <= kt[K - 1]) {
            code = (int)e.x;
            return true;
        }
        defer(F, t, (int)e.x, lower);
    }
    return false;
}

// Leaf record p against ray (o, d) over (tmin, tend) for a resumable call: 1 when it is a
// candidate (ts, id set), 2 when its t* lies in (tmin, tend) but not before `cut`, so that a
// later call of the segment may take it (ts set), 0 when it is a candidate of no call of the
// segment from this one on. Decides as leaf_candidate does.
PTIR_DEV int leaf_candidate3(const AccelView& A, int p, float3 o, float3 d, float tmin, float tend, float cut,
                             float& ts_out, unsigned& id_out) {
    const float4* rec = A.leaves + 4 * (size_t)p;
    const float4 r0 = __ldg(rec + 0), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
    const float3 od = make_float3(r0.x * o.x + r0.y * o.y + r0.z * o.z + r0.w,
                                  r1.x * o.x + r1.y * o.y + r1.z * o.z + r1.w,
                                  r2.x * o.x + r2.y * o.y + r2.z * o.z + r2.w);
    const float3 dd = make_float3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z,
                                  r2.x * d.x + r2.y * d.y + r2.z * d.z);
    const float den = 1.0f / dot(dd, dd);
    const float ts = -dot(od, dd) * den;
    if (!(ts > tmin && ts < tend)) return 0;
    ts_out = ts;
    if (!(ts < cut)) return 2;
    const float3 inv = make_float3(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    float b0, b1;
    slab(f3(-1.0f), f3(1.0f), od, inv, b0, b1);
    if (fmaxf(b0, tmin) > fminf(b1, tend)) return 0;
    const float3 c = cross(normalize_or_keep(dd), od);
    if (!(dot(c, c) * den < 9.0f)) return 0;
    id_out = __float_as_uint(__ldg(&rec[3].x));
    return 1;
}

// exact instance test of leaf record p in a resumable call (the k-buffer holds leaf record
// indices): a candidate is inserted, and what it pushes out of the buffer, or a leaf whose t*
// lies past the K-th distance, is set aside for the next call
template <int K>
PTIR_DEV void test_leaf_resume(const AccelView& A, int p, float3 o, float3 d, TraceState& t, float (&kt)[K],
                               unsigned (&kid)[K], const Frontier& F) {
    float ts;
    unsigned gid;
    const int r = leaf_candidate3(A, p, o, d, t.tmin, t.tend, kt[K - 1], ts, gid);
    if (r == 2) {
        defer(F, t, ~p, ts);
    } else if (r == 1) {
        float et;
        unsigned ep;
        kbuf_insert_evict(kt, kid, ts, (unsigned)p, et, ep);
        if (ep != kNoHit) defer(F, t, ~(int)ep, et);
    }
}

// Start a trace call of ray (o, d) over (tmin, tend). Returns true when node visits remain
// (trace_step), false when (kt, kid) is already final. With kResume (k-buffer of leaf record
// indices, frontier F) a call with `resume` continues from what the segment's previous call set
// aside, unless that overflowed F; a segment's first call starts from the root. `cap` seeds the
// call's cut (trace_continue takes over a seeded call that ends with its k-buffer not full).
template <int K, bool kLeafIndex = false, bool kResume = false, class Ids>
PTIR_DEV bool trace_start(const AccelView& A, float3 o, float3 d, float tmin, float tend, float (&kt)[K], Ids& kid,
                          TraceState& t, TraceCounters& ctr, const Frontier* F = nullptr, bool resume = false,
                          float cap = kFarT) {
    t.cap = cap;
    t.floor = -kFarT;
    static_assert(!kResume || kLeafIndex, "resumed calls keep leaf record indices in the k-buffer");
    if constexpr (kResume) {
        if (!resume) {
            t.fr_cur = 0;
            t.fr_n = 0;
            t.fr_pos = 0;
            t.fr_next = 0;
        }
    }
    kbuf_clear(kt, kid);
    ++ctr.calls;
    if (A.n <= 0) return false;
    if (A.n == 1) {
        ++ctr.leaves;
        test_leaf<K, kLeafIndex>(A, 0, o, d, tmin, tend, kt, kid);
        ctr.candidates += kbuf_count(kt);
        return false;
    }
    t.inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    t.tmin = tmin;
    t.tend = tend;
    t.slack = A.cull_slack > 0.0f ? A.cull_slack / sqrtf(dot(d, d)) : 0.0f;
    t.node = 0;
    t.sp = 0;
    if constexpr (kResume) {
        if (resume && t.fr_next <= F->cap) {
            t.fr_cur = 1 - t.fr_cur;
            t.fr_n = t.fr_next;
            t.fr_pos = 0;
            t.fr_next = 0;
            int code;
            if (!pull(*F, t, kt, code)) return false;  // nothing was set aside: no candidate remains
            t.node = code;
        } else {
            t.fr_n = 0;  // the previous call overflowed its frontier: from the root, recording anew
            t.fr_pos = 0;
            t.fr_next = 0;
        }
    }
    return true;
}

// One 4-wide node visit between its box tests and its descent, so that the leaf children can be
// tested in between (in the lane, or by the whole warp).
struct NodeVisit {
    int ch[4];           // children: >= 0 node, kNoChild empty, else leaf ~c
    float t0[4], key[4]; // cull distance (clipped entry, less the slack), visit order key
    unsigned hits;       // children whose box the ray crosses and whose cull distance is before t_K
};

// Box tests of the node t.node. Returns the mask of leaf children to test. With kResume the
// children whose box the ray crosses past the K-th distance are set aside in F. Without kSlack
// the cull slack (exact candidates) is not applied: a kernel built so holds neither its registers
// nor the kmax load.
template <int K, bool kResume = false, bool kSlack = true>
PTIR_DEV unsigned visit_node(const AccelView& A, float3 o, TraceState& t, const float (&kt)[K], NodeVisit& v,
                             TraceCounters& ctr, const Frontier* F = nullptr) {
    const float3 inv = t.inv;
    const float tmin = t.tmin, tend = t.tend;
    ++ctr.nodes;
    const float4* nd = A.nodes + 8 * (size_t)t.node;
    // near and far plane rows of each axis from the direction's signs (rows: lo.x lo.y lo.z
    // hi.x hi.y hi.z), so each slab interval needs no min / max of its two plane distances
    const int rx = inv.x >= 0.0f ? 0 : 3, ry = inv.y >= 0.0f ? 1 : 4, rz = inv.z >= 0.0f ? 2 : 5;
    const float4 nx = __ldg(nd + rx), ny = __ldg(nd + ry), nz = __ldg(nd + rz);
    const float4 fx = __ldg(nd + (3 - rx)), fy = __ldg(nd + (5 - ry)), fz = __ldg(nd + (7 - rz));
    const float4 cc = __ldg(nd + 6);
    float sl[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if constexpr (kSlack) {
        if (t.slack > 0.0f) {
            const float4 km = __ldg(nd + 7);
            sl[0] = km.x * t.slack; sl[1] = km.y * t.slack; sl[2] = km.z * t.slack; sl[3] = km.w * t.slack;
        }
    }
    const float nxa[4] = {nx.x, nx.y, nx.z, nx.w}, nya[4] = {ny.x, ny.y, ny.z, ny.w};
    const float nza[4] = {nz.x, nz.y, nz.z, nz.w}, fxa[4] = {fx.x, fx.y, fx.z, fx.w};
    const float fya[4] = {fy.x, fy.y, fy.z, fy.w}, fza[4] = {fz.x, fz.y, fz.z, fz.w};
    v.ch[0] = __float_as_int(cc.x);
    v.ch[1] = __float_as_int(cc.y);
    v.ch[2] = __float_as_int(cc.z);
    v.ch[3] = __float_as_int(cc.w);
    v.hits = 0;
    unsigned leaves = 0;
    // plane distance (p - o) / d as one FMA, p * inv - o * inv. A NaN (0 * inf, or inf - inf for a
    // ray parallel to an axis) leaves the axis unbounded, so the test stays conservative.
    const float3 oi = make_float3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        // clipped slab interval [a, b]
        const float a = max3f(fmaf(nxa[k], inv.x, -oi.x), fmaf(nya[k], inv.y, -oi.y),
                              fmaxf(fmaf(nza[k], inv.z, -oi.z), tmin));
        const float b = min3f(fmaf(fxa[k], inv.x, -oi.x), fmaf(fya[k], inv.y, -oi.y),
                              fminf(fmaf(fza[k], inv.z, -oi.z), tend));
        v.t0[k] = kSlack ? a - sl[k] : a;
        // visit order: the clipped entry, with a sixteenth of the clipped extent added so that
        // boxes that all enter at tmin (those containing the origin) go shorter first. Measured
        // on 2 views of 512x384x4 (1M Gaussians): the step took 163.7 ms with this key, 171.0
        // with the entry alone, 168.0 with a quarter of the extent and 178.6 with the middle.
        v.key[k] = 15.0f * a + b;
        // a continued call also culls what ends before its floor (t* lies in the box interval,
        // up to the grazing case; with the slack, within the slack of it)
        const bool crossed = v.ch[k] != kNoChild && a <= b && (kSlack ? b + sl[k] : b) >= t.floor;
        const bool h = crossed && v.t0[k] <= fminf(kt[K - 1], t.cap);
        if constexpr (kResume) {
            if (crossed && !h) defer(*F, t, v.ch[k], v.t0[k]);
        }
        v.hits |= h ? (1u << k) : 0u;
        leaves |= (h && v.ch[k] < 0) ? (1u << k) : 0u;
    }
    return leaves;
}

// Descent after the leaf tests: into the first internal child by key still in front of the K-th
// distance, the others pushed largest key first; else the next stacked subtree that can still hold
// a nearer candidate (then, with kResume, the next frontier entry that can). Returns false when
// no node visit remains. With kResume what is passed over for the K-th distance is set aside.
template <int K, bool kResume = false>
PTIR_DEV bool descend(TraceState& t, const NodeVisit& v, const float (&kt)[K], StackEntry* stack,
                      unsigned* err, TraceCounters& ctr, const Frontier* F = nullptr) {
    int sp = t.sp;
    int node = t.node;
    int best = -1;
    float bkey = 3.0e38f;
    unsigned inner = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool cand = ((v.hits >> k) & 1u) && v.ch[k] >= 0;
        const bool h = cand && v.t0[k] <= fminf(kt[K - 1], t.cap);
        if constexpr (kResume) {
            if (cand && !h) defer(*F, t, v.ch[k], v.t0[k]);  // passed over after the leaf tests
        }
        inner |= h ? (1u << k) : 0u;
        if (h && v.key[k] < bkey) {
            bkey = v.key[k];
            best = k;
        }
    }
    if (best >= 0) {
        inner &= ~(1u << best);
        const int np = __popc(inner);
        if (sp + np > kStackDepth) {
            atomicOr(err, kErrStackOverflow);
            return false;
        }
        while (inner) {
            // largest remaining key first
            int far = -1;
            float fkey = -3.0e38f;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if ((inner >> k) & 1u && v.key[k] > fkey) {
                    fkey = v.key[k];
                    far = k;
                }
            }
            inner &= ~(1u << far);
            stack[sp] = make_int2(far == 0 ? v.ch[0] : (far == 1 ? v.ch[1] : (far == 2 ? v.ch[2] : v.ch[3])),
                                  __float_as_int(far == 0 ? v.t0[0]
                                                          : (far == 1 ? v.t0[1] : (far == 2 ? v.t0[2] : v.t0[3]))));
            ++sp;
        }
        node = best == 0 ? v.ch[0] : (best == 1 ? v.ch[1] : (best == 2 ? v.ch[2] : v.ch[3]));
    } else {
        // pop the next subtree that can still hold a candidate nearer than the K-th
        bool found = false;
        while (sp > 0) {
            --sp;
            const StackEntry e = stack[sp];
            if (__int_as_float(e.y) <= fminf(kt[K - 1], t.cap)) {
                node = e.x;
                found = true;
                break;
            }
            if constexpr (kResume) defer(*F, t, e.x, __int_as_float(e.y));
        }
        if constexpr (kResume) {
            if (!found) found = pull(*F, t, kt, node);
        }
        if (!found) return false;
    }
    t.sp = sp;
    t.node = node;
    return true;
}

// One 4-wide node visit of a trace call with its leaf tests in the lane (with kResume, t.node < 0
// is a leaf set aside by the previous call, tested instead). Returns false when the call is
// complete.
template <int K, bool kLeafIndex = false, bool kResume = false, bool kSlack = true, class Ids>
PTIR_DEV bool trace_step(const AccelView& A, float3 o, float3 d, TraceState& t, float (&kt)[K], Ids& kid,
                         StackEntry* stack, unsigned* err, TraceCounters& ctr, const Frontier* F = nullptr) {
    NodeVisit v;
    unsigned leaves;
    if (kResume && t.node < 0) {
        ++ctr.leaves;
        if constexpr (kResume) test_leaf_resume(A, ~t.node, o, d, t, kt, kid, *F);
        v.ch[0] = v.ch[1] = v.ch[2] = v.ch[3] = kNoChild;
        v.hits = 0;
        leaves = 0;
    } else {
        leaves = visit_node<K, kResume, kSlack>(A, o, t, kt, v, ctr, F);
    }
    // leaf children: one test call site, looping over the mask
    while (leaves) {
        const int k = __ffs(leaves) - 1;
        leaves &= leaves - 1;
        const int c = k == 0 ? v.ch[0] : (k == 1 ? v.ch[1] : (k == 2 ? v.ch[2] : v.ch[3]));
        ++ctr.leaves;
        if constexpr (kResume) test_leaf_resume(A, ~c, o, d, t, kt, kid, *F);
        else test_leaf<K, kLeafIndex>(A, ~c, o, d, t.tmin, t.tend, kt, kid, t.cap, t.floor);
    }
    if (descend<K, kResume>(t, v, kt, stack, err, ctr, F)) return true;
    ctr.candidates += kbuf_count(kt);
    return false;
}

// A seeded call that ended with its k-buffer not full holds every candidate before its cap: it
// goes on from the root for the candidates from the cap on, keeping its k-buffer (the same call:
// its candidates are counted when it ends again).
template <int K>
PTIR_DEV void trace_continue(TraceState& t, const float (&kt)[K], TraceCounters& ctr) {
    ctr.candidates -= kbuf_count(kt);
    t.floor = t.cap;
    t.cap = kFarT;
    t.node = 0;
    t.sp = 0;
}

// Fill (kt, kid) with the K nearest candidates of ray (o, d) in (tmin, tend).
// `stack` holds kStackDepth entries.
template <int K>
PTIR_DEV void trace_kbuf(const AccelView& A, float3 o, float3 d, float tmin, float tend, float (&kt)[K],
                         unsigned (&kid)[K], StackEntry* stack, unsigned* err, TraceCounters& ctr) {
    TraceState t;
    if (!trace_start(A, o, d, tmin, tend, kt, kid, t, ctr)) return;
    while (trace_step(A, o, d, t, kt, kid, stack, err, ctr)) {
    }
}

}  // namespace ptir
