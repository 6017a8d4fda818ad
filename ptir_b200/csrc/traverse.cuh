// Software LBVH traversal with a register k-buffer: the replacement for OptiX's
// optixTrace + __intersection__is + __anyhit__ah of the reference
// (threedgptir_tracer/include/3dgptir/kernels/cuda/pathTracer.cuh:58-113,
//  src/kernels/cuda/referenceOptix.cu:73-133, gaussianParticles.cuh:484-500).
//
// One call returns the K candidates with the smallest closest-approach parameter t* in
// (tmin, tend), ascending. A Gaussian is a candidate when its object-space ray hits the unit
// instance box [-1,1]^3 within [tmin, tend] and passes the perpendicular-distance test.
//
// Culling follows the reference's traversal: subtrees are culled by their instance-box AABBs
// against [tmin, t_K], where t_K is the K-th distance found so far (the reference's any-hit
// program shrinks the ray's tmax to the 16th distance). This returns the K nearest candidates
// except for a Gaussian whose closest approach lies before its own box entry (a ray grazing a
// box corner, where the kernel response is below the acceptance threshold): like the
// reference, it is then kept only if reached before t_K drops below its box entry.
#pragma once

#include "device_types.h"
#include "vecmath.cuh"

namespace ptir {

constexpr int kKBuf = 16;            // reference MaxNumHitPerTrace; the kernels also build K = 8 and 32
constexpr int kStackDepth = 64;      // traversal stack entries
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

// number of filled slots
template <int K>
PTIR_DEV unsigned kbuf_count(const unsigned (&kid)[K]) {
    unsigned c = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) c += kid[j] != kNoHit ? 1u : 0u;
    return c;
}

// sorted insertion; an entry equal to an existing distance goes behind it
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

// ray vs AABB slab interval (inverse direction precomputed; NaNs from 0*inf are ignored by fmin/fmax)
PTIR_DEV void slab(float3 lo, float3 hi, float3 o, float3 inv, float& t0, float& t1) {
    const float ax = (lo.x - o.x) * inv.x, bx = (hi.x - o.x) * inv.x;
    const float ay = (lo.y - o.y) * inv.y, by = (hi.y - o.y) * inv.y;
    const float az = (lo.z - o.z) * inv.z, bz = (hi.z - o.z) * inv.z;
    t0 = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
    t1 = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
}

// exact instance test of leaf record p
template <int K>
PTIR_DEV void test_leaf(const AccelView& A, int p, float3 o, float3 d, float tmin, float tend, float (&kt)[K],
                        unsigned (&kid)[K]) {
    const float4* rec = A.leaves + 4 * (size_t)p;
    const float4 r0 = __ldg(rec + 0), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
    const float3 od = make_float3(r0.x * o.x + r0.y * o.y + r0.z * o.z + r0.w,
                                  r1.x * o.x + r1.y * o.y + r1.z * o.z + r1.w,
                                  r2.x * o.x + r2.y * o.y + r2.z * o.z + r2.w);
    const float3 dd = make_float3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z,
                                  r2.x * d.x + r2.y * d.y + r2.z * d.z);
    const float dd2 = dot(dd, dd);
    const float den = 1.0f / dd2;
    const float ts = -dot(od, dd) * den;
    if (!(ts > tmin && ts < tend && ts < kt[K - 1])) return;
    // object-space unit box within [tmin, tend]
    const float3 inv = make_float3(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    float b0, b1;
    slab(f3(-1.0f), f3(1.0f), od, inv, b0, b1);
    if (fmaxf(b0, tmin) > fminf(b1, tend)) return;
    const float3 c = cross(normalize_or_keep(dd), od);
    if (!(dot(c, c) * den < 9.0f)) return;
    const unsigned gid = __float_as_uint(__ldg(&rec[3].x));
    kbuf_insert(kt, kid, ts, gid);
}

// Fill (kt, kid) with the K nearest candidates of ray (o, d) in (tmin, tend).
// `stack` holds kStackDepth node indices, `stack_t` their entry distances.
template <int K>
PTIR_DEV void trace_kbuf(const AccelView& A, float3 o, float3 d, float tmin, float tend, float (&kt)[K],
                         unsigned (&kid)[K], int* stack, float* stack_t, unsigned* err, TraceCounters& ctr) {
    kbuf_clear(kt, kid);
    ++ctr.calls;
    if (A.n <= 0) return;
    if (A.n == 1) {
        ++ctr.leaves;
        test_leaf(A, 0, o, d, tmin, tend, kt, kid);
        ctr.candidates += kbuf_count(kid);
        return;
    }
    const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    int sp = 0;
    int node = 0;
    while (true) {
        ++ctr.nodes;
        const float4* nd = A.nodes + 4 * (size_t)node;
        const float4 a = __ldg(nd + 0), b = __ldg(nd + 1), c = __ldg(nd + 2), e = __ldg(nd + 3);
        const int left = __float_as_int(e.x), right = __float_as_int(e.y);
        float l0, l1, r0, r1;
        slab(make_float3(a.x, a.y, a.z), make_float3(a.w, b.x, b.y), o, inv, l0, l1);
        slab(make_float3(b.z, b.w, c.x), make_float3(c.y, c.z, c.w), o, inv, r0, r1);
        l0 = fmaxf(l0, tmin);
        r0 = fmaxf(r0, tmin);
        l1 = fminf(l1, tend);
        r1 = fminf(r1, tend);
        const float cut = kt[K - 1];
        bool hl = l0 <= l1 && l0 <= cut;
        bool hr = r0 <= r1 && r0 <= cut;
        if (hl && left < 0) {
            ++ctr.leaves;
            test_leaf(A, ~left, o, d, tmin, tend, kt, kid);
            hl = false;
        }
        if (hr && right < 0) {
            ++ctr.leaves;
            test_leaf(A, ~right, o, d, tmin, tend, kt, kid);
            hr = false;
        }
        if (hl && hr) {
            // nearer middle of the clipped interval first: boxes that contain the origin all
            // enter at tmin, their extent along the ray tells them apart
            const bool lfirst = (l0 + l1) <= (r0 + r1);
            if (sp >= kStackDepth) {
                atomicOr(err, kErrStackOverflow);
                break;
            }
            stack[sp] = lfirst ? right : left;
            stack_t[sp] = lfirst ? r0 : l0;
            ++sp;
            node = lfirst ? left : right;
        } else if (hl) {
            node = left;
        } else if (hr) {
            node = right;
        } else {
            // pop the next subtree that can still hold a candidate nearer than the K-th
            bool found = false;
            while (sp > 0) {
                --sp;
                if (stack_t[sp] <= kt[K - 1]) {
                    node = stack[sp];
                    found = true;
                    break;
                }
            }
            if (!found) break;
        }
    }
    ctr.candidates += kbuf_count(kid);
}

}  // namespace ptir
