// BVH build and refit over the Gaussian instance boxes of the tracer: Morton-sorted leaves, then
// PLOC (Meister and Bittner 2018, the default) or the Karras hierarchy (Karras 2012, "Maximizing
// Parallelism in the Construction of BVHs, Octrees, and k-d Trees"), collapsed to 4-wide nodes.
//
//   1. prep      per Gaussian: kernel support scale, world->instance map, instance AABB
//                (the instance transform of threedgptir_tracer/src/particlePrimitives.cu:543-610)
//   2. bounds    scene AABB = union of the instance AABBs (two-pass reduction)
//   3. morton    60-bit extended Morton key: AABB centre and size
//   4. sort      key/id radix sort (radix_sort.cuh: stable LSD, 8-bit digits)
//   5. gather    leaf records in key order
//   6. hierarchy internal nodes from the sorted keys (ties broken by position), or PLOC
//                (agglomerative clustering by surface area over the sorted leaves)
//   7. refit     bottom-up child boxes with arrival counters
//   8. collapse  4-wide nodes, greedy by surface area (rebuild only)
//   9. emit      the 4-wide node records the traversal reads
// A refit (rebuild == false, same n) redoes 1, 2, 5, 7 and 9 in the stored leaf order and topology.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "radix_sort.cuh"
#include "../../include/ptir_b200.h"
#include "accel.h"
#include "storage.cuh"
#include "vecmath.cuh"

namespace ptir {

namespace {

constexpr int kReduceBlocks = 296;  // 2 x 148 SMs
constexpr int kReduceThreads = 256;

// kernel support radius in units of the particle scale (particlePrimitives.cu:27-51)
__device__ float support_scale(float density, float min_response, int clamping, float degree) {
    const float modulation = clamping ? density : 1.0f;
    const float min_resp = fminf(min_response / modulation, 0.97f);
    if (degree < 0.0f) {
        const float k = fabsf(degree);
        const float s = 1.0f / powf(3.0f, k);
        return powf((1.0f / (logf(min_resp) - 1.0f) + 1.0f) / s, 1.0f / k);
    }
    if (degree == 0.0f) return ((1.0f - min_resp) / 3.0f) / -0.329630334487f;
    const float a = -4.5f / powf(3.0f, degree);
    return powf(logf(min_resp) / a, 1.0f / degree);
}

__global__ void k_prep(int n, const float* __restrict__ pos, const float* __restrict__ rot, const float* __restrict__ scl,
                       const float* __restrict__ dns, AccelBuildOptions opt, float4* __restrict__ inst,
                       float4* __restrict__ box) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    // the attributes as the tracer stores them (rounded in 16-bit storage)
    const auto in = [&](const float* v, int i) { return round_storage(opt.storage, v[i]); };
    const float4 q = make_float4(in(rot, 4 * g), in(rot, 4 * g + 1), in(rot, 4 * g + 2), in(rot, 4 * g + 3));
    const Mat3 R = quat_r(q);
    const float ks = support_scale(in(dns, g), opt.min_response, opt.density_clamping, opt.kernel_degree);
    const float3 k = make_float3(in(scl, 3 * g), in(scl, 3 * g + 1), in(scl, 3 * g + 2)) * ks;
    const float3 mu = make_float3(in(pos, 3 * g), in(pos, 3 * g + 1), in(pos, 3 * g + 2));
    // world = R diag(k) obj + mu  =>  obj = diag(1/k) R^T (world - mu)
    const float3 a0 = make_float3(R.r0.x, R.r1.x, R.r2.x) * (1.0f / k.x);
    const float3 a1 = make_float3(R.r0.y, R.r1.y, R.r2.y) * (1.0f / k.y);
    const float3 a2 = make_float3(R.r0.z, R.r1.z, R.r2.z) * (1.0f / k.z);
    const float kmax = fmaxf(k.x, fmaxf(k.y, k.z));
    float4* rec = inst + 4 * (size_t)g;
    rec[0] = make_float4(a0.x, a0.y, a0.z, -dot(a0, mu));
    rec[1] = make_float4(a1.x, a1.y, a1.z, -dot(a1, mu));
    rec[2] = make_float4(a2.x, a2.y, a2.z, -dot(a2, mu));
    rec[3] = make_float4(__uint_as_float((unsigned)g), kmax, 0.0f, 0.0f);
    // AABB of the 8 transformed corners of [-1,1]^3 (particlePrimitives.cu:585-594)
    float3 lo = f3(3.0e38f), hi = f3(-3.0e38f);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float3 corner = make_float3((c & 4) ? 1.0f : -1.0f, (c & 2) ? 1.0f : -1.0f, (c & 1) ? 1.0f : -1.0f);
        const float3 v = mul_rows(R, corner * k) + mu;
        lo = fmin3(lo, v);
        hi = fmax3(hi, v);
    }
    box[2 * (size_t)g] = make_float4(lo.x, lo.y, lo.z, kmax);
    box[2 * (size_t)g + 1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
}

__device__ void block_minmax(float3& lo, float3& hi) {
    __shared__ float3 slo[kReduceThreads / 32], shi[kReduceThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        lo.x = fminf(lo.x, __shfl_xor_sync(0xFFFFFFFFu, lo.x, off));
        lo.y = fminf(lo.y, __shfl_xor_sync(0xFFFFFFFFu, lo.y, off));
        lo.z = fminf(lo.z, __shfl_xor_sync(0xFFFFFFFFu, lo.z, off));
        hi.x = fmaxf(hi.x, __shfl_xor_sync(0xFFFFFFFFu, hi.x, off));
        hi.y = fmaxf(hi.y, __shfl_xor_sync(0xFFFFFFFFu, hi.y, off));
        hi.z = fmaxf(hi.z, __shfl_xor_sync(0xFFFFFFFFu, hi.z, off));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        slo[w] = lo;
        shi[w] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < kReduceThreads / 32; ++i) {
            lo = fmin3(lo, slo[i]);
            hi = fmax3(hi, shi[i]);
        }
    }
}

__global__ void k_bounds_partial(int n, const float4* __restrict__ box, float4* __restrict__ partial) {
    float3 lo = f3(3.0e38f), hi = f3(-3.0e38f);
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const float4 a = box[2 * (size_t)g], b = box[2 * (size_t)g + 1];
        lo = fmin3(lo, make_float3(a.x, a.y, a.z));
        hi = fmax3(hi, make_float3(b.x, b.y, b.z));
    }
    block_minmax(lo, hi);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        partial[2 * blockIdx.x + 1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    }
}

__global__ void k_bounds_final(int parts, const float4* __restrict__ partial, float4* __restrict__ bounds) {
    float3 lo = f3(3.0e38f), hi = f3(-3.0e38f);
    for (int i = threadIdx.x; i < parts; i += blockDim.x) {
        const float4 a = partial[2 * i], b = partial[2 * i + 1];
        lo = fmin3(lo, make_float3(a.x, a.y, a.z));
        hi = fmax3(hi, make_float3(b.x, b.y, b.z));
    }
    block_minmax(lo, hi);
    if (threadIdx.x == 0) {
        bounds[0] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        bounds[1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    }
}

// spread the low 16 bits of v to every fourth bit
__device__ unsigned long long spread4(unsigned long long v) {
    v &= 0xFFFFull;
    v = (v | (v << 24)) & 0x000000FF000000FFull;
    v = (v | (v << 12)) & 0x000F000F000F000Full;
    v = (v | (v << 6)) & 0x0303030303030303ull;
    v = (v | (v << 3)) & 0x1111111111111111ull;
    return v;
}

// Extended Morton key (Vinkler, Bittner and Havran 2017, "Extended Morton Codes for High
// Performance Bounding Volume Hierarchy Construction"): the AABB centre within the scene bounds
// and the AABB diagonal relative to the scene diagonal (weighted by kSizeWeight) as a fourth
// axis, 15 bits each, interleaved x y z size from the top. Large Gaussians then group apart
// from small neighbours instead of inflating every ancestor of a small-Gaussian subtree.
constexpr float kSizeWeight = 0.5f;
constexpr int kKeyBits = 60;

__global__ void k_morton(int n, const float4* __restrict__ box, const float4* __restrict__ bounds,
                         unsigned long long* __restrict__ keys, unsigned* __restrict__ ids) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const float4 a = box[2 * (size_t)g], b = box[2 * (size_t)g + 1];
    const float4 lo = bounds[0], hi = bounds[1];
    const float3 c = make_float3(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z));
    const float3 ext = make_float3(fmaxf(hi.x - lo.x, 1e-30f), fmaxf(hi.y - lo.y, 1e-30f), fmaxf(hi.z - lo.z, 1e-30f));
    const float3 e = make_float3(b.x - a.x, b.y - a.y, b.z - a.z);
    const float scale = 32767.0f;  // 2^15 - 1
    const unsigned long long qx = (unsigned long long)fminf(fmaxf((c.x - lo.x) / ext.x, 0.0f) * scale, scale);
    const unsigned long long qy = (unsigned long long)fminf(fmaxf((c.y - lo.y) / ext.y, 0.0f) * scale, scale);
    const unsigned long long qz = (unsigned long long)fminf(fmaxf((c.z - lo.z) / ext.z, 0.0f) * scale, scale);
    const float size = kSizeWeight * sqrtf(dot(e, e) / dot(ext, ext));
    const unsigned long long qs = (unsigned long long)fminf(fmaxf(size, 0.0f) * scale, scale);
    keys[g] = (spread4(qx) << 3) | (spread4(qy) << 2) | (spread4(qz) << 1) | spread4(qs);
    ids[g] = (unsigned)g;
}

__global__ void k_gather(int n, const unsigned* __restrict__ order, const float4* __restrict__ inst, float4* __restrict__ leaves) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned g = order[i];
    const float4* src = inst + 4 * (size_t)g;
    float4* dst = leaves + 4 * (size_t)i;
    dst[0] = src[0];
    dst[1] = src[1];
    dst[2] = src[2];
    dst[3] = src[3];
}

// common-prefix length of sorted keys i and j; equal keys fall back to the positions
__device__ __forceinline__ int prefix(const unsigned long long* __restrict__ keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz((unsigned)(i ^ j));
    return __clzll(a ^ b);
}

__global__ void k_hierarchy(int n, const unsigned long long* __restrict__ keys, float4* __restrict__ nodes, int* __restrict__ parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int dir = (prefix(keys, n, i, i + 1) - prefix(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = prefix(keys, n, i, i - dir);
    int lmax = 2;
    while (prefix(keys, n, i, i + lmax * dir) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (prefix(keys, n, i, i + (l + t) * dir) > dmin) l += t;
    const int j = i + l * dir;
    const int dnode = prefix(keys, n, i, j);
    int s = 0;
    for (int div = 2;; div <<= 1) {
        const int t = (l + div - 1) / div;
        if (prefix(keys, n, i, i + (s + t) * dir) > dnode) s += t;
        if (t <= 1) break;
    }
    const int split = i + s * dir + min(dir, 0);
    const int lo = min(i, j), hi = max(i, j);
    const int left = (lo == split) ? ~split : split;
    const int right = (hi == split + 1) ? ~(split + 1) : split + 1;
    nodes[4 * (size_t)i + 3] = make_float4(__int_as_float(left), __int_as_float(right), 0.0f, 0.0f);
    parent[left < 0 ? (n - 1) + ~left : left] = i;
    parent[right < 0 ? (n - 1) + ~right : right] = i;
    if (i == 0) parent[0] = -1;
}

// ---------------------------------------------------------------------------------------
// PLOC (Meister and Bittner 2018, "Parallel Locally-Ordered Clustering for Bounding Volume
// Hierarchy Construction"): an agglomerative build over the leaves in key order, in place of
// k_hierarchy. Every iteration, each cluster finds among the kPlocRadius clusters on either side
// of it in the current list the one whose union with it has the smallest box surface area;
// mutual nearest neighbours merge into a new binary node that takes the left one's place, and
// the list is compacted. Equal areas go to the nearer position in the list, then to the pair
// whose lower index is even, then to the smaller index: with the area this orders all pairs
// strictly, so the smallest pair of the list is always mutual and every iteration merges at
// least one pair, and coincident Gaussians (equal boxes) pair up all at once. Node indices are handed out from n - 2 down, so the last merge (the root)
// is node 0 as in the Karras hierarchy, and the binary nodes go through the same refit,
// collapse and emit.
constexpr int kPlocRadius = 16;
constexpr int kPlocThreads = 256;
constexpr int kPlocScanThreads = 1024;
constexpr int kPlocBatch = 4;  // iterations launched between reads of the cluster count

// surface area (halved) of the union of two boxes; the same value whichever box comes first
__device__ __forceinline__ float ploc_area(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    const float ex = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    const float ey = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    const float ez = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    const float a = ex * ey + ey * ez + ez * ex;
    return a == a ? a : INFINITY;  // a NaN box still pairs with someone
}

// the leaves in key order as the first clusters (cid ~i: leaf i), their instance boxes
__global__ void k_ploc_init(int n, const float4* __restrict__ box, const unsigned* __restrict__ order,
                            int* __restrict__ cid, float4* __restrict__ cb, unsigned* __restrict__ count,
                            unsigned* __restrict__ next_node) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *count = (unsigned)n;
        *next_node = (unsigned)(n - 1);
    }
    if (i >= n) return;
    const unsigned g = order[i];
    cid[i] = ~i;
    cb[2 * (size_t)i] = box[2 * (size_t)g];
    cb[2 * (size_t)i + 1] = box[2 * (size_t)g + 1];
}

// nearest neighbour of every cluster within kPlocRadius positions (-1 when alone)
__global__ void __launch_bounds__(kPlocThreads) k_ploc_nn(const unsigned* __restrict__ count_p,
                                                          const float4* __restrict__ cb, int* __restrict__ nn) {
    constexpr int kSpan = kPlocThreads + 2 * kPlocRadius;
    __shared__ float4 slo[kSpan], shi[kSpan];
    const int count = (int)*count_p;
    const int b0 = blockIdx.x * kPlocThreads;
    if (b0 >= count) return;
    for (int k = threadIdx.x; k < kSpan; k += kPlocThreads) {
        const int j = b0 - kPlocRadius + k;
        if (j >= 0 && j < count) {
            slo[k] = cb[2 * (size_t)j];
            shi[k] = cb[2 * (size_t)j + 1];
        }
    }
    __syncthreads();
    const int i = b0 + threadIdx.x;
    if (i >= count) return;
    const int s = threadIdx.x + kPlocRadius;
    const float4 lo = slo[s], hi = shi[s];
    int best = -1, bdist = 0, bmin = 0;
    float barea = INFINITY;
    for (int d = -kPlocRadius; d <= kPlocRadius; ++d) {
        const int j = i + d;
        if (d == 0 || j < 0 || j >= count) continue;
        const float a = ploc_area(lo, hi, slo[s + d], shi[s + d]);
        const int dist = d < 0 ? -d : d, mn = min(i, j);
        // pairs ordered by (area, list distance, parity of the lower index, lower index): equal
        // boxes (coincident Gaussians) then pair up as (0,1), (2,3), ... and halve every
        // iteration, where the smaller index alone would merge one pair an iteration
        const bool better = best < 0 || a < barea ||
                            (a == barea && (dist < bdist || (dist == bdist && ((mn & 1) < (bmin & 1) ||
                                                                               ((mn & 1) == (bmin & 1) && mn < bmin)))));
        if (better) {
            barea = a;
            best = j;
            bdist = dist;
            bmin = mn;
        }
    }
    nn[i] = best;
}

// number of clusters of a block that stay in the list (all but the right one of each merged pair)
__device__ __forceinline__ unsigned ploc_block_keep(bool keep, unsigned* wsum) {
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, keep);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    return bal;
}

// merge of mutual nearest neighbours: a binary node (left, right) with its parent links, in the
// left cluster's place; per block the number of clusters kept
__global__ void __launch_bounds__(kPlocThreads) k_ploc_merge(int n, const unsigned* __restrict__ count_p,
                                                             const int* __restrict__ nn, int* __restrict__ cid,
                                                             float4* __restrict__ cb, float4* __restrict__ nodes,
                                                             int* __restrict__ parent, unsigned* __restrict__ next_node,
                                                             unsigned* __restrict__ blk) {
    __shared__ unsigned wsum[kPlocThreads / 32];
    const int count = (int)*count_p;
    const int b0 = blockIdx.x * kPlocThreads;
    if (b0 >= count) return;
    const int i = b0 + threadIdx.x;
    bool keep = false;
    if (i < count) {
        const int j = nn[i];
        const bool mutual = j >= 0 && nn[j] == i;
        keep = !(mutual && j < i);
        if (mutual && i < j) {
            const int idx = (int)atomicSub(next_node, 1u) - 1;
            const int l = cid[i], r = cid[j];
            nodes[4 * (size_t)idx + 3] = make_float4(__int_as_float(l), __int_as_float(r), 0.0f, 0.0f);
            parent[l < 0 ? (n - 1) + ~l : l] = idx;
            parent[r < 0 ? (n - 1) + ~r : r] = idx;
            const float4 alo = cb[2 * (size_t)i], ahi = cb[2 * (size_t)i + 1];
            const float4 blo = cb[2 * (size_t)j], bhi = cb[2 * (size_t)j + 1];
            cb[2 * (size_t)i] = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f);
            cb[2 * (size_t)i + 1] = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f);
            cid[i] = idx;
        }
    }
    ploc_block_keep(keep, wsum);
    if (threadIdx.x == 0) {
        unsigned s = 0;
        for (int w = 0; w < kPlocThreads / 32; ++w) s += wsum[w];
        blk[blockIdx.x] = s;
    }
}

// exclusive scan of the per-block counts in one block; the total is the next cluster count
__global__ void __launch_bounds__(kPlocScanThreads) k_ploc_scan(const unsigned* __restrict__ count_p,
                                                                unsigned* __restrict__ blk,
                                                                unsigned* __restrict__ count_out) {
    __shared__ unsigned wsum[kPlocScanThreads / 32];
    const int count = (int)*count_p;
    const int nb = (count + kPlocThreads - 1) / kPlocThreads;
    const unsigned ln = threadIdx.x & 31u, w = threadIdx.x >> 5;
    unsigned carry = 0;
    for (int base = 0; base < nb; base += kPlocScanThreads) {
        const int k = base + (int)threadIdx.x;
        const unsigned v = k < nb ? blk[k] : 0u;
        unsigned x = v;  // inclusive scan within the warp
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (ln >= (unsigned)o) x += y;
        }
        if (ln == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            unsigned t = wsum[ln];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xFFFFFFFFu, t, o);
                if (ln >= (unsigned)o) t += y;
            }
            wsum[ln] = t;
        }
        __syncthreads();
        if (k < nb) blk[k] = carry + (w > 0 ? wsum[w - 1] : 0u) + x - v;
        carry += wsum[kPlocScanThreads / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *count_out = carry;
}

// the kept clusters, in order, into the other list
__global__ void __launch_bounds__(kPlocThreads) k_ploc_compact(const unsigned* __restrict__ count_p,
                                                               const int* __restrict__ nn, const int* __restrict__ cid,
                                                               const float4* __restrict__ cb,
                                                               const unsigned* __restrict__ blk, int* __restrict__ cid_out,
                                                               float4* __restrict__ cb_out) {
    __shared__ unsigned wsum[kPlocThreads / 32];
    const int count = (int)*count_p;
    const int b0 = blockIdx.x * kPlocThreads;
    if (b0 >= count) return;
    const int i = b0 + threadIdx.x;
    bool keep = false;
    if (i < count) {
        const int j = nn[i];
        keep = !(j >= 0 && j < i && nn[j] == i);
    }
    const unsigned bal = ploc_block_keep(keep, wsum);
    unsigned off = blk[blockIdx.x] + __popc(bal & ((1u << (threadIdx.x & 31u)) - 1u));
    for (unsigned w = 0; w < (threadIdx.x >> 5); ++w) off += wsum[w];
    if (keep) {
        cid_out[off] = cid[i];
        cb_out[2 * (size_t)off] = cb[2 * (size_t)i];
        cb_out[2 * (size_t)off + 1] = cb[2 * (size_t)i + 1];
    }
}

// box and kmax of child c of the hierarchy
__device__ __forceinline__ void child_box(const float4* __restrict__ sbox_unsorted, const unsigned* __restrict__ order,
                                          const float4* nodes, int c, float3& lo, float3& hi, float& kmax) {
    if (c < 0) {
        const unsigned g = order[~c];
        const float4 a = sbox_unsorted[2 * (size_t)g], b = sbox_unsorted[2 * (size_t)g + 1];
        lo = make_float3(a.x, a.y, a.z);
        hi = make_float3(b.x, b.y, b.z);
        kmax = a.w;
        return;
    }
    const float4* nd = nodes + 4 * (size_t)c;
    const float4 a = __ldcg(nd), b = __ldcg(nd + 1), e = __ldcg(nd + 2), f = __ldcg(nd + 3);
    lo = fmin3(make_float3(a.x, a.y, a.z), make_float3(b.z, b.w, e.x));
    hi = fmax3(make_float3(a.w, b.x, b.y), make_float3(e.y, e.z, e.w));
    kmax = fmaxf(f.z, f.w);
}

__global__ void k_refit(int n, const float4* __restrict__ box, const unsigned* __restrict__ order, float4* nodes,
                        const int* __restrict__ parent, unsigned* arrivals) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int p = parent[(n - 1) + j];
    while (p >= 0) {
        __threadfence();
        if (atomicAdd(arrivals + p, 1u) == 0u) return;  // the sibling subtree is not finished yet
        __threadfence();
        float4* nd = nodes + 4 * (size_t)p;
        const float4 f = __ldcg(nd + 3);
        const int left = __float_as_int(f.x), right = __float_as_int(f.y);
        float3 llo, lhi, rlo, rhi;
        float lk, rk;
        child_box(box, order, nodes, left, llo, lhi, lk);
        child_box(box, order, nodes, right, rlo, rhi, rk);
        __stcg(nd + 0, make_float4(llo.x, llo.y, llo.z, lhi.x));
        __stcg(nd + 1, make_float4(lhi.y, lhi.z, rlo.x, rlo.y));
        __stcg(nd + 2, make_float4(rlo.z, rhi.x, rhi.y, rhi.z));
        __stcg(nd + 3, make_float4(f.x, f.y, lk, rk));
        p = parent[p];
    }
}

// Collapse of the binary tree into 4-wide nodes, greedy by surface area: a 4-wide node starts
// from a binary node's two children and, while it has fewer than four, replaces the internal child
// with the largest box surface by that child's own two children. Its remaining internal children
// become the roots of further 4-wide nodes. Against taking every binary node at even depth with its
// grandchildren, this fills nodes whose children include leaves; a simulation of the tracer's
// traversal on the 1M-Gaussian scene (camera rays, k-buffer 16) measured 11 % fewer node visits.
// One block, level by level: wide node w has binary root wroot[w]; its children are recorded as
// binary references (wsrc, for refits) and as wide-node indices or leaves (wchild).
constexpr int kCollapseThreads = 1024;

__device__ __forceinline__ float box_area(float3 lo, float3 hi) {
    const float3 e = hi - lo;
    return e.x * e.y + e.y * e.z + e.z * e.x;
}

// child `side` (0 left, 1 right) of binary node record nd: its link and box
__device__ __forceinline__ void record_child(const float4* nd, int side, int& c, float3& lo, float3& hi) {
    const float4 a = nd[0], b = nd[1], e = nd[2], f = nd[3];
    if (side == 0) {
        c = __float_as_int(f.x);
        lo = make_float3(a.x, a.y, a.z);
        hi = make_float3(a.w, b.x, b.y);
    } else {
        c = __float_as_int(f.y);
        lo = make_float3(b.z, b.w, e.x);
        hi = make_float3(e.y, e.z, e.w);
    }
}

__global__ void __launch_bounds__(kCollapseThreads) k_collapse4(int n, const float4* __restrict__ nodes,
                                                                int* __restrict__ wroot, int* __restrict__ wsrc,
                                                                int* __restrict__ wchild, unsigned* __restrict__ wcount) {
    __shared__ unsigned tail;
    if (threadIdx.x == 0) {
        tail = 1u;
        wroot[0] = 0;
    }
    __syncthreads();
    unsigned head = 0;
    // every wave consumes at least one wide node and each binary node roots at most one, so the
    // loop ends after at most n - 1 waves
    for (int wave = 0; wave < n; ++wave) {
        const unsigned end = tail;
        __syncthreads();
        for (unsigned w = head + threadIdx.x; w < end; w += blockDim.x) {
            int ref[4];
            float area[4];
            int cnt = 2;
            const float4* nb = nodes + 4 * (size_t)wroot[w];
            for (int side = 0; side < 2; ++side) {
                float3 lo, hi;
                record_child(nb, side, ref[side], lo, hi);
                area[side] = box_area(lo, hi);
            }
            while (cnt < 4) {
                int best = -1;
                float barea = -1.0f;
                for (int k = 0; k < cnt; ++k)
                    if (ref[k] >= 0 && area[k] > barea) {
                        barea = area[k];
                        best = k;
                    }
                if (best < 0) break;
                const float4* nc = nodes + 4 * (size_t)ref[best];
                float3 lo, hi;
                record_child(nc, 0, ref[best], lo, hi);
                area[best] = box_area(lo, hi);
                record_child(nc, 1, ref[cnt], lo, hi);
                area[cnt] = box_area(lo, hi);
                ++cnt;
            }
            for (int k = 0; k < 4; ++k) {
                int src = kNoChild, link = kNoChild;
                if (k < cnt) {
                    src = link = ref[k];
                    if (ref[k] >= 0) {
                        const unsigned idx = atomicAdd(&tail, 1u);
                        wroot[idx] = ref[k];
                        link = (int)idx;
                    }
                }
                wsrc[4 * (size_t)w + k] = src;
                wchild[4 * (size_t)w + k] = link;
            }
        }
        __syncthreads();
        head = end;
        if (head == tail) break;
    }
    if (threadIdx.x == 0) *wcount = tail;
}

// 4-wide node w: the boxes of its children (binary references wsrc, from the refitted binary
// nodes or the instance boxes of leaves) and with each the largest kernel support radius (kmax)
// under it
__global__ void k_emit4(int n, const float4* __restrict__ nodes, const float4* __restrict__ sbox,
                        const unsigned* __restrict__ order, const int* __restrict__ wsrc,
                        const int* __restrict__ wchild, const unsigned* __restrict__ wcount,
                        float4* __restrict__ nodes4) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n - 1 || (unsigned)w >= *wcount) return;
    float lx[4], ly[4], lz[4], hx[4], hy[4], hz[4], km[4];
    int ch[4];
    for (int k = 0; k < 4; ++k) {
        const int src = wsrc[4 * (size_t)w + k];
        ch[k] = wchild[4 * (size_t)w + k];
        if (src == kNoChild) {
            lx[k] = ly[k] = lz[k] = hx[k] = hy[k] = hz[k] = km[k] = 0.0f;
            continue;
        }
        float3 lo, hi;
        child_box(sbox, order, nodes, src, lo, hi, km[k]);
        lx[k] = lo.x; ly[k] = lo.y; lz[k] = lo.z;
        hx[k] = hi.x; hy[k] = hi.y; hz[k] = hi.z;
    }
    float4* out = nodes4 + 8 * (size_t)w;
    out[0] = make_float4(lx[0], lx[1], lx[2], lx[3]);
    out[1] = make_float4(ly[0], ly[1], ly[2], ly[3]);
    out[2] = make_float4(lz[0], lz[1], lz[2], lz[3]);
    out[3] = make_float4(hx[0], hx[1], hx[2], hx[3]);
    out[4] = make_float4(hy[0], hy[1], hy[2], hy[3]);
    out[5] = make_float4(hz[0], hz[1], hz[2], hz[3]);
    out[6] = make_float4(__int_as_float(ch[0]), __int_as_float(ch[1]), __int_as_float(ch[2]), __int_as_float(ch[3]));
    out[7] = make_float4(km[0], km[1], km[2], km[3]);
}

template <class T>
cudaError_t grow(T*& ptr, size_t count, cudaStream_t s) {
    if (ptr) {
        cudaError_t e = cudaFreeAsync(ptr, s);
        if (e != cudaSuccess) return e;
        ptr = nullptr;
    }
    return cudaMallocAsync(reinterpret_cast<void**>(&ptr), count * sizeof(T), s);
}

// The binary nodes and parent links of a PLOC build over the n > 1 leaves in key order
// (st.ids[1]). Its scratch lives for the build only. Iterations are launched kPlocBatch at a
// time, then the cluster count is read back; at most n - 1 iterations are needed, since each
// merges at least one pair.
cudaError_t ploc_build(AccelState& st, int n, cudaStream_t s, std::string& err) {
    cudaError_t e = cudaSuccess;
    if (!st.ploc_host) {
        e = cudaMallocHost(reinterpret_cast<void**>(&st.ploc_host), 2 * sizeof(unsigned));
        if (e != cudaSuccess) {
            err = std::string("cudaMallocHost: ") + cudaGetErrorString(e);
            return e;
        }
    }
    const int nb = (n + kPlocThreads - 1) / kPlocThreads;
    // cluster boxes [2][2n] float4, cluster ids [2][n], neighbours [n], block counts [nb], counters [4]
    const size_t box_bytes = 2 * sizeof(float4) * (size_t)n;
    const size_t bytes = 2 * box_bytes + (3 * (size_t)n + (size_t)nb + 4) * sizeof(int) + 256;
    char* scratch = nullptr;
    e = cudaMallocAsync(reinterpret_cast<void**>(&scratch), bytes, s);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync (PLOC scratch): ") + cudaGetErrorString(e);
        return e;
    }
    float4* cb[2] = {reinterpret_cast<float4*>(scratch), reinterpret_cast<float4*>(scratch + box_bytes)};
    int* cid[2] = {reinterpret_cast<int*>(scratch + 2 * box_bytes), reinterpret_cast<int*>(scratch + 2 * box_bytes) + n};
    int* nn = cid[1] + n;
    unsigned* blk = reinterpret_cast<unsigned*>(nn + n);
    unsigned* cnt = blk + nb;  // [0], [1]: cluster counts of the two lists; [2]: next node index
    unsigned* next_node = cnt + 2;
    k_ploc_init<<<nb, kPlocThreads, 0, s>>>(n, st.box, st.ids[1], cid[0], cb[0], cnt, next_node);
    e = cudaGetLastError();
    int cur = 0;
    for (long long it = 0; e == cudaSuccess;) {
        for (int b = 0; b < kPlocBatch; ++b, ++it) {
            k_ploc_nn<<<nb, kPlocThreads, 0, s>>>(cnt + cur, cb[cur], nn);
            k_ploc_merge<<<nb, kPlocThreads, 0, s>>>(n, cnt + cur, nn, cid[cur], cb[cur], st.nodes, st.parent, next_node,
                                                     blk);
            k_ploc_scan<<<1, kPlocScanThreads, 0, s>>>(cnt + cur, blk, cnt + 1 - cur);
            k_ploc_compact<<<nb, kPlocThreads, 0, s>>>(cnt + cur, nn, cid[cur], cb[cur], blk, cid[1 - cur], cb[1 - cur]);
            cur = 1 - cur;
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(st.ploc_host, cnt + cur, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(st.ploc_host + 1, next_node, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            err = std::string("PLOC iteration: ") + cudaGetErrorString(e);
            break;
        }
        if (st.ploc_host[0] <= 1u) {
            if (st.ploc_host[1] != 0u) {  // n - 1 merges hand out every node index
                err = "PLOC ended with " + std::to_string(st.ploc_host[1]) + " node indices unused";
                e = cudaErrorUnknown;
            }
            break;
        }
        if (it > (long long)n + kPlocBatch) {
            err = "PLOC did not converge";
            e = cudaErrorUnknown;
            break;
        }
    }
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(st.parent, 0xFF, sizeof(int), s);  // the root (node 0) has no parent
        if (e != cudaSuccess) err = std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
    }
    const cudaError_t f = cudaFreeAsync(scratch, s);
    if (e == cudaSuccess && f != cudaSuccess) {
        err = std::string("cudaFreeAsync (PLOC scratch): ") + cudaGetErrorString(f);
        e = f;
    }
    return e;
}

}  // namespace

cudaError_t accel_build(AccelState& st, const AccelBuildOptions& opt, const float* pos, const float* rot,
                        const float* scl, const float* dns, int n, bool rebuild, cudaStream_t s, std::string& err) {
    cudaError_t e = cudaSuccess;
#define PTIR_TRY(expr)                                     \
    do {                                                   \
        e = (expr);                                        \
        if (e != cudaSuccess) {                            \
            err = std::string(#expr) + ": " + cudaGetErrorString(e); \
            st.valid = false;                              \
            return e;                                      \
        }                                                  \
    } while (0)
    if (n < 0) {
        err = "negative Gaussian count";
        return cudaErrorInvalidValue;
    }
    const bool refit = !rebuild && st.valid && st.n == n && n > 1;
    if (!refit && n > 1 && opt.builder == kBuilderPloc) {
        // refuse before anything is enqueued: a PLOC rebuild synchronises its stream
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        PTIR_TRY(cudaStreamIsCapturing(s, &cap));
        if (cap != cudaStreamCaptureStatusNone) {
            err = "a PLOC rebuild reads its cluster count back between iterations and cannot be captured in a CUDA "
                  "graph: rebuild before the capture and refit inside it";
            return cudaErrorStreamCaptureUnsupported;
        }
    }
    if (!st.bounds) PTIR_TRY(cudaMallocAsync(reinterpret_cast<void**>(&st.bounds), 2 * sizeof(float4), s));
    if (!st.partial) PTIR_TRY(cudaMallocAsync(reinterpret_cast<void**>(&st.partial), 2 * kReduceBlocks * sizeof(float4), s));
    st.n = n;
    if (n == 0) {
        st.valid = true;
        return cudaSuccess;
    }
    if ((size_t)n > st.capacity) {
        const size_t cap = (size_t)n;
        PTIR_TRY(grow(st.inst, 4 * cap, s));
        PTIR_TRY(grow(st.box, 2 * cap, s));
        PTIR_TRY(grow(st.keys[0], cap, s));
        PTIR_TRY(grow(st.keys[1], cap, s));
        PTIR_TRY(grow(st.ids[0], cap, s));
        PTIR_TRY(grow(st.ids[1], cap, s));
        PTIR_TRY(grow(st.leaves, 4 * cap, s));
        PTIR_TRY(grow(st.nodes, 4 * (cap > 1 ? cap - 1 : 1), s));
        PTIR_TRY(grow(st.parent, 2 * cap, s));
        PTIR_TRY(grow(st.arrivals, cap, s));
        PTIR_TRY(grow(st.wroot, cap, s));
        PTIR_TRY(grow(st.wsrc, 4 * cap, s));
        PTIR_TRY(grow(st.wchild, 4 * cap, s));
        if (!st.wcount) PTIR_TRY(cudaMallocAsync(reinterpret_cast<void**>(&st.wcount), sizeof(unsigned), s));
        PTIR_TRY(grow(st.nodes4, 8 * (cap > 1 ? cap - 1 : 1), s));
        st.capacity = cap;
        st.valid = false;
    }
    const int T = 256;
    const unsigned blocks = (unsigned)((n + T - 1) / T);
    k_prep<<<blocks, T, 0, s>>>(n, pos, rot, scl, dns, opt, st.inst, st.box);
    PTIR_TRY(cudaGetLastError());
    k_bounds_partial<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, st.box, st.partial);
    k_bounds_final<<<1, kReduceThreads, 0, s>>>(kReduceBlocks, st.partial, st.bounds);
    PTIR_TRY(cudaGetLastError());
    if (!refit) {
        k_morton<<<blocks, T, 0, s>>>(n, st.box, st.bounds, st.keys[0], st.ids[0]);
        PTIR_TRY(cudaGetLastError());
        const size_t need = radix_sort_temp_bytes<unsigned long long>(n);
        if (need > st.sort_temp_bytes) {
            if (st.sort_temp) PTIR_TRY(cudaFreeAsync(st.sort_temp, s));
            st.sort_temp = nullptr;
            PTIR_TRY(cudaMallocAsync(&st.sort_temp, need, s));
            st.sort_temp_bytes = need;
        }
        PTIR_TRY(radix_sort_pairs<unsigned long long>(st.sort_temp, st.sort_temp_bytes, st.keys[0], st.keys[1], st.ids[0],
                                                      st.ids[1], n, 0, kKeyBits, s));
        if (n > 1 && opt.builder == kBuilderPloc) {
            std::string perr;
            e = ploc_build(st, n, s, perr);
            if (e != cudaSuccess) {
                err = perr;
                st.valid = false;
                return e;
            }
        } else if (n > 1) {
            const unsigned iblocks = (unsigned)((n - 1 + T - 1) / T);
            k_hierarchy<<<iblocks, T, 0, s>>>(n, st.keys[1], st.nodes, st.parent);
            PTIR_TRY(cudaGetLastError());
        }
    }
    k_gather<<<blocks, T, 0, s>>>(n, st.ids[1], st.inst, st.leaves);
    PTIR_TRY(cudaGetLastError());
    if (n > 1) {
        PTIR_TRY(cudaMemsetAsync(st.arrivals, 0, sizeof(unsigned) * (size_t)(n - 1), s));
        k_refit<<<blocks, T, 0, s>>>(n, st.box, st.ids[1], st.nodes, st.parent, st.arrivals);
        PTIR_TRY(cudaGetLastError());
        if (!refit) {
            // the 4-wide topology (kept by refits)
            k_collapse4<<<1, kCollapseThreads, 0, s>>>(n, st.nodes, st.wroot, st.wsrc, st.wchild, st.wcount);
            PTIR_TRY(cudaGetLastError());
        }
        k_emit4<<<(unsigned)((n - 1 + T - 1) / T), T, 0, s>>>(n, st.nodes, st.box, st.ids[1], st.wsrc, st.wchild,
                                                             st.wcount, st.nodes4);
        PTIR_TRY(cudaGetLastError());
    }
    st.valid = true;
    return cudaSuccess;
#undef PTIR_TRY
}

void accel_free(AccelState& st) {
    auto rel = [](void* p) {
        if (p) cudaFree(p);
    };
    rel(st.inst);
    rel(st.box);
    rel(st.keys[0]);
    rel(st.keys[1]);
    rel(st.ids[0]);
    rel(st.ids[1]);
    rel(st.leaves);
    rel(st.nodes);
    rel(st.parent);
    rel(st.arrivals);
    rel(st.partial);
    rel(st.bounds);
    rel(st.sort_temp);
    rel(st.wroot);
    rel(st.wsrc);
    rel(st.wchild);
    rel(st.wcount);
    rel(st.nodes4);
    if (st.ploc_host) cudaFreeHost(st.ploc_host);
    st = AccelState();
}

// ---------------------------------------------------------------------------------------
// Allocation-free scene bounds (ptir_instance_bounds_noalloc).
//
// Some callers cannot allocate device memory once they are running. One example is a
// renderer or serving process that reserves all device memory for its own pool at start-up.
// Another is a plugin whose host forbids device allocation after initialisation. For them a
// cudaMalloc either fails, or synchronises the whole device in the middle of a frame.
// This entry point gives them the scene AABB of the Gaussians' instance boxes, the box every
// trace clips its rays to, with no allocation at all. Its only scratch is the file-scope array
// below.
//
// Limits. The array holds one partial AABB per block of kNoAllocItemsPerBlock Gaussians, for at
// most kNoAllocMaxBlocks blocks: N <= 8,388,608 Gaussians, 128 KiB of scratch. Every GPU that
// loads the library holds the array until the process exits. All calls share it. A call
// writes the partial of every block it launches before reading it, so nothing needs clearing
// between calls. Two calls that overlap on the GPU (unordered streams) race on it. The array's
// device address is looked up once per device and kept, so the library must not be used across
// a cudaDeviceReset (which unloads it from the device). With N = 0 the result is the empty box,
// lo = +3e38 and hi = -3e38 on every axis, which clips every ray to an empty interval.
namespace {

constexpr int kNoAllocItemsPerBlock = 2048;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float4 g_noalloc_partial[2 * kNoAllocMaxBlocks];

// the instance AABB of k_prep (8 transformed corners of [-1,1]^3), computed in place from the
// attributes as the tracer stores them (rounded to 16 bits with BF16 / FP16 storage, as k_prep does)
__device__ void instance_aabb(int g, const float* __restrict__ pos, const float* __restrict__ rot,
                              const float* __restrict__ scl, const float* __restrict__ dns, const AccelBuildOptions& opt,
                              float3& lo, float3& hi) {
    const auto in = [&](const float* v, int i) { return round_storage(opt.storage, v[i]); };
    const float4 q = make_float4(in(rot, 4 * g), in(rot, 4 * g + 1), in(rot, 4 * g + 2), in(rot, 4 * g + 3));
    const Mat3 R = quat_r(q);
    const float ks = support_scale(in(dns, g), opt.min_response, opt.density_clamping, opt.kernel_degree);
    const float3 k = make_float3(in(scl, 3 * g), in(scl, 3 * g + 1), in(scl, 3 * g + 2)) * ks;
    const float3 mu = make_float3(in(pos, 3 * g), in(pos, 3 * g + 1), in(pos, 3 * g + 2));
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float3 corner = make_float3((c & 4) ? 1.0f : -1.0f, (c & 2) ? 1.0f : -1.0f, (c & 1) ? 1.0f : -1.0f);
        const float3 v = mul_rows(R, corner * k) + mu;
        lo = fmin3(lo, v);
        hi = fmax3(hi, v);
    }
}

// one partial AABB per block of kNoAllocItemsPerBlock consecutive Gaussians
__global__ void k_bounds_noalloc_partial(int n, const float* __restrict__ pos, const float* __restrict__ rot,
                                         const float* __restrict__ scl, const float* __restrict__ dns,
                                         AccelBuildOptions opt, float4* __restrict__ partial) {
    const int first = blockIdx.x * kNoAllocItemsPerBlock;
    const int last = min(n, first + kNoAllocItemsPerBlock);
    float3 lo = f3(3.0e38f), hi = f3(-3.0e38f);
    for (int g = first + threadIdx.x; g < last; g += blockDim.x) instance_aabb(g, pos, rot, scl, dns, opt, lo, hi);
    block_minmax(lo, hi);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        partial[2 * blockIdx.x + 1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    }
}

std::mutex g_noalloc_mutex;
float4* g_noalloc_device_ptr[kMaxDevices] = {};

void set_error(char* buf, int len, const std::string& msg) {
    if (!buf || len <= 0) return;
    const size_t n = std::min<size_t>(msg.size(), (size_t)len - 1);
    std::memcpy(buf, msg.data(), n);
    buf[n] = '\0';
}

}  // namespace

}  // namespace ptir

extern "C" int ptir_instance_bounds_noalloc(float kernel_degree, float kernel_min_response, int32_t density_clamping,
                                            int32_t storage, const float* pos, const float* rot, const float* scl,
                                            const float* dns, int32_t n, float* bounds_out, void* stream, char* err,
                                            int32_t err_len) {
    using namespace ptir;
    if (storage != PTIR_STORAGE_FP32 && storage != PTIR_STORAGE_BF16 && storage != PTIR_STORAGE_FP16) {
        set_error(err, err_len, "storage must be PTIR_STORAGE_FP32, _BF16 or _FP16");
        return PTIR_EINVAL;
    }
    if (n < 0) {
        set_error(err, err_len, "negative Gaussian count");
        return PTIR_EINVAL;
    }
    if (n > kNoAllocItemsPerBlock * kNoAllocMaxBlocks) {
        set_error(err, err_len, "n = " + std::to_string(n) + " exceeds the allocation-free limit of " +
                                    std::to_string(kNoAllocItemsPerBlock * kNoAllocMaxBlocks) + " Gaussians");
        return PTIR_EINVAL;
    }
    if (!bounds_out || (reinterpret_cast<uintptr_t>(bounds_out) & 15u) != 0) {
        set_error(err, err_len, "bounds_out must be a 16-byte aligned device buffer of 8 floats");
        return PTIR_EINVAL;
    }
    if (n > 0 && (!pos || !rot || !scl || !dns)) {
        set_error(err, err_len, "null particle pointer");
        return PTIR_EINVAL;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(err, err_len, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return PTIR_ECUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(err, err_len, "device index " + std::to_string(dev) + " exceeds the limit of " +
                                    std::to_string(kMaxDevices) + " devices");
        return PTIR_EINVAL;
    }
    float4* scratch = nullptr;
    {
        // set-up, once per device (with that device current): the array's device address
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_device_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_partial);
            if (e != cudaSuccess) {
                set_error(err, err_len, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return PTIR_ECUDA;
            }
            g_noalloc_device_ptr[dev] = static_cast<float4*>(p);
        }
        scratch = g_noalloc_device_ptr[dev];
    }
    const AccelBuildOptions opt{kernel_degree, kernel_min_response, density_clamping, (unsigned)storage};
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int blocks = (n + kNoAllocItemsPerBlock - 1) / kNoAllocItemsPerBlock;
    if (blocks > 0) k_bounds_noalloc_partial<<<blocks, kReduceThreads, 0, s>>>(n, pos, rot, scl, dns, opt, scratch);
    k_bounds_final<<<1, kReduceThreads, 0, s>>>(blocks, scratch, reinterpret_cast<float4*>(bounds_out));
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(err, err_len, std::string("launch: ") + cudaGetErrorString(e));
        return PTIR_ECUDA;
    }
    set_error(err, err_len, "");
    return PTIR_OK;
}
