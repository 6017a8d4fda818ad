// Stable LSD radix sort of (key, value) pairs on the device: the sort of the LBVH build (60-bit
// Morton keys) and of the wavefront's ray order (28-bit keys).
//
// Each pass sorts by one 8-bit digit. The items are split into warp tiles of kRsItemsPerWarp
// consecutive items. A pass is three steps:
//   1. count: every warp counts its tile's digits in a shared-memory histogram and writes the
//      256 counts, digit-major (counts[digit * tiles + tile]);
//   2. scan: an exclusive prefix sum over those counts, so that counts[digit * tiles + tile]
//      becomes where the tile's first item of that digit goes (reduce, scan of the block sums,
//      apply);
//   3. scatter: every warp walks its tile again in order, 32 items at a time. Lanes with the same
//      digit find each other with __match_any_sync; an item's place is its digit's running
//      offset plus the number of same-digit lanes before it, and the highest of them advances
//      the running offset. Items keep their order within a digit, so the sort is stable.
// The passes alternate between the output arrays and the scratch copies so that the last pass
// writes the outputs.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ptir {

constexpr int kRsBits = 8;
constexpr int kRsBuckets = 1 << kRsBits;
constexpr int kRsWarps = 8;                // warps per block of the count and scatter kernels
constexpr int kRsItemsPerWarp = 2048;      // consecutive items of a warp tile
constexpr int kRsScanThreads = 1024;
constexpr int kRsScanItems = 4;            // per thread of a scan block
constexpr int kRsScanTile = kRsScanThreads * kRsScanItems;

inline long long rs_tiles(long long n) { return (n + kRsItemsPerWarp - 1) / kRsItemsPerWarp; }
inline long long rs_scan_blocks(long long m) { return (m + kRsScanTile - 1) / kRsScanTile; }

template <class Key>
__device__ __forceinline__ unsigned rs_digit(Key k, int shift, unsigned mask) {
    return (unsigned)(k >> shift) & mask;
}

template <class Key>
__global__ void __launch_bounds__(kRsWarps * 32) k_rs_count(const Key* __restrict__ keys, long long n, int shift,
                                                            unsigned mask, unsigned* __restrict__ counts,
                                                            long long tiles) {
    __shared__ unsigned hist[kRsWarps][kRsBuckets];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tile = (long long)blockIdx.x * kRsWarps + w;
    for (int d = lane; d < kRsBuckets; d += 32) hist[w][d] = 0u;
    __syncwarp();
    if (tile < tiles) {
        const long long begin = tile * kRsItemsPerWarp;
        const long long end = begin + kRsItemsPerWarp < n ? begin + kRsItemsPerWarp : n;
        for (long long i = begin + lane; i < end; i += 32) atomicAdd(&hist[w][rs_digit(keys[i], shift, mask)], 1u);
        __syncwarp();
        for (int d = lane; d < kRsBuckets; d += 32) counts[(long long)d * tiles + tile] = hist[w][d];
    }
}

// The scan kernels are static (internal linkage): every translation unit that sorts has its own.

// block sums of the scan tiles
static __global__ void __launch_bounds__(kRsScanThreads) k_rs_scan_reduce(const unsigned* __restrict__ v, long long m,
                                                                   unsigned* __restrict__ partial) {
    __shared__ unsigned warp_sums[kRsScanThreads / 32];
    const long long base = (long long)blockIdx.x * kRsScanTile;
    unsigned s = 0;
    for (int j = 0; j < kRsScanItems; ++j) {
        const long long i = base + (long long)j * kRsScanThreads + threadIdx.x;
        if (i < m) s += v[i];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned t = warp_sums[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xFFFFFFFFu, t, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = t;
    }
}

// exclusive scan of a block's kRsScanThreads values held one per thread; returns the total
static __device__ __forceinline__ unsigned rs_block_exclusive(unsigned x, unsigned* warp_sums, unsigned& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned inc = x;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sums[w] = inc;
    __syncthreads();
    if (w == 0) {
        unsigned t = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        warp_sums[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    total = warp_sums[(blockDim.x >> 5) - 1];
    const unsigned before = w > 0 ? warp_sums[w - 1] : 0u;
    __syncthreads();
    return before + inc - x;
}

// exclusive scan of the block sums, in place, by one block walking them in chunks
static __global__ void __launch_bounds__(kRsScanThreads) k_rs_scan_partials(unsigned* __restrict__ partial, long long nb) {
    __shared__ unsigned warp_sums[kRsScanThreads / 32];
    unsigned carry = 0;
    for (long long base = 0; base < nb; base += kRsScanThreads) {
        const long long i = base + threadIdx.x;
        const unsigned x = i < nb ? partial[i] : 0u;
        unsigned total;
        const unsigned ex = rs_block_exclusive(x, warp_sums, total);
        if (i < nb) partial[i] = carry + ex;
        carry += total;
    }
}

// exclusive scan of each tile, offset by its block's scanned sum
static __global__ void __launch_bounds__(kRsScanThreads) k_rs_scan_apply(unsigned* __restrict__ v, long long m,
                                                                  const unsigned* __restrict__ partial) {
    __shared__ unsigned warp_sums[kRsScanThreads / 32];
    const long long base = (long long)blockIdx.x * kRsScanTile;
    // each thread owns kRsScanItems consecutive values
    const long long first = base + (long long)threadIdx.x * kRsScanItems;
    unsigned x[kRsScanItems];
    unsigned sum = 0;
    for (int j = 0; j < kRsScanItems; ++j) {
        x[j] = first + j < m ? v[first + j] : 0u;
        sum += x[j];
    }
    unsigned total;
    unsigned run = partial[blockIdx.x] + rs_block_exclusive(sum, warp_sums, total);
    for (int j = 0; j < kRsScanItems; ++j) {
        if (first + j < m) v[first + j] = run;
        run += x[j];
    }
}

template <class Key>
__global__ void __launch_bounds__(kRsWarps * 32) k_rs_scatter(const Key* __restrict__ keys_in,
                                                              const unsigned* __restrict__ vals_in,
                                                              Key* __restrict__ keys_out, unsigned* __restrict__ vals_out,
                                                              long long n, int shift, unsigned mask,
                                                              const unsigned* __restrict__ offsets, long long tiles) {
    __shared__ unsigned run[kRsWarps][kRsBuckets];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tile = (long long)blockIdx.x * kRsWarps + w;
    if (tile >= tiles) return;  // whole warps leave together
    for (int d = lane; d < kRsBuckets; d += 32) run[w][d] = offsets[(long long)d * tiles + tile];
    __syncwarp();
    const unsigned below = (1u << lane) - 1u;
    const long long begin = tile * kRsItemsPerWarp;
    for (int c = 0; c < kRsItemsPerWarp; c += 32) {
        const long long i = begin + c + lane;
        const bool valid = i < n;
        Key k = Key(0);
        unsigned v = 0u;
        unsigned digit = kRsBuckets + (unsigned)lane;  // past the end: matches no other lane
        if (valid) {
            k = keys_in[i];
            v = vals_in[i];
            digit = rs_digit(k, shift, mask);
        }
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, digit);
        unsigned pos = 0u;
        if (valid) pos = run[w][digit] + (unsigned)__popc(peers & below);
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) run[w][digit] += (unsigned)__popc(peers);
        __syncwarp();
        if (valid) {
            keys_out[pos] = k;
            vals_out[pos] = v;
        }
        if (begin + c + 32 >= n) break;  // uniform: every lane sees the same bound
    }
}

// scratch bytes of radix_sort_pairs for n items with keys of type Key
template <class Key>
size_t radix_sort_temp_bytes(long long n) {
    const long long tiles = rs_tiles(n), m = (long long)kRsBuckets * tiles;
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return up(sizeof(Key) * (size_t)n) + up(sizeof(unsigned) * (size_t)n) + up(sizeof(unsigned) * (size_t)m) +
           up(sizeof(unsigned) * (size_t)rs_scan_blocks(m));
}

// Stable sort of (keys_in, vals_in) by bits [begin_bit, end_bit) of the keys into (keys_out,
// vals_out); `temp` holds radix_sort_temp_bytes<Key>(n) bytes.
template <class Key>
cudaError_t radix_sort_pairs(void* temp, size_t temp_bytes, const Key* keys_in, Key* keys_out,
                             const unsigned* vals_in, unsigned* vals_out, long long n, int begin_bit, int end_bit,
                             cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (temp_bytes < radix_sort_temp_bytes<Key>(n) || end_bit <= begin_bit || end_bit > (int)(8 * sizeof(Key)))
        return cudaErrorInvalidValue;
    const long long tiles = rs_tiles(n), m = (long long)kRsBuckets * tiles, nb = rs_scan_blocks(m);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    char* p = static_cast<char*>(temp);
    Key* alt_keys = reinterpret_cast<Key*>(p);
    p += up(sizeof(Key) * (size_t)n);
    unsigned* alt_vals = reinterpret_cast<unsigned*>(p);
    p += up(sizeof(unsigned) * (size_t)n);
    unsigned* counts = reinterpret_cast<unsigned*>(p);
    p += up(sizeof(unsigned) * (size_t)m);
    unsigned* partial = reinterpret_cast<unsigned*>(p);
    const int passes = (end_bit - begin_bit + kRsBits - 1) / kRsBits;
    const unsigned grid = (unsigned)((tiles + kRsWarps - 1) / kRsWarps);
    const Key* src_k = keys_in;
    const unsigned* src_v = vals_in;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = begin_bit + pass * kRsBits;
        const int bits = end_bit - shift < kRsBits ? end_bit - shift : kRsBits;
        const unsigned mask = (1u << bits) - 1u;
        // the last pass writes the outputs
        const bool to_out = ((passes - 1 - pass) & 1) == 0;
        Key* dst_k = to_out ? keys_out : alt_keys;
        unsigned* dst_v = to_out ? vals_out : alt_vals;
        k_rs_count<Key><<<grid, kRsWarps * 32, 0, s>>>(src_k, n, shift, mask, counts, tiles);
        k_rs_scan_reduce<<<(unsigned)nb, kRsScanThreads, 0, s>>>(counts, m, partial);
        k_rs_scan_partials<<<1, kRsScanThreads, 0, s>>>(partial, nb);
        k_rs_scan_apply<<<(unsigned)nb, kRsScanThreads, 0, s>>>(counts, m, partial);
        k_rs_scatter<Key><<<grid, kRsWarps * 32, 0, s>>>(src_k, src_v, dst_k, dst_v, n, shift, mask, counts, tiles);
        src_k = dst_k;
        src_v = dst_v;
    }
    return cudaGetLastError();
}

}  // namespace ptir
