// Environment importance table for NEE built on the device: the reference's
// build_environment_alias_table (threedgrut/model/aliastable.py:244-297) with its Vose alias
// construction (aliastable.py:49-116), which the reference runs in a host Python loop.
//
//   1. weights  per cell: equirect maps are area-averaged to the table size (cube maps, H == 6W,
//               are used as they are); Rec.709 luminance of the finite positive RGB times the
//               cell's solid angle (float32; solid angles evaluated in float64)
//   2. total    float64 sum of the weights (fixed order); all-zero or non-finite totals fall back
//               to the solid angles as weights, as the reference does
//   3. pdf      weight / (total * solid angle), per steradian
//   4. alias    scaled = w * n / total in float64; the small (< 1) and large (>= 1) lists in index
//               order, then Vose's pairing popping from the ends, on one thread: the pairing order
//               is sequential by construction and fixes the table
#include <cmath>
#include <cstdint>

#include "../../include/ptir_b200.h"

namespace ptir {

namespace {

constexpr int kEnvThreads = 1024;

__device__ double solid_angle_equirect(int row, int h, int w) {
    const double pi = 3.14159265358979323846;
    const double e0 = ((double)row / h - 0.5) * pi, e1 = ((double)(row + 1) / h - 0.5) * pi;
    return fmax((2.0 * pi / w) * (sin(e1) - sin(e0)), 0.0);
}

__device__ double solid_angle_cube(int u, int v, int fs) {
    auto area = [](double x, double y) { return atan2(x * y, sqrt(x * x + y * y + 1.0)); };
    const double u0 = -1.0 + 2.0 * u / fs, u1 = -1.0 + 2.0 * (u + 1) / fs;
    const double v0 = -1.0 + 2.0 * v / fs, v1 = -1.0 + 2.0 * (v + 1) / fs;
    return fmax(area(u1, v1) - area(u0, v1) - area(u1, v0) + area(u0, v0), 0.0);
}

// cell weights (float32, as the reference's float tensor) and solid angles
__global__ void k_env_weights(const float* __restrict__ env, int H, int W, int C, int th, int tw, int cube,
                              float* __restrict__ weight, float* __restrict__ solid) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= th * tw) return;
    const int oy = cell / tw, ox = cell - oy * tw;
    float rgb[3] = {0.0f, 0.0f, 0.0f};
    if (cube || (th == H && tw == W)) {
        const float* t = env + ((size_t)oy * W + ox) * C;
        rgb[0] = t[0];
        rgb[1] = t[1];
        rgb[2] = t[2];
    } else {
        // area average over the input rows [y0, y1) and columns [x0, x1) covered by the cell
        const int y0 = (int)(((long long)oy * H) / th), y1 = (int)((((long long)oy + 1) * H + th - 1) / th);
        const int x0 = (int)(((long long)ox * W) / tw), x1 = (int)((((long long)ox + 1) * W + tw - 1) / tw);
        float s[3] = {0.0f, 0.0f, 0.0f};
        for (int y = y0; y < y1; ++y)
            for (int x = x0; x < x1; ++x) {
                const float* t = env + ((size_t)y * W + x) * C;
                s[0] += t[0];
                s[1] += t[1];
                s[2] += t[2];
            }
        const float inv = 1.0f / (float)((y1 - y0) * (x1 - x0));
        rgb[0] = s[0] * inv;
        rgb[1] = s[1] * inv;
        rgb[2] = s[2] * inv;
    }
    for (int k = 0; k < 3; ++k) rgb[k] = (isfinite(rgb[k]) && rgb[k] > 0.0f) ? rgb[k] : 0.0f;
    const float lum = rgb[0] * 0.2126f + rgb[1] * 0.7152f + rgb[2] * 0.0722f;
    const double sa = cube ? solid_angle_cube(ox, oy % tw, tw) : solid_angle_equirect(oy, th, tw);
    solid[cell] = (float)sa;
    weight[cell] = lum * (float)sa;
}

// block-wide float64 sum in a fixed order
__device__ double block_sum(double v, double* red) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    __syncthreads();
    if (threadIdx.x == 0) red[0] = t;
    __syncthreads();
    t = red[0];
    __syncthreads();
    return t;
}

// exclusive scan of one count per thread (block order), returns this thread's offset and the total
__device__ int block_scan(int v, int* buf, int& total) {
    buf[threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            const int c = buf[i];
            buf[i] = acc;
            acc += c;
        }
        buf[blockDim.x] = acc;
    }
    __syncthreads();
    const int off = buf[threadIdx.x];
    total = buf[blockDim.x];
    __syncthreads();
    return off;
}

// One block: pdf, then the alias table. scratch: scaled [n] float64, small / large [n] int32.
__global__ void __launch_bounds__(kEnvThreads) k_env_alias(int n, float* __restrict__ weight,
                                                           const float* __restrict__ solid, double* __restrict__ scaled,
                                                           int* __restrict__ small, int* __restrict__ large,
                                                           float* __restrict__ out) {
    __shared__ double red[kEnvThreads / 32];
    __shared__ int scan[kEnvThreads + 1];
    float* prob = out;
    float* alias = out + n;
    float* pdf = out + 2 * n;
    // contiguous chunk of cells per thread, so that lists come out in index order
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int first = min(n, (int)threadIdx.x * per), last = min(n, first + per);

    double t = 0.0;
    for (int i = first; i < last; ++i) t += (double)weight[i];
    double total = block_sum(t, red);
    // float32 total as the reference's float tensor sum; fall back to the solid angles
    const bool fallback = !(isfinite((float)total) && (float)total > 0.0f);
    if (fallback) {
        for (int i = first; i < last; ++i) weight[i] = solid[i];
        __syncthreads();
        t = 0.0;
        for (int i = first; i < last; ++i) t += (double)weight[i];
        total = block_sum(t, red);
    }
    const float total_f = (float)total;
    for (int i = first; i < last; ++i) {
        const float s = solid[i];
        pdf[i] = s > 0.0f ? weight[i] / fmaxf(total_f * s, 1.17549435e-38f) : 0.0f;
    }
    // Vose (aliastable.py:49-116): float64 scaled weights, index-ordered lists
    int ns = 0, nl = 0;
    for (int i = first; i < last; ++i) {
        const float w = weight[i];
        const double v = (isfinite(w) && w > 0.0f) ? (double)w * ((double)n / total) : 0.0;
        scaled[i] = v;
        prob[i] = 1.0f;
        alias[i] = (float)i;
        if (total <= 0.0) continue;
        if (v < 1.0) ++ns; else ++nl;
    }
    int n_small = 0, n_large = 0;
    int so = block_scan(ns, scan, n_small);
    int lo = block_scan(nl, scan, n_large);
    if (total > 0.0) {
        for (int i = first; i < last; ++i) {
            if (scaled[i] < 1.0) small[so++] = i; else large[lo++] = i;
        }
    }
    __syncthreads();
    if (threadIdx.x != 0 || total <= 0.0) return;
    // pairing: pop from the ends; a large entry that drops below 1 joins the small list
    int top_s = n_small, top_l = n_large;
    for (int guard = 0; top_s > 0 && top_l > 0 && guard < 2 * n + 2; ++guard) {
        const int s = small[--top_s];
        const int g = large[--top_l];
        const double vs = scaled[s];
        prob[s] = (float)fmin(fmax(vs, 0.0), 1.0);
        alias[s] = (float)g;
        const double vg = scaled[g] - (1.0 - vs);
        scaled[g] = vg;
        if (vg < 1.0) small[top_s++] = g; else large[top_l++] = g;
    }
    // leftovers keep probability 1 and alias themselves (set above)
}

}  // namespace

}  // namespace ptir

extern "C" size_t ptir_env_table_scratch_bytes(int32_t cells) {
    return cells <= 0 ? 0 : (size_t)cells * (sizeof(double) + 2 * sizeof(int) + 2 * sizeof(float)) + 256;
}

extern "C" int ptir_build_env_table(const float* environment, int32_t env_h, int32_t env_w, int32_t channels,
                                    int32_t table_h, int32_t table_w, float* table_out, void* scratch,
                                    size_t scratch_bytes, void* stream) {
    if (!environment || !table_out || env_h <= 0 || env_w <= 0 || channels < 3) return PTIR_EINVAL;
    const bool cube = env_h == 6 * env_w;
    const int th = cube ? env_h : table_h, tw = cube ? env_w : table_w;
    if (th <= 0 || tw <= 0) return PTIR_EINVAL;
    const long long cells = (long long)th * tw;
    if (cells > (1ll << 30) || scratch_bytes < ptir_env_table_scratch_bytes((int32_t)cells) || !scratch)
        return PTIR_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char* p = static_cast<char*>(scratch);
    p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 15u) & ~uintptr_t(15));
    double* scaled = reinterpret_cast<double*>(p);
    int* small = reinterpret_cast<int*>(scaled + cells);
    int* large = small + cells;
    float* weight = reinterpret_cast<float*>(large + cells);
    float* solid = weight + cells;
    const int block = 256;
    ptir::k_env_weights<<<(unsigned)((cells + block - 1) / block), block, 0, s>>>(environment, env_h, env_w, channels,
                                                                                 th, tw, cube ? 1 : 0, weight, solid);
    ptir::k_env_alias<<<1, ptir::kEnvThreads, 0, s>>>((int)cells, weight, solid, scaled, small, large, table_out);
    return cudaGetLastError() == cudaSuccess ? PTIR_OK : PTIR_ECUDA;
}
