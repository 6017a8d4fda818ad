// Small float3 toolkit for the tracer kernels (device only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PTIR_DEV static __device__ __forceinline__

PTIR_DEV float3 f3(float a) { return make_float3(a, a, a); }
PTIR_DEV float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
PTIR_DEV float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
PTIR_DEV float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
PTIR_DEV float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
PTIR_DEV float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
PTIR_DEV float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
PTIR_DEV float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
PTIR_DEV float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
PTIR_DEV float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
PTIR_DEV float3& operator-=(float3& a, float3 b) { a = a - b; return a; }
PTIR_DEV float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
PTIR_DEV float3& operator*=(float3& a, float s) { a = a * s; return a; }
PTIR_DEV float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PTIR_DEV float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PTIR_DEV bool all_zero(float3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
PTIR_DEV float max3(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
PTIR_DEV float3 fmax3(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
PTIR_DEV float3 fmin3(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
// v/|v| when |v|^2 > 0, otherwise v
PTIR_DEV float3 normalize_or_keep(float3 v) {
    const float l = dot(v, v);
    return l > 0.0f ? v * rsqrtf(l) : v;
}
PTIR_DEV float3 ld3(const float* p) { return make_float3(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }

// 3x3 stored as three rows
struct Mat3 {
    float3 r0, r1, r2;
};
PTIR_DEV float3 mul_rows(const Mat3& m, float3 p) { return make_float3(dot(m.r0, p), dot(m.r1, p), dot(m.r2, p)); }
PTIR_DEV float3 mul_cols(const Mat3& m, float3 p) { return m.r0 * p.x + m.r1 * p.y + m.r2 * p.z; }

// Rows of R^T for a wxyz quaternion (w, x, y, z); the world->particle rotation.
PTIR_DEV Mat3 quat_rt(float4 q) {
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, rx = r * x, ry = r * y,
                rz = r * z;
    Mat3 m;
    m.r0 = make_float3(1.f - 2.f * (yy + zz), 2.f * (xy + rz), 2.f * (xz - ry));
    m.r1 = make_float3(2.f * (xy - rz), 1.f - 2.f * (xx + zz), 2.f * (yz + rx));
    m.r2 = make_float3(2.f * (xz + ry), 2.f * (yz - rx), 1.f - 2.f * (xx + yy));
    return m;
}
// Rows of R (particle->world rotation).
PTIR_DEV Mat3 quat_r(float4 q) {
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, rx = r * x, ry = r * y,
                rz = r * z;
    Mat3 m;
    m.r0 = make_float3(1.f - 2.f * (yy + zz), 2.f * (xy - rz), 2.f * (xz + ry));
    m.r1 = make_float3(2.f * (xy + rz), 1.f - 2.f * (xx + zz), 2.f * (yz - rx));
    m.r2 = make_float3(2.f * (xz - ry), 2.f * (yz + rx), 1.f - 2.f * (xx + yy));
    return m;
}

// Orthonormal basis around a unit vector (Duff et al. 2017, "Building an Orthonormal Basis, Revisited").
PTIR_DEV void onb(float3 n, float3& t, float3& b) {
    const float sign = copysignf(1.0f, n.z);
    const float a = -1.0f / (sign + n.z);
    const float c = n.x * n.y * a;
    t = make_float3(1.0f + sign * n.x * n.x * a, sign * c, -sign * n.x);
    b = make_float3(c, sign + n.y * n.y * a, -n.y);
}

// Index of the lowest set lane among `mask` that shares `key` (warp aggregation helper).
PTIR_DEV unsigned lane_id() { return threadIdx.x & 31u; }

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr float kInvPiF = 0.31830988618379067154f;
