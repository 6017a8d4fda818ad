// Light selection for next-event estimation: the environment, point, sphere and triangle-mesh
// lights of the reference's light sampler, in FP32.
//
//   top-level selection, per-type sampling and pdfs
//                        threedgptir_tracer/include/3dgptir/kernels/cuda/lightSampler.cuh:12-406
//   mesh triangles       threedgptir_tracer/include/3dgptir/kernels/cuda/meshLight.cuh:11-101
//   lights seen by rays  threedgptir_tracer/include/3dgptir/kernels/cuda/environment.cuh:491-634
//
// Random numbers are drawn in the reference's order (selection, then the light's own draws), so
// a path takes the same decisions. Triangle ranges are checked in 64 bits, so a packed table whose
// offset and count overflow 32 bits reads nothing instead of wrapping into the arrays.
#pragma once

#include "device_types.h"
#include "pcg.cuh"
#include "shading.cuh"
#include "vecmath.cuh"

namespace ptir {

enum LightType : unsigned { kLightEnv = 0u, kLightPoint = 1u, kLightSphere = 2u, kLightMesh = 3u };

struct LightSample {
    float3 wi, Li;
    float pdf;   // solid-angle pdf times the selection pdf (the selection pdf alone for point lights)
    float dist;  // distance to the sampled point, 1e20 for the environment
    unsigned type;
};

PTIR_DEV LightSample light_sample_empty() {
    LightSample ls;
    ls.wi = ls.Li = f3(0.0f);
    ls.pdf = 0.0f;
    ls.dist = 1e20f;
    ls.type = kLightEnv;
    return ls;
}

// float -> index as the reference's static_cast: toward zero, saturating, NaN -> 0
PTIR_DEV unsigned table_index(float v) { return __float2uint_rz(v + 0.5f); }

PTIR_DEV bool light_table_present(const LightView& L) { return L.entries > 0; }
PTIR_DEV bool mesh_lights_present(const LightView& L) {
    return L.num_mesh > 0 && L.num_vertices > 0 && L.num_triangles > 0 && L.tri_cols >= L.num_triangles;
}
PTIR_DEV float light_field(const LightView& L, unsigned id, int k) { return __ldg(L.lights + 9 * (size_t)id + k); }
PTIR_DEV unsigned light_type_of(const LightView& L, unsigned id) {
    return id < (unsigned)L.num_lights ? table_index(light_field(L, id, 0)) : 0xFFFFFFFFu;
}
PTIR_DEV float table_at(const LightView& L, int row, unsigned e) { return __ldg(L.table + (size_t)row * L.entries + e); }
PTIR_DEV float tri_table_at(const LightView& L, int row, unsigned t) {
    return __ldg(L.tri_table + (size_t)row * L.tri_cols + t);
}
PTIR_DEV float vlength(float3 v) { return sqrtf(dot(v, v)); }

// lightSampler.cuh:59-72
PTIR_DEV unsigned sample_light_entry(const LightView& L, Pcg32& rng) {
    const unsigned n = (unsigned)L.entries;
    const unsigned first = min(__float2uint_rz(rng.uniform() * (float)n), n - 1u);
    const unsigned other = min(table_index(table_at(L, 1, first)), n - 1u);
    return rng.uniform() < table_at(L, 0, first) ? first : other;
}

// lightSampler.cuh:74-91
PTIR_DEV LightSample sample_env_light(const EnvView& E, Pcg32& rng, float select, unsigned& lookups) {
    LightSample ls = light_sample_empty();
    if (!env_light_present(E)) return ls;
    float epdf = 0.0f;
    ls.wi = sample_env_direction(E, rng, epdf);
    ls.Li = env_radiance(E, ls.wi, lookups);
    ls.pdf = select * epdf;
    return ls;
}

// lightSampler.cuh:93-123
PTIR_DEV LightSample sample_point_light(const LightView& L, float3 pos, unsigned id, float select) {
    LightSample ls = light_sample_empty();
    if (id >= (unsigned)L.num_lights || light_type_of(L, id) != kLightPoint || select <= 0.0f) return ls;
    const float* r = L.lights + 9 * (size_t)id;
    const float3 to = ld3(r + 1) - pos;
    const float dist2 = dot(to, to);
    if (dist2 <= 1e-12f) return ls;
    const float dist = sqrtf(dist2);
    ls.wi = to / dist;
    ls.Li = ld3(r + 5) / dist2;
    ls.pdf = select;
    ls.dist = dist;
    ls.type = kLightPoint;
    return ls;
}

// lightSampler.cuh:125-179: a uniform point on the sphere, converted to solid angle
PTIR_DEV LightSample sample_sphere_light(const LightView& L, float3 pos, Pcg32& rng, unsigned id, float select) {
    LightSample ls = light_sample_empty();
    if (id >= (unsigned)L.num_lights || light_type_of(L, id) != kLightSphere) return ls;
    const float* r = L.lights + 9 * (size_t)id;
    const float radius = __ldg(r + 4);
    if (radius <= 0.0f) return ls;
    const float u1 = rng.uniform();
    const float u2 = rng.uniform();
    const float z = 1.0f - 2.0f * u1;
    const float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float sp, cp;
    sincosf(2.0f * kPiF * u2, &sp, &cp);
    const float3 nrm = make_float3(rr * cp, rr * sp, z);
    const float3 to = (ld3(r + 1) + radius * nrm) - pos;
    const float dist2 = dot(to, to);
    if (dist2 <= 1e-12f) return ls;
    const float dist = sqrtf(dist2);
    const float3 wi = to / dist;
    const float cos_l = fabsf(dot(nrm, -wi));
    if (cos_l <= 1e-6f) return ls;
    const float area = 4.0f * kPiF * radius * radius;
    ls.wi = wi;
    ls.Li = ld3(r + 5);
    ls.pdf = select * (1.0f / fmaxf(area, 1e-12f)) * dist2 / cos_l;
    ls.dist = dist;
    ls.type = kLightSphere;
    return ls;
}

// lightSampler.cuh:181-222: pdf of direction wi from pos under sphere sampling
PTIR_DEV float sphere_light_pdf(const LightView& L, float3 pos, float3 wi, unsigned id) {
    if (id >= (unsigned)L.num_lights || light_type_of(L, id) != kLightSphere) return 0.0f;
    const float* r = L.lights + 9 * (size_t)id;
    const float3 c = ld3(r + 1);
    const float radius = __ldg(r + 4);
    if (radius <= 0.0f) return 0.0f;
    const float3 oc = pos - c;
    const float b = dot(oc, wi);
    const float cc = dot(oc, oc) - radius * radius;
    const float disc = b * b - cc;
    if (disc <= 0.0f) return 0.0f;
    float t = -b - sqrtf(disc);
    if (t <= 1e-6f) t = -b + sqrtf(disc);
    if (t <= 1e-6f) return 0.0f;
    const float3 n = normalize_or_keep((pos + t * wi) - c);
    const float cos_l = fabsf(dot(n, -wi));
    if (cos_l <= 1e-6f) return 0.0f;
    const float area = 4.0f * kPiF * radius * radius;
    return (1.0f / fmaxf(area, 1e-12f)) * (t * t) / cos_l;
}

// meshLight.cuh:18-51
PTIR_DEV bool mesh_triangle(const LightView& L, unsigned tri, float3& v0, float3& v1, float3& v2) {
    if (tri >= (unsigned)L.num_triangles) return false;
    const int* t = L.triangles + 3 * (size_t)tri;
    const int i0 = __ldg(t), i1 = __ldg(t + 1), i2 = __ldg(t + 2);
    if (i0 < 0 || i1 < 0 || i2 < 0) return false;
    const unsigned nv = (unsigned)L.num_vertices;
    if ((unsigned)i0 >= nv || (unsigned)i1 >= nv || (unsigned)i2 >= nv) return false;
    v0 = ld3(L.vertices + 3 * (size_t)i0);
    v1 = ld3(L.vertices + 3 * (size_t)i1);
    v2 = ld3(L.vertices + 3 * (size_t)i2);
    return true;
}

// meshLight.cuh:53-84 (Moller-Trumbore; hits beyond 1e-5)
PTIR_DEV bool intersect_triangle(float3 o, float3 d, float3 v0, float3 v1, float3 v2, float& t) {
    const float3 e1 = v1 - v0, e2 = v2 - v0;
    const float3 pv = cross(d, e2);
    const float det = dot(e1, pv);
    if (fabsf(det) <= 1e-8f) return false;
    const float inv = 1.0f / det;
    const float3 tv = o - v0;
    const float u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const float3 qv = cross(tv, e1);
    const float v = dot(d, qv) * inv;
    if (v < 0.0f || (u + v) > 1.0f) return false;
    t = dot(e2, qv) * inv;
    return t > 1e-5f;
}

// triangle range of mesh light `id`; false when it lies outside the packed triangles
PTIR_DEV bool mesh_range(const LightView& L, unsigned id, unsigned& off, unsigned& count) {
    const float* m = L.mesh + 8 * (size_t)id;
    off = table_index(__ldg(m));
    count = table_index(__ldg(m + 1));
    return count != 0u && (unsigned long long)off + count <= (unsigned long long)L.num_triangles;
}

// cosine at the light of direction wi arriving on the triangle's plane; <= 1e-6 rejects
PTIR_DEV float mesh_cosine(float3 v0, float3 v1, float3 v2, float3 wi, bool two_sided, bool& ok) {
    const float3 nu = cross(v1 - v0, v2 - v0);
    const float nl = vlength(nu);
    ok = nl > 1e-12f;
    if (!ok) return 0.0f;
    const float c = dot(nu / nl, -wi);
    return two_sided ? fabsf(c) : c;
}

// meshLight.cuh:86-101
PTIR_DEV unsigned sample_mesh_triangle(const LightView& L, Pcg32& rng, unsigned off, unsigned count) {
    const unsigned local = min(__float2uint_rz(rng.uniform() * (float)count), count - 1u);
    const unsigned first = off + local;
    const unsigned other = min(table_index(tri_table_at(L, 1, first)), count - 1u);
    return rng.uniform() < tri_table_at(L, 0, first) ? first : off + other;
}

// lightSampler.cuh:224-293: a triangle by area, then a uniform point on it
PTIR_DEV LightSample sample_mesh_light(const LightView& L, float3 pos, Pcg32& rng, unsigned id, float select) {
    LightSample ls = light_sample_empty();
    if (!mesh_lights_present(L) || id >= (unsigned)L.num_mesh || select <= 0.0f) return ls;
    unsigned off, count;
    if (!mesh_range(L, id, off, count)) return ls;
    const unsigned tri = sample_mesh_triangle(L, rng, off, count);
    float3 v0, v1, v2;
    if (!mesh_triangle(L, tri, v0, v1, v2)) return ls;
    float u = rng.uniform();
    float v = rng.uniform();
    if (u + v > 1.0f) {
        u = 1.0f - u;
        v = 1.0f - v;
    }
    const float3 to = (v0 + u * (v1 - v0) + v * (v2 - v0)) - pos;
    const float dist2 = dot(to, to);
    if (dist2 <= 1e-12f) return ls;
    const float dist = sqrtf(dist2);
    const float3 wi = to / dist;
    const float* m = L.mesh + 8 * (size_t)id;
    bool ok;
    const float cos_l = mesh_cosine(v0, v1, v2, wi, __ldg(m + 7) > 0.5f, ok);
    if (!ok || cos_l <= 1e-6f) return ls;
    ls.wi = wi;
    ls.Li = ld3(m + 4);
    ls.pdf = select * tri_table_at(L, 2, tri) * dist2 / cos_l;
    ls.dist = dist;
    ls.type = kLightMesh;
    return ls;
}

// lightSampler.cuh:295-338: summed over every triangle the direction crosses
PTIR_DEV float mesh_light_pdf(const LightView& L, float3 pos, float3 wi, unsigned id) {
    if (!mesh_lights_present(L) || id >= (unsigned)L.num_mesh) return 0.0f;
    unsigned off, count;
    if (!mesh_range(L, id, off, count)) return 0.0f;
    const bool two_sided = __ldg(L.mesh + 8 * (size_t)id + 7) > 0.5f;
    float pdf = 0.0f;
    for (unsigned tri = off; tri < off + count; ++tri) {
        float3 v0, v1, v2;
        float t;
        if (!mesh_triangle(L, tri, v0, v1, v2) || !intersect_triangle(pos, wi, v0, v1, v2, t)) continue;
        bool ok;
        const float cos_l = mesh_cosine(v0, v1, v2, wi, two_sided, ok);
        if (!ok || cos_l <= 1e-6f) continue;
        pdf += tri_table_at(L, 2, tri) * (t * t) / cos_l;
    }
    return pdf;
}

// lightSampler.cuh:340-383
PTIR_DEV LightSample sample_light(const TraceParams& P, float3 pos, Pcg32& rng, unsigned& lookups) {
    const LightView& L = P.lights;
    if (!light_table_present(L)) return sample_env_light(P.env, rng, 1.0f, lookups);
    const unsigned e = sample_light_entry(L, rng);
    const unsigned type = table_index(table_at(L, 2, e));
    const unsigned id = table_index(table_at(L, 3, e));
    const float select = table_at(L, 4, e);
    switch (type) {
    case kLightEnv: return sample_env_light(P.env, rng, select, lookups);
    case kLightPoint: return sample_point_light(L, pos, id, select);
    case kLightSphere: return sample_sphere_light(L, pos, rng, id, select);
    case kLightMesh: return sample_mesh_light(L, pos, rng, id, select);
    default: return light_sample_empty();
    }
}

// lightSampler.cuh:385-406: pdf of sampling direction wi from pos (point lights, being delta
// lights, add nothing)
PTIR_DEV float light_sampler_pdf(const TraceParams& P, float3 pos, float3 wi) {
    const LightView& L = P.lights;
    if (!light_table_present(L)) return env_pdf(P.env, wi);
    float pdf = 0.0f;
    for (unsigned i = 0; i < (unsigned)L.entries; ++i) {
        const float select = table_at(L, 4, i);
        if (select <= 0.0f) continue;
        const unsigned type = table_index(table_at(L, 2, i));
        const unsigned id = table_index(table_at(L, 3, i));
        float p = 0.0f;
        if (type == kLightEnv) p = env_pdf(P.env, wi);
        else if (type == kLightSphere) p = sphere_light_pdf(L, pos, wi, id);
        else if (type == kLightMesh) p = mesh_light_pdf(L, pos, wi, id);
        pdf += select * p;
    }
    return pdf;
}

// environment.cuh:491-536
PTIR_DEV bool hit_sphere_light(const LightView& L, float3 o, float3 d, unsigned id, float& t, float3& radiance) {
    if (light_type_of(L, id) != kLightSphere) return false;
    const float* r = L.lights + 9 * (size_t)id;
    const float radius = __ldg(r + 4);
    if (radius <= 0.0f) return false;
    const float3 oc = o - ld3(r + 1);
    const float b = dot(oc, d);
    const float cc = dot(oc, oc) - radius * radius;
    const float disc = b * b - cc;
    if (disc <= 0.0f) return false;
    const float sq = sqrtf(disc);
    t = -b - sq;
    if (t <= 1e-5f) t = -b + sq;
    if (t <= 1e-5f) return false;
    radiance = ld3(r + 5);
    return !(radiance.x <= 0.0f && radiance.y <= 0.0f && radiance.z <= 0.0f);
}

// environment.cuh:538-597
PTIR_DEV bool hit_mesh_light(const LightView& L, float3 o, float3 d, unsigned id, float& t, float3& radiance) {
    if (!mesh_lights_present(L)) return false;
    unsigned off, count;
    if (!mesh_range(L, id, off, count)) return false;
    const float* m = L.mesh + 8 * (size_t)id;
    radiance = ld3(m + 4);
    if (radiance.x <= 0.0f && radiance.y <= 0.0f && radiance.z <= 0.0f) return false;
    const bool two_sided = __ldg(m + 7) > 0.5f;
    float nearest = 1e20f;
    for (unsigned tri = off; tri < off + count; ++tri) {
        float3 v0, v1, v2;
        float th;
        if (!mesh_triangle(L, tri, v0, v1, v2) || !intersect_triangle(o, d, v0, v1, v2, th)) continue;
        bool ok;
        const float cos_l = mesh_cosine(v0, v1, v2, d, two_sided, ok);
        if (!ok || cos_l <= 1e-6f) continue;
        nearest = fminf(nearest, th);
    }
    if (nearest >= 1e19f) return false;
    t = nearest;
    return true;
}

// environment.cuh:599-624 (render.visualize_lights): the nearest sphere or mesh light the ray
// (o, d) meets, wherever the Gaussians are; false when it meets none
PTIR_DEV bool visible_area_light(const LightView& L, float3 o, float3 d, float3& radiance) {
    float nearest = 1e20f;
    bool found = false;
    for (unsigned i = 0; i < (unsigned)L.num_lights; ++i) {
        float t;
        float3 r;
        if (hit_sphere_light(L, o, d, i, t, r) && t < nearest) {
            nearest = t;
            radiance = r;
            found = true;
        }
    }
    for (unsigned i = 0; i < (unsigned)L.num_mesh; ++i) {
        float t;
        float3 r;
        if (hit_mesh_light(L, o, d, i, t, r) && t < nearest) {
            nearest = t;
            radiance = r;
            found = true;
        }
    }
    return found;
}

}  // namespace ptir
