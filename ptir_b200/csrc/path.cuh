// Per-segment building blocks of the path tracer and its adjoint, shared by the megakernel
// (tracer.cu) and the wavefront stages (wavefront.cu).
#pragma once

#include "device_types.h"
#include "lights.cuh"
#include "pcg.cuh"
#include "shading.cuh"
#include "storage.cuh"
#include "traverse.cuh"
#include "vecmath.cuh"

namespace ptir {

// ------------------------------------------------------------------------------------
// per-segment state (the reference's rayPayload, threedgptir_tracer/include/3dgptir/payLoad.h:38-95)
struct Segment {
    float3 o, d;
    float3 radiance, normal, light, ray_dir_grad;
    float transmittance, depth, hit2, last_hit, distortion, hits_count;
    float scatter_pdf, light_pdf;
    bool hit, escaped;
    // interaction (interaction.h:22-76)
    bool ivalid;
    float3 pos, snrm, albedo;
    float rough, metal;
    float3 d_albedo;
    float d_rough, d_metal;
};

PTIR_DEV void segment_reset(Segment& s, float3 o, float3 d, float last_hit) {
    s.o = o;
    s.d = d;
    s.radiance = s.normal = s.light = s.ray_dir_grad = f3(0.0f);
    s.transmittance = 1.0f;
    s.depth = s.hit2 = s.distortion = s.hits_count = 0.0f;
    s.last_hit = last_hit;
    s.scatter_pdf = s.light_pdf = 0.0f;
    s.hit = s.escaped = false;
    s.ivalid = false;
    s.pos = s.snrm = s.albedo = f3(0.0f);
    s.rough = s.metal = 0.0f;
    s.d_albedo = f3(0.0f);
    s.d_rough = s.d_metal = 0.0f;
}

struct Emitter {
    float3 dir, contribution, light;
    float light_pdf, scatter_pdf;
    float tmax;  // shadow-ray end: short of a sampled point on a light, unbounded for the environment
};

struct PathState {
    unsigned active, bounces, max_bounces;
    unsigned sig;  // decision signature (kPathSig): FNV-1a over the path's discrete events
    float3 acc, acc_grad, acc_direct, acc_indirect, acc_light, acc_light_grad, throughput;
    Emitter em;
    // pending roughness gradient through the next direction (payLoad.h:97-138)
    bool pend_valid;
    float3 pend_o, pend_d, pend_dnext;
    float pend_opacity, pend_max_hit;
    unsigned pend_bounces;
};

template <int K_>
struct CtxT {
    static constexpr int K = K_;  // k-buffer size of the traversals
    const TraceParams& P;
    StackEntry* stack;
    TraceCounters& ctr;
};

// scene AABB interval, clamped at 0 (pathTracer.cuh:46-52)
PTIR_DEV float2 clip_scene(const TraceParams& P, float3 o, float3 d) {
    if (P.accel.n <= 0) return make_float2(1.0f, 0.0f);
    const float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const float4 lo = __ldg(P.accel.bounds), hi = __ldg(P.accel.bounds + 1);
    float t0, t1;
    slab(make_float3(lo.x, lo.y, lo.z), make_float3(hi.x, hi.y, hi.z), o, inv, t0, t1);
    return make_float2(fmaxf(0.0f, t0), t1);
}

// shared front of the hit evaluation: the particle frame, squared distance and response
struct Response {
    float3 gro, grd, scl;
    Mat3 rt;
    float d2, gres, alpha;
};

PTIR_DEV float kernel_response(int degree, float d2) {
    switch (degree) {
    case 8: { const float q = d2 * d2; return __expf(-0.000685871056241f * q * q); }
    case 5: return __expf(-0.0185185185185f * d2 * d2 * sqrtf(d2));
    case 4: return __expf(-0.0555555555556f * d2 * d2);
    case 3: return __expf(-0.166666666667f * d2 * sqrtf(d2));
    case 1: return __expf(-1.5f * sqrtf(d2));
    case 0: return fmaxf(1.0f - 0.329630334487f * sqrtf(d2), 0.0f);
    default: return __expf(-0.5f * d2);
    }
}

PTIR_DEV Response respond(const TraceParams& P, unsigned id, float3 o, float3 d, float& density) {
    const Geom g = load_geom(P.part, id);
    Response r;
    r.rt = quat_rt(g.quat);
    r.scl = g.scl;
    const float3 is = make_float3(1.0f / g.scl.x, 1.0f / g.scl.y, 1.0f / g.scl.z);
    r.gro = is * mul_rows(r.rt, o - g.pos);
    r.grd = normalize_or_keep(is * mul_rows(r.rt, d));
    const float3 cr = cross(r.grd, r.gro);
    r.d2 = dot(cr, cr);
    r.gres = kernel_response(P.kernel_degree, r.d2);
    density = g.dns;
    r.alpha = fminf(0.99f, r.gres * g.dns);
    return r;
}

// secondary rays skip Gaussians just in front of the origin whose shading normal faces along
// the ray (pathTracer.cuh:115-128)
PTIR_DEV bool self_occluded(const TraceParams& P, float t, unsigned id, float3 d) {
    if (t > (1e-1f - 2e-2f) || P.part.snrm == nullptr) return false;
    return dot(load_snrm(P.part, id), d) > 0.1f;
}

// SH coefficient k (0..15) of one Gaussian as an RGB triple: FP32 rows of the caller's tensor ...
struct ShRowF32 {
    const float* c;
    __device__ __forceinline__ float3 operator()(int k) const { return ld3(c + 3 * k); }
};

// ... or the 16-bit SH of a cold record
struct ShRow16 {
    const unsigned short* c;
    unsigned storage;
    __device__ __forceinline__ float at(int v) const { return widen(storage, __ldg(c + v)); }
    __device__ __forceinline__ float3 operator()(int k) const {
        return make_float3(at(3 * k), at(3 * k + 1), at(3 * k + 2));
    }
};

// SH radiance of degree <= 3 (+0.5 bias, clamped at 0) along direction d
template <class Coef>
PTIR_DEV float3 sh_eval(const Coef& c, int deg, float3 d) {
    float3 rad = c(0) * 0.28209479177387814f;
    if (deg > 0) {
        const float x = d.x, y = d.y, z = d.z;
        rad = rad - c(1) * (0.4886025119029199f * y) + c(2) * (0.4886025119029199f * z) -
              c(3) * (0.4886025119029199f * x);
        if (deg > 1) {
            const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            rad = rad + c(4) * (1.0925484305920792f * xy) + c(5) * (-1.0925484305920792f * yz) +
                  c(6) * (0.31539156525252005f * (2.0f * zz - xx - yy)) +
                  c(7) * (-1.0925484305920792f * xz) + c(8) * (0.5462742152960396f * (xx - yy));
            if (deg > 2) {
                rad = rad + c(9) * (-0.5900435899266435f * y * (3.0f * xx - yy)) +
                      c(10) * (2.890611442640554f * xy * z) +
                      c(11) * (-0.4570457994644658f * y * (4.0f * zz - xx - yy)) +
                      c(12) * (0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy)) +
                      c(13) * (-0.4570457994644658f * x * (4.0f * zz - xx - yy)) +
                      c(14) * (1.445305721320277f * z * (xx - yy)) +
                      c(15) * (-0.5900435899266435f * x * (xx - 3.0f * yy));
            }
        }
    }
    return relu3(rad + f3(0.5f));
}

PTIR_DEV float3 sh_radiance(const TraceParams& P, unsigned id, float3 d) {
    const int deg = P.part.sph_degree;
    if (P.part.storage == kStoreF32) return sh_eval(ShRowF32{P.part.sph + (size_t)id * P.part.sph_stride}, deg, d);
    const ShRow16 c{reinterpret_cast<const unsigned short*>(P.part.cold + (size_t)P.part.cold_stride * id + 1),
                    P.part.storage};
    return sh_eval(c, deg, d);
}

// Stochastic shadow transmittance: occluded at the first hit whose alpha beats a draw
// (pathTracer.cuh:130-214).
template <class Ctx>
PTIR_DEV bool shadow_occluded(const Ctx& C, float3 o, float3 d, float tmax, Pcg32& rng) {
    const TraceParams& P = C.P;
    const float2 clip = clip_scene(P, o, d);
    float start = fmaxf(0.0f, clip.x - 1e-9f);
    const float end = fminf(tmax, clip.y) + 1e-9f;
    if (start >= end) return false;
    float kt[Ctx::K];
    unsigned kid[Ctx::K];
    for (int round = 0; start < end; ++round) {
        if (round > (1 << 16)) {
            atomicOr(P.error_word, kErrLoopBound);
            break;
        }
        trace_kbuf(P.accel, o, d, start + 1e-9f, end, kt, kid, C.stack, P.error_word, C.ctr);
        if (kid[0] == kNoHit) break;
        float batch_end = start;
        bool stop = false;
#pragma unroll
        for (int i = 0; i < Ctx::K; ++i) {
            if (stop) continue;
            const unsigned id = kid[i];
            if (id == kNoHit || kt[i] > end) { stop = true; continue; }
            batch_end = fmaxf(batch_end, kt[i]);
            if (self_occluded(P, kt[i], id, d)) continue;
            float dns;
            const Response r = respond(P, id, o, d, dns);
            const float alpha = (r.gres > P.min_response && r.alpha > P.alpha_min) ? r.alpha : 0.0f;
            if (alpha > 0.0f && rng.uniform() < alpha) return true;
        }
        if (batch_end <= start || kid[Ctx::K - 1] == kNoHit) break;
        start = batch_end;
    }
    return false;
}

PTIR_DEV void shading_frame(const Segment& s, float3& n, float3& wo, float3& alb, float& met, bool metallic_on) {
    n = normalize_or(s.snrm, make_float3(0.0f, 0.0f, 1.0f));
    wo = normalize_or(-s.d, n);
    alb = saturate(s.albedo);
    met = metallic_on ? saturate(s.metal) : 0.0f;
}

PTIR_DEV void emitter_clear(Emitter& em) {
    em.contribution = em.light = f3(0.0f);
    em.light_pdf = 0.0f;
    em.scatter_pdf = 0.0f;
    em.dir = f3(0.0f);
    em.tmax = kFarT;
}

// ------------------------------------------------------------------------------------
// Decision signature of a path (diagnostics, P.flags & kPathSig): an FNV-1a hash over the events
// in which a float evaluation takes a discrete branch, in path order: per segment its accepted-hit
// count, interaction and escape flags; whether NEE casts a shadow ray and whether it is occluded;
// whether the path continues after each BRDF sample. Two evaluations of the same path (this
// tracer and the oracle, or two precisions) with equal signatures took the same branches.
PTIR_DEV unsigned sig_mix(unsigned h, unsigned v) { return (h ^ v) * 16777619u; }
PTIR_DEV unsigned sig_segment(const Segment& s) {
    const unsigned hits = (unsigned)fminf(fmaxf(s.hits_count, 0.0f), 65535.0f);
    return hits | (s.ivalid ? 1u << 16 : 0u) | (s.escaped ? 1u << 17 : 0u) | (s.hit ? 1u << 18 : 0u);
}
constexpr unsigned kSigNee = 0x100000u, kSigShadow = 0x200000u, kSigCont = 0x300000u;
PTIR_DEV void sig_event(const TraceParams& P, PathState& ps, unsigned v) {
    if (P.flags & kPathSig) ps.sig = sig_mix(ps.sig, v);
}
PTIR_DEV bool path_continues(const PathState& ps) { return ps.active && !(max3(ps.throughput) < 1e-4f); }

// Next-event estimation (pathTracer.cuh:461-504), first half: light sample, visibility-independent
// checks and BRDF. Fills the emitter as if unoccluded and returns true when a shadow ray has to
// decide it (nee_shadow).
template <class Ctx>
PTIR_DEV bool nee_prepare_light(const Ctx& C, PathState& ps, const Segment& s, Pcg32& rng) {
    const TraceParams& P = C.P;
    emitter_clear(ps.em);
    const LightSample ls = sample_light(P, s.pos, rng, C.ctr.env);
    const float lpdf = ls.pdf;
    const float3 wi = ls.wi, Li = ls.Li;
    if (lpdf <= 0.0f || all_zero(Li)) return false;
    if (dot(s.snrm, wi) <= 0.0f) return false;
    float3 n, wo, alb;
    float met;
    const bool metallic_on = (P.flags & kMetallic) != 0;
    shading_frame(s, n, wo, alb, met, metallic_on);
    float spdf;
    const BrdfTerms bc = eval_brdf<false>(wo, n, alb, met, clamp_rough(s.rough), wi, metallic_on, spdf);
    if (ls.type == kLightPoint) spdf = 0.0f;  // a delta light: no BRDF-side MIS weight
    ps.em.dir = wi;
    ps.em.tmax = ls.dist < 1e19f ? fmaxf(0.0f, ls.dist - 2e-2f) : kFarT;
    ps.em.light_pdf = lpdf;
    ps.em.scatter_pdf = spdf;
    ps.em.light = Li;
    ps.em.contribution = ps.throughput * bc.value * Li / fmaxf(lpdf, 1e-6f);
    return true;
}

template <class Ctx>
PTIR_DEV bool nee_prepare(const Ctx& C, PathState& ps, const Segment& s, Pcg32& rng) {
    const bool shadow = nee_prepare_light(C, ps, s, rng);
    sig_event(C.P, ps, kSigNee | (shadow ? 1u : 0u));
    return shadow;
}

// second half: the stochastic shadow ray from the interaction toward the sampled direction;
// an occluded sample leaves an empty emitter
template <class Ctx>
PTIR_DEV void nee_shadow(const Ctx& C, PathState& ps, const Segment& s, Pcg32& rng) {
    ++C.ctr.segments;
    const float3 wi = ps.em.dir;
    const bool occluded = shadow_occluded(C, s.pos + wi * 2e-2f, wi, ps.em.tmax, rng);
    sig_event(C.P, ps, kSigShadow | (occluded ? 1u : 0u));
    if (occluded) emitter_clear(ps.em);
}

template <class Ctx>
PTIR_DEV void sample_nee(const Ctx& C, PathState& ps, const Segment& s, Pcg32& rng) {
    if (nee_prepare(C, ps, s, rng)) nee_shadow(C, ps, s, rng);
}

// BRDF-sampled continuation (pathTracer.cuh:430-459)
template <class Ctx>
PTIR_DEV void sample_next(const Ctx& C, PathState& ps, Segment& s, Pcg32& rng) {
    const TraceParams& P = C.P;
    float3 n, wo, alb;
    float met;
    const bool metallic_on = (P.flags & kMetallic) != 0;
    shading_frame(s, n, wo, alb, met, metallic_on);
    float3 next = s.d;
    const float3 rnd = rng.uniform3();
    const BrdfSample b = sample_brdf<false>(wo, n, alb, met, clamp_rough(s.rough), rnd, metallic_on, next);
    const float3 nt = ps.throughput * b.value;
    if (all_zero(nt)) {
        ps.throughput = f3(0.0f);
        ps.active = 0u;
        return;
    }
    ps.throughput = nt;
    const float lpdf = (P.flags & kMis) ? light_sampler_pdf(P, s.pos, next) : 0.0f;
    const float3 origin = s.pos + normalize_or_keep(next) * 2e-2f;
    segment_reset(s, origin, next, 0.0f);
    if (P.flags & kMis) {
        s.scatter_pdf = b.pdf;
        s.light_pdf = lpdf;
    }
}

// What an escaped segment sees (environment.cuh:599-634): with render.visualize_lights the
// nearest sphere or mesh light along its ray, else the environment. 0: nothing, 1: a light
// (radiance in vr), 2: the environment (looked up by the caller).
template <class Ctx>
PTIR_DEV int escaped_light(const Ctx& C, const Segment& s, float3& vr) {
    const TraceParams& P = C.P;
    if ((P.flags & kVisualizeLights) && visible_area_light(P.lights, s.o, s.d, vr)) return 1;
    return env_present(P.env) ? 2 : 0;
}

// Radiance gathered at the end of a segment (environment.cuh:636-715)
template <class Ctx>
PTIR_DEV void accumulate_light(const Ctx& C, PathState& ps, Segment& s) {
    const TraceParams& P = C.P;
    const bool first = ps.bounces == 1u;
    const bool mis = (P.flags & kMis) != 0;
    float bmis = 1.0f, lmis = 1.0f;
    if (mis && first) {
        bmis = mis_weight(s.scatter_pdf, s.light_pdf);
        lmis = mis_weight(ps.em.light_pdf, ps.em.scatter_pdf);
    }
    const float3 nee = ps.em.contribution * lmis;
    if (P.render_opts == 1u) {
        if (mis && first) ps.acc += nee;
        if (ps.bounces > 0u && s.ivalid) {
            float3 contrib = ps.throughput * s.radiance;
            if (mis && first) contrib *= bmis;
            ps.acc += contrib;
            ps.acc_indirect += contrib;
        } else if (s.escaped) {
            float3 vr;
            const int seen = escaped_light(C, s, vr);
            if (seen == 0) return;
            if (seen == 2) vr = env_radiance(P.env, s.d, C.ctr.env);
            ps.throughput *= s.transmittance;
            s.light += vr;
            ps.acc_light += vr;
            float3 contrib = ps.throughput * s.light;
            if (mis && first) contrib *= bmis;
            ps.acc += contrib;
            ps.acc_direct += contrib;
        }
        return;
    }
    if (mis && first) {
        ps.acc += nee;
        ps.acc_direct += nee;
    }
    if (s.escaped) {
        float3 vr;
        const int seen = escaped_light(C, s, vr);
        if (seen == 0) return;
        if (seen == 2) vr = env_radiance(P.env, s.d, C.ctr.env);
        ps.throughput *= s.transmittance;
        s.light += vr;
        ps.acc_light += vr;
        float3 contrib = ps.throughput * s.light;
        if (mis && first) contrib *= bmis;
        s.radiance += contrib;
        ps.acc += contrib;
        if (ps.bounces < 2u) ps.acc_direct += contrib;
        else ps.acc_indirect += contrib;
    }
}

PTIR_DEV void path_init(PathState& ps, unsigned max_bounces) {
    ps.sig = 2166136261u;
    ps.active = 1u;
    ps.bounces = 0u;
    ps.max_bounces = max_bounces;
    ps.acc = ps.acc_grad = ps.acc_direct = ps.acc_indirect = ps.acc_light = ps.acc_light_grad = f3(0.0f);
    ps.throughput = f3(1.0f);
    ps.em.dir = ps.em.contribution = f3(0.0f);
    ps.em.light_pdf = ps.em.scatter_pdf = 0.0f;
    ps.pend_valid = false;
    ps.pend_o = ps.pend_d = ps.pend_dnext = f3(0.0f);
    ps.pend_opacity = ps.pend_max_hit = 0.0f;
    ps.pend_bounces = 0u;
}

// channels 0..2 of a strided per-sample array at element offset `off`
PTIR_DEV float3 ld_sample3(const float* a, const SampleLayout& L, long long off) {
    return make_float3(__ldg(a + off), __ldg(a + off + L.sc), __ldg(a + off + 2 * L.sc));
}

// world-space ray of sample (x, y, z) of launch `view` (flat index li)
PTIR_DEV void world_ray(const TraceParams& P, int view, unsigned x, unsigned y, unsigned z, size_t li, float3& o,
                        float3& d) {
    const float* m = P.views[view].to_world;
    const bool flat = P.flat_samples != 0;
    const float3 lo = ld_sample3(P.ray_ori, P.ray_ori_layout, sample_offset(P.ray_ori_layout, flat, z, y, x, li));
    const float3 ld = ld_sample3(P.ray_dir, P.ray_dir_layout, sample_offset(P.ray_dir_layout, flat, z, y, x, li));
    const float3 m0 = ld3(m), m1 = ld3(m + 4), m2 = ld3(m + 8);
    o = make_float3(dot(m0, lo) + __ldg(m + 3), dot(m1, lo) + __ldg(m + 7), dot(m2, lo) + __ldg(m + 11));
    d = make_float3(dot(m0, ld), dot(m1, ld), dot(m2, ld));
}

// The adjoint's per-sample inputs (the forward's pbr and light and their incoming gradients) into
// the path state, and the incoming material-output gradient onto the primary interaction.
PTIR_DEV void load_adjoint_inputs(const TraceParams& P, const BwdInputs& B, unsigned x, unsigned y, unsigned z,
                                  size_t li, PathState& ps) {
    const bool flat = P.flat_samples != 0;
    auto at = [&](const float* a, const SampleLayout& L) {
        return a ? ld_sample3(a, L, sample_offset(L, flat, z, y, x, li)) : f3(0.0f);
    };
    ps.acc = at(B.pbr, B.pbr_layout);
    ps.acc_grad = at(B.pbr_grad, B.pbr_grad_layout);
    ps.acc_light = at(B.light, B.light_layout);
    ps.acc_light_grad = at(B.light_grad, B.light_grad_layout);
}

PTIR_DEV void add_material_output_grad(const TraceParams& P, const BwdInputs& B, unsigned x, unsigned y, unsigned z,
                                       size_t li, Segment& s) {
    if (!s.ivalid || !B.material_grad) return;
    const SampleLayout& L = B.material_grad_layout;
    const long long off = sample_offset(L, P.flat_samples != 0, z, y, x, li);
    s.d_albedo += ld_sample3(B.material_grad, L, off);
    s.d_rough += __ldg(B.material_grad + off + 3 * L.sc);
    if (P.flags & kMetallic) s.d_metal += __ldg(B.material_grad + off + 4 * L.sc);
}

PTIR_DEV unsigned effective_bounces(const TraceParams& P) {
    return P.render_opts ? min(P.max_bounces, 2u) : P.max_bounces;
}

// Lane `lane` of 8x4 pixel tile `tile` of the batch: its view, launch index (x, y, z) within the
// view and flat launch index li; false past the last tile or outside the view's image.
PTIR_DEV bool tile_launch(const TraceParams& P, long long tile, unsigned lane, int& view, unsigned& x, unsigned& y,
                          unsigned& z, size_t& li) {
    if (tile < 0 || tile >= P.tiles) return false;
    int v = 0;
    while (v + 1 < P.nviews && P.views[v + 1].tile0 <= tile) ++v;
    const ViewDesc& V = P.views[v];
    const unsigned tiles_x = (unsigned)(V.w + 7) >> 3, tiles_y = (unsigned)(V.h + 3) >> 2;
    const unsigned long long local = (unsigned long long)(tile - V.tile0);
    const unsigned long long per_z = (unsigned long long)tiles_x * tiles_y;
    z = (unsigned)(local / per_z);
    const unsigned t = (unsigned)(local - (unsigned long long)z * per_z);
    const unsigned ty = t / tiles_x, tx = t - ty * tiles_x;
    x = (tx << 3) + (lane & 7u);
    y = (ty << 2) + (lane >> 3);
    view = v;
    li = (size_t)V.offset + ((size_t)z * V.h + y) * V.w + x;
    return z < (unsigned)V.z && x < (unsigned)V.w && y < (unsigned)V.h;
}

// launch index of this thread in the megakernel: warps own 8x4 pixel tiles
PTIR_DEV bool launch_index(const TraceParams& P, int& view, unsigned& x, unsigned& y, unsigned& z, size_t& li) {
    const long long warp = (long long)((blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5);
    return tile_launch(P, warp, threadIdx.x & 31u, view, x, y, z, li);
}

PTIR_DEV void flush_counters(const TraceParams& P, const TraceCounters& c) {
    if (P.counters == nullptr) return;
    const unsigned v[9] = {c.segments, c.calls, c.candidates, c.accepted, c.env, c.replay, c.replay_accepted, c.nodes,
                           c.leaves};
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const unsigned s = __reduce_add_sync(0xFFFFFFFFu, v[k]);
        if ((threadIdx.x & 31u) == 0u && s) atomicAdd(P.counters + k, (unsigned long long)s);
    }
}

// Front-to-back compositing of one segment over k-buffer batches (pathTracer.cuh:216-311 with
// processHit, gaussianParticles.cuh:343-440), split so that a schedule can interleave the trace
// calls of many segments: composite_begin, then while composite_open: one trace call over
// (composite_tmin, composite_tend), stop if it found nothing, composite_hits; then composite_end.
constexpr int kMaxRounds = 1 << 16;  // trace calls per segment before the loop-bound error

struct Composite {
    float3 o, d;
    float3 radiance, normal, albedo, snrm;
    float transmittance, depth, hit2, distortion, hits_count, rough, metal;
    float last_hit, clip_end;
    bool hit;
};

PTIR_DEV void composite_begin(const TraceParams& P, Composite& c, float3 o, float3 d) {
    const float2 clip = clip_scene(P, o, d);
    c.o = o;
    c.d = d;
    c.radiance = c.normal = c.albedo = c.snrm = f3(0.0f);
    c.transmittance = 1.0f;
    c.depth = c.hit2 = c.distortion = c.hits_count = c.rough = c.metal = 0.0f;
    c.last_hit = fmaxf(0.0f, clip.x - 1e-9f);
    c.clip_end = clip.y;
    c.hit = false;
}

PTIR_DEV bool composite_open(const TraceParams& P, const Composite& c) {
    return c.last_hit <= c.clip_end && c.transmittance > P.min_transmittance;
}
PTIR_DEV float composite_tmin(const Composite& c) { return c.last_hit + 1e-9f; }
PTIR_DEV float composite_tend(const Composite& c) { return c.clip_end + 1e-9f; }

// Composite candidate (t, id) of a batch. Accepted Gaussians are flagged in `vis` (when given)
// as int32 1 inside the float32 tensor, as the reference does (pathTracer.cuh:283-284).
template <bool kSelfOcc>
PTIR_DEV void composite_one(const TraceParams& P, TraceCounters& ctr, Composite& c, float t, unsigned id, float* vis) {
    if (id == kNoHit || !(c.transmittance > P.min_transmittance)) return;
    if (kSelfOcc && self_occluded(P, t, id, c.d)) {
        c.last_hit = fmaxf(c.last_hit, t);
        return;
    }
    float dns;
    const Response r = respond(P, id, c.o, c.d, dns);
    const bool accept = r.gres > P.min_response && r.alpha > P.alpha_min;
    if (accept) {
        ++ctr.accepted;
        const float w = r.alpha * c.transmittance;
        const float3 grds = r.scl * r.grd * dot(r.grd, -r.gro);
        const float hit_t = sqrtf(dot(grds, grds));
        c.radiance += sh_radiance(P, id, c.d) * w;
        float3 alb;
        float rgh, met;
        load_material(P.part, id, alb, rgh, met);
        c.albedo += alb * w;
        c.rough += rgh * w;
        c.metal += met * w;
        c.transmittance *= (1.0f - r.alpha);
        c.depth += hit_t * w;
        c.hit2 += hit_t * hit_t * w;
        if (P.flags & kNormals) {
            c.snrm += load_snrm(P.part, id) * w;
            const float3 srot = mul_cols(r.rt, r.scl);
            c.normal += normalize_or_keep((r.gro + r.grd * (dot(r.grd, -r.gro) - sqrtf(9.0f - r.d2))) * srot) * w;
        }
        c.hit = true;
        const float op = 1.0f - c.transmittance;
        c.distortion = fmaxf(op * c.hit2 - c.depth * c.depth, 0.0f);
        if (vis) vis[id] = __int_as_float(1);
    }
    c.last_hit = fmaxf(c.last_hit, t);
    c.hits_count += accept ? 1.0f : 0.0f;  // the output is written only with kHitCounts
}

// Composite one k-buffer batch held in registers.
template <bool kSelfOcc, int K>
PTIR_DEV void composite_hits(const TraceParams& P, TraceCounters& ctr, Composite& c, const float (&kt)[K],
                             const unsigned (&kid)[K], float* vis) {
#pragma unroll
    for (int i = 0; i < K; ++i) composite_one<kSelfOcc>(P, ctr, c, kt[i], kid[i], vis);
}

// Composite one k-buffer batch held in memory (entry i at kt[i * stride], kid[i * stride]).
template <bool kSelfOcc, int K>
PTIR_DEV void composite_hits_strided(const TraceParams& P, TraceCounters& ctr, Composite& c, const float* kt,
                                     const unsigned* kid, int stride, float* vis) {
#pragma unroll 1
    for (int i = 0; i < K; ++i) {
        const unsigned id = kid[i * stride];
        if (id == kNoHit) break;  // the batch is sorted: the rest is empty too
        composite_one<kSelfOcc>(P, ctr, c, kt[i * stride], id, vis);
    }
}

// Composite entries [from, to) of a batch held in memory whose entries are leaf-record indices
// (k-buffers filled with kLeafIndex).
template <bool kSelfOcc>
PTIR_DEV void composite_leaf_batch(const TraceParams& P, TraceCounters& ctr, Composite& c, const float* kt,
                                   const unsigned* kp, int stride, int from, int to, float* vis) {
#pragma unroll 1
    for (int i = from; i < to; ++i) {
        const unsigned p = kp[i * stride];
        if (p == kNoHit) break;
        composite_one<kSelfOcc>(P, ctr, c, kt[i * stride], leaf_gaussian(P.accel, p), vis);
    }
}

// The segment after compositing: every field reset but the MIS pdfs (kept when MIS is on),
// the interaction when the segment is opaque enough, else the escape draw.
PTIR_DEV void composite_end(const TraceParams& P, const Composite& c, float scatter_pdf, float light_pdf, Segment& s,
                            Pcg32& rng) {
    segment_reset(s, c.o, c.d, c.last_hit);
    if (P.flags & kMis) {
        s.scatter_pdf = scatter_pdf;
        s.light_pdf = light_pdf;
    }
    s.radiance = c.radiance;
    s.normal = c.normal;
    s.transmittance = c.transmittance;
    s.depth = c.depth;
    s.hit2 = c.hit2;
    s.distortion = c.distortion;
    s.hits_count = c.hits_count;
    s.hit = c.hit;
    const float op = 1.0f - s.transmittance;
    if (s.hit && op > 0.5f) {
        const float inv = 1.0f / fmaxf(op, 1e-12f);
        s.ivalid = true;
        s.pos = s.o + s.d * (s.depth * inv);
        s.snrm = c.snrm * inv;
        s.albedo = c.albedo * inv;
        s.rough = c.rough * inv;
        s.metal = c.metal * inv;
    } else {
        s.escaped = rng.uniform() < s.transmittance;
    }
}

template <bool kSelfOcc, class Ctx>
PTIR_DEV void intersect_mark(const Ctx& C, Segment& s, Pcg32& rng, float* vis) {
    const TraceParams& P = C.P;
    Composite c;
    composite_begin(P, c, s.o, s.d);
    float kt[Ctx::K];
    unsigned kid[Ctx::K];
    for (int round = 0; composite_open(P, c); ++round) {
        if (round > kMaxRounds) {
            atomicOr(P.error_word, kErrLoopBound);
            break;
        }
        trace_kbuf(P.accel, c.o, c.d, composite_tmin(c), composite_tend(c), kt, kid, C.stack, P.error_word,
                   C.ctr);
        if (kid[0] == kNoHit) break;
        composite_hits<kSelfOcc>(P, C.ctr, c, kt, kid, vis);
        // a k-buffer that is not full held every candidate of the call: a later call finds none
        if (kid[Ctx::K - 1] == kNoHit) break;
    }
    composite_end(P, c, s.scatter_pdf, s.light_pdf, s, rng);
}

// ------------------------------------------------------------------------------------
// Gradient scatter: a float atomic add, and with a compensation buffer the rounding error of
// that add (TwoSum of the value found and the term, in round-to-nearest) added to the buffer,
// so that sum + compensation carries the terms to about twice float precision however many
// paths hit the same Gaussian or texel.
PTIR_DEV void grad_add(float* g, float* comp, float v) {
    const float old = atomicAdd(g, v);
    if (!comp) return;
    const float s = __fadd_rn(old, v);
    const float bp = __fsub_rn(s, old);
    const float err = __fadd_rn(__fsub_rn(old, __fsub_rn(s, bp)), __fsub_rn(v, bp));
    if (err != 0.0f) atomicAdd(comp, err);
}

// Scatter of one row of gradient terms (a Gaussian's material row, an environment texel's
// colour), terms v[0..n). With kWarpAggregate the active lanes that add to the same row first
// combine their terms, by shuffles in lane order, and the lowest of them issues the row's
// atomics: the atomic traffic on a popular Gaussian or texel falls by the number of lanes that
// share it, and only the order of the float additions changes. With a compensation buffer the
// rounding errors of that combination (TwoSum) go to the buffer too, so the compensated sums
// keep their accuracy whichever lanes happen to meet.
template <int N>
PTIR_DEV void grad_add_row(unsigned flags, float* g, float* comp, float (&v)[N], int n) {
    float err[N];
#pragma unroll
    for (int k = 0; k < N; ++k) err[k] = 0.0f;
    if (flags & kWarpAggregate) {
        const unsigned lane = threadIdx.x & 31u;
        const unsigned peers = __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(g));
        if (peers != (1u << lane)) {
            float sum[N];
#pragma unroll
            for (int k = 0; k < N; ++k) sum[k] = 0.0f;
            for (unsigned m = peers; m; m &= m - 1u) {
                const int src = __ffs(m) - 1;
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    const float x = __shfl_sync(peers, v[k], src);
                    const float t = __fadd_rn(sum[k], x);
                    const float bp = __fsub_rn(t, sum[k]);
                    err[k] = __fadd_rn(err[k], __fadd_rn(__fsub_rn(sum[k], __fsub_rn(t, bp)), __fsub_rn(x, bp)));
                    sum[k] = t;
                }
            }
            if ((int)lane != __ffs(peers) - 1) return;
#pragma unroll
            for (int k = 0; k < N; ++k) v[k] = sum[k];
        }
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (k >= n) continue;
        grad_add(g + k, comp ? comp + k : nullptr, v[k]);
        if (comp && err[k] != 0.0f) atomicAdd(comp + k, err[k]);
    }
}

// ------------------------------------------------------------------------------------
// backward: path replay ("radiative backprop") of referenceBwdOptix.cu:27-74

// One re-traversal of a segment that scatters a material gradient onto its Gaussians
// (the arguments of the reference's rayIntersectBwd).
struct ReplayJob {
    float3 o, d, da;
    float opacity, max_hit, dr, dm;
    unsigned self_occ;
};

// A replay job in progress: its ray, the per-opacity material gradient it scatters, the
// interval still to re-traverse and the transmittance so far.
struct ReplayState {
    float3 o, d, da;
    float dr, dm, start, end, tr;
    bool self_occ;
};

PTIR_DEV void replay_begin(const TraceParams& P, const ReplayJob& j, ReplayState& r, TraceCounters& ctr) {
    ++ctr.replay;
    r.self_occ = j.self_occ != 0u;
    r.o = j.o;
    r.d = j.d;
    const float inv = 1.0f / fmaxf(j.opacity, 1e-12f);
    r.da = j.da * inv;
    r.dr = j.dr * inv;
    r.dm = j.dm * inv;
    const float2 clip = clip_scene(P, r.o, r.d);
    r.start = fmaxf(0.0f, clip.x - 1e-9f);
    // The reference ends the re-traversal at max_hit + 1e-9 in float: beyond t ~ 0.017 that is
    // max_hit itself, and with the strict t < tend test the segment's last composited Gaussian
    // gets no gradient. kExactReplay extends the end by one float step to include it.
    r.end = (P.flags & kExactReplay) ? nextafterf(fminf(j.max_hit, clip.y), 3.0e38f) : fminf(j.max_hit, clip.y) + 1e-9f;
    r.tr = 1.0f;
}

PTIR_DEV bool replay_open(const TraceParams& P, const ReplayState& r) {
    return r.start < r.end && r.tr > P.min_transmittance;
}

// Scatter the material gradient onto the accepted hits of one k-buffer batch, front to back
// (with kLeafIndex the batch holds leaf record indices).
template <int K, bool kLeafIndex = false>
PTIR_DEV void replay_batch(const TraceParams& P, const BwdInputs& B, ReplayState& r, const float (&kt)[K],
                           const unsigned (&kid)[K], TraceCounters& ctr) {
    const bool metallic_on = (P.flags & kMetallic) != 0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        if (kid[i] == kNoHit || !(r.tr > P.min_transmittance)) continue;
        const unsigned id = kLeafIndex ? leaf_gaussian(P.accel, kid[i]) : kid[i];
        if (r.self_occ && self_occluded(P, kt[i], id, r.d)) {
            r.start = fmaxf(r.start, kt[i]);
            continue;
        }
        float dns;
        const Response res = respond(P, id, r.o, r.d, dns);
        if (res.gres > P.min_response && res.alpha > P.alpha_min) {
            ++ctr.replay_accepted;
            const float w = res.alpha * r.tr;
            float* g = B.particle_material_grad + 5 * (size_t)id;
            float* cg = B.particle_material_comp ? B.particle_material_comp + 5 * (size_t)id : nullptr;
            float row[5] = {w * r.da.x, w * r.da.y, w * r.da.z, w * r.dr, w * r.dm};
            grad_add_row(P.flags, g, cg, row, metallic_on ? 5 : 4);
            r.tr *= (1.0f - res.alpha);
        }
        r.start = fmaxf(r.start, kt[i]);
    }
}

// pathTracer.cuh:313-390: one re-traversal that scatters a material gradient onto its Gaussians.
// With a frontier F (k-buffer 8 or 16) the rounds after the first resume from what the previous
// round set aside (traverse.cuh).
template <class Ctx>
PTIR_DEV void replay_material_grad(const Ctx& C, const BwdInputs& B, const ReplayJob& j, const Frontier* F = nullptr) {
    constexpr int K = Ctx::K;
    const TraceParams& P = C.P;
    ReplayState r;
    replay_begin(P, j, r, C.ctr);
    float kt[K];
    unsigned kid[K];
    TraceState t;
    for (int round = 0; replay_open(P, r); ++round) {
        if (round > (1 << 16)) {
            atomicOr(P.error_word, kErrLoopBound);
            break;
        }
        if constexpr (K <= 16) {
            if (F) {
                if (trace_start<K, true, true>(P.accel, r.o, r.d, r.start + 1e-9f, r.end, kt, kid, t, C.ctr, F,
                                               round > 0)) {
                    while (trace_step<K, true, true>(P.accel, r.o, r.d, t, kt, kid, C.stack, P.error_word,
                                                     C.ctr, F)) {
                    }
                }
                if (kid[0] == kNoHit) break;
                replay_batch<K, true>(P, B, r, kt, kid, C.ctr);
                if (kid[K - 1] == kNoHit) break;
                continue;
            }
        }
        trace_kbuf(P.accel, r.o, r.d, r.start + 1e-9f, r.end, kt, kid, C.stack, P.error_word, C.ctr);
        if (kid[0] == kNoHit) break;
        replay_batch(P, B, r, kt, kid, C.ctr);
        if (kid[K - 1] == kNoHit) break;
    }
}

// environment texel gradient of a bilinear lookup plus the finite-difference direction gradient
// (environment.cuh:89-114, 421-473)
template <class Ctx>
PTIR_DEV float3 env_radiance_bwd(const Ctx& C, const BwdInputs& B, float3 d, float3 cg, float3& dir_grad) {
    const EnvView& E = C.P.env;
    if (!env_present(E)) return f3(0.0f);
    const EnvRotation rot = env_rotation(E);
    const Footprint f = footprint_of(E, env_rotate(rot, d));
    const float3 bg = bilerp(E, f);
    ++C.ctr.env;
    if (B.environment_grad) {
        auto add = [&](int x, int y, float w) {
            const size_t texel = 4 * ((size_t)y * E.w + x);
            float* g = B.environment_grad + texel;
            float* c = B.environment_comp ? B.environment_comp + texel : nullptr;
            float row[3] = {w * cg.x, w * cg.y, w * cg.z};
            grad_add_row(C.P.flags, g, c, row, 3);
        };
        add(f.x0, f.y0, f.w00);
        add(f.x1, f.y0, f.w10);
        add(f.x0, f.y1, f.w01);
        add(f.x1, f.y1, f.w11);
    }
    const float3 u = normalize_or_keep(d);
    float3 t, b;
    onb(u, t, b);
    const float eps = 1e-3f;
    const float ps = rsqrtf(1.0f + eps * eps);
    const float3 tb = bilerp(E, footprint_of(E, env_rotate(rot, (u + t * eps) * ps)));
    const float3 bb = bilerp(E, footprint_of(E, env_rotate(rot, (u + b * eps) * ps)));
    C.ctr.env += 2;
    const float ie = 1.0f / eps;
    dir_grad += t * dot((tb - bg) * ie, cg) + b * dot((bb - bg) * ie, cg);
    return bg;
}

// environment.cuh:717-808
template <class Ctx>
PTIR_DEV void accumulate_light_bwd(const Ctx& C, const BwdInputs& B, PathState& ps, Segment& s) {
    const TraceParams& P = C.P;
    const bool first = ps.bounces == 1u;
    const bool mis = (P.flags & kMis) != 0;
    float bmis = 1.0f, lmis = 1.0f;
    if (mis && first) {
        bmis = mis_weight(s.scatter_pdf, s.light_pdf);
        lmis = mis_weight(ps.em.light_pdf, ps.em.scatter_pdf);
    }
    if (P.render_opts == 1u) {
        if (mis && first) ps.acc -= ps.em.contribution * lmis;
        if (ps.bounces > 0u && s.ivalid) {
            float3 contrib = ps.throughput * s.radiance;
            if (mis && first) contrib *= bmis;
            ps.acc -= contrib;
        } else if (s.escaped) {
            float3 vr;
            const int seen = escaped_light(C, s, vr);
            if (seen == 0) return;
            ps.throughput *= s.transmittance;
            float3 eg = ps.acc_grad * ps.throughput;
            if (mis && first) eg *= bmis;
            eg += ps.acc_light_grad;
            if (seen == 2) vr = env_radiance_bwd(C, B, s.d, eg, s.ray_dir_grad);
            float3 contrib = ps.throughput * vr;
            if (mis && first) contrib *= bmis;
            ps.acc -= contrib;
        }
        return;
    }
    if (mis && first) ps.acc -= ps.em.contribution * lmis;
    if (s.escaped) {
        float3 vr;
        const int seen = escaped_light(C, s, vr);
        if (seen == 0) return;
        ps.throughput *= s.transmittance;
        float3 eg = ps.acc_grad * ps.throughput;
        if (mis && first) eg *= bmis;
        eg += ps.acc_light_grad;
        if (seen == 2) vr = env_radiance_bwd(C, B, s.d, eg, s.ray_dir_grad);
        float3 contrib = ps.throughput * vr;
        if (mis && first) contrib *= bmis;
        s.radiance += contrib;
        ps.acc -= contrib;
    }
}

// pathTracer.cuh:392-428; `replay` receives the re-traversal (run now or queued)
template <class Replay>
PTIR_DEV void pending_bwd(PathState& ps, const Segment& s, Replay&& replay) {
    if (!ps.pend_valid) return;
    const float dr = dot(s.ray_dir_grad, ps.pend_dnext);
    ps.pend_valid = false;
    if (dr == 0.0f) return;
    replay(ReplayJob{ps.pend_o, ps.pend_d, f3(0.0f), ps.pend_opacity, ps.pend_max_hit, dr, 0.0f,
                     ps.pend_bounces > 1u ? 1u : 0u});
}

// pathTracer.cuh:506-548 (albedo only; the environment and roughness terms are disabled there).
// The reference weights the term by the environment's radiance in the sampled direction, whatever
// light was sampled; with exact_replay the sampled light's radiance is used, which is the same
// for environment samples and the derivative of the estimator for the other lights.
template <class Ctx>
PTIR_DEV void nee_grad_bwd(const Ctx& C, PathState& ps, Segment& s, const Segment& it) {
    const TraceParams& P = C.P;
    if (ps.bounces != 1u || ps.em.light_pdf <= 0.0f) return;
    float3 n, wo, alb;
    float met;
    const bool metallic_on = (P.flags & kMetallic) != 0;
    shading_frame(it, n, wo, alb, met, metallic_on);
    float spdf;
    const BrdfTerms g = eval_brdf<true>(wo, n, alb, met, it.rough, ps.em.dir, metallic_on, spdf);
    const float scale = mis_weight(ps.em.light_pdf, ps.em.scatter_pdf) / fmaxf(ps.em.light_pdf, 1e-6f);
    const float3 bgc = (P.flags & kExactReplay) ? ps.em.light : env_radiance(P.env, ps.em.dir, C.ctr.env);
    const float3 dl = ps.acc_grad * ps.throughput * bgc * scale;
    s.d_albedo += dl * g.d_albedo;
}

// pathTracer.cuh:551-634; `replay` receives the re-traversal of the scattering segment
template <class Ctx, class Replay>
PTIR_DEV void sample_next_bwd(const Ctx& C, PathState& ps, Segment& s, Pcg32& rng, Replay&& replay) {
    const TraceParams& P = C.P;
    const bool metallic_on = (P.flags & kMetallic) != 0;
    const bool mis = (P.flags & kMis) != 0;
    const Segment it = s;  // the interaction being scattered from
    float3 n, wo, alb;
    float met;
    shading_frame(it, n, wo, alb, met, metallic_on);
    float3 next = it.d;
    const float3 rnd = rng.uniform3();
    const BrdfSample b = sample_brdf<true>(wo, n, alb, met, it.rough, rnd, metallic_on, next);
    const float3 nt = ps.throughput * b.value;
    if (all_zero(nt)) {
        ps.throughput = f3(0.0f);
        ps.active = 0u;
        return;
    }
    float lpdf = 0.0f;
    bool first_nee = false;
    if (mis) {
        lpdf = light_sampler_pdf(P, it.pos, next);
        first_nee = ps.bounces == 1u && max3(nt) >= 1e-4f;
        if (first_nee) nee_grad_bwd(C, ps, s, it);
    }
    float3 dep = ps.acc;
    if (mis && first_nee) dep -= ps.em.contribution * mis_weight(ps.em.light_pdf, ps.em.scatter_pdf);
    const float3 num = ps.acc_grad * dep;
    const float3 dl = make_float3(b.value.x > kBrdfEps ? num.x / b.value.x : 0.0f,
                                  b.value.y > kBrdfEps ? num.y / b.value.y : 0.0f,
                                  b.value.z > kBrdfEps ? num.z / b.value.z : 0.0f);
    s.d_albedo += dl * b.d_albedo;
    s.d_rough += dot(dl, b.d_rough);
    if (metallic_on) s.d_metal += dot(dl, b.d_metallic);
    ps.pend_valid = dot(b.d_next_dir, b.d_next_dir) > 0.0f;
    ps.pend_o = it.o;
    ps.pend_d = it.d;
    ps.pend_opacity = 1.0f - it.transmittance;
    ps.pend_max_hit = it.last_hit;
    ps.pend_dnext = b.d_next_dir;
    ps.pend_bounces = ps.bounces;
    if (!all_zero(s.d_albedo) || s.d_rough != 0.0f || s.d_metal != 0.0f)
        replay(ReplayJob{it.o, it.d, s.d_albedo, 1.0f - it.transmittance, it.last_hit, s.d_rough, s.d_metal,
                         ps.bounces > 1u ? 1u : 0u});
    ps.throughput = nt;
    const float3 origin = it.pos + normalize_or_keep(next) * 2e-2f;
    segment_reset(s, origin, next, 0.0f);
    if (mis) {
        s.scatter_pdf = b.pdf;
        s.light_pdf = lpdf;
    }
}

}  // namespace ptir
