// Environment lighting and the "fast" GGX/Lambert BRDF used by the path tracer, in FP32.
//
// Behaviour follows the reference's device code:
//   environment lookups  threedgptir_tracer/include/3dgptir/kernels/cuda/environment.cuh:49-473
//   BRDF and its grads   threedgptir_tracer/include/3dgptir/kernels/cuda/material.cuh:40-634
#pragma once

#include "device_types.h"
#include "pcg.cuh"
#include "vecmath.cuh"

namespace ptir {

// ------------------------------------------------------------------------------------
// environment map (equirectangular [h, w] or cube map [6w, w]), bilinear with u wrap / v clamp
struct Footprint {
    int x0, x1, y0, y1;
    float w00, w10, w01, w11;
};

PTIR_DEV int wrap_index(int v, int n) {
    if (n <= 0) return 0;
    int r = v % n;
    return r < 0 ? r + n : r;
}
PTIR_DEV int clamp_index(int v, int lo, int hi) { return max(lo, min(v, hi)); }

PTIR_DEV Footprint footprint_equirect(const EnvView& E, float u, float v) {
    u = u - floorf(u);
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    const float x = u * (float)E.w - 0.5f, y = v * (float)E.h - 0.5f;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const float ax = x - (float)x0, ay = y - (float)y0;
    Footprint f;
    f.x0 = wrap_index(x0, E.w);
    f.x1 = wrap_index(x0 + 1, E.w);
    f.y0 = clamp_index(y0, 0, E.h - 1);
    f.y1 = clamp_index(y0 + 1, 0, E.h - 1);
    f.w00 = (1.0f - ax) * (1.0f - ay);
    f.w10 = ax * (1.0f - ay);
    f.w01 = (1.0f - ax) * ay;
    f.w11 = ax * ay;
    return f;
}

PTIR_DEV Footprint footprint_cube(const EnvView& E, int face, float u, float v) {
    const int fs = E.w;
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    const float x = u * (float)fs - 0.5f, y = v * (float)fs - 0.5f;
    const int x0 = (int)floorf(x), y0 = (int)floorf(y);
    const float ax = x - (float)x0, ay = y - (float)y0;
    const int yo = face * fs;
    Footprint f;
    f.x0 = clamp_index(x0, 0, fs - 1);
    f.x1 = clamp_index(x0 + 1, 0, fs - 1);
    f.y0 = clamp_index(y0 + yo, yo, yo + fs - 1);
    f.y1 = clamp_index(y0 + 1 + yo, yo, yo + fs - 1);
    f.w00 = (1.0f - ax) * (1.0f - ay);
    f.w10 = ax * (1.0f - ay);
    f.w01 = (1.0f - ax) * ay;
    f.w11 = ax * ay;
    return f;
}

// The environment's rotation about z by 2 pi offset_x + pi / 2, then about x by 2 pi offset_y,
// evaluated at each lookup with the device's sincosf from the offsets held in memory, as the
// reference evaluates it (environment.cuh:116-178). The rounding of those sines and cosines
// (cos(pi / 2) is not zero in float) shows in the bilinear weights and, amplified by 1 / eps, in
// the finite-difference direction gradient, so they are computed the same way here.
struct EnvRotation {
    float sz, cz, sx, cx;
};
PTIR_DEV EnvRotation env_rotation(const EnvView& E) {
    EnvRotation r;
    sincosf(E.offset_x * 2.0f * kPiF + 0.5f * kPiF, &r.sz, &r.cz);
    sincosf(E.offset_y * 2.0f * kPiF, &r.sx, &r.cx);
    return r;
}
PTIR_DEV float3 env_rotate(const EnvRotation& r, float3 d) {
    const float3 z = make_float3(d.x * r.cz - d.y * r.sz, d.x * r.sz + d.y * r.cz, d.z);
    return make_float3(z.x, z.y * r.cx - z.z * r.sx, z.y * r.sx + z.z * r.cx);
}
PTIR_DEV float3 env_rotate(const EnvView& E, float3 d) { return env_rotate(env_rotation(E), d); }
PTIR_DEV float3 env_unrotate(const EnvView& E, float3 e) {
    const EnvRotation r = env_rotation(E);
    const float3 x = make_float3(e.x, e.y * r.cx + e.z * r.sx, -e.y * r.sx + e.z * r.cx);
    return make_float3(x.x * r.cz + x.y * r.sz, -x.x * r.sz + x.y * r.cz, x.z);
}

PTIR_DEV void equirect_uv(float3 d, float& u, float& v) {
    const float theta = atan2f(d.x, d.y);
    const float phi = asinf(fminf(1.0f, fmaxf(-1.0f, -d.z)));
    u = (theta + kPiF) * (0.5f * kInvPiF);
    v = 0.5f + phi * kInvPiF;
}

PTIR_DEV void cube_face_uv(float3 d, int& face, float& u, float& v) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    float ma, sc, tc;
    if (ax >= ay && ax >= az) {
        ma = ax;
        if (d.x > 0.0f) { face = 0; sc = -d.z; tc = -d.y; } else { face = 1; sc = d.z; tc = -d.y; }
    } else if (ay >= ax && ay >= az) {
        ma = ay;
        if (d.y > 0.0f) { face = 2; sc = d.x; tc = d.z; } else { face = 3; sc = d.x; tc = -d.z; }
    } else {
        ma = az;
        if (d.z > 0.0f) { face = 4; sc = d.x; tc = -d.y; } else { face = 5; sc = -d.x; tc = -d.y; }
    }
    const float im = 1.0f / fmaxf(ma, 1e-12f);
    u = 0.5f * (sc * im + 1.0f);
    v = 0.5f * (tc * im + 1.0f);
}

PTIR_DEV Footprint footprint_of(const EnvView& E, float3 rotated_dir) {
    if (E.cube) {
        int face;
        float u, v;
        cube_face_uv(rotated_dir, face, u, v);
        return footprint_cube(E, face, u, v);
    }
    float u, v;
    equirect_uv(rotated_dir, u, v);
    return footprint_equirect(E, u, v);
}

PTIR_DEV float3 texel(const EnvView& E, int x, int y) {
    const float4 t = __ldg(E.data + (size_t)y * E.w + x);
    return make_float3(t.x, t.y, t.z);
}

PTIR_DEV float3 bilerp(const EnvView& E, const Footprint& f) {
    return texel(E, f.x0, f.y0) * f.w00 + texel(E, f.x1, f.y0) * f.w10 + texel(E, f.x0, f.y1) * f.w01 +
           texel(E, f.x1, f.y1) * f.w11;
}

PTIR_DEV bool env_present(const EnvView& E) { return E.data != nullptr && E.w > 0 && E.h > 0; }
PTIR_DEV bool env_light_present(const EnvView& E) { return env_present(E) && E.cells > 0; }

// radiance seen along world direction d (zero without an environment)
PTIR_DEV float3 env_radiance(const EnvView& E, float3 d, unsigned& lookups) {
    if (!env_present(E)) return f3(0.0f);
    ++lookups;
    return bilerp(E, footprint_of(E, env_rotate(E, d)));
}

// equirect (u, v) -> direction
PTIR_DEV float3 equirect_direction(float u, float v) {
    u = u - floorf(u);
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    const float theta = u * kTwoPiF - kPiF, phi = (v - 0.5f) * kPiF;
    float st, ct, sp, cp;
    sincosf(theta, &st, &ct);
    sincosf(phi, &sp, &cp);
    return make_float3(st * cp, ct * cp, -sp);
}

PTIR_DEV float3 cube_direction(int face, float u, float v) {
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    const float s = 2.0f * u - 1.0f, t = 2.0f * v - 1.0f;
    float3 d;
    switch (face) {
    case 0: d = make_float3(1.0f, -t, -s); break;
    case 1: d = make_float3(-1.0f, -t, s); break;
    case 2: d = make_float3(s, 1.0f, t); break;
    case 3: d = make_float3(s, -1.0f, -t); break;
    case 4: d = make_float3(s, -t, 1.0f); break;
    default: d = make_float3(-s, -t, -1.0f); break;
    }
    return normalize_or_keep(d);
}

// Importance-sample a direction from the alias table: 2 draws pick the cell (Walker/Vose),
// 2 draws jitter inside it. Returns the world direction and the per-steradian pdf.
PTIR_DEV float3 sample_env_direction(const EnvView& E, Pcg32& rng, float& pdf) {
    const int cells = E.cells;
    const int first = min((int)(rng.uniform() * (float)cells), cells - 1);
    const int other = clamp_index((int)(__ldg(E.alias + first) + 0.5f), 0, cells - 1);
    const int cell = rng.uniform() < __ldg(E.prob + first) ? first : other;
    const int x = cell % E.aw, y = cell / E.aw;
    const float ju = rng.uniform();
    const float jv = rng.uniform();
    float3 d;
    if (E.cube) {
        const int fs = E.aw;
        const int face = clamp_index(y / fs, 0, 5);
        const int fy = y - face * fs;
        d = cube_direction(face, ((float)x + ju) / (float)fs, ((float)fy + jv) / (float)fs);
    } else {
        d = equirect_direction(((float)x + ju) / (float)E.aw, ((float)y + jv) / (float)E.ah);
    }
    pdf = __ldg(E.pdf + cell);
    return env_unrotate(E, d);
}

// per-steradian pdf of the alias sampler for direction d (cell lookup, no interpolation)
PTIR_DEV float env_pdf(const EnvView& E, float3 rd) {
    if (!env_light_present(E)) return 0.0f;
    const float3 d = env_rotate(E, rd);
    int x, y;
    if (E.cube) {
        int face;
        float u, v;
        cube_face_uv(d, face, u, v);
        const int fs = E.aw;
        x = clamp_index((int)(u * (float)fs), 0, fs - 1);
        y = min(face * fs + clamp_index((int)(v * (float)fs), 0, fs - 1), E.ah - 1);
    } else {
        float u, v;
        equirect_uv(d, u, v);
        x = wrap_index((int)(u * (float)E.aw), E.aw);
        y = clamp_index((int)(v * (float)E.ah), 0, E.ah - 1);
    }
    return __ldg(E.pdf + (size_t)y * E.aw + x);
}

PTIR_DEV float mis_weight(float a, float b) {
    const float a2 = a * a, b2 = b * b;
    return a2 / fmaxf(a2 + b2, 1e-6f);
}

// ------------------------------------------------------------------------------------
// BRDF: 50/50 Lambert (cosine hemisphere) / GGX half-vector sampling, Smith-Schlick G,
// Schlick Fresnel, roughness clamped to [0.05, 1].
constexpr float kBrdfEps = 1e-6f;
constexpr float kMinRough = 0.05f;

PTIR_DEV float saturate(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
PTIR_DEV float3 saturate(float3 v) { return make_float3(saturate(v.x), saturate(v.y), saturate(v.z)); }
PTIR_DEV float clamp_rough(float r) { return fminf(fmaxf(r, kMinRough), 1.0f); }
PTIR_DEV float3 relu3(float3 v) { return make_float3(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f), fmaxf(v.z, 0.0f)); }
PTIR_DEV float3 pos_mask(float3 v) {
    return make_float3(v.x > 0.0f ? 1.0f : 0.0f, v.y > 0.0f ? 1.0f : 0.0f, v.z > 0.0f ? 1.0f : 0.0f);
}
PTIR_DEV float3 normalize_or(float3 v, float3 fallback) {
    const float l2 = dot(v, v);
    return l2 > kBrdfEps ? v * rsqrtf(l2) : fallback;
}
PTIR_DEV float3 from_normal_space(float3 n, float3 l) {
    float3 t, b;
    onb(n, t, b);
    return t * l.x + b * l.y + n * l.z;
}

PTIR_DEV float3 sample_cosine(float3 n, float u1, float u2) {
    const float xi = saturate(u1);
    const float r = sqrtf(xi);
    float s, c;
    sincosf(kTwoPiF * saturate(u2), &s, &c);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - xi));
    return from_normal_space(n, make_float3(r * c, r * s, z));
}

PTIR_DEV float3 sample_ggx_half(float3 n, float rough, float u1, float u2) {
    const float a = rough * rough, a2 = a * a;
    const float xi = saturate(u1);
    const float den = fmaxf(1.0f + (a2 - 1.0f) * xi, kBrdfEps);
    const float ct = sqrtf(fmaxf(0.0f, (1.0f - xi) / den));
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float s, c;
    sincosf(kTwoPiF * saturate(u2), &s, &c);
    return from_normal_space(n, make_float3(st * c, st * s, ct));
}

struct BrdfTerms {
    float3 value;      // f * cos
    float3 d_albedo;
    float3 d_metallic;
    float3 d_rough;
};

// f(wo, L) cos(theta_L) and the mixed sampling pdf; with kGrad also d/d{albedo, metallic, roughness}
template <bool kGrad>
PTIR_DEV BrdfTerms eval_brdf(float3 wo, float3 n, float3 albedo, float metallic, float roughness, float3 ldir, bool metallic_on,
                             float& pdf) {
    BrdfTerms r;
    r.value = r.d_albedo = r.d_metallic = r.d_rough = f3(0.0f);
    const float3 L = normalize_or(ldir, n);
    const float NdotV = saturate(dot(n, wo)), NdotL = saturate(dot(n, L));
    pdf = 0.0f;
    if (NdotV <= 0.0f || NdotL <= 0.0f) return r;
    const float rough = clamp_rough(roughness);
    const float3 f0 = f3(0.04f) + (albedo - f3(0.04f)) * metallic;
    const float3 H = normalize_or(wo + L, n);
    const float NdotH = saturate(dot(n, H)), VdotH = saturate(dot(wo, H));
    const float x = 1.0f - saturate(VdotH), x2 = x * x, q = x2 * x2 * x;
    const float3 F = f0 + (f3(1.0f) - f0) * q;
    const float omm = 1.0f - metallic;
    const float3 dcol = albedo * omm;
    const float dscale = NdotL * kInvPiF;
    const float3 diffuse = dcol * (f3(1.0f) - F) * dscale;
    const float a = rough * rough, a2 = a * a;
    const float dden = fmaxf(NdotH * NdotH * (a2 - 1.0f) + 1.0f, kBrdfEps);
    const float D = a2 * kInvPiF / fmaxf(dden * dden, kBrdfEps);
    const float k = 0.5f * rough * rough;
    const float Dv = fmaxf(NdotV * (1.0f - k) + k, kBrdfEps);
    const float Dl = fmaxf(NdotL * (1.0f - k) + k, kBrdfEps);
    const float Gv = NdotV / Dv, Gl = NdotL / Dl, G = Gv * Gl;
    const float inv4v = 1.0f / fmaxf(4.0f * NdotV, kBrdfEps);
    const float sscale = D * G * inv4v;
    const float3 spec = F * sscale;
    const float pd = NdotL * kInvPiF;
    const float ps = VdotH > 0.0f ? D * NdotH / fmaxf(4.0f * VdotH, kBrdfEps) : 0.0f;
    pdf = 0.5f * (pd + ps);
    const float3 value = diffuse + spec;
    r.value = relu3(value);
    if (kGrad) {
        const float3 mask = pos_mask(value);
        const float omq = 1.0f - q;
        const float dF_dA = metallic * omq;
        if (metallic_on) {
            const float3 dF_dM = (albedo - f3(0.04f)) * omq;
            const float3 dDiff_dM = (-albedo * (f3(1.0f) - F) - dcol * dF_dM) * dscale;
            r.d_metallic = (dDiff_dM + dF_dM * sscale) * mask;
        }
        r.d_albedo = (((f3(1.0f) - F) - albedo * dF_dA) * (omm * dscale) + f3(dF_dA * sscale)) * mask;
        const float dD_da2 =
            kInvPiF * (1.0f / fmaxf(dden * dden, kBrdfEps) - (2.0f * a2 * NdotH * NdotH) / fmaxf(dden * dden * dden, kBrdfEps));
        const float dD_dr = dD_da2 * (4.0f * rough * rough * rough);
        const float dGv_dk = -NdotV * (1.0f - NdotV) / (Dv * Dv);
        const float dGl_dk = -NdotL * (1.0f - NdotL) / (Dl * Dl);
        const float dG_dr = (Gl * dGv_dk + Gv * dGl_dk) * rough;
        const float dS_dr = (dD_dr * G + D * dG_dr) * inv4v;
        const float dr_din = (roughness > kMinRough && roughness < 1.0f) ? 1.0f : 0.0f;
        r.d_rough = F * (dS_dr * dr_din) * mask;
    }
    return r;
}

// d(mixed pdf)/d(roughness) for a fixed direction
PTIR_DEV float mixed_pdf_rough_grad(float3 wo, float3 n, float roughness, float3 ldir) {
    const float3 L = normalize_or(ldir, n);
    const float NdotV = saturate(dot(n, wo)), NdotL = saturate(dot(n, L));
    if (NdotV <= 0.0f || NdotL <= 0.0f) return 0.0f;
    if (!(roughness > kMinRough && roughness < 1.0f)) return 0.0f;
    const float rough = clamp_rough(roughness);
    const float3 H = normalize_or(wo + L, n);
    const float NdotH = saturate(dot(n, H)), VdotH = saturate(dot(wo, H));
    if (VdotH <= 0.0f) return 0.0f;
    const float a = rough * rough, a2 = a * a;
    const float dden = fmaxf(NdotH * NdotH * (a2 - 1.0f) + 1.0f, kBrdfEps);
    const float dD_da2 =
        kInvPiF * (1.0f / fmaxf(dden * dden, kBrdfEps) - (2.0f * a2 * NdotH * NdotH) / fmaxf(dden * dden * dden, kBrdfEps));
    const float dD_dr = dD_da2 * (4.0f * rough * rough * rough);
    return 0.5f * dD_dr * NdotH / fmaxf(4.0f * VdotH, kBrdfEps);
}

struct BrdfSample {
    float3 value;      // f cos / pdf (clamped >= 0)
    float3 d_albedo, d_metallic, d_rough, d_next_dir;
    float pdf;
};

// Draw the next direction: rnd.z < 0.5 -> cosine lobe, else GGX half vector reflected.
template <bool kGrad>
PTIR_DEV BrdfSample sample_brdf(float3 wo, float3 n, float3 albedo, float metallic, float roughness, float3 rnd,
                                bool metallic_on, float3& next) {
    BrdfSample s;
    s.value = s.d_albedo = s.d_metallic = s.d_rough = s.d_next_dir = f3(0.0f);
    s.pdf = 0.0f;
    const float rough = clamp_rough(roughness);
    float3 L;
    if (rnd.z < 0.5f) {
        L = sample_cosine(n, rnd.x, rnd.y);
        if (!kGrad && !(dot(n, L) > 0.0f)) return s;
    } else {
        const float3 H = sample_ggx_half(n, rough, rnd.x, rnd.y);
        L = H * (2.0f * dot(wo, H)) - wo;
        const bool ok = dot(n, L) > 0.0f;
        if (!kGrad && !ok) return s;
        if (kGrad && ok && roughness > kMinRough && roughness < 1.0f) {
            const float rs = clamp_rough(roughness + 1e-3f);
            const float step = rs - rough;
            if (step > kBrdfEps) {
                const float3 Hs = sample_ggx_half(n, rs, rnd.x, rnd.y);
                const float3 Ls = Hs * (2.0f * dot(wo, Hs)) - wo;
                if (dot(n, Ls) > 0.0f) s.d_next_dir = (Ls - L) / step;
            }
        }
    }
    next = L;
    if (dot(n, L) <= 0.0f) {
        s.d_next_dir = f3(0.0f);
        return s;
    }
    float pdf;
    const BrdfTerms t = eval_brdf<kGrad>(wo, n, albedo, metallic, roughness, L, metallic_on, pdf);
    if (pdf <= kBrdfEps) {
        s.d_next_dir = f3(0.0f);
        return s;
    }
    s.pdf = pdf;
    const float ip = 1.0f / fmaxf(pdf, kBrdfEps);
    const float3 value = t.value * ip;
    s.value = relu3(value);
    if (kGrad) {
        const float3 mask = pos_mask(value);
        const float dpdf = mixed_pdf_rough_grad(wo, n, roughness, L);
        s.d_albedo = t.d_albedo * ip * mask;
        s.d_rough = (t.d_rough * ip - t.value * (dpdf * ip * ip)) * mask;
        if (metallic_on) s.d_metallic = t.d_metallic * ip * mask;
    }
    return s;
}

}  // namespace ptir
