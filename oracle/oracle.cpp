// ORACLE — TEST INFRASTRUCTURE ONLY. See oracle.h for scope and the candidate semantics.
// Restates, per function, the reference files cited beside each definition.
#include "oracle.h"

#include <omp.h>

#include <array>
#include <initializer_list>
#include <limits>
#include <string>
#include <utility>

namespace oracle {

int kDrawOrder = 0;

// =======================================================================================
// acceleration structure (particlePrimitives.cu:27-51, 543-610; optixTracer.cpp:633-907)
template <class T>
static void bvh_build(Instances<T>& I, int node, int first, int count) {
    auto& nd = I.nodes[node];
    V3<T> lo = v3<T>(std::numeric_limits<T>::infinity()), hi = v3<T>(-std::numeric_limits<T>::infinity());
    V3<T> clo = lo, chi = hi;
    for (int i = first; i < first + count; ++i) {
        const int g = I.order[i];
        lo = {std::fmin(lo.x, I.lo[g].x), std::fmin(lo.y, I.lo[g].y), std::fmin(lo.z, I.lo[g].z)};
        hi = {std::fmax(hi.x, I.hi[g].x), std::fmax(hi.y, I.hi[g].y), std::fmax(hi.z, I.hi[g].z)};
        const V3<T> c = (I.lo[g] + I.hi[g]) * T(0.5);
        clo = {std::fmin(clo.x, c.x), std::fmin(clo.y, c.y), std::fmin(clo.z, c.z)};
        chi = {std::fmax(chi.x, c.x), std::fmax(chi.y, c.y), std::fmax(chi.z, c.z)};
    }
    // conservative padding so that rounding in the slab test never prunes a true candidate
    const V3<T> ext = hi - lo;
    const T pad = T(1e-5) * (std::fmax(ext.x, std::fmax(ext.y, ext.z)) + std::fmax(std::fabs(lo.x), std::fmax(std::fabs(hi.x), T(1))));
    nd.lo = lo - v3<T>(pad);
    nd.hi = hi + v3<T>(pad);
    nd.first = first;
    nd.count = count;
    nd.left = nd.right = -1;
    if (count <= 4) return;
    const V3<T> ce = chi - clo;
    const int axis = (ce.x >= ce.y && ce.x >= ce.z) ? 0 : (ce.y >= ce.z ? 1 : 2);
    auto key = [&](int g) {
        const V3<T> c = (I.lo[g] + I.hi[g]) * T(0.5);
        return axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
    };
    const int mid = first + count / 2;
    std::nth_element(I.order.begin() + first, I.order.begin() + mid, I.order.begin() + first + count,
                     [&](int a, int b) { return key(a) < key(b); });
    const int l = int(I.nodes.size());
    I.nodes.push_back({});
    I.nodes.push_back({});
    I.nodes[node].left = l;
    I.nodes[node].right = l + 1;
    bvh_build(I, l, first, mid - first);
    bvh_build(I, l + 1, mid, first + count - mid);
}

template <class T>
void build_instances(const Config& cfg, const Inputs& in, Instances<T>& I) {
    I.n = in.n;
    I.inv.resize(in.n);
    I.center.resize(in.n);
    I.lo.resize(in.n);
    I.hi.resize(in.n);
    const T inf = std::numeric_limits<T>::infinity();
    I.scene_lo = v3<T>(inf);
    I.scene_hi = v3<T>(-inf);
    for (int g = 0; g < in.n; ++g) {
        const T qw = in.brot[4 * g + 0], qx = in.brot[4 * g + 1], qy = in.brot[4 * g + 2], qz = in.brot[4 * g + 3];
        const M33<T> R = quat_to_r<T>(qw, qx, qy, qz);
        const T ks = kernel_scale<T>(T(in.bdns[g]), T(cfg.min_response), cfg.density_clamping != 0, cfg.kernel_degree);
        const V3<T> kscl = v3<T>(T(in.bscl[3 * g + 0]), T(in.bscl[3 * g + 1]), T(in.bscl[3 * g + 2])) * ks;
        const V3<T> mu = v3<T>(T(in.bpos[3 * g + 0]), T(in.bpos[3 * g + 1]), T(in.bpos[3 * g + 2]));
        // object space = diag(1/kscl) R^T (x - mu): inverse of world = R diag(kscl) obj + mu
        M33<T> A;
        for (int i = 0; i < 3; ++i) {
            const T inv_k = T(1) / (i == 0 ? kscl.x : (i == 1 ? kscl.y : kscl.z));
            A.r[i] = v3<T>(R.r[0].x, R.r[1].x, R.r[2].x);
            if (i == 1) A.r[i] = v3<T>(R.r[0].y, R.r[1].y, R.r[2].y);
            if (i == 2) A.r[i] = v3<T>(R.r[0].z, R.r[1].z, R.r[2].z);
            A.r[i] = A.r[i] * inv_k;
        }
        I.inv[g] = A;
        I.center[g] = mu;
        // world AABB of the 8 transformed box corners (particlePrimitives.cu:585-594)
        V3<T> lo = v3<T>(inf), hi = v3<T>(-inf);
        for (int c = 0; c < 8; ++c) {
            const V3<T> corner = v3<T>((c & 4) ? T(1) : T(-1), (c & 2) ? T(1) : T(-1), (c & 1) ? T(1) : T(-1));
            const V3<T> v = rowmul(R, corner * kscl) + mu;
            lo = {std::fmin(lo.x, v.x), std::fmin(lo.y, v.y), std::fmin(lo.z, v.z)};
            hi = {std::fmax(hi.x, v.x), std::fmax(hi.y, v.y), std::fmax(hi.z, v.z)};
        }
        I.lo[g] = lo;
        I.hi[g] = hi;
        I.scene_lo = {std::fmin(I.scene_lo.x, lo.x), std::fmin(I.scene_lo.y, lo.y), std::fmin(I.scene_lo.z, lo.z)};
        I.scene_hi = {std::fmax(I.scene_hi.x, hi.x), std::fmax(I.scene_hi.y, hi.y), std::fmax(I.scene_hi.z, hi.z)};
    }
    I.empty = in.n == 0;
    I.nodes.clear();
    I.order.resize(in.n);
    for (int g = 0; g < in.n; ++g) I.order[g] = g;
    if (in.n > 0) {
        I.nodes.reserve(2 * in.n);
        I.nodes.push_back({});
        bvh_build(I, 0, 0, in.n);
    }
}

template void build_instances<float>(const Config&, const Inputs&, Instances<float>&);
template void build_instances<double>(const Config&, const Inputs&, Instances<double>&);

// =======================================================================================
struct Hit {
    uint32_t id;
    double t;  // stored in double; comparisons are done in T by the caller
};
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kK = 16;  // pipelineParameters.h:79 MaxNumHitPerTrace

template <class T>
struct Ray {
    V3<T> o, d;
};

template <class T>
struct Interaction {  // interaction.h:22-76
    bool valid = false;
    V3<T> position{}, snormal{};
    V3<T> albedo{};
    T roughness = 0, metallic = 0;
    V3<T> d_albedo{};
    T d_roughness = 0, d_metallic = 0;
};

template <class T>
struct RayPayload {  // payLoad.h:38-95
    Ray<T> ray{};
    Interaction<T> inter{};
    V3<T> radiance{}, light{}, contribution{}, normal{};
    T transmittance = 1, hit_distance = 0, hit2 = 0, last_hit = 0, distortion = 0, hits_count = 0;
    T scatter_pdf = 0, light_pdf = 0;
    V3<T> ray_dir_grad{};
    unsigned hit = 0;
    bool valid = false;
    RayPayload() = default;
    RayPayload(const Ray<T>& r, T last) : ray(r), last_hit(last) {}
};

template <class T>
struct Pending {  // payLoad.h:97-138
    bool valid = false;
    Ray<T> ray{};
    T opacity = 0, max_hit = 0;
    V3<T> dnext{};
    unsigned bounces = 0;
};

template <class T>
struct Path {  // payLoad.h:140-168
    unsigned active = 1, bounces = 0, max_bounces = 0;
    // Decision signature (no counterpart in the reference; for parity diagnostics): an FNV-1a hash
    // over the events in which a path takes a discrete branch, in path order, computed the same
    // way by the GPU tracer (path.cuh, sig_*): each segment's accepted-hit count, interaction,
    // escape and hit flags; whether NEE casts a shadow ray and whether it is occluded; whether the
    // path continues after each BRDF sample.
    uint32_t sig = 2166136261u;
    void mix(uint32_t v) { sig = (sig ^ v) * 16777619u; }
    RayPayload<T> cur{}, emitter{};
    V3<T> acc{}, acc_grad{}, acc_direct{}, acc_indirect{}, acc_light{}, acc_light_grad{};
    V3<T> throughput = v3<T>(T(1));
    Pending<T> pending{};
};

template <class T>
struct BrdfGrad {  // material.cuh:311-317
    V3<T> value{}, d_albedo{}, d_metallic{}, d_roughness{}, d_next_dir{};
};

// ---------------------------------------------------------------------------------------
// The reference adds and subtracts its 1e-9 trace epsilons in float (pathTracer.cuh:167,221,326),
// where they vanish once |x| exceeds ~0.017: x + 1e-9f == x. The oracle applies the offset the
// float evaluation would produce, so that interval ends land where the reference's land (e.g.
// a backward replay ends exactly at the last composited hit and, the test being strict, never
// reaches it).
template <class T>
static inline T float_offset(T x, float e) {
    const float xf = float(x);
    volatile float y = xf + e;
    return x + T(float(y) - xf);
}

template <class T>
class Tracer {
public:
    const Config& cfg;
    const Inputs& in;
    const Instances<T>& I;
    EnvView<T> env;
    Stats st;
    // backward accumulation (per thread)
    std::vector<double>* mat_grad = nullptr;
    std::vector<double>* env_grad = nullptr;
    float* visibility = nullptr;
    // scene AABB (the emitted IAS AABB, optixTracer.cpp:901-903)
    V3<T> alo, ahi;
    T min_resp, alpha_min;

    Tracer(const Config& c, const Inputs& i, const Instances<T>& inst) : cfg(c), in(i), I(inst) {
        env.data = (in.env && in.eh > 0 && in.ew > 0) ? in.env : nullptr;
        env.w = in.ew;
        env.h = in.eh;
        env.cube = env.data && in.eh == 6 * in.ew;  // optixTracer.cpp:229-231
        if (in.alias && in.ah > 0 && in.aw > 0) {     // optixTracer.cpp:207-216
            env.cells = in.ah * in.aw;
            env.aw = in.aw;
            env.ah = in.ah;
            env.prob = in.alias;
            env.alias = in.alias + env.cells;
            env.pdf = in.alias + 2 * env.cells;
        }
        alo = I.scene_lo;
        ahi = I.scene_hi;
        min_resp = T(cfg.min_response);
        alpha_min = T(1.0f / 255.0f);
    }

    // pathTracer.cuh:46-52
    void clip_scene(const Ray<T>& r, T& t0, T& t1) const {
        const V3<T> a = (alo - r.o) / r.d;
        const V3<T> b = (ahi - r.o) / r.d;
        const V3<T> mx = {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)};
        const V3<T> mn = {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)};
        t0 = std::fmax(T(0), std::fmax(mn.x, std::fmax(mn.y, mn.z)));
        t1 = std::fmin(mx.x, std::fmin(mx.y, mx.z));
        if (I.empty) { t0 = T(1); t1 = T(0); }
    }

    // ---- candidate test of one Gaussian (object-space box + gaussianParticles.cuh:484-500)
    bool candidate(int g, const Ray<T>& r, T tmin, T tend, T& tstar) const {
        const M33<T>& A = I.inv[g];
        const V3<T> o = rowmul(A, r.o - I.center[g]);
        const V3<T> d = rowmul(A, r.d);
        // unit box [-1,1]^3 within [tmin, tend]
        T te = tmin, tx = tend;
        const T oc[3] = {o.x, o.y, o.z}, dc[3] = {d.x, d.y, d.z};
        for (int a = 0; a < 3; ++a) {
            if (dc[a] == T(0)) {
                if (oc[a] < T(-1) || oc[a] > T(1)) return false;
                continue;
            }
            const T inv = T(1) / dc[a];
            T t0 = (T(-1) - oc[a]) * inv, t1 = (T(1) - oc[a]) * inv;
            if (t0 > t1) std::swap(t0, t1);
            te = std::fmax(te, t0);
            tx = std::fmin(tx, t1);
        }
        if (te > tx) return false;
        return instance_hit(o, d, tmin, tend, tstar);
    }

    // intersectInstanceParticle (gaussianParticles.cuh:484-500), object-space ray (o, d)
    static bool instance_hit(const V3<T>& o, const V3<T>& d, T tmin, T tend, T& tstar) {
        const T dd = dot(d, d);
        const T den = T(1) / dd;
        tstar = -dot(o, d) * den;
        if (!(tstar > tmin && tstar < tend)) return false;
        const V3<T> c = cross(safe_normalize(d), o);
        return dot(c, c) * den < T(9);
    }

    static bool slab(const V3<T>& lo, const V3<T>& hi, const Ray<T>& r, T tmin, T tend) {
        T te = tmin, tx = tend;
        const T oc[3] = {r.o.x, r.o.y, r.o.z}, dc[3] = {r.d.x, r.d.y, r.d.z};
        const T l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
        for (int a = 0; a < 3; ++a) {
            if (dc[a] == T(0)) {
                if (oc[a] < l[a] || oc[a] > h[a]) return false;
                continue;
            }
            const T inv = T(1) / dc[a];
            T t0 = (l[a] - oc[a]) * inv, t1 = (h[a] - oc[a]) * inv;
            if (t0 > t1) std::swap(t0, t1);
            te = std::fmax(te, t0);
            tx = std::fmin(tx, t1);
        }
        return te <= tx;
    }

    // pathTracer.cuh:58-113 + referenceOptix.cu:73-133: the 16 nearest candidates in (tmin, tend)
    void trace(std::array<Hit, kK>& out, const Ray<T>& r, T tmin, T tend) {
        for (auto& h : out) h = {kInvalid, 1e20};
        st.trace_calls++;
        if (I.empty) return;
        std::vector<std::pair<T, uint32_t>> found;
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const auto& nd = I.nodes[stack[--sp]];
            if (!slab(nd.lo, nd.hi, r, tmin, tend)) continue;
            if (nd.left < 0) {
                for (int i = nd.first; i < nd.first + nd.count; ++i) {
                    const int g = I.order[i];
                    T ts;
                    if (candidate(g, r, tmin, tend, ts)) found.push_back({ts, uint32_t(g)});
                }
            } else {
                stack[sp++] = nd.left;
                stack[sp++] = nd.right;
            }
        }
        const size_t k = std::min<size_t>(kK, found.size());
        std::partial_sort(found.begin(), found.begin() + k, found.end(),
                          [](const auto& a, const auto& b) { return a.first < b.first || (a.first == b.first && a.second < b.second); });
        for (size_t i = 0; i < k; ++i) out[i] = {found[i].second, double(found[i].first)};
        st.candidates += k;
    }

    // ---- particle records
    struct Density { V3<T> pos; T dns; M33<T> rt; V3<T> scl; };
    Density fetch_density(uint32_t g) const {  // gaussianParticles.cuh:173-186
        const float* p = in.density + 12 * size_t(g);
        Density d;
        d.pos = v3<T>(p[0], p[1], p[2]);
        d.dns = p[3];
        d.rt = quat_to_rt<T>(p[4], p[5], p[6], p[7]);
        d.scl = v3<T>(p[8], p[9], p[10]);
        return d;
    }

    // the shared front of processHit / shadowHitAlpha / rayIntersectBwd
    // (gaussianParticles.cuh:384-396, pathTracer.cuh:146-158, 362-373)
    void response(const Density& D, const Ray<T>& r, V3<T>& gro, V3<T>& grd, T& d2, T& gres, T& galpha) const {
        const V3<T> giscl = v3<T>(T(1) / D.scl.x, T(1) / D.scl.y, T(1) / D.scl.z);
        gro = giscl * rowmul(D.rt, r.o - D.pos);
        grd = safe_normalize(giscl * rowmul(D.rt, r.d));
        const V3<T> c = cross(grd, gro);
        d2 = dot(c, c);
        gres = particle_response<T>(cfg.kernel_degree, d2);
        galpha = std::fmin(T(0.99), gres * D.dns);
    }

    // pathTracer.cuh:115-128
    bool self_occlusion(const Hit& h, const Ray<T>& r) const {
        if (T(h.t) > T(1e-1f - 2e-2f) || in.snrm == nullptr) return false;
        const float* n = in.snrm + 3 * size_t(h.id);
        return dot(v3<T>(n[0], n[1], n[2]), r.d) > T(0.1);
    }

    // gaussianParticles.cuh:55-87
    V3<T> sh_radiance(uint32_t g, V3<T> dir) const {
        const float* c = in.sph + size_t(g) * cfg.sph_max_coeffs * 3;
        auto C = [&](int i) { return v3<T>(c[3 * i], c[3 * i + 1], c[3 * i + 2]); };
        const int deg = in.sph_degree;
        V3<T> rad = C(0) * T(0.28209479177387814);
        if (deg > 0) {
            const T x = dir.x, y = dir.y, z = dir.z;
            const T c1 = T(0.4886025119029199);
            rad = rad - C(1) * (c1 * y) + C(2) * (c1 * z) - C(3) * (c1 * x);
            if (deg > 1) {
                const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
                rad = rad + C(4) * (T(1.0925484305920792) * xy) + C(5) * (T(-1.0925484305920792) * yz) +
                      C(6) * (T(0.31539156525252005) * (T(2) * zz - xx - yy)) + C(7) * (T(-1.0925484305920792) * xz) +
                      C(8) * (T(0.5462742152960396) * (xx - yy));
                if (deg > 2) {
                    rad = rad + C(9) * (T(-0.5900435899266435) * y * (T(3) * xx - yy)) +
                          C(10) * (T(2.890611442640554) * xy * z) +
                          C(11) * (T(-0.4570457994644658) * y * (T(4) * zz - xx - yy)) +
                          C(12) * (T(0.3731763325901154) * z * (T(2) * zz - T(3) * xx - T(3) * yy)) +
                          C(13) * (T(-0.4570457994644658) * x * (T(4) * zz - xx - yy)) +
                          C(14) * (T(1.445305721320277) * z * (xx - yy)) +
                          C(15) * (T(-0.5900435899266435) * x * (xx - T(3) * yy));
                }
            }
        }
        rad = rad + v3<T>(T(0.5));
        return {std::fmax(rad.x, T(0)), std::fmax(rad.y, T(0)), std::fmax(rad.z, T(0))};
    }

    // The compositing state of processHit (gaussianParticles.cuh:343-440): transmittance, radiance,
    // depth and its second moment, material and shading normal sums, normal.
    struct HitSums {
        T transmittance = 1, depth = 0, depth2 = 0, rgh = 0, met = 0;
        V3<T> radiance{}, alb{}, snrm{}, normal{};
    };

    // gaussianParticles.cuh:343-440: response of Gaussian `id` to the ray; when accepted, its
    // weighted contributions are added to the sums and the transmittance falls. Returns accepted.
    bool process_hit(uint32_t id, const Ray<T>& ray, HitSums& h) const {
        const Density D = fetch_density(id);
        V3<T> gro, grd; T d2, gres, ga;
        response(D, ray, gro, grd, d2, gres, ga);
        if (!(gres > min_resp && ga > alpha_min)) return false;
        const T wgt = ga * h.transmittance;
        const V3<T> grds = D.scl * grd * dot(grd, -gro);
        const T hit_t = std::sqrt(dot(grds, grds));
        h.radiance += sh_radiance(id, ray.d) * wgt;
        const float* m = in.material + 5 * size_t(id);
        h.alb += v3<T>(m[0], m[1], m[2]) * wgt;
        h.rgh += T(m[3]) * wgt;
        h.met += T(m[4]) * wgt;
        h.transmittance *= (T(1) - ga);
        h.depth += hit_t * wgt;
        h.depth2 += hit_t * hit_t * wgt;
        if (cfg.enable_normals) {
            const float* n = in.snrm + 3 * size_t(id);
            h.snrm += v3<T>(n[0], n[1], n[2]) * wgt;
            const V3<T> srot = colmul(D.rt, D.scl);
            h.normal += safe_normalize((gro + grd * (dot(grd, -gro) - std::sqrt(T(9) - d2))) * srot) * wgt;
        }
        return true;
    }

    // pathTracer.cuh:216-311 (+ processHit, gaussianParticles.cuh:343-440)
    void ray_intersect(bool self_occ, const Ray<T>& ray, RayPayload<T>& p, Sampler& s) {
        T t0, t1;
        clip_scene(ray, t0, t1);
        const T spdf = p.scatter_pdf, lpdf = p.light_pdf;
        p = RayPayload<T>(ray, std::fmax(T(0), float_offset(t0, -1e-9f)));
        if (cfg.enable_mis) { p.scatter_pdf = spdf; p.light_pdf = lpdf; }
        HitSums sums;
        std::array<Hit, kK> hits;
        while (p.last_hit <= t1 && sums.transmittance > T(in.min_transmittance)) {
            trace(hits, p.ray, float_offset(p.last_hit, 1e-9f), float_offset(t1, 1e-9f));
            if (hits[0].id == kInvalid) break;
            for (int i = 0; i < kK; ++i) {
                const Hit& h = hits[i];
                if (h.id == kInvalid || !(sums.transmittance > T(in.min_transmittance))) continue;
                if (self_occ && self_occlusion(h, p.ray)) { p.last_hit = std::fmax(p.last_hit, T(h.t)); continue; }
                const bool accept = process_hit(h.id, p.ray, sums);
                if (accept) {
                    st.accepted++;
                    p.hit = 1;
                    const T op = T(1) - sums.transmittance;
                    p.distortion = std::fmax(op * sums.depth2 - sums.depth * sums.depth, T(0));
                    if (visibility) visibility[h.id] = 1.0f;
                }
                p.last_hit = std::fmax(p.last_hit, T(h.t));
                p.hits_count += accept ? T(1) : T(0);  // output only with enable_hitcounts
            }
        }
        p.transmittance = sums.transmittance;
        p.radiance = sums.radiance;
        p.hit2 = sums.depth2;
        p.normal = sums.normal;
        const T op = T(1) - p.transmittance;
        p.hit_distance = sums.depth;
        p.valid = false;
        if (p.hit && op > T(0.5)) {
            const T inv = T(1) / std::fmax(op, T(1e-12));
            const T dd = sums.depth * inv;
            p.inter.valid = true;
            p.inter.position = p.ray.o + p.ray.d * dd;
            p.inter.snormal = sums.snrm * inv;
            p.inter.albedo = sums.alb * inv;
            p.inter.roughness = sums.rgh * inv;
            p.inter.metallic = sums.met * inv;
        } else {
            const T u = s.next_1d();
            p.valid = u < p.transmittance;
        }
    }

    // pathTracer.cuh:161-214 (+ shadowHitAlpha 130-159)
    bool shadow_occluded(const Ray<T>& ray, Sampler& s, T tmin, T tmax) {
        T c0, c1;
        clip_scene(ray, c0, c1);
        T start = std::fmax(tmin, float_offset(c0, -1e-9f));
        const T end = float_offset(std::fmin(tmax, c1), 1e-9f);
        if (start >= end) return false;
        std::array<Hit, kK> hits;
        while (start < end) {
            trace(hits, ray, float_offset(start, 1e-9f), end);
            if (hits[0].id == kInvalid) break;
            T batch_end = start;
            for (int i = 0; i < kK; ++i) {
                const Hit& h = hits[i];
                if (h.id == kInvalid) break;
                if (T(h.t) > end) break;
                batch_end = std::fmax(batch_end, T(h.t));
                if (self_occlusion(h, ray)) continue;
                const Density D = fetch_density(h.id);
                V3<T> gro, grd; T d2, gres, ga;
                response(D, ray, gro, grd, d2, gres, ga);
                const T alpha = (gres > min_resp && ga > alpha_min) ? ga : T(0);
                if (alpha > T(0) && T(s.next_1d()) < alpha) return true;
            }
            if (batch_end <= start) break;
            start = batch_end;
        }
        return false;
    }

    // ---- material.cuh
    static T sat(T v) { return std::fmin(std::fmax(v, T(0)), T(1)); }
    static V3<T> sat(V3<T> v) { return {sat(v.x), sat(v.y), sat(v.z)}; }
    static T clamp_rough(T r) { return std::fmin(std::fmax(r, T(0.05)), T(1)); }
    static V3<T> clamp_nonneg(V3<T> v) { return {std::fmax(v.x, T(0)), std::fmax(v.y, T(0)), std::fmax(v.z, T(0))}; }
    static V3<T> nonneg_mask(V3<T> v) { return {v.x > T(0) ? T(1) : T(0), v.y > T(0) ? T(1) : T(0), v.z > T(0) ? T(1) : T(0)}; }
    static V3<T> safe_norm_fb(V3<T> v, V3<T> fb) {  // material.cuh:77-89
        const T l2 = dot(v, v);
        return l2 > T(1e-6) ? v * (T(1) / std::sqrt(l2)) : fb;
    }
    static V3<T> to_normal_space(V3<T> n, V3<T> l) {  // material.cuh:95-106
        V3<T> t, b;
        branchless_onb(n, t, b);
        return t * l.x + b * l.y + n * l.z;
    }
    T effective_metallic(T m) const { return cfg.enable_metallic ? sat(m) : T(0); }

    V3<T> sample_diffuse(V3<T> n, T u1, T u2) const {  // material.cuh:127-145
        const T xi = sat(u1);
        const T r = std::sqrt(xi);
        const T phi = T(2 * kPi) * sat(u2);
        const T z = std::sqrt(std::fmax(T(0), T(1) - xi));
        return to_normal_space(n, v3<T>(r * std::cos(phi), r * std::sin(phi), z));
    }
    V3<T> sample_ggx_h(V3<T> n, T rough, T u1, T u2) const {  // material.cuh:147-173
        const T a = rough * rough, a2 = a * a;
        const T xi = sat(u1);
        const T den = std::fmax(T(1) + (a2 - T(1)) * xi, T(1e-6));
        const T ct = std::sqrt(std::fmax(T(0), (T(1) - xi) / den));
        const T stt = std::sqrt(std::fmax(T(0), T(1) - ct * ct));
        const T phi = T(2 * kPi) * sat(u2);
        return to_normal_space(n, v3<T>(stt * std::cos(phi), stt * std::sin(phi), ct));
    }

    // material.cuh:448-492
    V3<T> eval_brdf(V3<T> wo, V3<T> n, V3<T> albedo, T metallic, T roughness, V3<T> ldir, T& pdf) const {
        const V3<T> L = safe_norm_fb(ldir, n);
        const T NdotV = sat(dot(n, wo)), NdotL = sat(dot(n, L));
        pdf = 0;
        if (NdotV <= T(0) || NdotL <= T(0)) return {};
        const T rough = clamp_rough(roughness);
        const V3<T> f0 = v3<T>(T(0.04)) + (albedo - v3<T>(T(0.04))) * metallic;
        const V3<T> H = safe_norm_fb(wo + L, n);
        const T NdotH = sat(dot(n, H)), VdotH = sat(dot(wo, H));
        const T x = T(1) - sat(VdotH), x2 = x * x, x5 = x2 * x2 * x;
        const V3<T> F = f0 + (v3<T>(T(1)) - f0) * x5;
        const V3<T> diffuse = albedo * (T(1) - metallic) * (v3<T>(T(1)) - F) * (NdotL * T(1 / kPi));
        const T a = rough * rough, a2 = a * a;
        const T dden = std::fmax(NdotH * NdotH * (a2 - T(1)) + T(1), T(1e-6));
        const T D = a2 * T(1 / kPi) / std::fmax(dden * dden, T(1e-6));
        const T k = T(0.5) * rough * rough;
        const T Gv = NdotV / std::fmax(NdotV * (T(1) - k) + k, T(1e-6));
        const T Gl = NdotL / std::fmax(NdotL * (T(1) - k) + k, T(1e-6));
        const V3<T> spec = F * (D * Gv * Gl / std::fmax(T(4) * NdotV, T(1e-6)));
        const T pd = NdotL * T(1 / kPi);
        const T ps = VdotH > T(0) ? D * NdotH / std::fmax(T(4) * VdotH, T(1e-6)) : T(0);
        pdf = T(0.5) * (pd + ps);
        return clamp_nonneg(diffuse + spec);
    }

    // material.cuh:514-600
    BrdfGrad<T> eval_brdf_grad(V3<T> wo, V3<T> n, V3<T> albedo, T metallic, T roughness, V3<T> ldir, T& pdf) const {
        BrdfGrad<T> r;
        const V3<T> L = safe_norm_fb(ldir, n);
        const T NdotV = sat(dot(n, wo)), NdotL = sat(dot(n, L));
        pdf = 0;
        if (NdotV <= T(0) || NdotL <= T(0)) return r;
        const T rough = clamp_rough(roughness);
        const V3<T> f0 = v3<T>(T(0.04)) + (albedo - v3<T>(T(0.04))) * metallic;
        const V3<T> H = safe_norm_fb(wo + L, n);
        const T NdotH = sat(dot(n, H)), VdotH = sat(dot(wo, H));
        const T x = T(1) - sat(VdotH), x2 = x * x, q = x2 * x2 * x, omq = T(1) - q;
        const V3<T> F = f0 + (v3<T>(T(1)) - f0) * q;
        const T omm = T(1) - metallic;
        const V3<T> dcol = albedo * omm;
        const T dscale = NdotL * T(1 / kPi);
        const V3<T> diffuse = dcol * (v3<T>(T(1)) - F) * dscale;
        const T a = rough * rough, a2 = a * a;
        const T dden = std::fmax(NdotH * NdotH * (a2 - T(1)) + T(1), T(1e-6));
        const T D = a2 * T(1 / kPi) / std::fmax(dden * dden, T(1e-6));
        const T k = T(0.5) * rough * rough;
        const T Dv = std::fmax(NdotV * (T(1) - k) + k, T(1e-6));
        const T Dl = std::fmax(NdotL * (T(1) - k) + k, T(1e-6));
        const T Gv = NdotV / Dv, Gl = NdotL / Dl, G = Gv * Gl;
        const T sscale = D * G / std::fmax(T(4) * NdotV, T(1e-6));
        const V3<T> spec = F * sscale;
        const T pd = NdotL * T(1 / kPi);
        const T ps = VdotH > T(0) ? D * NdotH / std::fmax(T(4) * VdotH, T(1e-6)) : T(0);
        pdf = T(0.5) * (pd + ps);
        const V3<T> value = diffuse + spec;
        const V3<T> mask = nonneg_mask(value);
        r.value = clamp_nonneg(value);
        const T dF_dA = metallic * omq;
        if (cfg.enable_metallic) {
            const V3<T> dF_dM = (albedo - v3<T>(T(0.04))) * omq;
            const V3<T> dD_dM = (-albedo * (v3<T>(T(1)) - F) - dcol * dF_dM) * dscale;
            r.d_metallic = (dD_dM + dF_dM * sscale) * mask;
        }
        const V3<T> dDiff_dA = ((v3<T>(T(1)) - F) - albedo * dF_dA) * (omm * dscale);
        r.d_albedo = (dDiff_dA + v3<T>(dF_dA * sscale)) * mask;
        const T dD_da2 = T(1 / kPi) * (T(1) / std::fmax(dden * dden, T(1e-6)) -
                                       (T(2) * a2 * NdotH * NdotH) / std::fmax(dden * dden * dden, T(1e-6)));
        const T dD_dr = dD_da2 * (T(4) * rough * rough * rough);
        const T dGv_dk = -NdotV * (T(1) - NdotV) / (Dv * Dv);
        const T dGl_dk = -NdotL * (T(1) - NdotL) / (Dl * Dl);
        const T dG_dr = (Gl * dGv_dk + Gv * dGl_dk) * rough;
        const T dS_dr = (dD_dr * G + D * dG_dr) / std::fmax(T(4) * NdotV, T(1e-6));
        const T dr_din = (roughness > T(0.05) && roughness < T(1)) ? T(1) : T(0);
        r.d_roughness = F * (dS_dr * dr_din) * mask;
        return r;
    }

    // material.cuh:185-219
    T mixed_pdf_rough_grad(V3<T> wo, V3<T> n, T roughness, V3<T> ldir) const {
        const V3<T> L = safe_norm_fb(ldir, n);
        const T NdotV = sat(dot(n, wo)), NdotL = sat(dot(n, L));
        if (NdotV <= T(0) || NdotL <= T(0)) return 0;
        if (!(roughness > T(0.05) && roughness < T(1))) return 0;
        const T rough = clamp_rough(roughness);
        const V3<T> H = safe_norm_fb(wo + L, n);
        const T NdotH = sat(dot(n, H)), VdotH = sat(dot(wo, H));
        if (VdotH <= T(0)) return 0;
        const T a = rough * rough, a2 = a * a;
        const T dden = std::fmax(NdotH * NdotH * (a2 - T(1)) + T(1), T(1e-6));
        const T dD_da2 = T(1 / kPi) * (T(1) / std::fmax(dden * dden, T(1e-6)) -
                                       (T(2) * a2 * NdotH * NdotH) / std::fmax(dden * dden * dden, T(1e-6)));
        const T dD_dr = dD_da2 * (T(4) * rough * rough * rough);
        return T(0.5) * dD_dr * NdotH / std::fmax(T(4) * VdotH, T(1e-6));
    }

    // material.cuh:230-286
    V3<T> sample_brdf(V3<T> wo, V3<T> n, V3<T> albedo, T metallic, T roughness, V3<T> rnd, V3<T>& next, T& pdf) const {
        const T rough = clamp_rough(roughness);
        V3<T> L = n;
        pdf = 0;
        if (rnd.z < T(0.5)) {
            L = sample_diffuse(n, rnd.x, rnd.y);
            if (!(dot(n, L) > T(0))) { pdf = 0; return {}; }
        } else {
            const V3<T> H = sample_ggx_h(n, rough, rnd.x, rnd.y);
            L = H * (T(2) * dot(wo, H)) - wo;
            if (!(dot(n, L) > T(0))) { pdf = 0; return {}; }
        }
        next = L;
        if (dot(n, next) <= T(0)) { pdf = 0; return {}; }
        const V3<T> bc = eval_brdf(wo, n, albedo, metallic, roughness, next, pdf);
        if (pdf <= T(1e-6)) { pdf = 0; return {}; }
        return clamp_nonneg(bc / std::fmax(pdf, T(1e-6)));
    }

    // material.cuh:343-425
    BrdfGrad<T> sample_brdf_grad(V3<T> wo, V3<T> n, V3<T> albedo, T metallic, T roughness, V3<T> rnd, V3<T>& next, T& pdf) const {
        const T rough = clamp_rough(roughness);
        V3<T> dnext{};
        V3<T> L = n;
        pdf = 0;
        if (rnd.z < T(0.5)) {
            L = sample_diffuse(n, rnd.x, rnd.y);
        } else {
            const V3<T> H = sample_ggx_h(n, rough, rnd.x, rnd.y);
            L = H * (T(2) * dot(wo, H)) - wo;
            const bool valid = dot(n, L) > T(0);
            const T dr = (roughness > T(0.05) && roughness < T(1)) ? T(1) : T(0);
            if (dr > T(0) && valid) {
                const T rs = clamp_rough(roughness + T(1e-3));
                const T step = rs - rough;
                if (step > T(1e-6)) {
                    const V3<T> Hs = sample_ggx_h(n, rs, rnd.x, rnd.y);
                    const V3<T> Ls = Hs * (T(2) * dot(wo, Hs)) - wo;
                    if (dot(n, Ls) > T(0)) dnext = (Ls - L) / step;
                }
            }
        }
        BrdfGrad<T> r;
        r.d_next_dir = dnext;
        next = L;
        if (dot(n, next) <= T(0)) { pdf = 0; r.d_next_dir = {}; return r; }
        const BrdfGrad<T> bc = eval_brdf_grad(wo, n, albedo, metallic, roughness, next, pdf);
        if (pdf <= T(1e-6)) { pdf = 0; r.d_next_dir = {}; return r; }
        const T ip = T(1) / std::fmax(pdf, T(1e-6));
        const V3<T> value = bc.value * ip;
        const V3<T> mask = nonneg_mask(value);
        const T dpdf = mixed_pdf_rough_grad(wo, n, roughness, next);
        r.value = clamp_nonneg(value);
        r.d_albedo = bc.d_albedo * ip * mask;
        r.d_roughness = (bc.d_roughness * ip - bc.value * (dpdf * ip * ip)) * mask;
        if (cfg.enable_metallic) r.d_metallic = bc.d_metallic * ip * mask;
        return r;
    }

    void frame_of(const Interaction<T>& it, V3<T> raydir, V3<T>& n, V3<T>& wo, V3<T>& alb, T& met) const {
        n = safe_norm_fb(it.snormal, v3<T>(T(0), T(0), T(1)));
        wo = safe_norm_fb(-raydir, n);
        alb = sat(it.albedo);
        met = effective_metallic(it.metallic);
    }

    // ---- environment.cuh
    V3<T> env_texel(int x, int y) const {
        const float* p = env.data + 4 * (size_t(y) * env.w + x);
        return v3<T>(p[0], p[1], p[2]);
    }
    static int wrapi(int v, int n) { if (n <= 0) return 0; int r = v % n; return r < 0 ? r + n : r; }
    static int clampi(int v, int lo, int hi) { return std::max(lo, std::min(v, hi)); }
    Footprint fp_equirect(T u, T v) const {  // environment.cuh:49-74
        u = u - std::floor(u);
        v = std::fmin(std::fmax(v, T(0)), T(1));
        const T x = u * T(env.w) - T(0.5), y = v * T(env.h) - T(0.5);
        const int x0 = int(std::floor(x)), y0 = int(std::floor(y));
        const T ax = x - T(x0), ay = y - T(y0);
        Footprint f;
        f.x0 = wrapi(x0, env.w); f.x1 = wrapi(x0 + 1, env.w);
        f.y0 = clampi(y0, 0, env.h - 1); f.y1 = clampi(y0 + 1, 0, env.h - 1);
        f.w00 = double((T(1) - ax) * (T(1) - ay)); f.w10 = double(ax * (T(1) - ay));
        f.w01 = double((T(1) - ax) * ay); f.w11 = double(ax * ay);
        return f;
    }
    Footprint fp_cube(int face, T u, T v) const {  // environment.cuh:330-359
        const int fs = env.w;
        u = std::fmin(std::fmax(u, T(0)), T(1));
        v = std::fmin(std::fmax(v, T(0)), T(1));
        const T x = u * T(fs) - T(0.5), y = v * T(fs) - T(0.5);
        const int x0 = int(std::floor(x)), y0 = int(std::floor(y));
        const T ax = x - T(x0), ay = y - T(y0);
        const int yo = face * fs;
        Footprint f;
        f.x0 = clampi(x0, 0, fs - 1); f.x1 = clampi(x0 + 1, 0, fs - 1);
        f.y0 = clampi(y0 + yo, yo, yo + fs - 1); f.y1 = clampi(y0 + 1 + yo, yo, yo + fs - 1);
        f.w00 = double((T(1) - ax) * (T(1) - ay)); f.w10 = double(ax * (T(1) - ay));
        f.w01 = double((T(1) - ax) * ay); f.w11 = double(ax * ay);
        return f;
    }
    V3<T> bilinear(const Footprint& f) {  // environment.cuh:76-87
        st.env_lookups++;
        return env_texel(f.x0, f.y0) * T(f.w00) + env_texel(f.x1, f.y0) * T(f.w10) +
               env_texel(f.x0, f.y1) * T(f.w01) + env_texel(f.x1, f.y1) * T(f.w11);
    }
    void add_env_grad(const Footprint& f, V3<T> g) {  // environment.cuh:89-114
        if (!env_grad) return;
        auto add = [&](int x, int y, double w) {
            double* p = env_grad->data() + 4 * (size_t(y) * env.w + x);
            p[0] += w * double(g.x); p[1] += w * double(g.y); p[2] += w * double(g.z);
        };
        add(f.x0, f.y0, f.w00); add(f.x1, f.y0, f.w10); add(f.x0, f.y1, f.w01); add(f.x1, f.y1, f.w11);
    }
    // rotation by the environment offset, fixed to (0,0) by optixTracer.cpp:223
    // (environment.cuh:116-179): rotZ = pi/2, rotX = 0
    struct Rot { T sz, cz, sx, cx; };
    Rot rot() const { const T a = T(0.5 * kPi); return {std::sin(a), std::cos(a), T(0), T(1)}; }
    static V3<T> rotate(V3<T> d, const Rot& r) {
        const V3<T> z = {d.x * r.cz - d.y * r.sz, d.x * r.sz + d.y * r.cz, d.z};
        return {z.x, z.y * r.cx - z.z * r.sx, z.y * r.sx + z.z * r.cx};
    }
    static V3<T> inv_rotate(V3<T> e, const Rot& r) {
        const V3<T> x = {e.x, e.y * r.cx + e.z * r.sx, -e.y * r.sx + e.z * r.cx};
        return {x.x * r.cz + x.y * r.sz, -x.x * r.sz + x.y * r.cz, x.z};
    }
    static void equirect_uv(V3<T> d, T& u, T& v) {  // environment.cuh:361-366
        const T theta = std::atan2(d.x, d.y);
        const T phi = std::asin(std::fmin(T(1), std::fmax(T(-1), -d.z)));
        u = (theta + T(kPi)) * T(0.5 / kPi);
        v = T(0.5) + phi * T(1 / kPi);
    }
    static void cube_face_uv(V3<T> d, int& face, T& u, T& v) {  // environment.cuh:257-301
        const T ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
        T ma, sc, tc;
        if (ax >= ay && ax >= az) { ma = ax; if (d.x > T(0)) { face = 0; sc = -d.z; tc = -d.y; } else { face = 1; sc = d.z; tc = -d.y; } }
        else if (ay >= ax && ay >= az) { ma = ay; if (d.y > T(0)) { face = 2; sc = d.x; tc = d.z; } else { face = 3; sc = d.x; tc = -d.z; } }
        else { ma = az; if (d.z > T(0)) { face = 4; sc = d.x; tc = -d.y; } else { face = 5; sc = -d.x; tc = -d.y; } }
        const T im = T(1) / std::fmax(ma, T(1e-12));
        u = T(0.5) * (sc * im + T(1));
        v = T(0.5) * (tc * im + T(1));
    }
    Footprint footprint_rotated(V3<T> dir) const {
        if (env.cube) { int f; T u, v; cube_face_uv(dir, f, u, v); return fp_cube(f, u, v); }
        T u, v; equirect_uv(dir, u, v); return fp_equirect(u, v);
    }
    V3<T> background(V3<T> d) {  // environment.cuh:447-454
        if (!env.has_env()) return {};
        return bilinear(footprint_rotated(rotate(d, rot())));
    }
    // environment.cuh:421-445
    V3<T> dir_grad_fast(V3<T> d, V3<T> bg, V3<T> cg, const Rot& r) {
        const V3<T> u = safe_normalize(d);
        V3<T> t, b;
        branchless_onb(u, t, b);
        const T eps = T(1e-3);
        const T ps = T(1) / std::sqrt(T(1) + eps * eps);
        const V3<T> td = (u + t * eps) * ps, bd = (u + b * eps) * ps;
        const V3<T> tb = bilinear(footprint_rotated(rotate(td, r)));
        const V3<T> bb = bilinear(footprint_rotated(rotate(bd, r)));
        const T ie = T(1) / eps;
        return t * dot((tb - bg) * ie, cg) + b * dot((bb - bg) * ie, cg);
    }
    // environment.cuh:456-473
    V3<T> background_bwd(V3<T> d, V3<T> cg, V3<T>* dir_grad) {
        if (!env.has_env()) return {};
        const Rot r = rot();
        const Footprint f = footprint_rotated(rotate(d, r));
        const V3<T> bg = bilinear(f);
        add_env_grad(f, cg);
        if (dir_grad) *dir_grad += dir_grad_fast(d, bg, cg, r);
        return bg;
    }
    // environment.cuh:181-195
    static V3<T> equirect_dir(T u, T v) {
        u = u - std::floor(u);
        v = std::fmin(std::fmax(v, T(0)), T(1));
        const T theta = u * T(2 * kPi) - T(kPi), phi = (v - T(0.5)) * T(kPi);
        return {std::sin(theta) * std::cos(phi), std::cos(theta) * std::cos(phi), -std::sin(phi)};
    }
    // environment.cuh:197-225
    static V3<T> cube_dir(int face, T u, T v) {
        u = std::fmin(std::fmax(u, T(0)), T(1));
        v = std::fmin(std::fmax(v, T(0)), T(1));
        const T s = T(2) * u - T(1), t = T(2) * v - T(1);
        V3<T> d;
        switch (face) {
        case 0: d = {T(1), -t, -s}; break;
        case 1: d = {T(-1), -t, s}; break;
        case 2: d = {s, T(1), t}; break;
        case 3: d = {s, T(-1), -t}; break;
        case 4: d = {s, -t, T(1)}; break;
        default: d = {-s, -t, T(-1)}; break;
        }
        return safe_normalize(d);
    }
    // environment.cuh:227-255
    V3<T> sample_alias_dir(Sampler& s, T& pdf) {
        const int cells = env.cells;
        const float u0 = s.next_1d();
        const int ic = std::min(int(u0 * float(cells)), cells - 1);
        const int ac = clampi(int(env.alias[ic] + 0.5f), 0, cells - 1);
        const float u1 = s.next_1d();
        const int cell = u1 < env.prob[ic] ? ic : ac;
        const int x = cell % env.aw, y = cell / env.aw;
        float ju, jv;
        next_2(s, ju, jv);
        V3<T> d;
        if (env.cube) {
            const int fs = env.aw;
            const int face = clampi(y / fs, 0, 5);
            const int fy = y - face * fs;
            d = cube_dir(face, (T(x) + T(ju)) / T(fs), (T(fy) + T(jv)) / T(fs));
        } else {
            d = equirect_dir((T(x) + T(ju)) / T(env.aw), (T(y) + T(jv)) / T(env.ah));
        }
        pdf = env.pdf[cell];
        return inv_rotate(d, rot());
    }
    // environment.cuh:303-328
    T alias_pdf(V3<T> rd) const {
        const V3<T> d = rotate(rd, rot());
        int x, y;
        if (env.cube) {
            int face; T u, v;
            cube_face_uv(d, face, u, v);
            const int fs = env.aw;
            x = clampi(int(u * T(fs)), 0, fs - 1);
            y = face * fs + clampi(int(v * T(fs)), 0, fs - 1);
        } else {
            T u, v;
            equirect_uv(d, u, v);
            x = wrapi(int(u * T(env.aw)), env.aw);
            y = clampi(int(v * T(env.ah)), 0, env.ah - 1);
        }
        return env.pdf[size_t(y) * env.aw + x];
    }
    // ---- punctual and area lights (lightSampler.cuh:12-406, meshLight.cuh:11-101)
    struct LightSample {
        V3<T> wi{}, Li{};
        T pdf = 0, dist = T(1e20);
        unsigned type = 0;  // 0 environment, 1 point, 2 sphere, 3 mesh
    };
    // the reference's static_cast<unsigned>(v + 0.5f) on the device: toward zero, saturating, NaN -> 0
    static unsigned table_index(float v) {
        const float f = v + 0.5f;
        if (!(f > 0.0f)) return 0u;
        if (f >= 4294967296.0f) return 0xFFFFFFFFu;
        return unsigned(f);
    }
    static unsigned scaled_index(float u, unsigned n) {  // min(unsigned(u * n), n - 1)
        const float f = u * float(n);
        const unsigned i = !(f > 0.0f) ? 0u : (f >= 4294967296.0f ? 0xFFFFFFFFu : unsigned(f));
        return std::min(i, n - 1u);
    }
    bool has_table() const { return in.light_entries > 0; }
    bool has_mesh() const {
        return in.num_mesh_lights > 0 && in.num_mesh_vertices > 0 && in.num_mesh_triangles > 0 &&
               in.mesh_tri_cols >= in.num_mesh_triangles;
    }
    float table(int row, unsigned e) const { return in.light_table[size_t(row) * in.light_entries + e]; }
    float tri_table(int row, unsigned t) const { return in.mesh_tri_table[size_t(row) * in.mesh_tri_cols + t]; }
    const float* light_row(unsigned id) const { return in.lights + 9 * size_t(id); }
    const float* mesh_row(unsigned id) const { return in.mesh_lights + 8 * size_t(id); }
    unsigned light_type(unsigned id) const {
        return id < unsigned(in.num_lights) ? table_index(light_row(id)[0]) : 0xFFFFFFFFu;
    }
    static V3<T> f3(const float* p) { return {T(p[0]), T(p[1]), T(p[2])}; }
    static T length(V3<T> v) { return std::sqrt(dot(v, v)); }

    // lightSampler.cuh:59-72
    unsigned sample_entry(Sampler& s) const {
        const unsigned n = unsigned(in.light_entries);
        const unsigned first = scaled_index(s.next_1d(), n);
        const unsigned other = std::min(table_index(table(1, first)), n - 1u);
        return s.next_1d() < table(0, first) ? first : other;
    }
    // lightSampler.cuh:74-91
    LightSample sample_env_light(Sampler& s, T select) {
        LightSample ls;
        if (!env.has_light()) return ls;
        T epdf = 0;
        ls.wi = sample_alias_dir(s, epdf);
        ls.Li = background(ls.wi);
        ls.pdf = select * epdf;
        return ls;
    }
    // lightSampler.cuh:93-123
    LightSample sample_point(V3<T> pos, unsigned id, T select) const {
        LightSample ls;
        if (id >= unsigned(in.num_lights) || light_type(id) != 1u || select <= T(0)) return ls;
        const float* r = light_row(id);
        const V3<T> to = f3(r + 1) - pos;
        const T d2 = dot(to, to);
        if (d2 <= T(1e-12)) return ls;
        const T dist = std::sqrt(d2);
        ls.wi = to / dist;
        ls.Li = f3(r + 5) / d2;
        ls.pdf = select;
        ls.dist = dist;
        ls.type = 1;
        return ls;
    }
    // lightSampler.cuh:125-179
    LightSample sample_sphere(V3<T> pos, Sampler& s, unsigned id, T select) const {
        LightSample ls;
        if (id >= unsigned(in.num_lights) || light_type(id) != 2u) return ls;
        const float* r = light_row(id);
        const T radius = T(r[4]);
        if (radius <= T(0)) return ls;
        const float u1 = s.next_1d();
        const float u2 = s.next_1d();
        const T z = T(1) - T(2) * T(u1);
        const T rr = std::sqrt(std::fmax(T(0), T(1) - z * z));
        const T phi = T(2) * T(kPi) * T(u2);
        const V3<T> nrm{rr * std::cos(phi), rr * std::sin(phi), z};
        const V3<T> to = (f3(r + 1) + nrm * radius) - pos;
        const T d2 = dot(to, to);
        if (d2 <= T(1e-12)) return ls;
        const T dist = std::sqrt(d2);
        const V3<T> wi = to / dist;
        const T cl = std::fabs(dot(nrm, -wi));
        if (cl <= T(1e-6)) return ls;
        const T area = T(4) * T(kPi) * radius * radius;
        ls.wi = wi;
        ls.Li = f3(r + 5);
        ls.pdf = select * (T(1) / std::fmax(area, T(1e-12))) * d2 / cl;
        ls.dist = dist;
        ls.type = 2;
        return ls;
    }
    // lightSampler.cuh:181-222
    T sphere_pdf(V3<T> pos, V3<T> wi, unsigned id) const {
        if (id >= unsigned(in.num_lights) || light_type(id) != 2u) return T(0);
        const float* r = light_row(id);
        const T radius = T(r[4]);
        if (radius <= T(0)) return T(0);
        const V3<T> oc = pos - f3(r + 1);
        const T b = dot(oc, wi);
        const T c = dot(oc, oc) - radius * radius;
        const T disc = b * b - c;
        if (disc <= T(0)) return T(0);
        T t = -b - std::sqrt(disc);
        if (t <= T(1e-6)) t = -b + std::sqrt(disc);
        if (t <= T(1e-6)) return T(0);
        const V3<T> n = safe_normalize((pos + wi * t) - f3(r + 1));
        const T cl = std::fabs(dot(n, -wi));
        if (cl <= T(1e-6)) return T(0);
        const T area = T(4) * T(kPi) * radius * radius;
        return (T(1) / std::fmax(area, T(1e-12))) * (t * t) / cl;
    }
    // meshLight.cuh:18-51
    bool mesh_triangle(unsigned tri, V3<T>& v0, V3<T>& v1, V3<T>& v2) const {
        if (tri >= unsigned(in.num_mesh_triangles)) return false;
        const int* t = in.mesh_triangles + 3 * size_t(tri);
        if (t[0] < 0 || t[1] < 0 || t[2] < 0) return false;
        const unsigned nv = unsigned(in.num_mesh_vertices);
        if (unsigned(t[0]) >= nv || unsigned(t[1]) >= nv || unsigned(t[2]) >= nv) return false;
        v0 = f3(in.mesh_vertices + 3 * size_t(t[0]));
        v1 = f3(in.mesh_vertices + 3 * size_t(t[1]));
        v2 = f3(in.mesh_vertices + 3 * size_t(t[2]));
        return true;
    }
    // meshLight.cuh:53-84
    static bool intersect_triangle(V3<T> o, V3<T> d, V3<T> v0, V3<T> v1, V3<T> v2, T& t) {
        const V3<T> e1 = v1 - v0, e2 = v2 - v0;
        const V3<T> pv = cross(d, e2);
        const T det = dot(e1, pv);
        if (std::fabs(det) <= T(1e-8)) return false;
        const T inv = T(1) / det;
        const V3<T> tv = o - v0;
        const T u = dot(tv, pv) * inv;
        if (u < T(0) || u > T(1)) return false;
        const V3<T> qv = cross(tv, e1);
        const T v = dot(d, qv) * inv;
        if (v < T(0) || (u + v) > T(1)) return false;
        t = dot(e2, qv) * inv;
        return t > T(1e-5);
    }
    // triangle range of a mesh light (checked in 64 bits)
    bool mesh_range(unsigned id, unsigned& off, unsigned& count) const {
        const float* m = mesh_row(id);
        off = table_index(m[0]);
        count = table_index(m[1]);
        return count != 0u && uint64_t(off) + count <= uint64_t(in.num_mesh_triangles);
    }
    // cosine at the light; ok = false for a degenerate triangle
    static T mesh_cosine(V3<T> v0, V3<T> v1, V3<T> v2, V3<T> wi, bool two_sided, bool& ok) {
        const V3<T> nu = cross(v1 - v0, v2 - v0);
        const T nl = length(nu);
        ok = nl > T(1e-12);
        if (!ok) return T(0);
        const T c = dot(nu / nl, -wi);
        return two_sided ? std::fabs(c) : c;
    }
    // meshLight.cuh:86-101
    unsigned sample_triangle(Sampler& s, unsigned off, unsigned count) const {
        const unsigned first = off + scaled_index(s.next_1d(), count);
        const unsigned other = std::min(table_index(tri_table(1, first)), count - 1u);
        return s.next_1d() < tri_table(0, first) ? first : off + other;
    }
    // lightSampler.cuh:224-293
    LightSample sample_mesh(V3<T> pos, Sampler& s, unsigned id, T select) const {
        LightSample ls;
        if (!has_mesh() || id >= unsigned(in.num_mesh_lights) || select <= T(0)) return ls;
        unsigned off, count;
        if (!mesh_range(id, off, count)) return ls;
        const unsigned tri = sample_triangle(s, off, count);
        V3<T> v0, v1, v2;
        if (!mesh_triangle(tri, v0, v1, v2)) return ls;
        float u = s.next_1d();
        float v = s.next_1d();
        if (u + v > 1.0f) { u = 1.0f - u; v = 1.0f - v; }
        const V3<T> to = (v0 + (v1 - v0) * T(u) + (v2 - v0) * T(v)) - pos;
        const T d2 = dot(to, to);
        if (d2 <= T(1e-12)) return ls;
        const T dist = std::sqrt(d2);
        const V3<T> wi = to / dist;
        bool ok;
        const T cl = mesh_cosine(v0, v1, v2, wi, mesh_row(id)[7] > 0.5f, ok);
        if (!ok || cl <= T(1e-6)) return ls;
        ls.wi = wi;
        ls.Li = f3(mesh_row(id) + 4);
        ls.pdf = select * T(tri_table(2, tri)) * d2 / cl;
        ls.dist = dist;
        ls.type = 3;
        return ls;
    }
    // lightSampler.cuh:295-338
    T mesh_pdf(V3<T> pos, V3<T> wi, unsigned id) const {
        if (!has_mesh() || id >= unsigned(in.num_mesh_lights)) return T(0);
        unsigned off, count;
        if (!mesh_range(id, off, count)) return T(0);
        const bool two = mesh_row(id)[7] > 0.5f;
        T pdf = 0;
        for (unsigned tri = off; tri < off + count; ++tri) {
            V3<T> v0, v1, v2;
            T t;
            if (!mesh_triangle(tri, v0, v1, v2) || !intersect_triangle(pos, wi, v0, v1, v2, t)) continue;
            bool ok;
            const T cl = mesh_cosine(v0, v1, v2, wi, two, ok);
            if (!ok || cl <= T(1e-6)) continue;
            pdf += T(tri_table(2, tri)) * (t * t) / cl;
        }
        return pdf;
    }
    // lightSampler.cuh:340-383
    LightSample sample_light(V3<T> pos, Sampler& s) {
        if (!has_table()) return sample_env_light(s, T(1));
        const unsigned e = sample_entry(s);
        const unsigned type = table_index(table(2, e)), id = table_index(table(3, e));
        const T select = T(table(4, e));
        switch (type) {
        case 0: return sample_env_light(s, select);
        case 1: return sample_point(pos, id, select);
        case 2: return sample_sphere(pos, s, id, select);
        case 3: return sample_mesh(pos, s, id, select);
        default: return LightSample();
        }
    }
    // lightSampler.cuh:385-406 (point lights are delta lights and add nothing)
    T light_pdf(V3<T> pos, V3<T> wi) const {
        if (!has_table()) return env.has_light() ? alias_pdf(wi) : T(0);
        T pdf = 0;
        for (unsigned i = 0; i < unsigned(in.light_entries); ++i) {
            const T select = T(table(4, i));
            if (select <= T(0)) continue;
            const unsigned type = table_index(table(2, i)), id = table_index(table(3, i));
            T p = 0;
            if (type == 0) p = env.has_light() ? alias_pdf(wi) : T(0);
            else if (type == 2) p = sphere_pdf(pos, wi, id);
            else if (type == 3) p = mesh_pdf(pos, wi, id);
            pdf += select * p;
        }
        return pdf;
    }
    // environment.cuh:491-536
    bool hit_sphere_light(const Ray<T>& r, unsigned id, T& t, V3<T>& rad) const {
        if (light_type(id) != 2u) return false;
        const float* L = light_row(id);
        const T radius = T(L[4]);
        if (radius <= T(0)) return false;
        const V3<T> oc = r.o - f3(L + 1);
        const T b = dot(oc, r.d);
        const T c = dot(oc, oc) - radius * radius;
        const T disc = b * b - c;
        if (disc <= T(0)) return false;
        const T sq = std::sqrt(disc);
        t = -b - sq;
        if (t <= T(1e-5)) t = -b + sq;
        if (t <= T(1e-5)) return false;
        rad = f3(L + 5);
        return !(rad.x <= T(0) && rad.y <= T(0) && rad.z <= T(0));
    }
    // environment.cuh:538-597
    bool hit_mesh_light(const Ray<T>& r, unsigned id, T& t, V3<T>& rad) const {
        if (!has_mesh()) return false;
        unsigned off, count;
        if (!mesh_range(id, off, count)) return false;
        rad = f3(mesh_row(id) + 4);
        if (rad.x <= T(0) && rad.y <= T(0) && rad.z <= T(0)) return false;
        const bool two = mesh_row(id)[7] > 0.5f;
        T nearest = T(1e20);
        for (unsigned tri = off; tri < off + count; ++tri) {
            V3<T> v0, v1, v2;
            T th;
            if (!mesh_triangle(tri, v0, v1, v2) || !intersect_triangle(r.o, r.d, v0, v1, v2, th)) continue;
            bool ok;
            const T cl = mesh_cosine(v0, v1, v2, r.d, two, ok);
            if (!ok || cl <= T(1e-6)) continue;
            nearest = std::fmin(nearest, th);
        }
        if (nearest >= T(1e19)) return false;
        t = nearest;
        return true;
    }
    // environment.cuh:599-634: what an escaped ray sees. 0 nothing, 1 a sphere or mesh light
    // (render.visualize_lights only; radiance in rad), 2 the environment
    int escaped_light(const Ray<T>& r, V3<T>& rad) const {
        if (cfg.visualize_lights) {
            T nearest = T(1e20);
            bool found = false;
            for (unsigned i = 0; i < unsigned(in.num_lights); ++i) {
                T t; V3<T> c;
                if (hit_sphere_light(r, i, t, c) && t < nearest) { nearest = t; rad = c; found = true; }
            }
            for (unsigned i = 0; i < unsigned(in.num_mesh_lights); ++i) {
                T t; V3<T> c;
                if (hit_mesh_light(r, i, t, c) && t < nearest) { nearest = t; rad = c; found = true; }
            }
            if (found) return 1;
        }
        return env.has_env() ? 2 : 0;
    }

    static T mis(T a, T b) { const T a2 = a * a, b2 = b * b; return a2 / std::fmax(a2 + b2, T(1e-6)); }

    // pathTracer.cuh:461-504 (+ lightSampler.cuh:74-91, 359-383)
    void sample_nee(Path<T>& P, Sampler& s) {
        const Interaction<T> it = P.cur.inter;
        T spdf = 0;
        const LightSample ls = sample_light(it.position, s);
        const T lpdf = ls.pdf;
        const V3<T> wi = ls.wi, Li = ls.Li;
        if (lpdf <= T(0) || is_zero(Li) || dot(it.snormal, wi) <= T(0)) {
            P.emitter = RayPayload<T>();
            P.mix(kSigNee);
            return;
        }
        P.mix(kSigNee | 1u);
        V3<T> n, wo, alb; T met;
        frame_of(it, P.cur.ray.d, n, wo, alb, met);
        const V3<T> bc = eval_brdf(wo, n, alb, met, clamp_rough(it.roughness), wi, spdf);
        if (ls.type == 1u) spdf = T(0);
        const Ray<T> lr{it.position + wi * T(2e-2), wi};
        const T tmax = ls.dist < T(1e19) ? std::fmax(T(0), ls.dist - T(2e-2)) : T(1e20);
        st.segments++;
        const bool occluded = shadow_occluded(lr, s, T(0), tmax);
        P.mix(kSigShadow | (occluded ? 1u : 0u));
        if (occluded) { P.emitter = RayPayload<T>(); return; }
        P.emitter = RayPayload<T>(lr, T(0));
        P.emitter.light_pdf = lpdf;
        P.emitter.scatter_pdf = spdf;
        P.emitter.light = Li;
        P.emitter.contribution = P.throughput * bc * Li / std::fmax(lpdf, T(1e-6));
    }

    // pathTracer.cuh:430-459
    void sample_next(Path<T>& P, Sampler& s) {
        const Ray<T> cr = P.cur.ray;
        const Interaction<T> it = P.cur.inter;
        V3<T> next = cr.d;
        T spdf = 0;
        V3<T> n, wo, alb; T met;
        frame_of(it, cr.d, n, wo, alb, met);
        const V3<T> rnd = next_3d<T>(s);
        const V3<T> bt = sample_brdf(wo, n, alb, met, clamp_rough(it.roughness), rnd, next, spdf);
        const V3<T> nt = P.throughput * bt;
        if (is_zero(nt)) { P.throughput = {}; P.active = 0; return; }
        P.throughput = nt;
        const Ray<T> nr{it.position + safe_normalize(next) * T(2e-2), next};
        P.cur = RayPayload<T>(nr, T(0));
        if (cfg.enable_mis) { P.cur.scatter_pdf = spdf; P.cur.light_pdf = light_pdf(it.position, next); }
    }

    // environment.cuh:636-715
    void accumulate_light(Path<T>& P) {
        P.cur.contribution = {};
        const bool first = P.bounces == 1u;
        T bmis = 1, lmis = 1;
        V3<T> nee{};
        if (cfg.enable_mis) {
            if (first) { bmis = mis(P.cur.scatter_pdf, P.cur.light_pdf); lmis = mis(P.emitter.light_pdf, P.emitter.scatter_pdf); }
            nee = P.emitter.contribution * lmis;
        }
        if (in.render_opts == 1) {
            if (cfg.enable_mis && first) P.acc += nee;
            if (P.bounces > 0u && P.cur.inter.valid) {
                P.cur.contribution = P.throughput * P.cur.radiance;
                if (cfg.enable_mis && first) P.cur.contribution *= bmis;
                P.acc += P.cur.contribution;
                P.acc_indirect += P.cur.contribution;
            } else if (P.cur.valid) {
                V3<T> vr{};
                const int seen = escaped_light(P.cur.ray, vr);
                if (seen == 0) return;
                if (seen == 2) vr = background(P.cur.ray.d);
                P.throughput *= P.cur.transmittance;
                P.cur.light += vr;
                P.acc_light += vr;
                P.cur.contribution = P.throughput * P.cur.light;
                if (cfg.enable_mis && first) P.cur.contribution *= bmis;
                P.acc += P.cur.contribution;
                P.acc_direct += P.cur.contribution;
            }
            return;
        }
        if (cfg.enable_mis && first) { P.acc += nee; P.acc_direct += nee; }
        if (P.cur.valid) {
            V3<T> vr{};
            const int seen = escaped_light(P.cur.ray, vr);
            if (seen == 0) return;
            if (seen == 2) vr = background(P.cur.ray.d);
            P.throughput *= P.cur.transmittance;
            P.cur.light += vr;
            P.acc_light += vr;
            P.cur.contribution = P.throughput * P.cur.light;
            if (cfg.enable_mis && first) P.cur.contribution *= bmis;
            P.cur.radiance += P.cur.contribution;
            P.acc += P.cur.contribution;
            if (P.bounces < 2u) P.acc_direct += P.cur.contribution;
            else P.acc_indirect += P.cur.contribution;
        }
    }

    // ---- backward (referenceBwdOptix.cu, pathTracer.cuh:313-634, environment.cuh:717-808)
    void add_mat_grad(uint32_t g, V3<T> da, T dr, T dm) {
        if (!mat_grad) return;
        double* p = mat_grad->data() + 5 * size_t(g);
        p[0] += double(da.x); p[1] += double(da.y); p[2] += double(da.z); p[3] += double(dr);
        if (cfg.enable_metallic) p[4] += double(dm);
    }

    // pathTracer.cuh:313-390
    void ray_intersect_bwd(bool self_occ, const Ray<T>& ray, T opacity, T max_hit, V3<T> da, T dr, T dm) {
        st.replay_segments++;
        const T inv = T(1) / std::fmax(opacity, T(1e-12));
        da = da * inv; dr = dr * inv; dm = dm * inv;
        T c0, c1;
        clip_scene(ray, c0, c1);
        T start = std::fmax(T(0), float_offset(c0, -1e-9f));
        const T end = float_offset(std::fmin(max_hit, c1), 1e-9f);
        T tr = 1;
        std::array<Hit, kK> hits;
        while (start < end && tr > T(in.min_transmittance)) {
            trace(hits, ray, float_offset(start, 1e-9f), end);
            if (hits[0].id == kInvalid) break;
            for (int i = 0; i < kK; ++i) {
                const Hit& h = hits[i];
                if (h.id == kInvalid || !(tr > T(in.min_transmittance))) continue;
                if (self_occ && self_occlusion(h, ray)) { start = std::fmax(start, T(h.t)); continue; }
                const Density D = fetch_density(h.id);
                V3<T> gro, grd; T d2, gres, ga;
                response(D, ray, gro, grd, d2, gres, ga);
                if (gres > min_resp && ga > alpha_min) {
                    const T wgt = ga * tr;
                    add_mat_grad(h.id, da * wgt, dr * wgt, dm * wgt);
                    tr *= (T(1) - ga);
                }
                start = std::fmax(start, T(h.t));
            }
        }
    }

    // pathTracer.cuh:392-428
    void pending_bwd(Path<T>& P) {
        Pending<T>& pd = P.pending;
        if (!pd.valid) return;
        const T dr = dot(P.cur.ray_dir_grad, pd.dnext);
        const Pending<T> c = pd;
        pd = Pending<T>();
        if (dr == T(0)) return;
        ray_intersect_bwd(c.bounces > 1u, c.ray, c.opacity, c.max_hit, V3<T>{}, dr, T(0));
    }

    // pathTracer.cuh:506-548
    void nee_grad_bwd(Path<T>& P, const Ray<T>& cr, const Interaction<T>& it) {
        if (P.bounces != 1u) return;
        if (P.emitter.light_pdf <= T(0)) return;
        T spdf = 0;
        const V3<T> L = P.emitter.ray.d;
        V3<T> n, wo, alb; T met;
        frame_of(it, cr.d, n, wo, alb, met);
        const BrdfGrad<T> bg = eval_brdf_grad(wo, n, alb, met, it.roughness, L, spdf);
        const T lmis = mis(P.emitter.light_pdf, P.emitter.scatter_pdf);
        const T scale = lmis / std::fmax(P.emitter.light_pdf, T(1e-6));
        const V3<T> b = background(L);
        const V3<T> dl = P.acc_grad * P.throughput * b * scale;
        P.cur.inter.d_albedo += dl * bg.d_albedo;
    }

    // pathTracer.cuh:551-634
    void sample_next_bwd(Path<T>& P, Sampler& s) {
        const Ray<T> cr = P.cur.ray;
        const Interaction<T> it = P.cur.inter;
        V3<T> next = cr.d;
        T spdf = 0;
        V3<T> n, wo, alb; T met;
        frame_of(it, cr.d, n, wo, alb, met);
        const V3<T> rnd = next_3d<T>(s);
        const BrdfGrad<T> bt = sample_brdf_grad(wo, n, alb, met, it.roughness, rnd, next, spdf);
        const V3<T> nt = P.throughput * bt.value;
        if (is_zero(nt)) { P.throughput = {}; P.active = 0; return; }
        T lpdf = 0;
        bool first_nee = false;
        if (cfg.enable_mis) {
            lpdf = light_pdf(it.position, next);
            first_nee = P.bounces == 1u && vmax(nt) >= T(1e-4);
            if (first_nee) nee_grad_bwd(P, cr, it);
        }
        V3<T> dep = P.acc;
        if (cfg.enable_mis && first_nee) dep -= P.emitter.contribution * mis(P.emitter.light_pdf, P.emitter.scatter_pdf);
        const V3<T> num = P.acc_grad * dep;
        const V3<T> dl = {bt.value.x > T(1e-6) ? num.x / bt.value.x : T(0),
                          bt.value.y > T(1e-6) ? num.y / bt.value.y : T(0),
                          bt.value.z > T(1e-6) ? num.z / bt.value.z : T(0)};
        P.cur.inter.d_albedo += dl * bt.d_albedo;
        P.cur.inter.d_roughness += dot(dl, bt.d_roughness);
        if (cfg.enable_metallic) P.cur.inter.d_metallic += dot(dl, bt.d_metallic);
        {
            const V3<T> g = bt.d_next_dir;
            P.pending.valid = dot(g, g) > T(0);
            P.pending.ray = cr;
            P.pending.opacity = T(1) - P.cur.transmittance;
            P.pending.max_hit = P.cur.last_hit;
            P.pending.dnext = g;
            P.pending.bounces = P.bounces;
        }
        ray_intersect_bwd(P.bounces > 1u, cr, T(1) - P.cur.transmittance, P.cur.last_hit, P.cur.inter.d_albedo,
                          P.cur.inter.d_roughness, P.cur.inter.d_metallic);
        P.throughput = nt;
        const Ray<T> nr{it.position + safe_normalize(next) * T(2e-2), next};
        P.cur = RayPayload<T>(nr, T(0));
        if (cfg.enable_mis) { P.cur.scatter_pdf = spdf; P.cur.light_pdf = lpdf; }
    }

    // environment.cuh:717-808
    void accumulate_light_bwd(Path<T>& P) {
        P.cur.contribution = {};
        const bool first = P.bounces == 1u;
        T bmis = 1, lmis = 1;
        if (cfg.enable_mis && first) { bmis = mis(P.cur.scatter_pdf, P.cur.light_pdf); lmis = mis(P.emitter.light_pdf, P.emitter.scatter_pdf); }
        if (in.render_opts == 1) {
            if (cfg.enable_mis && first) P.acc -= P.emitter.contribution * lmis;
            if (P.bounces > 0u && P.cur.inter.valid) {
                P.cur.contribution = P.throughput * P.cur.radiance;
                if (cfg.enable_mis && first) P.cur.contribution *= bmis;
                P.acc -= P.cur.contribution;
            } else if (P.cur.valid) {
                V3<T> vr{};
                const int seen = escaped_light(P.cur.ray, vr);
                if (seen == 0) return;
                P.throughput *= P.cur.transmittance;
                V3<T> eg = P.acc_grad * P.throughput;
                if (cfg.enable_mis && first) eg *= bmis;
                eg += P.acc_light_grad;
                if (seen == 2) vr = background_bwd(P.cur.ray.d, eg, &P.cur.ray_dir_grad);
                P.cur.contribution = P.throughput * vr;
                if (cfg.enable_mis && first) P.cur.contribution *= bmis;
                P.acc -= P.cur.contribution;
            }
            return;
        }
        if (cfg.enable_mis && first) P.acc -= P.emitter.contribution * lmis;
        if (P.cur.valid) {
            V3<T> vr{};
            const int seen = escaped_light(P.cur.ray, vr);
            if (seen == 0) return;
            P.throughput *= P.cur.transmittance;
            V3<T> eg = P.acc_grad * P.throughput;
            if (cfg.enable_mis && first) eg *= bmis;
            eg += P.acc_light_grad;
            if (seen == 2) vr = background_bwd(P.cur.ray.d, eg, &P.cur.ray_dir_grad);
            P.cur.contribution = P.throughput * vr;
            if (cfg.enable_mis && first) P.cur.contribution *= bmis;
            P.cur.radiance += P.cur.contribution;
            P.acc -= P.cur.contribution;
        }
    }

    // ---- launch index → world ray (pipelineParameters.h:93-111)
    Ray<T> world_ray(size_t li) const {
        const float* o = in.ray_ori + 3 * li;
        const float* d = in.ray_dir + 3 * li;
        const float* m = in.ray_to_world;
        Ray<T> r;
        r.o = {T(m[0]) * o[0] + T(m[1]) * o[1] + T(m[2]) * o[2] + T(m[3]),
               T(m[4]) * o[0] + T(m[5]) * o[1] + T(m[6]) * o[2] + T(m[7]),
               T(m[8]) * o[0] + T(m[9]) * o[1] + T(m[10]) * o[2] + T(m[11])};
        r.d = {T(m[0]) * d[0] + T(m[1]) * d[1] + T(m[2]) * d[2],
               T(m[4]) * d[0] + T(m[5]) * d[1] + T(m[6]) * d[2],
               T(m[8]) * d[0] + T(m[9]) * d[1] + T(m[10]) * d[2]};
        return r;
    }

    static uint32_t sig_segment(const RayPayload<T>& p) {
        const double hc = std::fmin(std::fmax(double(p.hits_count), 0.0), 65535.0);
        return uint32_t(hc) | (p.inter.valid ? 1u << 16 : 0u) | (p.valid ? 1u << 17 : 0u) | (p.hit ? 1u << 18 : 0u);
    }
    static constexpr uint32_t kSigNee = 0x100000u, kSigShadow = 0x200000u, kSigCont = 0x300000u;

    unsigned max_bounces() const {  // optixTracer.cpp:959
        return in.render_opts ? std::min(in.max_bounces, 2u) : in.max_bounces;
    }

    // referenceOptix.cu:27-71
    void forward_one(size_t li, uint32_t x, uint32_t y, uint32_t z, const FwdOut& out) {
        Sampler s;
        s.init_launch(x, y, z, in.frame);
        Path<T> P;
        P.max_bounces = max_bounces();
        const Ray<T> ray = world_ray(li);
        st.segments++;
        ray_intersect(false, ray, P.cur, s);
        P.mix(sig_segment(P.cur));
        if (out.path_sig) out.path_sig[li] = P.sig;
        // pathTracer.cuh:636-663
        auto put = [](float* dst, size_t li, int c, std::initializer_list<T> v) {
            if (!dst) return;
            int k = 0;
            for (T e : v) dst[li * c + k++] = float(e);
        };
        const RayPayload<T>& p = P.cur;
        put(out.radiance, li, 3, {p.radiance.x, p.radiance.y, p.radiance.z});
        put(out.density, li, 1, {T(1) - p.transmittance});
        put(out.hit, li, 2, {p.hit_distance, p.last_hit});
        put(out.hit2, li, 1, {p.hit2});
        put(out.distortion, li, 1, {p.distortion});
        if (cfg.enable_normals) {
            put(out.normal, li, 3, {p.normal.x, p.normal.y, p.normal.z});
            put(out.snormal, li, 3, {p.inter.snormal.x, p.inter.snormal.y, p.inter.snormal.z});
        } else {
            put(out.normal, li, 3, {T(0), T(0), T(0)});
            put(out.snormal, li, 3, {T(0), T(0), T(0)});
        }
        put(out.material, li, 5, {p.inter.albedo.x, p.inter.albedo.y, p.inter.albedo.z, p.inter.roughness, p.inter.metallic});
        put(out.hits_count, li, 1, {cfg.enable_hitcounts ? p.hits_count : T(0)});
        put(out.pbr, li, 3, {T(0), T(0), T(0)});
        put(out.light, li, 3, {T(0), T(0), T(0)});
        put(out.components, li, 6, {T(0), T(0), T(0), T(0), T(0), T(0)});
        if (!cfg.visualize_lights && !P.cur.inter.valid) return;
        if (cfg.enable_mis) sample_nee(P, s);
        for (unsigned depth = 0; depth < P.max_bounces && P.active; ++depth) {
            accumulate_light(P);
            P.active &= unsigned((depth + 1u < P.max_bounces) && P.cur.inter.valid);
            if (!P.active) break;
            P.bounces = depth + 1u;
            sample_next(P, s);
            const bool cont = P.active && !(vmax(P.throughput) < T(1e-4));
            P.mix(kSigCont | (cont ? 1u : 0u));
            if (!cont) break;
            st.segments++;
            ray_intersect(true, P.cur.ray, P.cur, s);
            P.mix(sig_segment(P.cur));
        }
        if (out.path_sig) out.path_sig[li] = P.sig;
        // pathTracer.cuh:665-681
        put(out.pbr, li, 3, {P.acc.x, P.acc.y, P.acc.z});
        put(out.light, li, 3, {P.acc_light.x, P.acc_light.y, P.acc_light.z});
        put(out.components, li, 6, {P.acc_direct.x, P.acc_direct.y, P.acc_direct.z, P.acc_indirect.x, P.acc_indirect.y,
                                    P.acc_indirect.z});
    }

    // referenceBwdOptix.cu:27-74
    void backward_one(size_t li, uint32_t x, uint32_t y, uint32_t z, const BwdIn& bi) {
        Sampler s;
        s.init_launch(x, y, z, in.frame);
        Path<T> P;
        P.max_bounces = max_bounces();
        auto g3 = [&](const float* a) { return a ? v3<T>(a[3 * li], a[3 * li + 1], a[3 * li + 2]) : V3<T>{}; };
        P.acc = g3(bi.pbr);
        P.acc_grad = g3(bi.pbr_grad);
        P.acc_light = g3(bi.light);
        P.acc_light_grad = g3(bi.light_grad);
        const Ray<T> ray = world_ray(li);
        ray_intersect(false, ray, P.cur, s);
        if (P.cur.inter.valid && bi.material_grad) {
            const float* mg = bi.material_grad + 5 * li;
            P.cur.inter.d_albedo += v3<T>(mg[0], mg[1], mg[2]);
            P.cur.inter.d_roughness += T(mg[3]);
            if (cfg.enable_metallic) P.cur.inter.d_metallic += T(mg[4]);
        }
        if (!cfg.visualize_lights && !P.cur.inter.valid) return;
        if (cfg.enable_mis) sample_nee(P, s);
        for (unsigned depth = 0; depth < P.max_bounces && P.active; ++depth) {
            accumulate_light_bwd(P);
            pending_bwd(P);
            P.active &= unsigned((depth + 1u < P.max_bounces) && P.cur.inter.valid);
            if (!P.active) break;
            P.bounces = depth + 1u;
            sample_next_bwd(P, s);
            if (vmax(P.throughput) < T(1e-4)) break;
            ray_intersect(true, P.cur.ray, P.cur, s);
        }
    }
};

}  // namespace oracle

// =======================================================================================
// C API for ctypes (tests and bench CPU legs only)
using namespace oracle;

extern "C" {

struct orc_config {
    int kernel_degree;
    float min_response;
    int density_clamping;
    int sph_max_coeffs;
    int enable_normals, enable_hitcounts, enable_mis, enable_metallic, visualize_lights;
    int draw_order;
};

struct orc_scene {
    int n;
    const float *bpos, *brot, *bscl, *bdns;
    const float *density, *material, *sph, *snrm;
    const float* env;
    int eh, ew;
    const float* alias;
    int ah, aw;
    const float* ray_to_world;  // 12 floats (3x4)
    const float *ray_ori, *ray_dir;
    int nz, h, w;
    unsigned frame;
    int sph_degree;
    float min_transmittance;
    unsigned max_bounces;
    unsigned render_opts;
    const float* lights;
    const float* light_table;
    const float* mesh_vertices;
    const int* mesh_triangles;
    const float* mesh_lights;
    const float* mesh_tri_table;
    int num_lights, light_entries, num_mesh_vertices, num_mesh_triangles, num_mesh_lights, mesh_tri_cols;
};

struct orc_fwd_out {
    float *radiance, *density, *hit, *hit2, *distortion, *normal, *snormal, *material, *hits_count, *pbr, *light,
        *components, *visibility;
    uint32_t* path_sig;
};

struct orc_bwd_in {
    const float *pbr, *light, *pbr_grad, *light_grad, *material_grad;
};

struct orc_stats {
    unsigned long long segments, trace_calls, candidates, accepted, env_lookups, replay_segments;
};

}  // extern "C"

static Config to_cfg(const orc_config* c) {
    Config k;
    k.kernel_degree = c->kernel_degree;
    k.min_response = c->min_response;
    k.density_clamping = c->density_clamping;
    k.sph_max_coeffs = c->sph_max_coeffs;
    k.enable_normals = c->enable_normals;
    k.enable_hitcounts = c->enable_hitcounts;
    k.enable_mis = c->enable_mis;
    k.enable_metallic = c->enable_metallic;
    k.visualize_lights = c->visualize_lights;
    kDrawOrder = c->draw_order;
    return k;
}

static Inputs to_in(const orc_scene* s) {
    Inputs in;
    in.n = s->n;
    in.bpos = s->bpos; in.brot = s->brot; in.bscl = s->bscl; in.bdns = s->bdns;
    in.density = s->density; in.material = s->material; in.sph = s->sph; in.snrm = s->snrm;
    in.env = s->env; in.eh = s->eh; in.ew = s->ew;
    in.alias = s->alias; in.ah = s->ah; in.aw = s->aw;
    if (s->ray_to_world) std::memcpy(in.ray_to_world, s->ray_to_world, 12 * sizeof(float));
    in.ray_ori = s->ray_ori; in.ray_dir = s->ray_dir;
    in.nz = s->nz; in.h = s->h; in.w = s->w;
    in.frame = s->frame;
    in.sph_degree = s->sph_degree;
    in.min_transmittance = s->min_transmittance;
    in.max_bounces = s->max_bounces;
    in.render_opts = s->render_opts;
    in.lights = s->lights; in.light_table = s->light_table; in.mesh_vertices = s->mesh_vertices;
    in.mesh_triangles = s->mesh_triangles; in.mesh_lights = s->mesh_lights; in.mesh_tri_table = s->mesh_tri_table;
    in.num_lights = s->lights ? s->num_lights : 0;
    in.light_entries = s->light_table ? s->light_entries : 0;
    in.num_mesh_vertices = s->mesh_vertices ? s->num_mesh_vertices : 0;
    in.num_mesh_triangles = s->mesh_triangles ? s->num_mesh_triangles : 0;
    in.num_mesh_lights = s->mesh_lights ? s->num_mesh_lights : 0;
    in.mesh_tri_cols = s->mesh_tri_table ? s->mesh_tri_cols : 0;
    return in;
}

static void add_stats(orc_stats* o, const Stats& s) {
    if (!o) return;
    o->segments += s.segments; o->trace_calls += s.trace_calls; o->candidates += s.candidates;
    o->accepted += s.accepted; o->env_lookups += s.env_lookups; o->replay_segments += s.replay_segments;
}

template <class T>
static int run_fwd(const orc_config* c, const orc_scene* s, const orc_fwd_out* o, int nthreads, long long stride,
                   orc_stats* stats) {
    const Config cfg = to_cfg(c);
    const Inputs in = to_in(s);
    Instances<T> I;
    build_instances<T>(cfg, in, I);
    FwdOut out;
    out.radiance = o->radiance; out.density = o->density; out.hit = o->hit; out.hit2 = o->hit2;
    out.distortion = o->distortion; out.normal = o->normal; out.snormal = o->snormal; out.material = o->material;
    out.hits_count = o->hits_count; out.pbr = o->pbr; out.light = o->light; out.components = o->components;
    out.path_sig = o->path_sig;
    if (o->visibility) std::fill(o->visibility, o->visibility + in.n, 0.0f);
    const long long total = (long long)in.nz * in.h * in.w;
    if (stride < 1) stride = 1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    std::vector<Stats> st(omp_get_max_threads());
#pragma omp parallel
    {
        Tracer<T> tr(cfg, in, I);
        tr.visibility = o->visibility;  // idempotent writes of 1.0f
#pragma omp for schedule(dynamic, 64)
        for (long long li = 0; li < total; li += stride) {
            const uint32_t x = uint32_t(li % in.w), y = uint32_t((li / in.w) % in.h), z = uint32_t(li / ((long long)in.w * in.h));
            tr.forward_one(size_t(li), x, y, z, out);
        }
        st[omp_get_thread_num()] = tr.st;
    }
    for (auto& e : st) add_stats(stats, e);
    return 0;
}

template <class T>
static int run_bwd(const orc_config* c, const orc_scene* s, const orc_bwd_in* b, double* mat_grad, double* env_grad,
                   int nthreads, long long stride, orc_stats* stats) {
    const Config cfg = to_cfg(c);
    const Inputs in = to_in(s);
    Instances<T> I;
    build_instances<T>(cfg, in, I);
    BwdIn bi;
    bi.pbr = b->pbr; bi.light = b->light; bi.pbr_grad = b->pbr_grad; bi.light_grad = b->light_grad;
    bi.material_grad = b->material_grad;
    const long long total = (long long)in.nz * in.h * in.w;
    if (stride < 1) stride = 1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int nt = omp_get_max_threads();
    std::vector<std::vector<double>> mg(nt), eg(nt);
    std::vector<Stats> st(nt);
#pragma omp parallel
    {
        const int t = omp_get_thread_num();
        mg[t].assign(size_t(in.n) * 5, 0.0);
        eg[t].assign(size_t(std::max(in.eh, 0)) * std::max(in.ew, 0) * 4, 0.0);
        Tracer<T> tr(cfg, in, I);
        tr.mat_grad = &mg[t];
        tr.env_grad = &eg[t];
#pragma omp for schedule(dynamic, 64)
        for (long long li = 0; li < total; li += stride) {
            const uint32_t x = uint32_t(li % in.w), y = uint32_t((li / in.w) % in.h), z = uint32_t(li / ((long long)in.w * in.h));
            tr.backward_one(size_t(li), x, y, z, bi);
        }
        st[t] = tr.st;
    }
    if (mat_grad) {
        std::fill(mat_grad, mat_grad + size_t(in.n) * 5, 0.0);
        for (auto& v : mg) for (size_t i = 0; i < v.size(); ++i) mat_grad[i] += v[i];
    }
    if (env_grad) {
        const size_t ne = size_t(std::max(in.eh, 0)) * std::max(in.ew, 0) * 4;
        std::fill(env_grad, env_grad + ne, 0.0);
        for (auto& v : eg) for (size_t i = 0; i < v.size(); ++i) env_grad[i] += v[i];
    }
    for (auto& e : st) add_stats(stats, e);
    return 0;
}

extern "C" {

int orc_trace_f64(const orc_config* c, const orc_scene* s, const orc_fwd_out* o, int nthreads, long long stride,
                  orc_stats* stats) {
    return run_fwd<double>(c, s, o, nthreads, stride, stats);
}
int orc_trace_f32(const orc_config* c, const orc_scene* s, const orc_fwd_out* o, int nthreads, long long stride,
                  orc_stats* stats) {
    return run_fwd<float>(c, s, o, nthreads, stride, stats);
}
int orc_trace_bwd_f64(const orc_config* c, const orc_scene* s, const orc_bwd_in* b, double* mat_grad, double* env_grad,
                      int nthreads, long long stride, orc_stats* stats) {
    return run_bwd<double>(c, s, b, mat_grad, env_grad, nthreads, stride, stats);
}
int orc_trace_bwd_f32(const orc_config* c, const orc_scene* s, const orc_bwd_in* b, double* mat_grad, double* env_grad,
                      int nthreads, long long stride, orc_stats* stats) {
    return run_bwd<float>(c, s, b, mat_grad, env_grad, nthreads, stride, stats);
}

// candidate lists of single trace() calls, for traversal tests: rays [m,6] (o,d), tmin/tend [m];
// out_ids [m,16] (0xFFFFFFFF = empty), out_t [m,16]
int orc_trace_candidates(const orc_config* c, const orc_scene* s, int m, const float* rays, const float* tmin,
                         const float* tend, unsigned* out_ids, double* out_t) {
    const Config cfg = to_cfg(c);
    const Inputs in = to_in(s);
    Instances<double> I;
    build_instances<double>(cfg, in, I);
    Tracer<double> tr(cfg, in, I);
    std::array<Hit, kK> hits;
    for (int i = 0; i < m; ++i) {
        Ray<double> r{{rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]}, {rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]}};
        tr.trace(hits, r, tmin[i], tend[i]);
        for (int k = 0; k < kK; ++k) { out_ids[16 * i + k] = hits[k].id; out_t[16 * i + k] = hits[k].t; }
    }
    return 0;
}

// scene AABB and per-Gaussian kernel scale / world AABB (build_bvh parity): aabb[6], kscl[n], lo/hi [n,3]
int orc_instances(const orc_config* c, const orc_scene* s, double* aabb, double* kscl, double* lo, double* hi) {
    const Config cfg = to_cfg(c);
    const Inputs in = to_in(s);
    Instances<double> I;
    build_instances<double>(cfg, in, I);
    aabb[0] = I.scene_lo.x; aabb[1] = I.scene_lo.y; aabb[2] = I.scene_lo.z;
    aabb[3] = I.scene_hi.x; aabb[4] = I.scene_hi.y; aabb[5] = I.scene_hi.z;
    for (int g = 0; g < in.n; ++g) {
        if (kscl) kscl[g] = kernel_scale<double>(in.bdns[g], cfg.min_response, cfg.density_clamping != 0, cfg.kernel_degree);
        if (lo) { lo[3 * g] = I.lo[g].x; lo[3 * g + 1] = I.lo[g].y; lo[3 * g + 2] = I.lo[g].z; }
        if (hi) { hi[3 * g] = I.hi[g].x; hi[3 * g + 1] = I.hi[g].y; hi[3 * g + 2] = I.hi[g].z; }
    }
    return 0;
}

// PCG32 stream of a launch index: out[count] u32 values after init (sampler.cuh:43-72)
int orc_sampler_stream(unsigned x, unsigned y, unsigned z, unsigned frame, int count, unsigned* out) {
    Sampler s;
    s.init_launch(x, y, z, frame);
    for (int i = 0; i < count; ++i) out[i] = s.next_u32();
    return 0;
}

unsigned long long orc_launch_seed(unsigned x, unsigned y, unsigned z, unsigned frame) {
    return Sampler::seed_of(x, y, z, frame);
}

int orc_num_threads(void) { return omp_get_max_threads(); }

// Light samples from positions pos [m,3], sample i drawn from the launch stream (i, 0, 0, frame):
// out [m,9] = wi xyz, Li rgb, pdf, dist, type; eval_pdf [m] = the light sampler's pdf of the
// sampled direction (lightSampler.cuh:340-406). FP64.
}  // extern "C"

// Known-answer evaluations of single reference functions in scalar type T (see orc_kat).
template <class T>
static int kat_impl(const orc_config* c, const orc_scene* sc, const char* name, int n, const float* in, double* out,
                    double* env_grad) {
    const Config cfg = to_cfg(c);
    const Inputs inp = to_in(sc);
    Instances<T> I;
    build_instances<T>(cfg, inp, I);
    Tracer<T> tr(cfg, inp, I);
    std::vector<double> eg(size_t(std::max(inp.eh, 0)) * std::max(inp.ew, 0) * 4, 0.0);
    tr.env_grad = &eg;
    using V = V3<T>;
    const std::string what(name);
    auto v3f = [](const float* p) { return V{T(p[0]), T(p[1]), T(p[2])}; };
    auto put3 = [](double* o, const V& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; };
    for (int i = 0; i < n; ++i) {
        if (what == "process_hit") {
            const float* a = in + 8 * size_t(i);
            typename Tracer<T>::HitSums h;
            h.transmittance = a[7];
            const bool acc = tr.process_hit(uint32_t(a[6]), Ray<T>{v3f(a), v3f(a + 3)}, h);
            double* o = out + 18 * size_t(i);
            o[0] = acc ? 1.0 : 0.0; o[1] = h.transmittance; put3(o + 2, h.radiance); o[5] = h.depth; o[6] = h.depth2;
            put3(o + 7, h.alb); o[10] = h.rgh; o[11] = h.met; put3(o + 12, h.snrm); put3(o + 15, h.normal);
        } else if (what == "intersect") {
            const float* a = in + 8 * size_t(i);
            T t = T(0);
            const bool hit = Tracer<T>::instance_hit(v3f(a), v3f(a + 3), T(a[6]), T(a[7]), t);
            out[2 * size_t(i)] = hit ? 1.0 : 0.0;
            out[2 * size_t(i) + 1] = t;
        } else if (what == "brdf_sample" || what == "brdf_eval" || what == "brdf_grads") {
            const float* a = in + 16 * size_t(i);
            const V wo = v3f(a), nrm = v3f(a + 3), alb = v3f(a + 6), r3 = v3f(a + 11);
            T pdf = T(0);
            if (what == "brdf_eval") {
                put3(out + 4 * size_t(i), tr.eval_brdf(wo, nrm, alb, T(a[9]), T(a[10]), r3, pdf));
                out[4 * size_t(i) + 3] = pdf;
            } else if (what == "brdf_sample") {
                V next{};
                const V v = tr.sample_brdf(wo, nrm, alb, T(a[9]), T(a[10]), r3, next, pdf);
                double* o = out + 7 * size_t(i);
                put3(o, v); put3(o + 3, next); o[6] = pdf;
            } else {
                V next{};
                const BrdfGrad<T> g = tr.sample_brdf_grad(wo, nrm, alb, T(a[9]), T(a[10]), r3, next, pdf);
                double* o = out + 19 * size_t(i);
                put3(o, g.value); put3(o + 3, g.d_albedo); put3(o + 6, g.d_metallic); put3(o + 9, g.d_roughness);
                put3(o + 12, g.d_next_dir); put3(o + 15, next); o[18] = pdf;
            }
        } else if (what == "env_lookup") {
            const V d = v3f(in + 3 * size_t(i));
            put3(out + 4 * size_t(i), tr.background(d));
            out[4 * size_t(i) + 3] = inp.ah > 0 ? tr.alias_pdf(d) : 0.0;
        } else if (what == "env_bwd") {
            const float* a = in + 6 * size_t(i);
            V dir_grad{};
            put3(out + 6 * size_t(i), tr.background_bwd(v3f(a), v3f(a + 3), &dir_grad));
            put3(out + 6 * size_t(i) + 3, dir_grad);
        } else if (what == "env_sample") {
            const float* a = in + 4 * size_t(i);
            Sampler s;
            s.init_launch(unsigned(a[0]), unsigned(a[1]), unsigned(a[2]), unsigned(a[3]));
            T pdf = T(0);
            put3(out + 4 * size_t(i), tr.sample_alias_dir(s, pdf));
            out[4 * size_t(i) + 3] = pdf;
        } else if (what == "light_sample") {
            const float* a = in + 7 * size_t(i);
            Sampler s;
            s.init_launch(unsigned(a[3]), unsigned(a[4]), unsigned(a[5]), unsigned(a[6]));
            const auto ls = tr.sample_light(v3f(a), s);
            double* o = out + 9 * size_t(i);
            put3(o, ls.wi); put3(o + 3, ls.Li); o[6] = ls.pdf; o[7] = ls.dist; o[8] = double(ls.type);
        } else if (what == "light_pdf") {
            const float* a = in + 6 * size_t(i);
            out[i] = tr.light_pdf(v3f(a), v3f(a + 3));
        } else {
            return 1;
        }
    }
    if (env_grad) std::copy(eg.begin(), eg.end(), env_grad);
    return 0;
}

extern "C" {

// Known-answer evaluations of single reference functions, the cases of tests/golden/device_kat.npz
// (inputs and outputs laid out as the reference kernels of oracle/ref_device_kat.cu lay them out),
// in FP64, or with fp32 != 0 in the FP32 instantiation. env_grad [eh, ew, 4] receives the
// environment gradient of "env_bwd".
int orc_kat(const orc_config* c, const orc_scene* sc, const char* name, int n, const float* in, double* out,
            double* env_grad, int fp32) {
    return fp32 ? kat_impl<float>(c, sc, name, n, in, out, env_grad) : kat_impl<double>(c, sc, name, n, in, out, env_grad);
}

int orc_light_samples(const orc_config* c, const orc_scene* sc, int m, const float* pos, double* out,
                      double* eval_pdf) {
    const Config cfg = to_cfg(c);
    const Inputs in = to_in(sc);
    Instances<double> I;
    build_instances<double>(cfg, in, I);
    Tracer<double> tr(cfg, in, I);
    for (int i = 0; i < m; ++i) {
        Sampler s;
        s.init_launch(unsigned(i), 0u, 0u, in.frame);
        const V3<double> p{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        const auto ls = tr.sample_light(p, s);
        double* o = out + 9 * size_t(i);
        o[0] = ls.wi.x; o[1] = ls.wi.y; o[2] = ls.wi.z;
        o[3] = ls.Li.x; o[4] = ls.Li.y; o[5] = ls.Li.z;
        o[6] = ls.pdf; o[7] = ls.dist; o[8] = double(ls.type);
        eval_pdf[i] = ls.pdf > 0.0 ? tr.light_pdf(p, ls.wi) : 0.0;
    }
    return 0;
}

}  // extern "C"
