// Forward path tracer and path-replay adjoint through the Gaussian field (FP32, sm_100a).
//
// One thread runs one path of one launch index (x, y, z = sample * B + view), as the
// reference raygen programs do (threedgptir_tracer/src/kernels/cuda/referenceOptix.cu:27-71,
// referenceBwdOptix.cu:27-74). Each warp covers an 8x4 pixel tile so primary rays of a warp
// are coherent. Candidate gathering is the software LBVH traversal of traverse.cuh.
#include "path.cuh"
#include "stages.h"

namespace ptir {

constexpr int kWarpsPerBlock = 4;  // one 8x4 pixel tile per warp

// ------------------------------------------------------------------------------------
// forward (referenceOptix.cu:27-71)
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_trace_fwd(TraceParams P, FwdOutputs O) {
    StackEntry stack[kStackDepth];
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    CtxT<kKBuf> C{P, stack, ctr};
    unsigned x, y, z;
    int view;
    size_t li;
    if (launch_index(P, view, x, y, z, li)) {
        Pcg32 rng;
        rng.seed(x, y, z, P.views[view].frame);
        PathState ps;
        path_init(ps, effective_bounces(P));
        Segment s;
        float3 o, d;
        world_ray(P, view, x, y, z, li, o, d);
        segment_reset(s, o, d, 0.0f);
        ++ctr.segments;
        intersect_mark<false>(C, s, rng, O.visibility);
        sig_event(P, ps, sig_segment(s));
        // primary outputs (pathTracer.cuh:636-663)
        {
            float* r = O.radiance + 3 * li;
            r[0] = s.radiance.x; r[1] = s.radiance.y; r[2] = s.radiance.z;
            O.density[li] = 1.0f - s.transmittance;
            O.hit[2 * li] = s.depth;
            O.hit[2 * li + 1] = s.last_hit;
            O.hit2[li] = s.hit2;
            O.distortion[li] = s.distortion;
            const bool nrm = (P.flags & kNormals) != 0;
            float* n = O.normal + 3 * li;
            n[0] = nrm ? s.normal.x : 0.0f; n[1] = nrm ? s.normal.y : 0.0f; n[2] = nrm ? s.normal.z : 0.0f;
            float* sn = O.snormal + 3 * li;
            sn[0] = nrm ? s.snrm.x : 0.0f; sn[1] = nrm ? s.snrm.y : 0.0f; sn[2] = nrm ? s.snrm.z : 0.0f;
            float* m = O.material + 5 * li;
            m[0] = s.albedo.x; m[1] = s.albedo.y; m[2] = s.albedo.z; m[3] = s.rough; m[4] = s.metal;
            O.hits_count[li] = (P.flags & kHitCounts) ? s.hits_count : 0.0f;
        }
        if ((P.flags & kVisualizeLights) || s.ivalid) {
            if (P.flags & kMis) sample_nee(C, ps, s, rng);
            for (unsigned depth = 0; depth < ps.max_bounces && ps.active; ++depth) {
                accumulate_light(C, ps, s);
                ps.active &= (unsigned)((depth + 1u < ps.max_bounces) && s.ivalid);
                if (!ps.active) break;
                ps.bounces = depth + 1u;
                sample_next(C, ps, s, rng);
                const bool cont = path_continues(ps);
                sig_event(P, ps, kSigCont | (cont ? 1u : 0u));
                if (!cont) break;
                ++ctr.segments;
                intersect_mark<true>(C, s, rng, O.visibility);
                sig_event(P, ps, sig_segment(s));
            }
        }
        if (O.path_sig) O.path_sig[li] = ps.sig;
        // PBR outputs (pathTracer.cuh:665-681); zero when the primary ray found no surface
        float* pb = O.pbr + 3 * li;
        pb[0] = ps.acc.x; pb[1] = ps.acc.y; pb[2] = ps.acc.z;
        float* lg = O.light + 3 * li;
        lg[0] = ps.acc_light.x; lg[1] = ps.acc_light.y; lg[2] = ps.acc_light.z;
        float* cp = O.components + 6 * li;
        cp[0] = ps.acc_direct.x; cp[1] = ps.acc_direct.y; cp[2] = ps.acc_direct.z;
        cp[3] = ps.acc_indirect.x; cp[4] = ps.acc_indirect.y; cp[5] = ps.acc_indirect.z;
    }
    flush_counters(P, ctr);
}

// ------------------------------------------------------------------------------------
// backward (referenceBwdOptix.cu:27-74)
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_trace_bwd(TraceParams P, BwdInputs B) {
    StackEntry stack[kStackDepth];
    TraceCounters ctr = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    CtxT<kKBuf> C{P, stack, ctr};
    unsigned x, y, z;
    int view;
    size_t li;
    if (launch_index(P, view, x, y, z, li)) {
        Pcg32 rng;
        rng.seed(x, y, z, P.views[view].frame);
        PathState ps;
        path_init(ps, effective_bounces(P));
        load_adjoint_inputs(P, B, x, y, z, li, ps);
        Segment s;
        float3 o, d;
        world_ray(P, view, x, y, z, li, o, d);
        segment_reset(s, o, d, 0.0f);
        ++ctr.segments;
        intersect_mark<false>(C, s, rng, nullptr);
        add_material_output_grad(P, B, x, y, z, li, s);
        if ((P.flags & kVisualizeLights) || s.ivalid) {
            if (P.flags & kMis) sample_nee(C, ps, s, rng);
            for (unsigned depth = 0; depth < ps.max_bounces && ps.active; ++depth) {
                accumulate_light_bwd(C, B, ps, s);
                const auto run_replay = [&](const ReplayJob& j) { replay_material_grad(C, B, j); };
                pending_bwd(ps, s, run_replay);
                ps.active &= (unsigned)((depth + 1u < ps.max_bounces) && s.ivalid);
                if (!ps.active) break;
                ps.bounces = depth + 1u;
                sample_next_bwd(C, ps, s, rng, run_replay);
                if (max3(ps.throughput) < 1e-4f) break;
                ++ctr.segments;
                intersect_mark<true>(C, s, rng, nullptr);
            }
        }
    }
    flush_counters(P, ctr);
}

cudaError_t launch_trace_fwd(const TraceParams& p, const FwdOutputs& o, const StageCtx& sc, cudaStream_t s) {
    const long long tiles = p.tiles;
    if (tiles <= 0) return cudaSuccess;
    const long long blocks = (tiles + kWarpsPerBlock - 1) / kWarpsPerBlock;
    sc.run(kStageMegakernel, p, s, [&](const TraceParams& q) {
        k_trace_fwd<<<(unsigned)blocks, 32 * kWarpsPerBlock, 0, s>>>(q, o);
    });
    return cudaGetLastError();
}

cudaError_t launch_trace_bwd(const TraceParams& p, const BwdInputs& b, const StageCtx& sc, cudaStream_t s) {
    const long long tiles = p.tiles;
    if (tiles <= 0) return cudaSuccess;
    const long long blocks = (tiles + kWarpsPerBlock - 1) / kWarpsPerBlock;
    sc.run(kStageMegakernel, p, s, [&](const TraceParams& q) {
        k_trace_bwd<<<(unsigned)blocks, 32 * kWarpsPerBlock, 0, s>>>(q, b);
    });
    return cudaGetLastError();
}

}  // namespace ptir
