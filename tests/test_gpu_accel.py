"""The LBVH that replaces the reference's OptiX instance acceleration structure
(OptixTracer::buildBVH, optixTracer.cpp:633-907, with the instance transforms of
particlePrimitives.cu:543-610): its structure, walked from ptir_debug_accel, and a refit after the
Gaussians move (the reference's OPTIX_BUILD_OPERATION_UPDATE, done every training step).

Binary node record (16 floats): left box lo.xyz, left box hi.xyz, right box lo.xyz, right box
hi.xyz, left child, right child (int32 bits: >= 0 a node, else leaf ~c), left kmax, right kmax.
Leaf record (16 floats): the world -> instance affine map [A | b] as three rows, then
(Gaussian id as uint32 bits, kmax, 0, 0).
"""
import numpy as np
import pytest
import torch

from oracle import compare as K
from oracle import oracle as O
from tests.scenes import _light_tensors, gpu_trace_bwd, make_tracer, small_scene, to_torch

pytestmark = pytest.mark.gpu

CORNERS = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64)


def _leaf_box(rec):
    m = rec[:12].astype(np.float64).reshape(3, 4)
    A, b = m[:, :3], m[:, 3]
    world = (np.linalg.inv(A) @ (CORNERS - b).T).T
    return world.min(0), world.max(0)


def _walk(nodes, leaves):
    """Check the tree and its boxes; returns (leaf ids in leaf order, node topology)."""
    n = leaves.shape[0]
    ids = leaves[:, 12].copy().view(np.uint32)
    assert np.array_equal(np.sort(ids), np.arange(n, dtype=np.uint32)), "leaves are not a permutation"
    leaf_boxes = [_leaf_box(leaves[i]) for i in range(n)]
    kmax_leaf = leaves[:, 13].astype(np.float64)
    topo = nodes[:, 12:14].copy().view(np.int32)

    def node_box(i):
        r = nodes[i].astype(np.float64)
        return (np.minimum(r[0:3], r[6:9]), np.maximum(r[3:6], r[9:12])), max(r[14], r[15])

    seen_nodes, seen_leaves = np.zeros(n - 1, bool), np.zeros(n, bool)
    stack = [0]
    while stack:
        i = stack.pop()
        assert not seen_nodes[i], f"node {i} reached twice"
        seen_nodes[i] = True
        r = nodes[i].astype(np.float64)
        for c, lo, hi, k in ((topo[i, 0], r[0:3], r[3:6], r[14]), (topo[i, 1], r[6:9], r[9:12], r[15])):
            if c >= 0:
                (clo, chi), ck = node_box(c)
                stack.append(c)
            else:
                leaf = ~c
                assert not seen_leaves[leaf], f"leaf {leaf} reached twice"
                seen_leaves[leaf] = True
                clo, chi = leaf_boxes[leaf]
                ck = kmax_leaf[leaf]
            tol = 1e-5 * (1.0 + np.abs(clo).max() + np.abs(chi).max())
            assert np.all(lo <= clo + tol) and np.all(hi >= chi - tol), (i, c, lo, hi, clo, chi)
            assert k >= ck * (1 - 1e-6), (i, c, k, ck)
    assert seen_nodes.all() and seen_leaves.all()
    return ids, topo


def _oracle_boxes_match(leaves, s):
    """Every leaf's box is its Gaussian's instance AABB as the oracle computes it (FP64)."""
    _, _, lo, hi = O.instances(O.OracleConfig(), s)
    ids = leaves[:, 12].copy().view(np.uint32)
    for i in range(leaves.shape[0]):
        blo, bhi = _leaf_box(leaves[i])
        g = ids[i]
        scale = 1e-4 * (1.0 + np.abs(hi[g]).max())
        assert np.allclose(blo, lo[g], atol=scale) and np.allclose(bhi, hi[g], atol=scale), (g, blo, lo[g], bhi, hi[g])


def _moved(s, frac=0.25, seed=3):
    """A seeded subset of the Gaussians moved, rescaled and re-opacified."""
    rng = np.random.default_rng(seed)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in s.items()}
    n = s["build_pos"].shape[0]
    sel = rng.random(n) < frac
    m = int(sel.sum())
    s["build_pos"][sel] += rng.normal(0.0, 0.05, (m, 3)).astype(np.float32)
    s["build_scl"][sel] *= np.exp(rng.normal(0.0, 0.2, (m, 3))).astype(np.float32)
    s["build_dns"][sel] = (1.0 / (1.0 + np.exp(-rng.standard_normal((m, 1))))).astype(np.float32)
    d = s["density"]
    d[:, 0:3], d[:, 3:4], d[:, 8:11] = s["build_pos"], s["build_dns"], s["build_scl"]
    return s


def _trace(tr, S, build, rebuild):
    zhw = tuple(S["ray_ori"].shape[:3])
    sig = torch.zeros(zhw, dtype=torch.int32, device="cuda")
    if build:
        tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], rebuild, True)
    out = tr.trace(S["frame"], S["ray_to_world"], S["ray_ori"], S["ray_dir"], S["density"], S["material"], S["sph"],
                   S["shading_normal"], S["environment"], S["alias_table"], *_light_tensors(S), S["render_opts"],
                   S["sph_degree"], S["min_transmittance"], S["max_bounces"], path_signature=sig)
    return out, sig.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("case", [
    dict(n=3000, w=32, h=24, spp=1, max_bounces=3),
    dict(n=4000, w=32, h=24, spp=1, max_bounces=3, layout="cluster_shell", scale_range=(0.002, 0.2)),
])
@pytest.mark.parametrize("builder", ["morton", "ploc"])
def test_structure_contains_every_box(cuda_device, case, builder):
    s = small_scene(**case)
    S = to_torch(s)
    tr = make_tracer(bvh_builder=builder)
    tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
    nodes, leaves = (t.numpy() for t in tr.debug_accel())
    _walk(nodes, leaves)
    _oracle_boxes_match(leaves, s)


@pytest.mark.parametrize("builder", ["morton", "ploc"])
def test_refit_after_motion_matches_rebuild_and_oracle(cuda_device, builder):
    s0 = small_scene(n=3000, w=40, h=32, spp=2, max_bounces=3)
    s1 = _moved(s0)
    S0, S1 = to_torch(s0), to_torch(s1)
    tr = make_tracer(bvh_builder=builder)
    tr.build_bvh(S0["build_pos"], S0["build_rot"], S0["build_scl"], S0["build_dns"], True, True)
    _, topo0 = _walk(*(t.numpy() for t in tr.debug_accel()))
    ids0 = tr.debug_accel()[1].numpy()[:, 12].copy().view(np.uint32)
    # refit: same count, rebuild = False, allow_update = True
    out_r, sig_r = _trace(tr, S1, build=True, rebuild=False)
    nodes, leaves = (t.numpy() for t in tr.debug_accel())
    ids1, topo1 = _walk(nodes, leaves)
    assert np.array_equal(topo0, topo1) and np.array_equal(ids0, ids1), "a refit keeps the topology and leaf order"
    _oracle_boxes_match(leaves, s1)
    # a fresh rebuild of the moved scene
    tr_b = make_tracer(bvh_builder=builder)
    out_b, sig_b = _trace(tr_b, S1, build=True, rebuild=True)
    torch.cuda.synchronize()
    assert tr.device_status() == 0 and tr_b.device_status() == 0
    same = sig_r == sig_b
    assert same.mean() >= 0.995, same.mean()
    for k in (0, 1, 7, 10, 11):
        a, b = out_r[k].cpu().numpy(), out_b[k].cpu().numpy()
        ok = K.within(a.reshape(*sig_r.shape, -1), b.reshape(*sig_r.shape, -1))
        assert ok[same].mean() >= 0.999, (k, ok[same].mean())
    # and the refit traces stay within parity of the oracle on the moved scene
    ref, _, _ = O.trace(O.OracleConfig(), s1, "f64")
    agree = sig_r == ref["path_sig"]
    assert agree.mean() >= 0.99, agree.mean()
    ok = K.within(out_r[10].cpu().numpy(), ref["pbr"])
    assert ok[agree].mean() >= 0.998, ok[agree].mean()
    # the scene bounds follow the motion
    lo, hi = tr.scene_bounds().numpy().reshape(2, 3)
    aabb, _, _, _ = O.instances(O.OracleConfig(), s1)
    assert np.allclose(np.concatenate([lo, hi]), aabb, atol=1e-4)


@pytest.mark.parametrize("case", [
    dict(n=3000, w=48, h=40, spp=2, max_bounces=3),
    dict(n=6000, w=40, h=32, spp=2, max_bounces=4, layout="cluster_shell", scale_range=(0.002, 0.2)),
    dict(n=4000, w=32, h=32, spp=4, max_bounces=3, scale_range=(0.05, 0.3)),
])
@pytest.mark.parametrize("kbuffer", [8, 16])
def test_resumed_calls_match_calls_from_the_root(cuda_device, case, kbuffer):
    """A segment's k-buffer rounds after its first resumed from what the previous round set aside
    (traverse.cuh, resume_rounds = 2) against every round from the root (resume_rounds = 1): the
    same candidates, so the same paths and, path by path, bitwise the same outputs, and the same
    adjoint up to the order of the gradient atomics. Only a grazing Gaussian (closest approach
    before its box entry) can be kept by one order and not the other."""
    s = small_scene(**case)
    S = to_torch(s)
    root = make_tracer(kbuffer=kbuffer, resume_rounds=1)
    resumed = make_tracer(kbuffer=kbuffer, resume_rounds=2)
    out_a, sig_a = _trace(root, S, build=True, rebuild=True)
    out_b, sig_b = _trace(resumed, S, build=True, rebuild=True)
    torch.cuda.synchronize()
    assert root.device_status() == 0 and resumed.device_status() == 0
    same = sig_a == sig_b
    print(f"k{kbuffer} {case}: {same.mean():.6f} of paths take the same decisions; node visits "
          f"{root.counters()['node_visits']} from the root, {resumed.counters()['node_visits']} resumed")
    assert same.mean() >= 0.999, same.mean()
    for k in (0, 1, 2, 3, 4, 5, 6, 7, 8, 10, 11, 12):
        a = out_a[k].cpu().numpy().reshape(*sig_a.shape, -1)
        b = out_b[k].cpu().numpy().reshape(*sig_b.shape, -1)
        eq = np.all(a == b, axis=-1)
        assert eq[same].mean() >= 0.999, (k, eq[same].mean())
    assert resumed.counters()["node_visits"] < root.counters()["node_visits"]
    # the backward replay's rounds (resumed by default)
    g = torch.from_numpy(np.random.default_rng(3).standard_normal(tuple(sig_a.shape) + (3,)).astype(np.float32)).cuda()
    g = torch.where(torch.from_numpy(same).cuda()[..., None], g, torch.zeros_like(g))
    grads = []
    for tr, out in ((root, out_a), (resumed, out_b)):
        _, mg, _, _, eg = gpu_trace_bwd(tr, S, list(out), g)
        grads.append((mg.cpu().numpy(), eg.cpu().numpy()))
    torch.cuda.synchronize()
    for a, b in zip(grads[0], grads[1]):
        rel, cos = K.rel_cos(a, b)
        assert rel <= 3e-5 and cos >= 0.99999, (rel, cos)


@pytest.mark.parametrize("case", [
    dict(n=3000, w=48, h=40, spp=2, max_bounces=3),
    dict(n=6000, w=40, h=32, spp=2, max_bounces=4, layout="cluster_shell", scale_range=(0.002, 0.2)),
    dict(n=40000, w=32, h=24, spp=1, max_bounces=3, layout="cluster_shell", scale_range=(0.002, 0.2)),
])
def test_ploc_tree_traces_as_the_morton_tree(cuda_device, case):
    """The PLOC hierarchy (agglomerative clustering by surface area, accel.cu) against the Karras
    hierarchy over the same sorted leaves: every trace call returns the K nearest candidates of its
    interval whatever the tree, so the paths take the same decisions and their outputs are bitwise
    equal, up to the order-dependent grazing case. The forward and the adjoint are compared."""
    s = small_scene(**case)
    S = to_torch(s)
    morton = make_tracer(bvh_builder="morton", collect_counters=True)
    ploc = make_tracer(bvh_builder="ploc", collect_counters=True)
    out_a, sig_a = _trace(morton, S, build=True, rebuild=True)
    out_b, sig_b = _trace(ploc, S, build=True, rebuild=True)
    torch.cuda.synchronize()
    assert morton.device_status() == 0 and ploc.device_status() == 0
    _walk(*(t.numpy() for t in ploc.debug_accel()))
    same = sig_a == sig_b
    ca, cb = morton.counters(), ploc.counters()
    print(f"{case}: {same.mean():.6f} of paths take the same decisions; node visits / leaf tests "
          f"morton {ca['node_visits']} / {ca['leaf_tests']}, ploc {cb['node_visits']} / {cb['leaf_tests']}")
    assert same.mean() >= 0.999, same.mean()
    for k in (0, 1, 2, 3, 4, 5, 6, 7, 8, 10, 11, 12):
        a = out_a[k].cpu().numpy().reshape(*sig_a.shape, -1)
        b = out_b[k].cpu().numpy().reshape(*sig_b.shape, -1)
        eq = np.all(a == b, axis=-1)
        assert eq[same].mean() >= 0.999, (k, eq[same].mean())
    g = torch.from_numpy(np.random.default_rng(5).standard_normal(tuple(sig_a.shape) + (3,)).astype(np.float32)).cuda()
    g = torch.where(torch.from_numpy(same).cuda()[..., None], g, torch.zeros_like(g))
    grads = []
    for tr, out in ((morton, out_a), (ploc, out_b)):
        _, mg, _, _, eg = gpu_trace_bwd(tr, S, list(out), g)
        grads.append((mg.cpu().numpy(), eg.cpu().numpy()))
    torch.cuda.synchronize()
    for a, b in zip(grads[0], grads[1]):
        rel, cos = K.rel_cos(a, b)
        assert rel <= 1e-5 and cos >= 0.99999, (rel, cos)


def test_ploc_rebuild_under_capture_fails_cleanly(cuda_device):
    """A PLOC rebuild synchronises its stream, so under CUDA-graph capture ptir_build_bvh refuses it
    before it enqueues anything: the call raises, the capture ends empty, and the structure built
    before stays in use (the same traces as before the attempt)."""
    from ptir_b200._native import PtirError

    s = small_scene(n=2000, w=16, h=16, spp=1, max_bounces=2)
    S = to_torch(s)
    tr = make_tracer(bvh_builder="ploc")
    out0, sig0 = _trace(tr, S, build=True, rebuild=True)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with pytest.raises(PtirError, match="cannot be captured"):
        with torch.cuda.graph(graph):
            tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
    torch.cuda.synchronize()
    del graph
    out1, sig1 = _trace(tr, S, build=False, rebuild=False)
    torch.cuda.synchronize()
    assert tr.device_status() == 0
    assert np.array_equal(sig0, sig1)
    assert torch.equal(out0[10], out1[10])


def test_ploc_coincident_gaussians_build_a_balanced_tree(cuda_device):
    """Coincident Gaussians give equal union areas for every pair of them. The PLOC tie-break pairs
    equal boxes up all at once ((0,1), (2,3), ... in the list), so 30,000 copies of one Gaussian
    build in a few iterations into a balanced tree, not a chain of one merge per iteration (which
    would also overflow the traversal stack). The tree is walked and a trace runs without a loop
    bound or stack overflow."""
    import time

    s = small_scene(n=30000, w=16, h=16, spp=1, max_bounces=2)
    for k in ("build_pos", "build_rot", "build_scl", "build_dns", "density", "material", "sph", "shading_normal"):
        s[k][1:] = s[k][0]  # every Gaussian a copy of the first
    S = to_torch(s)
    warm = make_tracer(bvh_builder="ploc")
    warm.build_bvh(S["build_pos"][:64], S["build_rot"][:64], S["build_scl"][:64], S["build_dns"][:64], True, True)
    torch.cuda.synchronize()
    tr = make_tracer(bvh_builder="ploc")
    t0 = time.perf_counter()
    tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    assert seconds < 3.0, seconds
    nodes, leaves = (t.numpy() for t in tr.debug_accel())
    _, topo = _walk(nodes, leaves)
    depth, stack = 0, [(0, 1)]
    while stack:
        i, dep = stack.pop()
        depth = max(depth, dep)
        stack += [(c, dep + 1) for c in topo[i] if c >= 0]
    assert depth <= 40, depth  # log2(30000) ~ 15
    _trace(tr, S, build=False, rebuild=False)
    torch.cuda.synchronize()
    assert tr.device_status() == 0
