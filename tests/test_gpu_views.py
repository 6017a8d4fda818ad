"""Batched views: views of different resolution and sample count traced in one launch sequence
(ptir_trace_views) give each view exactly the outputs of its own trace() call, and the whole
forward + adjoint of a batch replays from a captured CUDA graph with the eager results.

Forward outputs must be bitwise equal (every path is seeded and traced as in its own launch);
visibility is the union of the views' flags. Gradients are sums over views of float32 atomics in
a different order: relative L2 <= 1e-5.
"""
import numpy as np
import pytest
import torch

from ptir_b200 import synthetic
from ptir_b200.optix_tracer import split_views
from tests.scenes import make_tracer, small_scene, to_torch

pytestmark = pytest.mark.gpu

VIEWS = [(24, 16, 2, 3), (40, 32, 1, 5), (16, 16, 4, 3)]  # w, h, spp, frame


def _batch(S, device):
    eyes = synthetic.camera_positions(len(VIEWS), seed=4)
    views, oris, dirs = [], [], []
    for (w, h, spp, frame), eye in zip(VIEWS, eyes):
        o, d = synthetic.view_rays(w, h, spp, eye)
        oris.append(o.to(device))
        dirs.append(d.to(device))
        views.append((frame, S["ray_to_world"], spp, h, w))
    flat_o = torch.cat([o.reshape(-1, 3) for o in oris])
    flat_d = torch.cat([d.reshape(-1, 3) for d in dirs])
    return views, oris, dirs, flat_o, flat_d


def _scene_args(S):
    e = lambda *shape, dt=torch.float32: torch.empty(shape, dtype=dt, device=S["density"].device)  # noqa: E731
    return (S["density"], S["material"], S["sph"], S["shading_normal"], S["environment"], S["alias_table"],
            e(0, 9), e(5, 0), e(0, 3), e(0, 3, dt=torch.int32), e(0, 8), e(3, 0))


def _tail(S):
    return (S["render_opts"], S["sph_degree"], S["min_transmittance"], S["max_bounces"])


@pytest.mark.parametrize("schedule", ["wavefront", "megakernel"])
def test_views_match_separate_traces(cuda_device, schedule):
    s = small_scene(n=2500, max_bounces=3)
    S = to_torch(s)
    tr = make_tracer(schedule=schedule, chunk_tiles=7)
    tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
    views, oris, dirs, flat_o, flat_d = _batch(S, cuda_device)
    batch = [t.clone() for t in tr.trace_views(views, flat_o, flat_d, *_scene_args(S), *_tail(S))]
    vis_union = torch.zeros_like(batch[9].view(torch.int32))
    for k, (view, o, d) in enumerate(zip(views, oris, dirs)):
        single = tr.trace(view[0], view[1], o, d, *_scene_args(S), *_tail(S))
        vis_union |= single[9].view(torch.int32)
        for i, (b, x) in enumerate(zip(batch, single)):
            if i == 9:
                continue
            assert torch.equal(split_views(b, views)[k], x), (k, i)
    assert torch.equal(batch[9].view(torch.int32), vis_union)
    assert tr.device_status() == 0

    # adjoint: the batch gradient is the sum of the views' gradients
    rng = np.random.default_rng(2)
    g = torch.from_numpy(rng.standard_normal(batch[10].shape).astype(np.float32)).to(cuda_device)
    z = torch.zeros_like
    bwd = tr.trace_bwd_views(views, flat_o, flat_d, *batch[:8], batch[10], batch[11], *_scene_args(S)[:6],
                             *_scene_args(S)[6:], z(batch[0]), z(batch[1]), z(batch[2]), z(batch[3]), z(batch[4]),
                             z(batch[5]), z(batch[6]), z(batch[7]), g, z(batch[11]), *_tail(S))
    mg_sum, eg_sum = torch.zeros_like(bwd[1]), torch.zeros_like(bwd[4])
    for k, (view, o, d) in enumerate(zip(views, oris, dirs)):
        fw = [split_views(t, views)[k] for t in batch[:9]] + [batch[9]] + [split_views(t, views)[k] for t in batch[10:]]
        gk = split_views(g, views)[k]
        res = tr.trace_bwd(view[0], view[1], o, d, *fw[:8], fw[10], fw[11], *_scene_args(S), z(fw[0]), z(fw[1]),
                           z(fw[2]), z(fw[3]), z(fw[4]), z(fw[5]), z(fw[6]), z(fw[7]), gk, z(fw[11]), *_tail(S))
        mg_sum += res[1]
        eg_sum += res[4]
    for a, b in ((bwd[1], mg_sum), (bwd[4], eg_sum)):
        assert (a - b).double().norm() <= 1e-5 * b.double().norm() + 1e-12


def test_views_iteration_replays_from_cuda_graph(cuda_device):
    s = small_scene(n=2000, max_bounces=3)
    S = to_torch(s)
    tr = make_tracer()
    tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
    views, _, _, flat_o, flat_d = _batch(S, cuda_device)
    z = torch.zeros_like

    def iteration():
        tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], False, True)
        f = tr.trace_views(views, flat_o, flat_d, *_scene_args(S), *_tail(S))
        g = torch.sign(f[10] - 0.5) * 1e-3
        b = tr.trace_bwd_views(views, flat_o, flat_d, *f[:8], f[10], f[11], *_scene_args(S), z(f[0]), z(f[1]),
                               z(f[2]), z(f[3]), z(f[4]), z(f[5]), z(f[6]), z(f[7]), g, z(f[11]), *_tail(S))
        return f[0], f[10], b[1], b[4]

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            eager = [t.clone() for t in iteration()]
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        captured = iteration()
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(captured[0], eager[0]) and torch.equal(captured[1], eager[1])
    for a, b in zip(captured[2:], eager[2:]):
        assert (a - b).double().norm() <= 1e-5 * b.double().norm() + 1e-12
    assert tr.device_status() == 0
