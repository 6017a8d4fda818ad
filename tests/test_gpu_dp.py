"""The data-parallel training step (bench.py's multi-GPU step), run as two gloo ranks that share
cuda:0 (their kernels never wait on each other): each rank traces its share of the views
(ptir_b200.dist.shard_weighted, by samples), runs the adjoint, and the ranks sum the material and
environment gradients with one all-reduce of a persistent flat buffer (GradientBucket). The sum
must equal the adjoint of one process over all the views: the views are traced as a batch
(trace_views), where each view's paths are seeded from the view alone, so the split changes only
the order of the float additions (relative L2 <= 1e-5).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

VIEWS = [(24, 16, 2, 3), (40, 32, 1, 5), (16, 16, 4, 3), (32, 24, 1, 7)]  # w, h, spp, frame


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _adjoint(view_ids):
    """Forward + adjoint of the given views as one batch on cuda:0; (material grad, env grad)."""
    from ptir_b200 import synthetic
    from tests.scenes import gpu_trace_bwd, make_tracer, small_scene, to_torch  # noqa: F401
    from tests.test_gpu_views import _scene_args, _tail

    s = small_scene(n=2000, w=8, h=8, spp=1, max_bounces=3)
    S = to_torch(s, "cuda")
    eyes = synthetic.camera_positions(len(VIEWS), seed=4)
    views, oris, dirs, grads = [], [], [], []
    for v in view_ids:
        w, h, spp, frame = VIEWS[v]
        o, d = synthetic.view_rays(w, h, spp, eyes[v])
        oris.append(o.reshape(-1, 3))
        dirs.append(d.reshape(-1, 3))
        views.append((frame, S["ray_to_world"], spp, h, w))
        g = np.random.default_rng(100 + v).standard_normal((spp * h * w, 3)).astype(np.float32)
        grads.append(torch.from_numpy(g))
    ori, drs = torch.cat(oris).cuda(), torch.cat(dirs).cuda()
    tr = make_tracer()
    tr.build_bvh(S["build_pos"], S["build_rot"], S["build_scl"], S["build_dns"], True, True)
    fwd = tr.trace_views(views, ori, drs, *_scene_args(S), *_tail(S))
    (rad, dns, hit, hit2, dist, nrm, snrm, mat, hits, vis, pbr, light, comps) = fwd
    z = torch.zeros_like
    g = torch.cat(grads).cuda()
    out = tr.trace_bwd_views(views, ori, drs, rad, dns, hit, hit2, dist, nrm, snrm, mat, pbr, light,
                             *_scene_args(S), z(rad), z(dns), z(hit), z(hit2), z(dist), z(nrm), z(snrm), z(mat), g,
                             z(light), *_tail(S))
    torch.cuda.synchronize()
    assert tr.device_status() == 0
    return out[1], out[4]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from ptir_b200 import dist as pdist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = pdist.shard_weighted([w * h * spp for w, h, spp, _ in VIEWS], rank, world)
        mg, eg = _adjoint(mine)
        bucket = pdist.GradientBucket()
        # gloo sums host tensors; NCCL (bench.py) sums the device tensors in place
        mg_h, eg_h = mg.cpu(), eg.cpu()
        bucket.allreduce([mg_h, eg_h])
        flat_before = bucket.flat.data_ptr()
        bucket.allreduce([mg.cpu(), eg.cpu()])  # a second step reuses the buffer
        out[rank] = (mine, mg_h, eg_h, flat_before == bucket.flat.data_ptr())
    finally:
        dist.destroy_process_group()


def test_data_parallel_adjoint_equals_single_process(cuda_device):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assigned = sorted(res[0][0] + res[1][0])
    assert assigned == list(range(len(VIEWS))) and res[0][0] and res[1][0]
    assert res[0][3] and res[1][3], "the all-reduce buffer is reused across steps"
    mg_all, eg_all = (t.cpu() for t in _adjoint(list(range(len(VIEWS)))))
    for r in (0, 1):
        for got, ref in ((res[r][1], mg_all), (res[r][2], eg_all)):
            a, b = got.double().reshape(-1), ref.double().reshape(-1)
            rel = float((a - b).norm() / b.norm().clamp_min(1e-30))
            assert rel <= 1e-5, rel
