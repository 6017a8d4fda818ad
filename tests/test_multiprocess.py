"""Multi-process (gloo, world size 2, CPU) coverage of the data-parallel path."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from ptir_b200 import dist as pdist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        views = list(pdist.shard(8, rank, world))
        mat = torch.full((5, 5), float(rank + 1))
        env = torch.arange(12, dtype=torch.float32).reshape(1, 3, 4) * (rank + 1)
        pdist.allreduce_gradients([mat, env])
        out[rank] = (views, mat.clone(), env.clone())
    finally:
        dist.destroy_process_group()


def test_shard_partitions_views():
    for count in (0, 1, 7, 8, 17):
        for world in (1, 2, 3, 8):
            got = [list(pdist.shard(count, r, world)) for r in range(world)]
            flat = [v for g in got for v in g]
            assert flat == list(range(count))
            assert max(map(len, got)) - min(map(len, got)) <= 1
    with pytest.raises(ValueError):
        pdist.shard(4, 2, 2)


def test_gradient_allreduce_gloo_world2():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0][0] == [0, 1, 2, 3] and res[1][0] == [4, 5, 6, 7]
    for r in (0, 1):
        assert torch.equal(res[r][1], torch.full((5, 5), 3.0))
        assert torch.equal(res[r][2], torch.arange(12, dtype=torch.float32).reshape(1, 3, 4) * 3)


def test_weighted_shards_balance_segments():
    from ptir_b200.dist import shard_weighted

    w = [256 * 256, 800 * 800 * 16, 400 * 400 * 2, 512 * 512 * 4, 800 * 800, 256 * 256 * 16, 512 * 512, 400 * 400]
    for world in (1, 2, 3, 4, 8):
        got = [shard_weighted(w, r, world) for r in range(world)]
        assert sorted(i for g in got for i in g) == list(range(len(w)))
        loads = [sum(w[i] for i in g) for g in got]
        # largest-first greedy: within 4/3 of the best (>= max(total / world, largest item))
        assert max(loads) <= 4.0 / 3.0 * max(sum(w) / world, max(w)) + 1e-9
    assert shard_weighted([1.0] * 8, 0, 2) == [0, 2, 4, 6]
    with pytest.raises(ValueError):
        shard_weighted([1.0, -1.0], 0, 2)
