"""The multi-process path of bench.py on CPU (gloo, world size 2): ranks
render different cameras of the same scene (weak scaling, no data-path
collective), and the reported time is the maximum over ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path[:0] = [ROOT, os.path.join(ROOT, "del-splat_b200")]
    import bench
    from dsplat import scenes
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 + rank, world, torch.device("cpu"))
        bench.barrier(world)
        base = scenes.config3(seed=3, n=256, views=4)
        cams = bench.rank_cameras(base, rank, 4)
        out[rank] = (t, np.stack([c.mvp for c in cams]), base.means.copy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_views_and_time_by_the_slowest_rank():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (t0, mvp0, means0), (t1, mvp1, means1) = res[0], res[1]
    assert t0 == t1 == 11.0  # max over ranks, identical on every rank
    assert np.array_equal(means0, means1)  # the same scene
    assert mvp0.shape == mvp1.shape == (4, 16)
    assert not np.allclose(mvp0, mvp1)  # each rank its own cameras
