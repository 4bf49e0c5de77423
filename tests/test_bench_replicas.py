"""bench.py's multi-GPU plumbing on CPU: N replicas over a world-size-2 gloo
process group; the job's time is the maximum over ranks and the throughput
counts every rank's views (weak scaling)."""
from __future__ import annotations

import importlib.util
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench = _bench()
        mine = [100.0 + 50 * rank, 200.0 - 30 * rank]   # per-rank device and e2e milliseconds
        out[rank] = bench.max_over_ranks(mine, world, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_with_gloo():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        results = dict(out)
    assert results[0] == results[1] == [150.0, 200.0]


def test_single_rank_is_identity():
    assert _bench().max_over_ranks([3.0, 4.0], 1, "cpu") == [3.0, 4.0]


def test_level_sizes_follow_the_reference_pyramid():
    bench = _bench()
    assert bench.level_sizes(1600, 1200, 1) == [(800, 600), (1600, 1200)]
    assert bench.level_sizes(1280, 960, 4) == [(320, 240)]
    assert bench.level_sizes(3072, 2048, 1) == [(768, 512), (1536, 1024), (3072, 2048)]
    # one 800x600 and one 1600x1200 level: photometric + 1 prior + 3 geometric runs, then
    # hierarchy + 2 prior + 3 geometric runs
    assert bench.view_pixel_runs(1600, 1200, 1) == 800 * 600 * 5 + 1600 * 1200 * 6


def test_depth_accuracy_at_scaled_working_sizes():
    """The accuracy the bench reports: maps at the truth's size are compared pixel by pixel; maps
    smaller by an integer factor f (--initial-image-scale f) against truth pixel (f*x, f*y), the
    pixel whose ray the scaled camera's pixel x looks along; other sizes give None."""
    import numpy as np

    bench = _bench()

    class View:
        pass

    class Scene:
        pass

    v = View()
    yy, xx = np.mgrid[0:96, 0:128].astype(np.float32)
    v.depth = 10.0 + 0.05 * xx + 0.02 * yy
    v.depth[:8] = 0.0  # no truth there
    sc = Scene()
    sc.views = [v]
    assert bench.depth_accuracy([v.depth.copy()], sc) == 1.0
    quarter = v.depth[::4, ::4].copy()
    assert bench.depth_accuracy([quarter], sc) == 1.0
    assert bench.depth_accuracy([quarter * 1.02], sc) == 0.0  # every depth 2 % off
    assert bench.depth_accuracy([np.zeros((50, 60), np.float32)], sc) is None
