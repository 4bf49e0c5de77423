"""hpm_eval_costs_noalloc: the fixed-hypothesis cost evaluation for callers that
cannot have the library allocate device memory while they run (cudaMalloc and
cudaFree can synchronise the whole device and can fail when another allocator
owns the process's device memory).  Its staging is one fixed 4 MiB array per
GPU.

Checked through the C ABI against hpm_eval_costs on the same inputs, on two
calls in a row (the second reuses the array the first one left behind), with
the tolerance of the other cost tests (1e-4 absolute); at the exact capacity
of the array and one hypothesis past it; and for the property the entry point
exists for: a warm call leaves the device's free memory unchanged.  The file
sorts last so that a run stopping at the first failure has run every other test
before it.
"""
from __future__ import annotations

import numpy as np
import pytest

import hpm_b200
from conftest import scene_cams, scene_grays

pytestmark = pytest.mark.gpu

COST_TOL = 1e-4


def _hypotheses(scene, cams, n, seed):
    v0 = scene.views[0]
    H, W = v0.depth.shape
    rng = np.random.default_rng(seed)
    px = np.stack([rng.integers(0, W, n), rng.integers(0, H, n)], 1).astype(np.int32)
    nrm = rng.standard_normal((n, 3))
    nrm[:, 2] = -np.abs(nrm[:, 2]) - 0.5
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    depth = rng.uniform(cams[0].depth_min, cams[0].depth_max, n)
    Kinv = np.linalg.inv(v0.K.astype(np.float64))
    X = depth[:, None] * (np.concatenate([px, np.ones((n, 1))], 1) @ Kinv.T)
    w = -(nrm * X).sum(1)
    return px, np.concatenate([nrm, w[:, None]], 1).astype(np.float32)


def test_noalloc_costs_match_allocating_entry_point(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    with hpm_b200.Context(0) as ctx:
        for i, (g, c) in enumerate(zip(grays, cams)):
            ctx.set_view(i, g, c)
        # two calls in a row with different sizes: the second must not see the first one's leftovers
        for n, seed in ((3000, 21), (1200, 22)):
            px, planes = _hypotheses(small_scene, cams, n, seed)
            ref = ctx.eval_costs(0, srcs, params, px, planes)
            got = ctx.eval_costs_noalloc(0, srcs, params, px, planes)
            d = np.abs(got - ref)
            print(f"n={n}: max |noalloc - eval_costs| = {d.max():.3g}")
            assert got.shape == ref.shape
            assert (d <= COST_TOL).all(), d.max()


def test_noalloc_rejects_oversize_requests(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    with hpm_b200.Context(0) as ctx:
        for i, (g, c) in enumerate(zip(grays, cams)):
            ctx.set_view(i, g, c)
        n = (4 << 20) // (24 + 4 * len(srcs)) + 1000  # past the fixed staging size
        px = np.zeros((n, 2), np.int32)
        planes = np.tile(np.array([[0, 0, -1, 1]], np.float32), (n, 1))
        with pytest.raises(hpm_b200.HPMError, match="staging"):
            ctx.eval_costs_noalloc(0, srcs, params, px, planes)


def _scene10():
    """11 small views, 10 sources for view 0: the source count the capacity is quoted for."""
    from hpm_b200 import synth

    return synth.make_scene(n_views=11, width=64, height=48, layout="hemisphere", n_src=10, seed=31)


def test_noalloc_exact_capacity_and_one_past_it():
    scene = _scene10()
    cams = scene_cams(scene)
    grays = scene_grays(scene)
    srcs = [j for j, _ in scene.pairs[0]]
    assert len(srcs) == 10
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    with hpm_b200.Context(0) as ctx:
        for i, (g, c) in enumerate(zip(grays, cams)):
            ctx.set_view(i, g, c)
        # 65,536 x (16 + 8 + 4 * 10) bytes = 4 MiB exactly, every part a multiple of 256
        n = 65536
        px, planes = _hypotheses(scene, cams, n, 41)
        ref = ctx.eval_costs(0, srcs, params, px, planes)
        got = ctx.eval_costs_noalloc(0, srcs, params, px, planes)
        assert (np.abs(got - ref) <= COST_TOL).all()
        px1, planes1 = _hypotheses(scene, cams, n + 1, 42)
        with pytest.raises(hpm_b200.HPMError, match="staging"):
            ctx.eval_costs_noalloc(0, srcs, params, px1, planes1)
        # the rejected call left the context usable
        again = ctx.eval_costs_noalloc(0, srcs, params, px[:100], planes[:100])
        assert (np.abs(again - ref[:100]) <= COST_TOL).all()


def test_warm_noalloc_call_leaves_free_device_memory_unchanged():
    import torch

    scene = _scene10()
    cams = scene_cams(scene)
    grays = scene_grays(scene)
    srcs = [j for j, _ in scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    with hpm_b200.Context(0) as ctx:
        for i, (g, c) in enumerate(zip(grays, cams)):
            ctx.set_view(i, g, c)
        # first call: loads the kernel and looks the array's address up; then a larger call, warm
        px, planes = _hypotheses(scene, cams, 40000, 43)
        ctx.eval_costs_noalloc(0, srcs, params, px[:500], planes[:500])
        ctx.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        got = ctx.eval_costs_noalloc(0, srcs, params, px, planes)
        ctx.synchronize()
        free1 = torch.cuda.mem_get_info(0)[0]
        print(f"free device memory around a warm call: {free0} -> {free1} bytes")
        assert free1 == free0
        assert got.shape == (40000, 10)
