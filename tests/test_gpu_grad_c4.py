"""Differentiation form at its workload size: 20 views of 1024x768, 10 sources.

- The adjoint of the bilateral NCC (hpm_eval_cost_grad, FP32 on the B200) at
  10,000 random pixels of view 0 under seeded, sub-pixel-jittered ground-truth
  planes (depth x (1 + 0.3 %), normal tilted by about 1 degree), against FP64
  central finite differences (h = 1e-4 on depth, nx and ny) of the FP64 cost
  and against the FP64 analytic gradient (oracle/hpm_oracle_grad.c).
- Gauss-Newton refinement (hpm_gn_refine, 3 steps) beside the random-
  perturbation refinement of PlaneHypothesisRefinement (HPM.cu:765-841): from
  the state after k PatchMatch iterations, one more iteration of propagation and
  random refinement against 3 Gauss-Newton steps, on depth error and device
  time.
"""
from __future__ import annotations

import cv2
import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora

pytestmark = pytest.mark.gpu

N_PIX = 10_000
H_FD = 1e-4


@pytest.fixture(scope="module")
def c4():
    from hpm_b200 import synth

    scene = synth.make_config("c4", seed=404, device="cuda:0")
    cams = [hpm_b200.Camera.make(v.K, v.R, v.t, v.image.shape[1], v.image.shape[0], v.depth_min, v.depth_max)
            for v in scene.views]
    grays = [synth.gray_float(v.image) for v in scene.views]
    ctx = hpm_b200.Context(0)
    for i, (g, c) in enumerate(zip(grays, cams)):
        ctx.set_view(i, g, c)
    ctx.set_canny(0, cv2.Canny(scene.views[0].image, 50, 150))
    yield scene, cams, grays, ctx
    ctx.close()


def _jittered_planes(v, xs, ys, rng):
    th = np.zeros((len(xs), 3))
    for k, (x, y) in enumerate(zip(xs, ys)):
        n = v.R.astype(np.float64) @ v.normal[y, x].astype(np.float64)
        if n[2] > 0:
            n = -n
        n = n + rng.normal(0, 0.012, 3)
        n /= np.linalg.norm(n)
        if n[2] > 0:
            n = -n
        th[k] = [v.depth[y, x] * (1 + rng.normal(0, 0.003)), n[0], n[1]]
    return th


def test_adjoint_against_fp64_central_differences_10k_pixels(c4):
    scene, cams, grays, ctx = c4
    v0 = scene.views[0]
    srcs = [j for j, _ in scene.pairs[0]]
    assert len(srcs) == 10
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    rng = np.random.default_rng(404)
    H, W = v0.depth.shape
    inner = np.zeros((H, W), bool)
    inner[8:H - 8, 8:W - 8] = True
    ys, xs = np.nonzero((v0.depth > 0) & inner)
    pick = rng.choice(len(xs), N_PIX, replace=False)
    xs, ys = xs[pick], ys[pick]
    th = _jittered_planes(v0, xs, ys, rng).astype(np.float32)
    px = np.stack([xs, ys], 1).astype(np.int32)
    cost, grad = ctx.eval_cost_grad(0, srcs, params, px, th)
    fd_ok = fd_total = gpu_ok = gpu_total = 0
    cerr, fd_rel, gpu_rel = [], [], []
    for k in range(N_PIX):
        t64 = th[k].astype(np.float64)
        for j, s in enumerate(srcs):
            c64, g64 = ora.cost_grad64(grays[0], cams[0], grays[s], cams[s], params, int(xs[k]), int(ys[k]), t64)
            cerr.append(abs(c64 - cost[k, j]))
            if not (0.0 < c64 < 2.0):
                continue
            for a in range(3):
                e = np.zeros(3)
                e[a] = H_FD
                cp, _ = ora.cost_grad64(grays[0], cams[0], grays[s], cams[s], params, int(xs[k]), int(ys[k]),
                                        t64 + e, with_grad=False)
                cm, _ = ora.cost_grad64(grays[0], cams[0], grays[s], cams[s], params, int(xs[k]), int(ys[k]),
                                        t64 - e, with_grad=False)
                if not (0.0 < cp < 2.0 and 0.0 < cm < 2.0):
                    continue
                fd = (cp - cm) / (2 * H_FD)
                fd_total += 1
                fd_ok += abs(fd - g64[a]) <= 1e-2 * abs(g64[a]) + 1e-3
                fd_rel.append(abs(fd - g64[a]) / (abs(g64[a]) + 1e-3))
                gpu_total += 1
                gpu_ok += abs(grad[k, j, a] - g64[a]) <= 2e-3 * abs(g64[a]) + 2e-4
                gpu_rel.append(abs(grad[k, j, a] - g64[a]) / (abs(g64[a]) + 1e-3))
    cerr = np.asarray(cerr)
    print(f"C4 adjoint, {N_PIX} pixels x {len(srcs)} sources: cost |fp32 - fp64| p99 {np.quantile(cerr, 0.99):.3g}; "
          f"FP64 gradient vs central differences {fd_ok}/{fd_total}; CUDA adjoint vs FP64 gradient "
          f"{gpu_ok}/{gpu_total}")
    fd_rel, gpu_rel = np.asarray(fd_rel), np.asarray(gpu_rel)
    print("relative error quantiles (50/75/90/99 %): FD vs FP64 analytic "
          f"{np.round(np.quantile(fd_rel, [0.5, 0.75, 0.9, 0.99]), 5)}, CUDA vs FP64 analytic "
          f"{np.round(np.quantile(gpu_rel, [0.5, 0.75, 0.9, 0.99]), 5)}")
    assert np.quantile(cerr, 0.99) < 2e-4
    # the exactly bilinear cost has kinks at texel boundaries: a central difference that straddles one differs
    # from the one-sided analytic derivative, so the FD check holds for the bulk, not for every triple
    assert fd_total > 100_000 and np.median(fd_rel) < 2e-3
    assert gpu_ok >= 0.95 * gpu_total and np.median(gpu_rel) < 1e-3


def test_gauss_newton_beside_random_refinement(c4):
    import torch

    scene, cams, grays, ctx = c4
    v0 = scene.views[0]
    srcs = [j for j, _ in scene.pairs[0]]
    valid = v0.depth > 0
    stream = torch.cuda.ExternalStream(ctx.stream_handle())

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    def err(d):
        return np.abs(d - v0.depth)[valid] / v0.depth[valid]

    # first launches of each kernel (module load, shared-memory configuration) are not timed
    pw = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    pw.max_iterations = 1
    ctx.run_patchmatch(0, srcs, pw, seed=77)
    ctx.set_map(0, hpm_b200.MAP_DEPTH_GEOM, ctx.get_map(0, hpm_b200.MAP_DEPTH))
    ctx.gn_refine(0, srcs, pw, hpm_b200.MAP_DEPTH_GEOM, steps=1)
    rows = []
    for iters in (1, 2):
        p = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
        p.max_iterations = iters
        ms_pm = timed(lambda: ctx.run_patchmatch(0, srcs, p, seed=77))
        d0 = ctx.get_map(0, hpm_b200.MAP_DEPTH).copy()
        n0 = ctx.get_map(0, hpm_b200.MAP_NORMAL).copy()
        # one more iteration of propagation + random refinement, from scratch to iters + 1 (same seed)
        p1 = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
        p1.max_iterations = iters + 1
        ms_pm1 = timed(lambda: ctx.run_patchmatch(0, srcs, p1, seed=77))
        d1 = ctx.get_map(0, hpm_b200.MAP_DEPTH).copy()
        # three Gauss-Newton steps from the iters-iteration state
        ctx.set_map(0, hpm_b200.MAP_DEPTH_GEOM, d0)
        ctx.set_map(0, hpm_b200.MAP_NORMAL, n0)
        ms_gn = timed(lambda: ctx.gn_refine(0, srcs, p, hpm_b200.MAP_DEPTH_GEOM, steps=3))
        dg = ctx.get_map(0, hpm_b200.MAP_DEPTH_GEOM).copy()
        e0, e1, eg = err(d0), err(d1), err(dg)
        near = e0 < 0.02  # pixels already on the surface: where a local method can help
        rows.append((iters, ms_pm, ms_pm1 - ms_pm, ms_gn, np.median(e0[near]), np.median(e1[near]),
                     np.median(eg[near]), (e0 < 0.005).mean(), (e1 < 0.005).mean(), (eg < 0.005).mean()))
    print("\n| PatchMatch iterations | run ms | + 1 iteration (random refinement) ms | + 3 GN steps ms | "
          "median error (on-surface pixels): after k / k+1 / GN | within 0.5 %: after k / k+1 / GN |")
    for r in rows:
        print(f"| {r[0]} | {r[1]:.1f} | {r[2]:.1f} | {r[3]:.1f} | {r[4]:.4f} / {r[5]:.4f} / {r[6]:.4f} | "
              f"{r[7]:.3f} / {r[8]:.3f} / {r[9]:.3f} |")
    for r in rows:
        assert r[6] < r[4]  # Gauss-Newton lowers the error of pixels on the surface
