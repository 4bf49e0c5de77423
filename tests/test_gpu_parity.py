"""GPU parity of the PatchMatch hot path against the CPU oracle (B200).

Tolerances: per-hypothesis bilateral NCC within 1e-4 absolute (fixed-hypothesis
mode); integer state (per-pixel draw counters, view masks) bit-exact after
initialisation; end-to-end depth maps within 0.5 % relative depth and 2 degrees
normal angle on >= 99 % of pixels where the oracle converged.
"""
from __future__ import annotations

import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora
from conftest import scene_cams, scene_grays

pytestmark = pytest.mark.gpu

COST_TOL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    c = hpm_b200.Context(0)
    yield c
    c.close()


def _load_views(ctx, scene):
    cams = scene_cams(scene)
    grays = scene_grays(scene)
    for i, (g, c) in enumerate(zip(grays, cams)):
        ctx.set_view(i, g, c)
    return cams, grays


def test_texture_filter_model(ctx):
    """tex2D linear filtering equals the oracle's 8-bit-weight model (HPM.cu:409)."""
    rng = np.random.default_rng(5)
    img = rng.uniform(0, 255, (29, 37)).astype(np.float32)
    cam = hpm_b200.Camera.make(np.eye(3), np.eye(3), np.zeros(3), 37, 29, 1, 2)
    ctx.set_view(200, img, cam)
    xy = np.stack([rng.uniform(-3, 40, 4000), rng.uniform(-3, 32, 4000)], 1).astype(np.float32)
    xy = np.concatenate([xy, np.array([[np.nan, 3.0], [3.0, np.nan], [np.inf, 2.0], [-np.inf, 2.0], [1e30, 1e30]],
                                      np.float32)])
    gpu = ctx.sample_view(200, xy)
    errs = {}
    for model in (0, 1):
        ora.set_texture_model(model)
        cpu = np.array([ora.tex2d(img, x, y) for x, y in xy], np.float32)
        errs[model] = float(np.abs(cpu - gpu).max())
    ora.set_texture_model(0)
    print("texture model max errors (B200 model, separable model):", errs)
    assert errs[0] < 5e-5, errs


def test_wrap_mode_behaves_as_clamp(ctx):
    """HPM.cpp:760-761 asks for wrap with unnormalised coordinates."""
    rng = np.random.default_rng(6)
    img = rng.uniform(0, 255, (16, 20)).astype(np.float32)
    cam = hpm_b200.Camera.make(np.eye(3), np.eye(3), np.zeros(3), 20, 16, 1, 2)
    xy = np.stack([rng.uniform(-30, 50, 2000), rng.uniform(-30, 46, 2000)], 1).astype(np.float32)
    ctx.set_address_mode(1)
    ctx.set_view(201, img, cam)
    wrap = ctx.sample_view(201, xy)
    ctx.set_address_mode(0)
    ctx.set_view(201, img, cam)
    clamp = ctx.sample_view(201, xy)
    diff = float(np.abs(wrap - clamp).max())
    print("wrap vs clamp max difference:", diff)
    assert diff == 0.0


def test_eval_costs_match_oracle(ctx, small_scene):
    cams, grays = _load_views(ctx, small_scene)
    v0 = small_scene.views[0]
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    rng = np.random.default_rng(9)
    H, W = v0.depth.shape
    n = 3000
    px = np.stack([rng.integers(0, W, n), rng.integers(0, H, n)], 1).astype(np.int32)
    # random planes facing the camera plus ground-truth planes
    nrm = rng.standard_normal((n, 3))
    nrm[:, 2] = -np.abs(nrm[:, 2]) - 0.5
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    depth = rng.uniform(cams[0].depth_min, cams[0].depth_max, n)
    Kinv = np.linalg.inv(v0.K.astype(np.float64))
    X = depth[:, None] * (np.concatenate([px, np.ones((n, 1))], 1) @ Kinv.T)
    w = -(nrm * X).sum(1)
    planes = np.concatenate([nrm, w[:, None]], 1).astype(np.float32)
    gt = v0.depth[px[:, 1], px[:, 0]] > 0
    for k in np.nonzero(gt)[0][: n // 2]:
        x, y = px[k]
        ncam = v0.R @ v0.normal[y, x]
        Xg = v0.depth[y, x] * (Kinv @ np.array([x, y, 1.0]))
        planes[k] = [ncam[0], ncam[1], ncam[2], -float(ncam @ Xg)]
    gpu = ctx.eval_costs(0, srcs, params, px, planes)
    cpu = ora.eval_costs([grays[0]] + [grays[j] for j in srcs], [cams[0]] + [cams[j] for j in srcs], params, px,
                         planes)
    d = np.abs(gpu - cpu)
    print("eval_costs |gpu-oracle|: max %.3g  p99.9 %.3g  frac>1e-4 %.4g  (%d costs, %.1f%% < 2)" % (
        d.max(), np.quantile(d, 0.999), (d > COST_TOL).mean(), d.size, 100 * (cpu < 2).mean()))
    assert (d <= COST_TOL).mean() >= 0.999, d.max()
    assert np.median(d) < 1e-5


def _oracle_state_after(scene, cams, grays, params, seed, n_half):
    import cv2
    srcs = [j for j, _ in scene.pairs[0]]
    W, H = cams[0].width, cams[0].height
    st = ora.RunState(W, H)
    st.canny[:] = cv2.Canny(scene.views[0].image, 50, 150)
    imgs = [grays[0]] + [grays[j] for j in srcs]
    cs = [cams[0]] + [cams[j] for j in srcs]
    ora.random_init(imgs, cs, params, st, seed, 0)
    for k in range(n_half):
        ora.half_sweep(imgs, None, cs, params, st, k & 1, k >> 1, seed, 0)
    return st


def test_random_init_matches_oracle(ctx, small_scene):
    import cv2
    cams, grays = _load_views(ctx, small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    ctx.set_canny(0, cv2.Canny(small_scene.views[0].image, 50, 150))
    g = ctx.run_partial(0, srcs, params, 0, seed=21)
    st = _oracle_state_after(small_scene, cams, grays, params, 21, 0)
    np.testing.assert_array_equal(g["rng_draw"], st.rng_draw)
    sel_eq = (g["selected_views"] == st.selected_views).mean()
    dp = np.abs(g["planes"] - st.planes).max()
    dc = np.abs(g["costs"] - st.costs)
    print("init: view-mask agreement %.6f  max plane diff %.3g  max cost diff %.3g" % (sel_eq, dp, dc.max()))
    assert sel_eq >= 0.999
    assert dp < 1e-4
    assert (dc <= COST_TOL).mean() >= 0.999


def test_first_half_sweep_matches_oracle(ctx, small_scene):
    import cv2
    cams, grays = _load_views(ctx, small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    ctx.set_canny(0, cv2.Canny(small_scene.views[0].image, 50, 150))
    g = ctx.run_partial(0, srcs, params, 1, seed=22)
    st = _oracle_state_after(small_scene, cams, grays, params, 22, 1)
    same_draws = (g["rng_draw"] == st.rng_draw).mean()
    same_sel = (g["selected_views"] == st.selected_views).mean()
    close = np.all(np.abs(g["planes"] - st.planes) <= 1e-4 * np.maximum(1, np.abs(st.planes)), axis=-1).mean()
    print("after one half-sweep: draws equal %.5f  masks equal %.5f  planes close %.5f" % (same_draws, same_sel, close))
    assert same_draws >= 0.99 and same_sel >= 0.99 and close >= 0.99


def depth_normal_agreement(d1, n1, d2, n2, valid):
    rel = np.abs(d1 - d2) / np.maximum(np.abs(d2), 1e-6)
    cosang = np.clip((n1 * n2).sum(-1), -1, 1)
    ang = np.degrees(np.arccos(cosang))
    ok = (rel < 0.005) & (ang < 2.0)
    return ok[valid].mean()


def test_photometric_run_matches_oracle(ctx, small_scene):
    import cv2
    cams, grays = _load_views(ctx, small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    canny = cv2.Canny(small_scene.views[0].image, 50, 150)
    ctx.set_canny(0, canny)
    ctx.run_patchmatch(0, srcs, params, texture_level=0, seed=33)
    depth = ctx.get_map(0, hpm_b200.MAP_DEPTH)
    normal = ctx.get_map(0, hpm_b200.MAP_NORMAL)
    tex = ctx.get_map(0, hpm_b200.MAP_TEXTURE0)
    st = ora.RunState(cams[0].width, cams[0].height)
    st.canny[:] = canny
    ora.run_patchmatch([grays[0]] + [grays[j] for j in srcs], None, [cams[0]] + [cams[j] for j in srcs], params, st,
                       33, 0)
    np.testing.assert_allclose(tex, st.texture, rtol=1e-6)
    gt = small_scene.views[0].depth
    ocd = st.planes[..., 3]
    converged = (gt > 0) & (np.abs(ocd - gt) / np.maximum(gt, 1e-6) < 0.01)
    agree = depth_normal_agreement(depth, normal, ocd, st.planes[..., :3], converged)
    agree_all = depth_normal_agreement(depth, normal, ocd, st.planes[..., :3], np.ones_like(gt, bool))
    gpu_gt = (np.abs(depth - gt) / np.maximum(gt, 1e-6) < 0.01)[gt > 0].mean()
    print("photometric run: agreement on oracle-converged px %.4f, on all px %.4f; gpu within 1%% of GT %.4f" % (
        agree, agree_all, gpu_gt))
    assert agree >= 0.99
