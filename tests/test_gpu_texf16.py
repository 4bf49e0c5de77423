"""Half-precision and 8-bit source textures (hpm_set_texture_format) on the B200.

HPM_TEX_U8 stores the grey levels exactly in one byte and reads them back as
grey / 255; the NCC is scale-free, so only its flat-source threshold is
rescaled.  Its per-hypothesis cost error against the FP64 exact-bilinear cost
matches the float-texel path's, and so does the reconstruction accuracy.

The grey levels of 8-bit images (integers 0..255) are stored exactly in half
precision, but the texture unit returns a filtered half texel rounded to half
precision: up to 1/16 of a grey level off the float-texel result.  Measured
here: the samples stay within 0.0625 of the float-texel ones; against the FP64
exact-bilinear cost (oracle/hpm_oracle_grad.c) the per-hypothesis cost error
stays within 1.5x that of float texels plus 2e-3 at the 99th percentile; a whole
reconstruction keeps its accuracy against the rendered ground truth within 2
points.
"""
from __future__ import annotations

import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora
from conftest import scene_cams, scene_grays

pytestmark = pytest.mark.gpu


def test_half_texels_within_a_sixteenth_of_a_level():
    rng = np.random.default_rng(21)
    img = rng.integers(0, 256, (61, 83)).astype(np.float32)
    cam = hpm_b200.Camera.make(np.eye(3), np.eye(3), np.zeros(3), 83, 61, 1, 2)
    xy = np.stack([rng.uniform(-3, 86, 20000), rng.uniform(-3, 64, 20000)], 1).astype(np.float32)
    out = {}
    with hpm_b200.Context(0) as ctx:
        for fmt in (hpm_b200.TEX_F32, hpm_b200.TEX_F16):
            ctx.set_texture_format(fmt)
            ctx.set_view(3, img, cam)
            out[fmt] = ctx.sample_view(3, xy)
    d = np.abs(out[hpm_b200.TEX_F32] - out[hpm_b200.TEX_F16])
    print(f"identical samples {np.mean(d == 0):.3f}, max |f16 - f32| {d.max():.4f}")
    assert d.max() <= 0.0625


def test_cost_error_against_fp64(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    v0 = small_scene.views[0]
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    rng = np.random.default_rng(22)
    ys, xs = np.nonzero(v0.depth > 0)
    pick = rng.choice(len(xs), 400, replace=False)
    px = np.stack([xs[pick], ys[pick]], 1).astype(np.int32)
    Kinv = np.linalg.inv(v0.K.astype(np.float64))
    planes, thetas = [], []
    for x, y in px:
        n = v0.R @ v0.normal[y, x]
        n = -n if n[2] > 0 else n
        d = v0.depth[y, x]
        X = d * (Kinv @ np.array([x, y, 1.0]))
        planes.append([n[0], n[1], n[2], -float(n @ X)])
        thetas.append([d, n[0], n[1]])
    planes = np.asarray(planes, np.float32)
    errs = {}
    with hpm_b200.Context(0) as ctx:
        for fmt in (hpm_b200.TEX_F32, hpm_b200.TEX_F16, hpm_b200.TEX_U8):
            ctx.set_texture_format(fmt)
            for i, (g, c) in enumerate(zip(grays, cams)):
                ctx.set_view(i, g, c)
            got = ctx.eval_costs(0, srcs, params, px, planes)
            e = []
            for k, (x, y) in enumerate(px):
                for j, s in enumerate(srcs):
                    c64, _ = ora.cost_grad64(grays[0], cams[0], grays[s], cams[s], params, int(x), int(y),
                                             np.asarray(thetas[k], np.float64), with_grad=False)
                    if 0 < c64 < 2 and 0 < got[k, j] < 2:
                        e.append(abs(got[k, j] - c64))
            errs[fmt] = np.asarray(e)
    p32, p16, p8 = (np.quantile(errs[f], 0.99) for f in (hpm_b200.TEX_F32, hpm_b200.TEX_F16, hpm_b200.TEX_U8))
    print(f"cost error vs FP64 exact bilinear, p99: f32 texels {p32:.2e}, f16 texels {p16:.2e}, u8 texels {p8:.2e}; "
          f"median: {np.median(errs[hpm_b200.TEX_F32]):.2e}, {np.median(errs[hpm_b200.TEX_F16]):.2e}, "
          f"{np.median(errs[hpm_b200.TEX_U8]):.2e}")
    assert p16 <= 1.5 * p32 + 2e-3
    assert p8 <= 1.5 * p32 + 2e-3


def test_reconstruction_accuracy_with_half_texels():
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=5, width=160, height=120, seed=1, n_src=4)
    cams = scene_cams(sc)
    srcs = [[j for j, _ in p] for p in sc.pairs]
    acc = {}
    for fmt in (hpm_b200.TEX_F32, hpm_b200.TEX_F16, hpm_b200.TEX_U8):
        with hpm_b200.Context(0) as ctx:
            ctx.set_texture_format(fmt)
            for i, v in enumerate(sc.views):
                ctx.set_image(i, v.image)
            ctx.reconstruct(cams, srcs, initial_image_scale=1, seed=5, fuse=False)
            a = []
            for i, v in enumerate(sc.views):
                d = ctx.get_map(i, hpm_b200.MAP_DEPTH)  # after the prior passes
                ok = v.depth > 0
                a.append(float((np.abs(d - v.depth)[ok] / v.depth[ok] < 0.01).mean()))
            acc[fmt] = np.mean(a)
    print(f"pixels within 1 % of the true depth: f32 texels {acc[hpm_b200.TEX_F32]:.3f}, "
          f"f16 texels {acc[hpm_b200.TEX_F16]:.3f}, u8 texels {acc[hpm_b200.TEX_U8]:.3f}")
    assert acc[hpm_b200.TEX_F16] >= acc[hpm_b200.TEX_F32] - 0.02
    assert acc[hpm_b200.TEX_U8] >= acc[hpm_b200.TEX_F32] - 0.02
