"""GPU parity of the stages around PatchMatch: joint bilateral upsampling,
the consistency check (ConfidenceEvaluation) and fusion, against the oracle's
restatement of the reference's sequential loops.  Integer results (accepted
pixels, point order and count) must be identical; float results bit-identical
up to the rare double-rounding case noted in include/hpm_fp.h."""
from __future__ import annotations

import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora
from conftest import scene_cams, scene_grays

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = hpm_b200.Context(0)
    yield c
    c.close()


def noisy_maps(scene, seed=0, noise=0.004, ang=0.03):
    """Ground-truth depth/normal maps with multiplicative depth noise and normal jitter."""
    rng = np.random.default_rng(seed)
    depths, normals = [], []
    for v in scene.views:
        d = v.depth * (1.0 + noise * rng.standard_normal(v.depth.shape))
        d = np.where(v.depth > 0, d, 0.0).astype(np.float32)
        n = v.normal + ang * rng.standard_normal(v.normal.shape)
        n /= np.maximum(np.linalg.norm(n, axis=-1, keepdims=True), 1e-9)
        n = np.where(v.depth[..., None] > 0, n, np.array([0, 0, 1.0])).astype(np.float32)
        depths.append(d)
        normals.append(n)
    return depths, normals


def load(ctx, scene, depths, normals, kind):
    cams = scene_cams(scene)
    for i, (g, c) in enumerate(zip(scene_grays(scene), cams)):
        ctx.set_view(i, g, c)
        ctx.set_map(i, kind, depths[i])
        ctx.set_map(i, hpm_b200.MAP_NORMAL, normals[i])
        ctx.set_color(i, scene.views[i].image)
    return cams


@pytest.mark.parametrize("seed", [0, 1])
def test_confidence_matches_oracle(ctx, small_scene, seed):
    depths, normals = noisy_maps(small_scene, seed)
    cams = load(ctx, small_scene, depths, normals, hpm_b200.MAP_DEPTH)
    srcs = [[j for j, _ in p] for p in small_scene.pairs]
    iters = ctx.confidence_eval(srcs, hpm_b200.MAP_DEPTH)
    gpu = [ctx.get_map(i, hpm_b200.MAP_CONF) for i in range(len(srcs))]
    ref = ora.confidence_eval(cams, depths, normals, srcs)
    for i in range(len(srcs)):
        nz = ref[i] > 0
        print(f"view {i}: consistent px {nz.mean():.3f}, equal {np.mean(gpu[i] == ref[i]):.6f}, iterations {iters}")
        np.testing.assert_array_equal(gpu[i] > 0, ref[i] > 0)
        np.testing.assert_array_equal(gpu[i], ref[i])


def test_fusion_matches_oracle(ctx, small_scene):
    depths, normals = noisy_maps(small_scene, 5)
    cams = load(ctx, small_scene, depths, normals, hpm_b200.MAP_DEPTH_GEOM)
    srcs = [[j for j, _ in p] for p in small_scene.pairs]
    pts, n = ctx.fuse(srcs, hpm_b200.MAP_DEPTH_GEOM)
    ref, n_ref = ora.fusion(cams, depths, normals, [v.image for v in small_scene.views], srcs)
    print(f"fusion: gpu {n} points, oracle {n_ref}")
    if n != n_ref:
        for k in range(1, len(srcs) + 1):
            _, nk = ora.fusion(cams[:k], depths[:k], normals[:k], [v.image for v in small_scene.views][:k],
                               [[j for j in s if j < k] for s in srcs[:k]])
            print(f"  oracle with {k} views: {nk}")
        print("  gpu first points", pts[:3], "\n  oracle first points", ref[:3])
    assert n == n_ref
    np.testing.assert_array_equal(pts, ref)


def test_fusion_sky_variant(ctx, small_scene):
    depths, normals = noisy_maps(small_scene, 6)
    cams = load(ctx, small_scene, depths, normals, hpm_b200.MAP_DEPTH_GEOM)
    srcs = [[j for j, _ in p] for p in small_scene.pairs]
    rng = np.random.default_rng(3)
    sky = []
    for v in small_scene.views:
        m = np.zeros_like(v.image)
        m[: v.image.shape[0] // 3] = (234, 235, 55)
        m[rng.random(m.shape[:2]) < 0.1] = (234, 0, 0)
        sky.append(m)
    pts, n = ctx.fuse(srcs, hpm_b200.MAP_DEPTH_GEOM, sky_masks=sky)
    ref, n_ref = ora.fusion(cams, depths, normals, [v.image for v in small_scene.views], srcs, sky_masks=sky)
    assert n == n_ref
    np.testing.assert_array_equal(pts, ref)


def test_jbu_matches_oracle(ctx, small_scene):
    cams = scene_cams(small_scene)
    g = scene_grays(small_scene)[0]
    ctx.set_view(0, g, cams[0])
    v = small_scene.views[0]
    coarse_d = v.depth[::2, ::2].copy()
    coarse_n = v.normal[::2, ::2].copy()
    coarse_d[5, 7] = np.nan
    out = ctx.jbu_maps(0, coarse_d)
    ref = ora.jbu(g, coarse_d)
    np.testing.assert_array_equal(out, ref)
    od, on = ctx.jbu_maps(0, coarse_d, coarse_n)
    rd, rn = ora.jbu_prior(g, coarse_d, coarse_n)
    np.testing.assert_array_equal(od, rd)
    np.testing.assert_array_equal(on, rn)
