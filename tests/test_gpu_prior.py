"""GPU planar prior against the oracle: support points (exact list and
order), raster + double-precision plane fits + prior mask (exact), and the
distance-1 path (downsampling, prior JBU, reload; exact)."""
from __future__ import annotations

import cv2
import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora
from conftest import scene_cams, scene_grays
from test_delaunay import cv2_triangles

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = hpm_b200.Context(0)
    yield c
    c.close()


def prior_inputs(scene, seed=0):
    rng = np.random.default_rng(seed)
    v = scene.views[0]
    depth = np.where(v.depth > 0, v.depth * (1 + 0.002 * rng.standard_normal(v.depth.shape)), 0).astype(np.float32)
    cost = np.where(v.depth > 0, rng.uniform(0.0, 0.4, v.depth.shape), 2.0).astype(np.float32)
    conf = np.where(rng.random(v.depth.shape) < 0.5, rng.uniform(0.0, 1.5, v.depth.shape), 0.0).astype(np.float32)
    return depth, cost, conf


def load(ctx, scene, depth, cost, conf):
    cams = scene_cams(scene)
    g = scene_grays(scene)[0]
    ctx.set_view(0, g, cams[0])
    ctx.set_map(0, hpm_b200.MAP_DEPTH, depth)
    ctx.set_map(0, hpm_b200.MAP_COST, cost)
    ctx.set_map(0, hpm_b200.MAP_CONF, conf)
    return cams[0], g


def test_support_points_match_oracle(ctx, small_scene):
    depth, cost, conf = prior_inputs(small_scene)
    cam, _ = load(ctx, small_scene, depth, cost, conf)
    pts, (w, h) = ctx.support_points(0, 0)
    ref = ora.support_points(cost, conf, cam.width, cam.height)
    print(f"support points: {len(pts)}")
    np.testing.assert_array_equal(pts, ref)
    pts1, (w1, h1) = ctx.support_points(0, 1)
    hw, hh = int(round(cam.width * 0.5)), int(round(cam.height * 0.5))
    assert (w1, h1) == (hw, hh)
    ref1 = ora.support_points(ora.resize_linear(cost, hw, hh), ora.resize_linear(conf, hw, hh), int(cam.width * 0.5),
                              int(cam.height * 0.5))
    np.testing.assert_array_equal(pts1, ref1)


def test_prior_distance0_matches_oracle(ctx, small_scene):
    depth, cost, conf = prior_inputs(small_scene, 1)
    cam, _ = load(ctx, small_scene, depth, cost, conf)
    pts = ora.support_points(cost, conf, cam.width, cam.height)
    tris = np.asarray([sum(t, ()) for t in cv2_triangles(pts, cam.width, cam.height)], np.int32).reshape(-1, 6)
    ctx.prior_from_triangles(0, 0, tris)
    planes, mask = ctx.get_prior(0)
    dmin, dmax = hpm_b200.widened_range(cam)
    label, fits, pdepth, _ = ora.planar_prior(tris, depth, cam, 1.0, dmin, dmax, 0)
    ref_mask = (label > 0).astype(np.uint8)
    ref_planes = np.zeros_like(planes)
    lab = label.astype(np.int64)
    ref_planes[lab > 0] = fits[lab[lab > 0] - 1]
    print(f"prior d0: {len(tris)} triangles, masked px {ref_mask.mean():.3f}")
    np.testing.assert_array_equal(mask, ref_mask)
    np.testing.assert_array_equal(planes, ref_planes)


def test_prior_distance1_matches_oracle(ctx, small_scene):
    depth, cost, conf = prior_inputs(small_scene, 2)
    cam, gray = load(ctx, small_scene, depth, cost, conf)
    hw, hh = int(round(cam.width * 0.5)), int(round(cam.height * 0.5))
    dd = ora.resize_linear(depth, hw, hh)
    pts = ora.support_points(ora.resize_linear(cost, hw, hh), ora.resize_linear(conf, hw, hh), int(cam.width * 0.5),
                             int(cam.height * 0.5))
    tris = np.asarray([sum(t, ()) for t in cv2_triangles(pts, hw, hh)], np.int32).reshape(-1, 6)
    ctx.prior_from_triangles(0, 1, tris)
    planes, mask = ctx.get_prior(0)
    dmin, dmax = hpm_b200.widened_range(cam)
    _, _, pdepth, pnormal = ora.planar_prior(tris, dd, cam, 0.5, dmin, dmax, 1)
    ud, un = ora.jbu_prior(gray, pdepth, pnormal)
    ref_planes, ref_mask = ora.prior_reload(ud, un, cam, dmin, dmax)
    print(f"prior d1: {len(tris)} triangles, masked px {ref_mask.mean():.3f}")
    np.testing.assert_array_equal(mask, ref_mask)
    np.testing.assert_array_equal(planes, ref_planes)


def test_build_prior_runs(ctx, small_scene):
    depth, cost, conf = prior_inputs(small_scene, 3)
    load(ctx, small_scene, depth, cost, conf)
    n_p, n_t = ctx.build_prior(0, 0)
    _, mask = ctx.get_prior(0)
    assert n_p > 50 and n_t > 50 and mask.mean() > 0.2
