"""Whole-schedule parity on the B200: pyramid images and hpm_reconstruct.

Level images (cv::resize INTER_LINEAR 8UC3, cvtColor BGR2GRAY, Canny(50,150);
main.cpp:107-161, HPM.cpp:658-662, main.cpp:287) are compared with cv2, the
library the reference calls: bit-exact for integer factors, the pyramid's case.

hpm_reconstruct (main.cpp:1143-1364) is compared with the oracle pipeline
driven with the same triangulator as the product (hpm_delaunay); with that
one input shared, every map of every view must agree bit for bit.  The same
pipeline with cv2.Subdiv2D triangles differs only where Subdiv2D orders or
splits cocircular support points differently.
"""
from __future__ import annotations

import cv2
import numpy as np
import pytest

import hpm_b200
from conftest import scene_cams

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = hpm_b200.Context(0)
    yield c
    c.close()


def _color(h, w, seed):
    rng = np.random.default_rng(seed)
    base = cv2.GaussianBlur(rng.integers(0, 256, (h, w, 3)).astype(np.uint8), (5, 5), 1.5)
    return np.ascontiguousarray(base)


@pytest.mark.parametrize("size,target", [((160, 120), (80, 60)), ((333, 250), (333, 250)), ((400, 300), (100, 75))])
def test_level_image_matches_cv2(ctx, size, target):
    w0, h0 = size
    w, h = target
    img = _color(h0, w0, w0)
    ctx.set_image(7, img)
    cam = hpm_b200.Camera.make(np.diag([w, w, 1.0]), np.eye(3), np.zeros(3), w, h, 1, 5)
    ctx.prepare_level(7, w, h, cam)
    bgr, gray, edges = ctx.get_level(7)
    ref = img if (w, h) == (w0, h0) else cv2.resize(img, (w, h), interpolation=cv2.INTER_LINEAR)
    assert np.array_equal(bgr, ref)
    assert np.array_equal(gray, cv2.cvtColor(ref, cv2.COLOR_BGR2GRAY).astype(np.float32))
    assert np.array_equal(edges, cv2.Canny(ref, 50, 150))


def test_canny_hysteresis_follows_a_long_weak_chain(ctx):
    """A weak edge (Sobel L1 magnitude 80, between the thresholds 50 and 150) that winds across the
    whole image as a serpentine, joined to strong edges only at its start: hysteresis must carry
    the strong label along all of it, through hundreds of tile crossings, as cv2.Canny's flood
    fill does."""
    w, h = 1024, 768
    img = np.full((h, w, 3), 100, np.uint8)
    rows = list(range(20, h - 20, 38))
    for k, y in enumerate(rows):
        cv2.rectangle(img, (20, y), (w - 21, y + 4), (120, 120, 120), -1)
        if k + 1 < len(rows):
            x = w - 25 if k % 2 == 0 else 20
            cv2.rectangle(img, (x, y), (x + 4, rows[k + 1] + 4), (120, 120, 120), -1)
    cv2.rectangle(img, (14, 14), (30, 30), (230, 230, 230), -1)  # the strong start
    ctx.set_image(7, img)
    cam = hpm_b200.Camera.make(np.diag([w, w, 1.0]), np.eye(3), np.zeros(3), w, h, 1, 5)
    ctx.prepare_level(7, w, h, cam)
    _, _, edges = ctx.get_level(7)
    ref = cv2.Canny(img, 50, 150)
    assert (ref > 0).sum() > 20000  # the chain is kept, not only the start
    assert np.array_equal(edges, ref)


def _scene(w, h, seed=1):
    from hpm_b200 import synth
    return synth.make_scene(n_views=5, width=w, height=h, seed=seed, n_src=4)


@pytest.mark.parametrize("level_max_side", [0, 100])
def test_reconstruct_matches_oracle_pipeline(ctx, level_max_side):
    import pipeline as op

    sc = _scene(160, 120)
    cams = scene_cams(sc)
    srcs = [[j for j, _ in p] for p in sc.pairs]
    for i, v in enumerate(sc.views):
        ctx.set_image(i, v.image)
    n_pts = ctx.reconstruct(cams, srcs, initial_image_scale=1, seed=11, fuse=True, level_max_side=level_max_side)
    P = op.OraclePipeline([v.image for v in sc.views], cams, srcs, initial_image_scale=1, seed=11,
                          triangulate=hpm_b200.delaunay, level_max_side=level_max_side or 1000)
    pts, n_ref = P.reconstruct(fuse=True)
    for i, v in enumerate(P.views):
        for kind, key in ((hpm_b200.MAP_DEPTH_GEOM, "depth_geom"), (hpm_b200.MAP_NORMAL, "normal"),
                          (hpm_b200.MAP_COST, "cost"), (hpm_b200.MAP_DEPTH, "depth")):
            g = ctx.get_map(i, kind)
            o = np.ascontiguousarray(v.maps[key], np.float32)
            assert g.shape == o.shape
            # bitwise, except that any NaN equals any NaN (x86 and the GPU make NaNs with different payloads)
            eq = (g.view(np.uint32) == o.view(np.uint32)) | (np.isnan(g) & np.isnan(o))
            same = float(eq.all(axis=-1).mean() if g.ndim == 3 else eq.mean())
            print(f"view {i} {key}: identical {same:.5f}")
            assert same == 1.0, (i, key, same)
    assert n_pts == n_ref
    got = ctx.get_points()
    assert np.array_equal(got, pts.reshape(got.shape), equal_nan=True)


def test_c1_configuration_matches_oracle_pipeline(ctx):
    """The reference's small configuration: 5 views of 1280x960 on a 30-degree arc, 4 sources each,
    --initial-image-scale 4 (320x240 working size, one level), the whole schedule with fusion."""
    import pipeline as op
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=5, width=1280, height=960, layout="arc", n_src=4, seed=17)
    cams = scene_cams(sc)
    srcs = [[j for j, _ in p] for p in sc.pairs]
    for i, v in enumerate(sc.views):
        ctx.set_image(i, v.image)
    n_pts = ctx.reconstruct(cams, srcs, initial_image_scale=4, seed=23, fuse=True)
    P = op.OraclePipeline([v.image for v in sc.views], cams, srcs, initial_image_scale=4, seed=23,
                          triangulate=hpm_b200.delaunay)
    pts, n_ref = P.reconstruct(fuse=True)
    for i, v in enumerate(P.views):
        for kind, key in ((hpm_b200.MAP_DEPTH_GEOM, "depth_geom"), (hpm_b200.MAP_NORMAL, "normal")):
            g = ctx.get_map(i, kind)
            o = np.ascontiguousarray(v.maps[key], np.float32)
            assert g.shape == o.shape == ((240, 320, 3) if key == "normal" else (240, 320))
            eq = (g.view(np.uint32) == o.view(np.uint32)) | (np.isnan(g) & np.isnan(o))
            assert eq.all(), (i, key, float(eq.mean()))
    assert n_pts == n_ref
