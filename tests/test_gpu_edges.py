"""Edge cases of a PatchMatch run against the oracle, bit for bit (B200).

- every specialisation of the kernels on the number of sources: S = 1, 4, 10,
  12, 20, 31 (the NS = 4 / 10 / 16 / 31 builds and their block sizes);
- odd heights, whose last row the reference's checkerboard grid covers or not
  (HPM.cu:3004-3011), and a view smaller than the 11 x 11 patch;
- sources whose size differs from the reference's (uneven resolutions);
- geometric mode with the sources' depth maps.
Every map of the run (depth, normal, cost) must equal the oracle's bits, NaNs
compared as NaN.
"""
from __future__ import annotations

import cv2
import numpy as np
import pytest

import hpm_b200
import hpm_oracle as ora

pytestmark = pytest.mark.gpu


def _same(a, b):
    return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())


def _views(n, w, h, seed, sizes=None):
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=n, width=w, height=h, layout="hemisphere", seed=seed, n_src=min(n - 1, 31),
                          sizes=sizes)
    cams, grays = [], []
    for v in sc.views:
        hh, ww = v.image.shape[:2]
        cams.append(hpm_b200.Camera.make(v.K, v.R, v.t, ww, hh, v.depth_min, v.depth_max))
        grays.append(synth.gray_float(v.image))
    return sc, cams, grays


def _run_both(ctx, sc, cams, grays, srcs, mode, seed, depths=None):
    for i, (g, c) in enumerate(zip(grays, cams)):
        ctx.set_view(i, g, c)
    ref = sc.views[0]
    canny = cv2.Canny(ref.image, 50, 150)
    ctx.set_canny(0, canny)
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]), mode=mode)
    H, W = grays[0].shape
    st = ora.RunState(W, H)
    st.canny[:] = canny
    if mode & hpm_b200.MODE_GEOM:
        nrm = ref.normal.astype(np.float32)
        cost = np.full((H, W), 0.5, np.float32)
        for i in range(len(grays)):
            ctx.set_map(i, hpm_b200.MAP_DEPTH, depths[i])
        ctx.set_map(0, hpm_b200.MAP_NORMAL, nrm)
        ctx.set_map(0, hpm_b200.MAP_COST, cost)
        st.planes[..., :3] = nrm
        st.planes[..., 3] = depths[0]
        st.costs[:] = cost
    ctx.run_patchmatch(0, srcs, params, texture_level=0, seed=seed)
    kind = hpm_b200.MAP_DEPTH_GEOM if mode & hpm_b200.MODE_GEOM else hpm_b200.MAP_DEPTH
    got = (ctx.get_map(0, kind), ctx.get_map(0, hpm_b200.MAP_NORMAL), ctx.get_map(0, hpm_b200.MAP_COST))
    dl = None if depths is None else [None] + [depths[j] for j in srcs]
    ora.run_patchmatch([grays[0]] + [grays[j] for j in srcs], dl, [cams[0]] + [cams[j] for j in srcs], params, st,
                       seed, 0)
    return got, (st.planes[..., 3], st.planes[..., :3], st.costs)


@pytest.fixture(scope="module")
def ctx():
    c = hpm_b200.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("n_src", [1, 12, 20, 31])
def test_source_count_specialisations(ctx, n_src):
    sc, cams, grays = _views(n_src + 1, 64, 48, seed=40 + n_src)
    srcs = list(range(1, n_src + 1))
    got, want = _run_both(ctx, sc, cams, grays, srcs, 0, seed=7)
    for g, w, name in zip(got, want, ("depth", "normal", "cost")):
        assert _same(g, w), (n_src, name)


@pytest.mark.parametrize("size", [(67, 41), (50, 33), (9, 7)])
def test_odd_and_tiny_sizes(ctx, size):
    w, h = size
    sc, cams, grays = _views(4, w, h, seed=w)
    got, want = _run_both(ctx, sc, cams, grays, [1, 2, 3], 0, seed=8)
    for g, wnt, name in zip(got, want, ("depth", "normal", "cost")):
        assert _same(g, wnt), (size, name)


def test_uneven_source_sizes_and_geometric_mode(ctx):
    sizes = [(80, 60), (64, 48), (96, 72), (80, 60)]
    sc, cams, grays = _views(4, 80, 60, seed=3, sizes=sizes)
    got, want = _run_both(ctx, sc, cams, grays, [1, 2, 3], 0, seed=9)
    for g, w, name in zip(got, want, ("depth", "normal", "cost")):
        assert _same(g, w), ("photometric", name)
    depths = [v.depth.astype(np.float32) for v in sc.views]
    got, want = _run_both(ctx, sc, cams, grays, [1, 2, 3], hpm_b200.MODE_GEOM, seed=10, depths=depths)
    for g, w, name in zip(got, want, ("depth", "normal", "cost")):
        assert _same(g, w), ("geometric", name)
