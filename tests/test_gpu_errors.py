"""Error behaviour of the C ABI on the B200: every misuse returns an HPM_E_* code
with a message (the reference prints and exits, HPM.cpp:68-101), and the
context keeps working afterwards."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import hpm_b200
from conftest import scene_cams, scene_grays

pytestmark = pytest.mark.gpu


def _raises(fn, code_text):
    with pytest.raises(hpm_b200.HPMError) as e:
        fn()
    assert code_text in str(e.value), str(e.value)
    return str(e.value)


def test_misuse_is_reported_and_the_context_survives(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    srcs = [j for j, _ in small_scene.pairs[0]]
    with hpm_b200.Context(0) as ctx:
        p = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
        # nothing uploaded yet
        _raises(lambda: ctx.run_patchmatch(0, srcs, p), "not set")
        for i, (g, c) in enumerate(zip(grays, cams)):
            ctx.set_view(i, g, c)
        # no Canny map for the reference
        _raises(lambda: ctx.run_patchmatch(0, srcs, p), "Canny")
        import cv2
        ctx.set_canny(0, cv2.Canny(small_scene.views[0].image, 50, 150))
        # source counts and params that disagree
        _raises(lambda: ctx.run_patchmatch(0, [], hpm_b200.Params.make(1, 1, 2)), "source views")
        _raises(lambda: ctx.run_patchmatch(0, srcs, hpm_b200.Params.make(len(srcs), 1, 2)), "num_images")
        _raises(lambda: ctx.run_patchmatch(0, [0] * 32, hpm_b200.Params.make(33, 1, 2)), "source views")
        # mandatory consistency without the geometric mode, geometric mode without depth maps
        _raises(lambda: ctx.run_patchmatch(0, srcs, hpm_b200.Params.make(len(srcs) + 1, 1, 2,
                                                                          mode=hpm_b200.MODE_MAND)), "geometric")
        with pytest.raises(hpm_b200.HPMError):
            ctx.run_patchmatch(0, srcs, hpm_b200.Params.make(len(srcs) + 1, 1, 2, mode=hpm_b200.MODE_GEOM))
        # fixed-hypothesis costs outside the image, oversize no-alloc request
        _raises(lambda: ctx.eval_costs(0, srcs, p, np.array([[-1, 0]]), np.zeros((1, 4))), "outside")
        # maps that do not exist
        _raises(lambda: ctx.get_map(3, hpm_b200.MAP_CONF), "no map")
        # fusion of a map kind that is not a depth map, and of an out-of-range kind
        _raises(lambda: ctx.fuse([srcs] * 5, depth_kind=hpm_b200.MAP_COST, capacity=16), "depth_kind")
        _raises(lambda: ctx.fuse([srcs] * 5, depth_kind=99, capacity=16), "depth_kind")
        # a whole reconstruction with a bad scale
        for i, v in enumerate(small_scene.views):
            ctx.set_image(i, v.image)
        _raises(lambda: ctx.reconstruct(cams, [[1]] * 5, initial_image_scale=0), "at least 1")
        # raw ABI: null context, bad texture format
        lib = hpm_b200.load_library()
        assert lib.hpm_run_patchmatch(None, 0, None, 0, None, 0, ctypes.c_uint64(0)) == 1
        _raises(lambda: ctx.set_texture_format(7), "texture format")
        # the context still runs a valid pass, bit-identically to a fresh one
        ctx.run_patchmatch(0, srcs, p, seed=5)
        d1 = ctx.get_map(0, hpm_b200.MAP_DEPTH)
    with hpm_b200.Context(0) as fresh:
        for i, (g, c) in enumerate(zip(grays, cams)):
            fresh.set_view(i, g, c)
        fresh.set_canny(0, cv2.Canny(small_scene.views[0].image, 50, 150))
        fresh.run_patchmatch(0, srcs, p, seed=5)
        d2 = fresh.get_map(0, hpm_b200.MAP_DEPTH)
    assert np.array_equal(d1.view(np.uint32), d2.view(np.uint32))
