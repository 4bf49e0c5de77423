"""The FP64 gradient of the differentiable bilateral NCC (oracle/hpm_oracle_grad.c)
against FP64 central finite differences, h = 1e-4 in each of (depth, nx, ny).
CPU only.  Bilinear sampling is piecewise linear: a difference whose step moves
one of the 36 samples across a texel edge averages two slopes.  At h = 1e-4
that happens for a few percent of the components, so there at least 95 % must
agree to 2e-3 relative; at h = 1e-6, where edge crossings are rare, at least
99 % must agree to 1e-4 relative (plus 1e-7 absolute)."""
from __future__ import annotations

import numpy as np

import hpm_b200
import hpm_oracle as ora
from conftest import scene_cams, scene_grays


def _theta_from_gt(v, x, y, rng, jitter=0.02):
    n = v.R @ v.normal[y, x]
    if n[2] > 0:
        n = -n
    n = n + rng.normal(0, jitter, 3)
    n /= np.linalg.norm(n)
    if n[2] > 0:
        n = -n
    return np.array([v.depth[y, x] * (1 + rng.normal(0, 0.005)), n[0], n[1]])


def test_fp64_gradient_matches_central_differences(small_scene):
    cams = scene_cams(small_scene)
    grays = scene_grays(small_scene)
    v0 = small_scene.views[0]
    srcs = [j for j, _ in small_scene.pairs[0]]
    params = hpm_b200.Params.make(len(srcs) + 1, *hpm_b200.widened_range(cams[0]))
    rng = np.random.default_rng(3)
    H, W = v0.depth.shape
    ys, xs = np.nonzero(v0.depth > 0)
    pick = rng.choice(len(xs), 150, replace=False)
    ok = {1e-4: 0, 1e-6: 0}
    total = 0
    for k in pick:
        x, y = int(xs[k]), int(ys[k])
        th = _theta_from_gt(v0, x, y, rng)
        for j in srcs[:2]:
            c, g = ora.cost_grad64(grays[0], cams[0], grays[j], cams[j], params, x, y, th)
            if not (0.0 < c < 2.0):
                continue
            for a in range(3):
                total += 1
                for h, rel, absol in ((1e-4, 2e-3, 1e-6), (1e-6, 1e-4, 1e-7)):
                    tp, tm = th.copy(), th.copy()
                    tp[a] += h
                    tm[a] -= h
                    fd = (ora.cost_grad64(grays[0], cams[0], grays[j], cams[j], params, x, y, tp, False)[0] -
                          ora.cost_grad64(grays[0], cams[0], grays[j], cams[j], params, x, y, tm, False)[0]) / (2 * h)
                    ok[h] += abs(fd - g[a]) <= rel * max(abs(g[a]), abs(fd)) + absol
    print(f"FD agreement: h=1e-4 {ok[1e-4]}/{total}, h=1e-6 {ok[1e-6]}/{total}")
    assert total > 300
    assert ok[1e-4] >= 0.95 * total
    assert ok[1e-6] >= 0.99 * total
