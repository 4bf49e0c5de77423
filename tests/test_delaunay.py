"""Host Delaunay triangulation (hpm_delaunay) against cv2.Subdiv2D, the
library HPM::DelaunayTriangulation calls (HPM.cpp:1075-1097).  CPU only.

The prior raster lets the last triangle win on shared edges (main.cpp:398-404)
and the plane fits round by vertex order, so what must agree is the triangle
LIST: the same triangles in the same order, each with the same first vertex --
on random points, on points aligned to the 5-pixel support-point grid (many
cocircular and collinear quadruples), on points lying on earlier edges, with
repeated points, and at the 1600 x 1200 working size."""
from __future__ import annotations

import cv2
import numpy as np

import hpm_b200


def cv2_triangles(xy, w, h):
    sub = cv2.Subdiv2D((0, 0, w, h))
    for x, y in xy:
        sub.insert((float(x), float(y)))
    out = []
    for t in sub.getTriangleList():
        pts = [int(t[0]), int(t[1]), int(t[2]), int(t[3]), int(t[4]), int(t[5])]
        if all(0 <= pts[2 * k] < w and 0 <= pts[2 * k + 1] < h for k in range(3)):
            out.append(pts)
    return np.asarray(out, np.int32).reshape(-1, 6)


def _same_list(xy, w, h):
    ours = hpm_b200.delaunay(np.asarray(xy, np.int32), w, h)
    ref = cv2_triangles(xy, w, h)
    return ours.shape == ref.shape and bool((ours == ref).all()), len(ref)


def test_random_points_same_list_as_subdiv2d():
    for seed in range(12):
        rng = np.random.default_rng(seed)
        w, h = 640, 480
        xy = np.stack([rng.integers(0, w, 1500), rng.integers(0, h, 1500)], 1)
        same, n = _same_list(xy, w, h)
        assert same, (seed, n)


def test_dense_points_with_repeats_same_list():
    """Dense integer points (many on earlier edges, collinear and cocircular) with repeats, some immediate."""
    for seed in range(20):
        rng = np.random.default_rng(100 + seed)
        pts = [(int(a), int(b)) for a, b in zip(rng.integers(0, 64, 150), rng.integers(0, 48, 150))]
        for _ in range(15):
            j = int(rng.integers(0, len(pts)))
            pts.insert(int(rng.integers(j, len(pts) + 1)), pts[j])
        same, n = _same_list(pts, 64, 48)
        assert same, (seed, n)


def test_support_point_grid_same_list_at_working_size():
    rng = np.random.default_rng(1)
    for (w, h), keep in (((320, 240), 0.6), ((1600, 1200), 0.05)):
        # one point per kept 5x5 block, anywhere in the block or at its centre, as
        # GetSupportPoints_Classify_Check produces; block order as it scans
        pts = []
        for c in range(0, w, 5):
            for r in range(0, h, 5):
                if rng.random() < keep:
                    pts.append((c + 2, r + 2) if rng.random() < 0.5 else (c + int(rng.integers(0, 5)),
                                                                          r + int(rng.integers(0, 5))))
        same, n = _same_list(pts, w, h)
        print(f"support-point grid {w}x{h}: {n} triangles, identical list: {same}")
        assert same


def test_duplicates_and_degenerate_inputs():
    assert hpm_b200.delaunay(np.zeros((0, 2), np.int32), 10, 10).shape == (0, 6)
    t = hpm_b200.delaunay(np.array([[1, 1], [1, 1], [8, 1], [4, 7], [4, 7]]), 10, 10)
    assert t.shape == (1, 6)
    # collinear points produce no triangle inside the image
    t = hpm_b200.delaunay(np.array([[1, 1], [3, 3], [6, 6]]), 10, 10)
    assert len(t) == 0
    # points outside the rectangle (which Subdiv2D rejects) are skipped
    t = hpm_b200.delaunay(np.array([[1, 1], [8, 1], [4, 7], [12, 3], [-1, 2]]), 10, 10)
    assert t.shape == (1, 6)


def test_plane_fits_match_opencv_svd():
    """HPM::GetPriorPlaneParams (HPM.cpp:1132-1166) fits each triangle's plane with
    cv::SVD::solveZ on the 3x4 float matrix of its camera-frame points.  The
    restatement takes the exact null space in double; against OpenCV's own float
    SVD (cv2.SVDecomp, full UV, last row of V^T, then the reference's sign rule and
    normalisation) the plane parameters agree to 1e-4 relative."""
    import hpm_oracle as ora
    from hpm_b200 import synth
    from conftest import scene_cams

    sc = synth.make_scene(n_views=5, width=320, height=240, seed=1, n_src=4)
    cam = scene_cams(sc)[0]
    depth = np.where(sc.views[0].depth > 0, sc.views[0].depth, 6.0).astype(np.float32)
    rng = np.random.default_rng(0)
    pts = np.unique(np.stack([rng.integers(0, 320, 900), rng.integers(0, 240, 900)], 1), axis=0).astype(np.int32)
    tris = np.asarray(hpm_b200.delaunay(pts, 320, 240), np.int32).reshape(-1, 6)
    _, planes, _, _ = ora.planar_prior(tris, depth, cam, 1.0, 0.1, 100.0, 0)
    K = np.array(cam.K, np.float32).reshape(3, 3)
    f32 = np.float32

    def point(x, y):  # Get3DPointonRefCam (HPM.cpp:258-267), float arithmetic
        d = depth[y, x]
        return [f32(d * f32(f32(x) - K[0, 2])) / K[0, 0], f32(d * f32(f32(y) - K[1, 2])) / K[1, 1], d]

    worst = 0.0
    for t, pl in zip(tris, planes):
        A = np.ones((3, 4), np.float32)
        for r in range(3):
            A[r, :3] = point(t[2 * r], t[2 * r + 1])
        B = cv2.SVDecomp(A, flags=cv2.SVD_FULL_UV)[2][-1].astype(np.float32)
        norm = f32(np.sqrt(np.float64(B[0]) ** 2 + np.float64(B[1]) ** 2 + np.float64(B[2]) ** 2))
        ref = (B / (-norm if B[3] < 0 else norm)).astype(np.float32)
        worst = max(worst, float(np.abs(ref - pl).max()) / max(1.0, abs(float(ref[3]))))
    print(f"plane fits vs cv2 SVD over {len(tris)} triangles: worst relative difference {worst:.2e}")
    assert worst <= 1e-4
