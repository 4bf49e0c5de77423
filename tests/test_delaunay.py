"""Host Delaunay triangulation (hpm_delaunay) against cv2.Subdiv2D, the
library HPM::DelaunayTriangulation calls (HPM.cpp:1075-1097).  CPU only.

For points in general position the Delaunay triangulation is unique, so the
triangle sets must agree (away from the hull, where Subdiv2D's finite enclosing
triangle can change hull triangles).  Support points are integer and often
cocircular; there the triangulation is not unique and only the fraction of
shared triangles is reported and bounded."""
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
        pts = [(int(t[0]), int(t[1])), (int(t[2]), int(t[3])), (int(t[4]), int(t[5]))]
        if all(0 <= x < w and 0 <= y < h for x, y in pts):
            out.append(pts)
    return out


def canon(tris):
    return {tuple(sorted(map(tuple, np.asarray(t).reshape(3, 2).tolist()))) for t in tris}


def test_general_position_matches_subdiv2d():
    rng = np.random.default_rng(0)
    w, h = 640, 480
    xy = np.unique(np.stack([rng.integers(5, w - 5, 1500), rng.integers(5, h - 5, 1500)], 1), axis=0)
    rng.shuffle(xy)
    ours = canon(hpm_b200.delaunay(xy, w, h))
    ref = canon(cv2_triangles(xy, w, h))
    inter = len(ours & ref)
    print(f"general position: ours {len(ours)}, cv2 {len(ref)}, shared {inter}")
    assert inter >= 0.98 * len(ref)


def test_duplicates_and_degenerate_inputs():
    assert hpm_b200.delaunay(np.zeros((0, 2), np.int32), 10, 10).shape == (0, 6)
    t = hpm_b200.delaunay(np.array([[1, 1], [1, 1], [8, 1], [4, 7], [4, 7]]), 10, 10)
    assert t.shape == (1, 6)
    # collinear points produce no triangle inside the image
    t = hpm_b200.delaunay(np.array([[1, 1], [3, 3], [6, 6]]), 10, 10)
    assert len(t) == 0


def test_support_point_grid_agreement():
    rng = np.random.default_rng(1)
    w, h = 320, 240
    # one or two points per 5x5 block, as GetSupportPoints_Classify_Check produces
    pts = []
    for c in range(0, w, 5):
        for r in range(0, h, 5):
            if rng.random() < 0.6:
                pts.append((c + rng.integers(0, 5), r + rng.integers(0, 5)))
    xy = np.asarray(pts, np.int32)
    ours = canon(hpm_b200.delaunay(xy, w, h))
    ref = canon(cv2_triangles(xy, w, h))
    inter = len(ours & ref)
    print(f"support-point grid: ours {len(ours)}, cv2 {len(ref)}, shared {inter / max(1, len(ref)):.3f}")
    assert inter >= 0.9 * len(ref)


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
