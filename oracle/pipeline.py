"""CPU ORACLE of the whole schedule -- test infrastructure only.

Restates main() of HPM-MVS++ (main.cpp:1143-1364) and ProcessProblem
(main.cpp:237-634) over in-memory maps instead of .dmb files, using the C
oracle for every kernel and host loop, and OpenCV (cv2) where the reference
calls OpenCV: cv::resize of the pyramid images, cvtColor, Canny and
Subdiv2D.  Seeds follow the same per-(pass, view) derivation as the CUDA
pipeline so both draw identical random streams.
"""
from __future__ import annotations

import math
from typing import List, Sequence

import cv2
import numpy as np

import hpm_oracle as ora

MASK64 = (1 << 64) - 1

MODE_GEOM, MODE_PRIOR, MODE_MULTIGEOM, MODE_HIERARCHY, MODE_UPSAMPLE, MODE_MAND = 1, 2, 4, 8, 16, 32


def mix_seed(base: int, a: int, b: int) -> int:
    z = (base ^ ((a * 0x9E3779B97F4A7C15) & MASK64) ^ ((b * 0xBF58476D1CE4E5B9) & MASK64)) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def f32(x) -> float:
    return float(np.float32(x))


def cv2_triangles(xy: np.ndarray, w: int, h: int) -> np.ndarray:
    sub = cv2.Subdiv2D((0, 0, w, h))
    for x, y in xy:
        sub.insert((float(x), float(y)))
    out = []
    for t in sub.getTriangleList():
        pts = [int(t[0]), int(t[1]), int(t[2]), int(t[3]), int(t[4]), int(t[5])]
        out.append(pts)
    return np.asarray(out, np.int32).reshape(-1, 6)


class View:
    def __init__(self, image: np.ndarray, cam):
        self.orig = image
        self.cam0 = ora.to_cam(cam)
        self.maps: dict = {}


class OraclePipeline:
    def __init__(self, images: Sequence[np.ndarray], cams, src_lists: Sequence[Sequence[int]], initial_image_scale=4,
                 seed=0, geom_iterations=3, triangulate=None, level_max_side=1000):
        """triangulate(points (n,2) int32, w, h) -> (m,6) int32 triangles; defaults to cv2.Subdiv2D, the
        library HPM::DelaunayTriangulation calls (HPM.cpp:1075-1097)."""
        self.triangulate = triangulate or cv2_triangles
        self.size_bound = level_max_side
        self.views = [View(im, c) for im, c in zip(images, cams)]
        self.srcs = [list(s) for s in src_lists]
        self.scale = initial_image_scale
        self.seed = seed
        self.geom_iterations = geom_iterations
        self.pass_id = 0

    # ---- level preparation (PrepareScaleImages + InuputInitialization) ----
    def prepare_level(self, i: int, target: int) -> None:
        v = self.views[i]
        h0, w0 = v.orig.shape[:2]
        w, h = w0, h0
        img = v.orig
        if max(w0, h0) > target:
            factor = min(np.float32(target) / np.float32(w0), np.float32(target) / np.float32(h0))
            w = max(1, int(round(float(np.float32(w0) * np.float32(factor)))))
            h = max(1, int(round(float(np.float32(h0) * np.float32(factor)))))
            img = cv2.resize(v.orig, (w, h), interpolation=cv2.INTER_LINEAR)
        cam = ora.to_cam(v.cam0)
        sx = np.float32(w) / np.float32(w0)
        sy = np.float32(h) / np.float32(h0)
        cam.K[0] = f32(np.float32(cam.K[0]) * sx)
        cam.K[2] = f32(np.float32(cam.K[2]) * sx)
        cam.K[4] = f32(np.float32(cam.K[4]) * sy)
        cam.K[5] = f32(np.float32(cam.K[5]) * sy)
        cam.width, cam.height = w, h
        v.cam = cam
        v.color = img
        v.gray = cv2.cvtColor(img, cv2.COLOR_BGR2GRAY).astype(np.float32)
        v.canny = cv2.Canny(img, 50, 150)
        v.w, v.h = w, h

    # ---- one ProcessProblem PatchMatch run ----
    def run(self, i: int, mode: int, level: int) -> None:
        v = self.views[i]
        srcs = self.srcs[i]
        W, H = v.w, v.h
        p = ora.Params()
        p.max_iterations, p.patch_size, p.num_images, p.radius_increment = 3, 11, len(srcs) + 1, 2
        p.sigma_spatial, p.sigma_color, p.top_k = 5.0, 3.0, 4
        p.depth_min = f32(np.float32(v.cam.depth_min) * np.float32(0.6))
        p.depth_max = f32(np.float32(v.cam.depth_max) * np.float32(1.2))
        p.scaled_cols = p.scaled_rows = 0
        st = ora.RunState(W, H)
        st.canny[:] = v.canny
        geom, prior = bool(mode & MODE_GEOM), bool(mode & MODE_PRIOR)
        hier, mand = bool(mode & MODE_HIERARCHY), bool(mode & MODE_MAND)
        dkind = "depth_geom" if mode & MODE_MULTIGEOM else "depth"
        if geom or prior:
            st.planes[..., :3] = v.maps["normal"]
            st.planes[..., 3] = v.maps[dkind]
            st.costs[:] = v.maps["cost"]
        if prior or mand:
            st.confidences[:] = v.maps["conf"]
        if prior:
            st.prior_planes[:] = v.prior
            st.plane_masks[:] = v.prior_mask
        if hier and not geom and not prior:
            n, c, d = v.maps["normal"], v.maps["cost"], v.maps["depth"]
            nh, nw = n.shape[:2]
            upsample = (nw != H or nh != W)
            sp = np.zeros((nh, nw, 4), np.float32)
            sp[..., :3] = n
            sp[..., 3] = c if upsample else d
            st.scaled_planes = sp
            st.planes[..., 3] = d
            p.scaled_cols, p.scaled_rows = nw, nh
            if upsample:
                mode |= MODE_UPSAMPLE
        p.mode = mode
        depths = None
        if geom:
            depths = [None] + [self.views[j].maps[dkind] for j in srcs]
        imgs = [v.gray] + [self.views[j].gray for j in srcs]
        cams = [v.cam] + [self.views[j].cam for j in srcs]
        ora.run_patchmatch(imgs, depths, cams, p, st, mix_seed(self.seed, self.pass_id, i), i)
        v.maps["depth_geom" if geom else "depth"] = st.planes[..., 3].copy()
        v.maps["normal"] = st.planes[..., :3].copy()
        v.maps["cost"] = st.costs.copy()
        if not prior and not mand:
            v.maps[f"texture{level}"] = st.texture.copy()

    def confidence(self, kind: str) -> None:
        confs = ora.confidence_eval([v.cam for v in self.views], [v.maps[kind] for v in self.views],
                                    [v.maps["normal"] for v in self.views], self.srcs)
        for v, c in zip(self.views, confs):
            v.maps["conf"] = c

    def build_prior(self, i: int, distance: int) -> None:
        v = self.views[i]
        W, H = v.w, v.h
        dmin = f32(np.float32(v.cam.depth_min) * np.float32(0.6))
        dmax = f32(np.float32(v.cam.depth_max) * np.float32(1.2))
        depth, cost, conf = v.maps["depth"], v.maps["cost"], v.maps["conf"]
        if distance == 0:
            pts = ora.support_points(cost, conf, W, H)
            tris = self.triangulate(pts, W, H)
            label, fits, _, _ = ora.planar_prior(tris, depth, v.cam, 1.0, dmin, dmax, 0)
            lab = label.astype(np.int64)
            prior = np.zeros((H, W, 4), np.float32)
            prior[lab > 0] = fits[lab[lab > 0] - 1]
            mask = (lab > 0).astype(np.uint32)
        else:
            f = np.float32(1.0) / np.float32(distance * 2)
            hw, hh = int(round(float(np.float32(W) * f))), int(round(float(np.float32(H) * f)))
            dd = ora.resize_linear(depth, hw, hh)
            pts = ora.support_points(ora.resize_linear(cost, hw, hh), ora.resize_linear(conf, hw, hh),
                                     int(np.float32(W) * f), int(np.float32(H) * f))
            tris = self.triangulate(pts, hw, hh)
            _, _, pdepth, pnormal = ora.planar_prior(tris, dd, v.cam, float(f), dmin, dmax, 1)
            if max(H // hh, W // hw) == 1:
                ud, un = np.zeros((H, W), np.float32), np.zeros((H, W, 3), np.float32)
            else:
                ud, un = ora.jbu_prior(v.gray, pdepth, pnormal)
            prior, m8 = ora.prior_reload(ud, un, v.cam, dmin, dmax)
            mask = m8.astype(np.uint32)
        v.prior, v.prior_mask = prior, mask

    # ---- main() ----
    def reconstruct(self, fuse: bool = True):
        n = len(self.views)
        init_side, nds = [], []
        for v in self.views:
            h, w = v.orig.shape[:2]
            s = max(1, (max(w, h) + self.scale // 2) // self.scale)
            k, side = 0, s
            while side > self.size_bound:
                side //= 2
                k += 1
            init_side.append(s)
            nds.append(k)
        max_nd = max(nds)
        max_hpm = max_nd
        cur = [0] * n
        first = True
        while max_nd >= 0:
            for i in range(n):
                if nds[i] >= 0:
                    cur[i] = int(init_side[i] / math.pow(2, nds[i]))
                    nds[i] -= 1
            for i in range(n):
                self.prepare_level(i, cur[i])
            level = max_nd
            if first:
                first = False
                self.pass_id += 1
                for i in range(n):
                    self.run(i, 0, level)
            else:
                for i, v in enumerate(self.views):
                    src = v.maps["depth_geom"]
                    if max(v.h // src.shape[0], v.w // src.shape[1]) != 1:
                        v.maps["depth"] = ora.jbu(v.gray, src)
                self.pass_id += 1
                for i in range(n):
                    self.run(i, MODE_HIERARCHY, level)
            for hpm_scale in range(max_hpm, level - 1, -1):
                self.confidence("depth")
                self.pass_id += 1
                for i in range(n):
                    self.build_prior(i, hpm_scale - nds[i] - 1)
                    self.run(i, MODE_PRIOR, level)
            for it in range(self.geom_iterations):
                mode = MODE_GEOM
                if it > 0:
                    mode |= MODE_MULTIGEOM | MODE_MAND
                    self.confidence("depth_geom")
                self.pass_id += 1
                for i in range(n):
                    self.run(i, mode, level)
            max_nd -= 1
        if not fuse:
            return None, 0
        return ora.fusion([v.cam for v in self.views], [v.maps["depth_geom"] for v in self.views],
                          [v.maps["normal"] for v in self.views], [v.color for v in self.views], self.srcs)
