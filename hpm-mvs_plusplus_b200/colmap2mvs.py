#!/usr/bin/env python3
"""COLMAP sparse model -> the HPM-MVS++ dense-folder inputs (cams/, pair.txt, images/).

Does what the reference's colmap2mvsnet_acm.py does (colmap2mvsnet_acm.py:305-451)
for the files main.cpp reads (cams/%08d_cam.txt, HPM.cpp:159-184; pair.txt,
main.cpp:171-200; images/%08d.jpg):

  * reads cameras, images and points3D of a COLMAP model in the text or the
    binary format (COLMAP's documented layouts);
  * intrinsics from the camera model's leading parameters (f or fx/fy, cx, cy;
    distortion terms are not applied, as in the reference);
  * images renumbered 0..n-1 in increasing COLMAP image id; extrinsics
    [R | t] from each image's unit quaternion (w, x, y, z) and translation;
  * depth range per image from the camera-frame depths of the 3D points it
    observes: the 1st percentile x 0.75 and the 99th percentile x 1.25 (index
    int(n * q) of the sorted depths); the number of depth planes is --max_d, or
    with --max_d 0 the inverse-depth count for a one-pixel step at depth_min;
    interval = (max - min) / (planes - 1) / --interval_scale;
  * view selection: the score of a pair is the number of the first image's
    observations (with multiplicity, unobserved -1 entries skipped) whose 3D
    point the second image also sees, set to 0 when the 75th-percentile
    triangulation angle of those points is below 1 degree; every view lists
    the min(20, n - 1) highest scores (numpy's argsort order, reversed);
  * images are copied when they are .jpg, else re-encoded as JPEG.

The pair scores are counted for all pairs at once from the points' tracks
(a sparse image x point incidence product) instead of per-pair list scans.

    python colmap2mvs.py --dense_folder DIR --save_folder OUT [--model_ext .txt|.bin]
"""
from __future__ import annotations

import argparse
import os
import shutil
import struct
from dataclasses import dataclass
from typing import Dict, List, Tuple

import numpy as np

# COLMAP camera models: id -> (name, parameter names)
CAMERA_MODELS = {
    0: ("SIMPLE_PINHOLE", ("f", "cx", "cy")),
    1: ("PINHOLE", ("fx", "fy", "cx", "cy")),
    2: ("SIMPLE_RADIAL", ("f", "cx", "cy", "k")),
    3: ("RADIAL", ("f", "cx", "cy", "k1", "k2")),
    4: ("OPENCV", ("fx", "fy", "cx", "cy", "k1", "k2", "p1", "p2")),
    5: ("OPENCV_FISHEYE", ("fx", "fy", "cx", "cy", "k1", "k2", "k3", "k4")),
    6: ("FULL_OPENCV", ("fx", "fy", "cx", "cy", "k1", "k2", "p1", "p2", "k3", "k4", "k5", "k6")),
    7: ("FOV", ("fx", "fy", "cx", "cy", "omega")),
    8: ("SIMPLE_RADIAL_FISHEYE", ("f", "cx", "cy", "k")),
    9: ("RADIAL_FISHEYE", ("f", "cx", "cy", "k1", "k2")),
    10: ("THIN_PRISM_FISHEYE", ("fx", "fy", "cx", "cy", "k1", "k2", "p1", "p2", "k3", "k4", "sx1", "sy1")),
}
MODEL_BY_NAME = {name: (mid, params) for mid, (name, params) in CAMERA_MODELS.items()}


@dataclass
class Camera:
    model: str
    width: int
    height: int
    params: np.ndarray


@dataclass
class Image:
    qvec: np.ndarray      # w, x, y, z
    tvec: np.ndarray
    camera_id: int
    name: str
    point3D_ids: np.ndarray  # -1: keypoint without a 3D point


# ---------------------------------------------------------------- readers

def _text_lines(path: str):
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if line and not line.startswith("#"):
                yield line


def read_cameras_text(path: str) -> Dict[int, Camera]:
    out = {}
    for line in _text_lines(path):
        f = line.split()
        out[int(f[0])] = Camera(f[1], int(f[2]), int(f[3]), np.array([float(x) for x in f[4:]]))
    return out


def read_images_text(path: str) -> Dict[int, Image]:
    out = {}
    # two lines per image: the pose line and the 2D points line, which may be empty
    with open(path) as fh:
        raw = [ln.rstrip("\n") for ln in fh if not ln.startswith("#")]
    k = 0
    while k < len(raw):
        head = raw[k].split()
        if not head:
            k += 1
            continue
        pts = raw[k + 1].split() if k + 1 < len(raw) else []
        k += 2
        iid = int(head[0])
        out[iid] = Image(np.array([float(x) for x in head[1:5]]), np.array([float(x) for x in head[5:8]]),
                         int(head[8]), " ".join(head[9:]), np.array([int(x) for x in pts[2::3]], np.int64))
    return out


def read_points3d_text(path: str) -> Dict[int, np.ndarray]:
    out = {}
    for line in _text_lines(path):
        f = line.split()
        out[int(f[0])] = np.array([float(f[1]), float(f[2]), float(f[3])])
    return out


class _Bin:
    def __init__(self, path: str):
        with open(path, "rb") as fh:
            self.b = fh.read()
        self.p = 0

    def take(self, fmt: str):
        n = struct.calcsize("<" + fmt)
        v = struct.unpack_from("<" + fmt, self.b, self.p)
        self.p += n
        return v

    def cstring(self) -> str:
        end = self.b.index(b"\x00", self.p)
        s = self.b[self.p:end].decode("utf-8")
        self.p = end + 1
        return s


def read_cameras_binary(path: str) -> Dict[int, Camera]:
    r = _Bin(path)
    out = {}
    (n,) = r.take("Q")
    for _ in range(n):
        cid, mid, w, h = r.take("iiQQ")
        name, pnames = CAMERA_MODELS[mid]
        out[cid] = Camera(name, w, h, np.array(r.take("d" * len(pnames))))
    return out


def read_images_binary(path: str) -> Dict[int, Image]:
    r = _Bin(path)
    out = {}
    (n,) = r.take("Q")
    for _ in range(n):
        vals = r.take("idddddddi")
        iid, q, t, cid = vals[0], vals[1:5], vals[5:8], vals[8]
        name = r.cstring()
        (npts,) = r.take("Q")
        pts = np.frombuffer(r.b, dtype=np.dtype([("x", "<f8"), ("y", "<f8"), ("id", "<i8")]), count=npts,
                            offset=r.p)
        r.p += 24 * npts
        out[iid] = Image(np.array(q), np.array(t), cid, name, pts["id"].astype(np.int64))
    return out


def read_points3d_binary(path: str) -> Dict[int, np.ndarray]:
    r = _Bin(path)
    out = {}
    (n,) = r.take("Q")
    for _ in range(n):
        pid, x, y, z = r.take("Qddd")
        r.take("BBBd")  # colour, reprojection error
        (tl,) = r.take("Q")
        r.p += 8 * tl  # track: (image id, point2D index) int32 pairs
        out[pid] = np.array([x, y, z])
    return out


def read_model(folder: str, ext: str):
    if ext == ".txt":
        return (read_cameras_text(os.path.join(folder, "cameras.txt")),
                read_images_text(os.path.join(folder, "images.txt")),
                read_points3d_text(os.path.join(folder, "points3D.txt")))
    return (read_cameras_binary(os.path.join(folder, "cameras.bin")),
            read_images_binary(os.path.join(folder, "images.bin")),
            read_points3d_binary(os.path.join(folder, "points3D.bin")))


# ---------------------------------------------------------------- geometry

def quat_to_rot(q: np.ndarray) -> np.ndarray:
    """Rotation matrix of the unit quaternion (w, x, y, z) (Hamilton convention, as COLMAP stores it), in the
    expanded textbook form with the reference converter's product order, so the camera files carry the same
    doubles (colmap2mvsnet_acm.py:253-263)."""
    w, x, y, z = (float(v) for v in q)
    return np.array([
        [1 - 2 * y ** 2 - 2 * z ** 2, 2 * x * y - 2 * w * z, 2 * z * x + 2 * w * y],
        [2 * x * y + 2 * w * z, 1 - 2 * x ** 2 - 2 * z ** 2, 2 * y * z - 2 * w * x],
        [2 * z * x - 2 * w * y, 2 * y * z + 2 * w * x, 1 - 2 * x ** 2 - 2 * y ** 2],
    ])


def intrinsic_matrix(cam: Camera) -> np.ndarray:
    names = MODEL_BY_NAME[cam.model][1]
    p = dict(zip(names, cam.params))
    fx = p.get("fx", p.get("f"))
    fy = p.get("fy", p.get("f"))
    return np.array([[fx, 0.0, p["cx"]], [0.0, fy, p["cy"]], [0.0, 0.0, 1.0]])


def depth_range(ext: np.ndarray, K: np.ndarray, xyz: np.ndarray, max_d: int, interval_scale: float):
    """(depth_min, interval, planes, depth_max) of one image from the world points it observes."""
    if len(xyz) == 0:
        raise ValueError("an image observes no 3D point; its depth range is undefined")
    z = np.sort(xyz @ ext[:3, :3].T[:, 2] + ext[2, 3])
    n = len(z)
    dmin = z[int(n * 0.01)] * 0.75
    dmax = z[int(n * 0.99)] * 1.25
    if max_d == 0:
        Kinv = np.linalg.inv(K)
        R, t = ext[:3, :3], ext[:3, 3]
        Rinv = np.linalg.inv(R)
        a = Rinv @ (Kinv @ np.array([K[0, 2], K[1, 2], 1.0]) * dmin - t)
        b = Rinv @ (Kinv @ np.array([K[0, 2] + 1, K[1, 2], 1.0]) * dmin - t)
        planes = (1 / dmin - 1 / dmax) / (1 / dmin - 1 / (dmin + np.linalg.norm(b - a)))
    else:
        planes = max_d
    return dmin, (dmax - dmin) / (planes - 1) / interval_scale, planes, dmax


def pair_scores(images: List[Image], centres: np.ndarray, points: Dict[int, np.ndarray]) -> np.ndarray:
    """n x n view-selection scores (symmetric; see the module docstring)."""
    n = len(images)
    score = np.zeros((n, n))
    # observations (image, point) with multiplicity, unobserved entries dropped
    obs_img, obs_pid = [], []
    for i, im in enumerate(images):
        ids = im.point3D_ids[im.point3D_ids != -1]
        obs_img.append(np.full(len(ids), i, np.int64))
        obs_pid.append(ids)
    obs_img = np.concatenate(obs_img) if obs_img else np.zeros(0, np.int64)
    obs_pid = np.concatenate(obs_pid) if obs_pid else np.zeros(0, np.int64)
    if obs_img.size == 0:
        return score
    # per point: the images that see it (each once) -> all (first image observation, second image) pairs
    uniq_pts, inv = np.unique(obs_pid, return_inverse=True)
    seen = np.unique(np.stack([inv, obs_img], 1), axis=0)  # (point index, image) presence
    order = np.argsort(seen[:, 0], kind="stable")
    seen = seen[order]
    starts = np.searchsorted(seen[:, 0], np.arange(len(uniq_pts)))
    ends = np.searchsorted(seen[:, 0], np.arange(len(uniq_pts)), side="right")
    xyz = np.array([points[int(p)] for p in uniq_pts])
    # every observation (i, point) pairs with each image j > i that sees the point
    ob_pt = inv
    counts = ends[ob_pt] - starts[ob_pt]
    rep_obs = np.repeat(np.arange(len(obs_img)), counts)
    offs = np.arange(len(rep_obs)) - np.repeat(np.cumsum(counts) - counts, counts)
    j = seen[starts[ob_pt[rep_obs]] + offs, 1]
    i = obs_img[rep_obs]
    keep = j > i
    i, j, pt = i[keep], j[keep], ob_pt[rep_obs[keep]]
    if i.size == 0:
        return score
    p = xyz[pt]
    a = centres[i] - p
    b = centres[j] - p
    cosang = np.sum(a * b, 1) / np.linalg.norm(a, axis=1) / np.linalg.norm(b, axis=1)
    theta = (180.0 / np.pi) * np.arccos(np.clip(cosang, -1.0, 1.0))
    key = i * n + j
    o = np.lexsort((theta, key))
    key, theta = key[o], theta[o]
    uk, first, cnt = np.unique(key, return_index=True, return_counts=True)
    q75 = theta[first + (cnt * 0.75).astype(np.int64)]
    val = np.where(q75 < 1.0, 0.0, cnt.astype(np.float64))
    ii, jj = uk // n, uk % n
    score[ii, jj] = val
    score[jj, ii] = val
    return score


# ---------------------------------------------------------------- writer

def convert(dense_folder: str, save_folder: str, max_d: int = 192, interval_scale: float = 1.0,
            model_ext: str = ".txt") -> None:
    cams, imgs, pts = read_model(os.path.join(dense_folder, "sparse"), model_ext)
    images = [imgs[k] for k in sorted(imgs)]
    n = len(images)
    K = {cid: intrinsic_matrix(c) for cid, c in cams.items()}
    ext = []
    for im in images:
        e = np.eye(4)
        e[:3, :3] = quat_to_rot(im.qvec)
        e[:3, 3] = im.tvec
        ext.append(e)
    ranges = []
    for im, e in zip(images, ext):
        ids = im.point3D_ids[im.point3D_ids != -1]
        xyz = np.array([pts[int(p)] for p in ids]).reshape(-1, 3)
        ranges.append(depth_range(e, K[im.camera_id], xyz, max_d, interval_scale))
    centres = np.array([-e[:3, :3].T @ e[:3, 3] for e in ext])
    score = pair_scores(images, centres, pts)
    n_sel = min(20, n - 1)

    os.makedirs(save_folder, exist_ok=True)
    cam_dir = os.path.join(save_folder, "cams")
    img_dir = os.path.join(save_folder, "images")
    for d in (cam_dir, img_dir):
        if os.path.exists(d):
            shutil.rmtree(d)
        os.makedirs(d)
    for i, (im, e) in enumerate(zip(images, ext)):
        Ki = K[im.camera_id]
        rows = ["extrinsic"] + ["".join(f"{v} " for v in e[r]) for r in range(4)] + ["", "intrinsic"]
        rows += ["".join(f"{v} " for v in Ki[r]) for r in range(3)]
        dmin, interval, planes, dmax = ranges[i]
        rows += ["", "%f %f %f %f" % (dmin, interval, planes, dmax)]
        with open(os.path.join(cam_dir, f"{i:08d}_cam.txt"), "w") as fh:
            fh.write("\n".join(rows) + "\n")
    with open(os.path.join(save_folder, "pair.txt"), "w") as fh:
        fh.write(f"{n}\n")
        for i in range(n):
            sel = np.argsort(score[i])[::-1][:n_sel]
            fh.write(f"{i}\n{len(sel)} " + "".join("%d %d " % (k, score[i, k]) for k in sel) + "\n")
    for i, im in enumerate(images):
        src = os.path.join(dense_folder, "images", im.name)
        dst = os.path.join(img_dir, f"{i:08d}.jpg")
        if src.endswith(".jpg"):
            shutil.copyfile(src, dst)
        else:
            import cv2  # only for re-encoding non-JPEG inputs
            img = cv2.imread(src)
            if img is None:
                raise ValueError(f"cannot read {src}")
            cv2.imwrite(dst, img)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--dense_folder", required=True)
    ap.add_argument("--save_folder", required=True)
    ap.add_argument("--max_d", type=int, default=192)
    ap.add_argument("--interval_scale", type=float, default=1.0)
    ap.add_argument("--model_ext", default=".txt", choices=(".txt", ".bin"))
    a = ap.parse_args(argv)
    convert(a.dense_folder, a.save_folder, a.max_d, a.interval_scale, a.model_ext)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
