"""Golden fixture of the COLMAP converter: a small synthetic COLMAP model and
the reference's own colmap2mvsnet_acm.py output for it.

Writes tests/golden/colmap/:
  dense/sparse/{cameras,images,points3D}.txt   an 8-view model of a seeded synthetic
                                               scene (PINHOLE, SIMPLE_PINHOLE and
                                               SIMPLE_RADIAL cameras; ground-truth
                                               surface points with their tracks)
  dense/images/*                               the views (.jpg copied, .png re-encoded)
  expected/cams/%08d_cam.txt, expected/pair.txt the reference converter's output

Run in the development container, where the reference sources are mounted:
    python tests/golden/make_colmap_golden.py /path/to/reference
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "colmap")


def rot_to_quat(R: np.ndarray) -> np.ndarray:
    """Unit quaternion (w, x, y, z) of a rotation matrix (Shepperd's method)."""
    t = np.trace(R)
    if t > 0:
        s = 2.0 * np.sqrt(1.0 + t)
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    else:
        k = int(np.argmax(np.diag(R)))
        i, j, l = k, (k + 1) % 3, (k + 2) % 3
        s = 2.0 * np.sqrt(1.0 + R[i, i] - R[j, j] - R[l, l])
        q = [0.0, 0.0, 0.0, 0.0]
        q[0] = (R[l, j] - R[j, l]) / s
        q[1 + i] = 0.25 * s
        q[1 + j] = (R[j, i] + R[i, j]) / s
        q[1 + l] = (R[l, i] + R[i, l]) / s
    q = np.asarray(q)
    return q / np.linalg.norm(q)


def build_model(folder: str, seed: int = 7) -> None:
    import cv2

    spec = importlib.util.spec_from_file_location("hpm_b200", os.path.join(ROOT, "hpm-mvs_plusplus_b200",
                                                                           "__init__.py"),
                                                  submodule_search_locations=[os.path.join(ROOT,
                                                                                           "hpm-mvs_plusplus_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hpm_b200"] = mod
    spec.loader.exec_module(mod)
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=8, width=96, height=72, layout="hemisphere", n_src=7, seed=seed)
    rng = np.random.default_rng(seed)
    os.makedirs(os.path.join(folder, "sparse"), exist_ok=True)
    os.makedirs(os.path.join(folder, "images"), exist_ok=True)
    # points: ground-truth surface points of random pixels, tracked into every view that sees them
    pts, tracks = [], []
    for i, v in enumerate(sc.views):
        ys, xs = np.nonzero(v.depth > 0)
        pick = rng.choice(len(xs), 60, replace=False)
        Kinv = np.linalg.inv(v.K.astype(np.float64))
        for x, y in zip(xs[pick], ys[pick]):
            Xc = v.depth[y, x] * (Kinv @ np.array([x, y, 1.0]))
            X = v.R.T.astype(np.float64) @ (Xc - v.t.astype(np.float64))
            obs = []
            for j, u in enumerate(sc.views):
                p = u.K.astype(np.float64) @ (u.R.astype(np.float64) @ X + u.t)
                if p[2] <= 0:
                    continue
                uu, vv = p[0] / p[2], p[1] / p[2]
                xi, yi = int(round(uu)), int(round(vv))
                if 0 <= xi < u.depth.shape[1] and 0 <= yi < u.depth.shape[0] and \
                        abs(u.depth[yi, xi] - p[2]) < 0.01 * p[2]:
                    obs.append((j, uu, vv))
            if len(obs) >= 2:
                pts.append(X)
                tracks.append(obs)
    models = ["PINHOLE", "SIMPLE_PINHOLE", "SIMPLE_RADIAL"]
    with open(os.path.join(folder, "sparse", "cameras.txt"), "w") as fh:
        fh.write("# Camera list with one line of data per camera:\n")
        for i, v in enumerate(sc.views):
            K = v.K.astype(np.float64)
            m = models[i % 3]
            h, w = v.image.shape[:2]
            params = {"PINHOLE": [K[0, 0], K[1, 1], K[0, 2], K[1, 2]],
                      "SIMPLE_PINHOLE": [K[0, 0], K[0, 2], K[1, 2]],
                      "SIMPLE_RADIAL": [K[0, 0], K[0, 2], K[1, 2], 0.0]}[m]
            fh.write(f"{i + 1} {m} {w} {h} " + " ".join(repr(float(p)) for p in params) + "\n")
    # image ids out of order on purpose (the converter sorts them); per image its 2D points
    obs_lists = [[] for _ in sc.views]
    for pid, obs in enumerate(tracks):
        for j, uu, vv in obs:
            obs_lists[j].append((uu, vv, pid + 1))
    ids = [10 * (i + 1) + (7 if i % 2 else 0) for i in range(len(sc.views))]
    with open(os.path.join(folder, "sparse", "images.txt"), "w") as fh:
        fh.write("# Image list with two lines of data per image:\n")
        for i, v in enumerate(sc.views):
            q = rot_to_quat(v.R.astype(np.float64))
            t = v.t.astype(np.float64)
            name = f"view_{i:02d}." + ("jpg" if i % 2 == 0 else "png")
            fh.write(f"{ids[i]} " + " ".join(repr(float(x)) for x in (*q, *t)) + f" {i + 1} {name}\n")
            entries = list(obs_lists[i]) + [(1.5, 2.5, -1)]  # a keypoint without a 3D point
            fh.write(" ".join(f"{float(u)!r} {float(w)!r} {p}" for u, w, p in entries) + "\n")
            path = os.path.join(folder, "images", name)
            if name.endswith(".jpg"):
                cv2.imwrite(path, v.image, [cv2.IMWRITE_JPEG_QUALITY, 95])
            else:
                cv2.imwrite(path, v.image)
    with open(os.path.join(folder, "sparse", "points3D.txt"), "w") as fh:
        fh.write("# 3D point list with one line of data per point:\n")
        for pid, (X, obs) in enumerate(zip(pts, tracks)):
            track = " ".join(f"{ids[j]} 0" for j, _, _ in obs)
            fh.write(f"{pid + 1} {float(X[0])!r} {float(X[1])!r} {float(X[2])!r} 128 128 128 0.5 {track}\n")


def run_reference(ref_dir: str, dense: str, out: str) -> None:
    sys.path.insert(0, ref_dir)  # importable by name: its worker processes unpickle its functions
    import colmap2mvsnet_acm as mod
    args = argparse.Namespace(dense_folder=dense, save_folder=out, max_d=192, interval_scale=1.0, theta0=5,
                              sigma1=1, sigma2=10, model_ext=".txt")
    os.makedirs(out, exist_ok=True)
    mod.processing_single_scene(args)


def main() -> None:
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HPM_REFERENCE_DIR", "")
    if not ref_dir or not os.path.isdir(ref_dir):
        raise SystemExit("usage: make_colmap_golden.py <reference source tree>")
    if os.path.isdir(OUT):
        shutil.rmtree(OUT)
    dense = os.path.join(OUT, "dense")
    build_model(dense)
    tmp = os.path.join(OUT, "_ref_out")
    run_reference(ref_dir, dense, tmp)
    exp = os.path.join(OUT, "expected")
    os.makedirs(os.path.join(exp, "cams"))
    for f in sorted(os.listdir(os.path.join(tmp, "cams"))):
        shutil.copyfile(os.path.join(tmp, "cams", f), os.path.join(exp, "cams", f))
    shutil.copyfile(os.path.join(tmp, "pair.txt"), os.path.join(exp, "pair.txt"))
    shutil.rmtree(tmp)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
