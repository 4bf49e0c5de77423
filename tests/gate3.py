"""Per-run agreement of two PatchMatch results from identical inputs (test helper).

The end-to-end accuracy gate compares depth maps pixel by pixel: a pixel agrees
when its depths are within 0.5 % of each other and its normals within 2 degrees.
Every pixel that does not agree is put in the first class that describes it:

  garbage     the reference wrote a non-unit normal or a non-finite depth: its
              uninitialised plane_hypotheses_now (HPM.cu:1844-1871) when the
              minimum-cost direction lies outside the image
  band        within 6 pixels of the image border, where that happens
  edge_on     either plane is within 6 degrees of containing the pixel's ray:
              the homography is nearly singular and the NCC ill-conditioned
  flat        the reference patch is flat (11 x 11 grey standard deviation < 4,
              i.e. sensor noise only): no texture decides the depth
  unresolved  neither result is within 1 % of the true depth: PatchMatch found
              no stable answer and rounding picked one of several
  surface     both results are within 1 % of the true depth: two points of the
              same surface, apart by refinement noise
  unexplained the rest -- one result on the surface and the other not
"""
from __future__ import annotations

import math

import numpy as np

CLASSES = ("garbage", "band", "edge_on", "flat", "unresolved", "surface", "unexplained")
DEPTH_TOL = 0.005
ANGLE_TOL_DEG = 2.0
BAND = 6
EDGE_ON_DEG = 6.0
FLAT_STD = 4.0
GT_TOL = 0.01


def local_std(gray: np.ndarray, radius: int = 5) -> np.ndarray:
    """Standard deviation of the (2r+1)^2 window around every pixel (edge-replicated)."""
    g = np.asarray(gray, np.float64)
    k = 2 * radius + 1
    p = np.pad(g, radius, mode="edge")
    c1 = np.pad(np.cumsum(np.cumsum(p, 0), 1), ((1, 0), (1, 0)))
    c2 = np.pad(np.cumsum(np.cumsum(p * p, 0), 1), ((1, 0), (1, 0)))
    H, W = g.shape

    def box(c):
        return c[k:k + H, k:k + W] - c[:H, k:k + W] - c[k:k + H, :W] + c[:H, :W]

    n = k * k
    m = box(c1) / n
    return np.sqrt(np.maximum(box(c2) / n - m * m, 0.0))


def view_rays(cam, W: int, H: int) -> np.ndarray:
    """Unit viewing rays in the world frame, H x W x 3 (R^T K^-1 (x, y, 1))."""
    K = np.asarray(cam.K[:], np.float64).reshape(3, 3)
    R = np.asarray(cam.R[:], np.float64).reshape(3, 3)
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float64)
    d = np.stack([(xs - K[0, 2]) / K[0, 0], (ys - K[1, 2]) / K[1, 1], np.ones_like(xs)], -1)
    d = d @ R  # (R^T d) row-wise
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


def classify(d_ref, n_ref, d_ours, n_ours, gray, cam, gt_depth=None) -> dict:
    """Counts of agreeing pixels and of each disagreement class (all pixels of the map)."""
    d_ref = np.asarray(d_ref, np.float64)
    d_ours = np.asarray(d_ours, np.float64)
    n_ref = np.asarray(n_ref, np.float64)
    n_ours = np.asarray(n_ours, np.float64)
    H, W = d_ref.shape
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        rel = np.abs(d_ours - d_ref) / np.abs(d_ref)
        nr = np.linalg.norm(n_ref, axis=-1)
        no = np.linalg.norm(n_ours, axis=-1)
        cosang = np.sum(n_ref * n_ours, -1) / (nr * no)
        ang = np.degrees(np.arccos(np.clip(cosang, -1.0, 1.0)))
    agree = (rel <= DEPTH_TOL) & (ang <= ANGLE_TOL_DEG)
    left = ~agree
    out = {"pixels": int(H * W), "agree": int(agree.sum())}
    garbage = left & (~np.isfinite(d_ref) | (np.abs(nr - 1.0) > 1e-3) | ~np.isfinite(nr))
    out["garbage"] = int(garbage.sum())
    left &= ~garbage
    ys, xs = np.mgrid[0:H, 0:W]
    band = (xs < BAND) | (ys < BAND) | (xs >= W - BAND) | (ys >= H - BAND)
    out["band"] = int((left & band).sum())
    left &= ~band
    rays = view_rays(cam, W, H)
    with np.errstate(invalid="ignore", divide="ignore"):
        c_ref = np.abs(np.sum(rays * n_ref, -1)) / nr
        c_ours = np.abs(np.sum(rays * n_ours, -1)) / no
    s = math.sin(math.radians(EDGE_ON_DEG))
    edge = (c_ref < s) | (c_ours < s)
    out["edge_on"] = int((left & edge).sum())
    left &= ~edge
    flat = local_std(gray) < FLAT_STD
    out["flat"] = int((left & flat).sum())
    left &= ~flat
    if gt_depth is not None:
        gt = np.asarray(gt_depth, np.float64)
        with np.errstate(invalid="ignore", divide="ignore"):
            on_ref = (gt > 0) & (np.abs(d_ref - gt) <= GT_TOL * gt)
            on_ours = (gt > 0) & (np.abs(d_ours - gt) <= GT_TOL * gt)
        unres = left & ~on_ref & ~on_ours
        out["unresolved"] = int(unres.sum())
        left &= ~unres
        surf = left & on_ref & on_ours
        out["surface"] = int(surf.sum())
        left &= ~surf
    else:
        out["unresolved"] = out["surface"] = 0
    out["unexplained"] = int(left.sum())
    return out


def add(total: dict, part: dict) -> dict:
    for k, v in part.items():
        total[k] = total.get(k, 0) + v
    return total


def fractions(c: dict) -> dict:
    n = max(c.get("pixels", 0), 1)
    return {k: c.get(k, 0) / n for k in ("agree",) + CLASSES}


def table(rows: dict, title: str) -> str:
    """Markdown table: one row per mode, shares of all pixels."""
    head = "| mode | pixels | agree | " + " | ".join(CLASSES) + " |"
    sep = "|" + "---|" * (3 + len(CLASSES))
    lines = [title, "", head, sep]
    for mode, c in rows.items():
        f = fractions(c)
        lines.append(f"| {mode} | {c['pixels']} | {100 * f['agree']:.2f} % | " +
                     " | ".join(f"{100 * f[k]:.2f} %" for k in CLASSES) + " |")
    return "\n".join(lines)
