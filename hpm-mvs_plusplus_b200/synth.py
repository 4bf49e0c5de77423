"""Seeded synthetic multi-view scenes with ground truth (stand-ins for real data).

A scene is a textured ground plane, five random planar patches and an
axis-aligned box (six planes plus a box), ray-cast into pinhole views.  Texture
is band-limited noise attached to each surface (so it is consistent across
views) plus per-view Gaussian noise; the views are 8-bit grey replicated into
BGR.  Cameras follow the reference's conventions: x_cam = R x_world + t,
K = [[f, 0, cx], [0, f, cy], [0, 0, 1]], depth range from the scene bounds in
each cam file (HPM.cpp:159-184).

Layouts:
  * `arc`        -- views on an arc of `arc_deg` degrees at distance 4, all looking
                    at the scene centre (the 5-view 1280x960 configuration);
  * `hemisphere` -- two rings plus a top view (the 49-view configuration);
  * `mixed`      -- several rings with uneven resolutions (the 120-view one).
`textureless_frac` > 0 flattens that fraction of surfaces to texture std <= 2.

Rendering uses torch on any device; the same seed gives the same scene.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch


@dataclass
class SceneView:
    image: np.ndarray          # H x W x 3 uint8 (BGR, grey replicated)
    K: np.ndarray              # 3x3 float32
    R: np.ndarray              # 3x3 float32
    t: np.ndarray              # 3 float32
    depth: np.ndarray          # H x W float32 ground truth (0 = background)
    normal: np.ndarray         # H x W x 3 world normals
    depth_min: float
    depth_max: float


@dataclass
class Scene:
    views: List[SceneView]
    pairs: List[List[tuple]]   # per view: [(src_id, score), ...] sorted by score
    seed: int
    meta: dict = field(default_factory=dict)


def _bandlimited_texture(rng: np.random.Generator, size: int, lo: float, hi: float) -> np.ndarray:
    """Noise with spatial frequencies in [lo, hi] cycles/texel, scaled to 0..1."""
    white = rng.standard_normal((size, size))
    f = np.fft.fftfreq(size)
    fx, fy = np.meshgrid(f, f)
    r = np.sqrt(fx * fx + fy * fy)
    band = ((r >= lo) & (r <= hi)).astype(np.float64)
    tex = np.real(np.fft.ifft2(np.fft.fft2(white) * band))
    tex -= tex.min()
    tex /= max(tex.max(), 1e-12)
    return tex.astype(np.float32)


def _look_at(C: np.ndarray, target: np.ndarray) -> tuple:
    z = target - C
    z = z / np.linalg.norm(z)
    down = np.array([0.0, -1.0, 0.0])
    x = np.cross(down, z)
    if np.linalg.norm(x) < 1e-6:
        x = np.array([1.0, 0.0, 0.0])
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z]).astype(np.float64)
    t = -R @ C
    return R, t


def _camera_centres(layout: str, n_views: int, radius: float, arc_deg: float) -> np.ndarray:
    if layout == "arc":
        az = np.deg2rad(np.linspace(-arc_deg / 2, arc_deg / 2, n_views))
        el = np.deg2rad(25.0)
        return np.stack([radius * np.cos(el) * np.sin(az), np.full_like(az, radius * np.sin(el)),
                         radius * np.cos(el) * np.cos(az)], 1)
    if layout in ("hemisphere", "mixed"):
        rings = [(20.0, 0.5), (45.0, 0.5)] if layout == "hemisphere" else [(15.0, 1 / 3), (35.0, 1 / 3), (55.0, 1 / 3)]
        n_top = 1 if layout == "hemisphere" else 0
        n_ring = n_views - n_top
        counts = [int(round(n_ring * w)) for _, w in rings]
        counts[-1] = n_ring - sum(counts[:-1])
        out = []
        for (el_deg, _), cnt in zip(rings, counts):
            el = np.deg2rad(el_deg)
            for k in range(cnt):
                a = 2 * np.pi * k / cnt + (0.13 if el_deg > 30 else 0.0)
                out.append([radius * np.cos(el) * np.sin(a), radius * np.sin(el), radius * np.cos(el) * np.cos(a)])
        if n_top:
            out.append([0.05, radius, 0.0])
        return np.asarray(out, np.float64)
    raise ValueError(layout)


class _Primitive:
    def __init__(self, kind: str, **kw):
        self.kind = kind
        self.__dict__.update(kw)


def _make_primitives(rng: np.random.Generator, textureless_frac: float, n_boxes: int = 1,
                     box_spread: float = 1.0) -> list:
    prims = []
    tex_size = 512
    # ground plane y = 0 over [-3, 3]^2
    prims.append(_Primitive("rect", c=np.array([0.0, 0.0, 0.0]), u=np.array([1.0, 0.0, 0.0]),
                            v=np.array([0.0, 0.0, 1.0]), a=3.0, b=3.0, tscale=3.0))
    for _ in range(5):
        c = np.array([rng.uniform(-1.1, 1.1), rng.uniform(0.25, 0.9), rng.uniform(-1.1, 1.1)])
        n = rng.standard_normal(3)
        n[1] = abs(n[1]) * 0.6
        n /= np.linalg.norm(n)
        u = np.cross(n, np.array([0.0, 1.0, 0.0]))
        if np.linalg.norm(u) < 1e-3:
            u = np.array([1.0, 0.0, 0.0])
        u /= np.linalg.norm(u)
        v = np.cross(n, u)
        prims.append(_Primitive("rect", c=c, u=u, v=v, a=rng.uniform(0.25, 0.5), b=rng.uniform(0.2, 0.45),
                                tscale=1.0))
    for _ in range(n_boxes):
        half = np.array([rng.uniform(0.15, 0.35), rng.uniform(0.15, 0.4), rng.uniform(0.15, 0.35)])
        c = np.array([rng.uniform(-box_spread, box_spread), half[1], rng.uniform(-box_spread, box_spread)])
        prims.append(_Primitive("box", c=c, half=half, tscale=1.0))
    for p in prims:
        p.tex = _bandlimited_texture(rng, tex_size, 0.012, 0.06)
        p.lo, p.hi = 40.0, 215.0
        if textureless_frac > 0 and rng.uniform() < textureless_frac:
            p.lo, p.hi = 126.0, 130.0  # std <= 2 grey levels
    return prims


def _sample_tex(tex: torch.Tensor, u: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """Bilinear lookup with wrap-around; u, v in texture units (texels)."""
    S = tex.shape[0]
    u = torch.remainder(u, S)
    v = torch.remainder(v, S)
    x0 = torch.floor(u)
    y0 = torch.floor(v)
    fx = u - x0
    fy = v - y0
    x0 = x0.long() % S
    y0 = y0.long() % S
    x1 = (x0 + 1) % S
    y1 = (y0 + 1) % S
    t00 = tex[y0, x0]
    t10 = tex[y0, x1]
    t01 = tex[y1, x0]
    t11 = tex[y1, x1]
    return (t00 * (1 - fx) + t10 * fx) * (1 - fy) + (t01 * (1 - fx) + t11 * fx) * fy


def render_view(prims, K, R, t, W, H, noise_rng: np.random.Generator, device, supersample: int = 2,
                ids_only: bool = False):
    """Grey image, depth and normals of one view; with ids_only, the index of the primitive seen at each
    pixel (-1: background) instead."""
    dev = torch.device(device)
    dt = torch.float64
    Kt = torch.tensor(K, dtype=dt, device=dev)
    Rt = torch.tensor(R, dtype=dt, device=dev)
    tt = torch.tensor(t, dtype=dt, device=dev)
    C = -(Rt.T @ tt)
    ss = supersample
    ys, xs = torch.meshgrid(torch.arange(H * ss, device=dev, dtype=dt), torch.arange(W * ss, device=dev, dtype=dt),
                            indexing="ij")
    px = (xs + 0.5) / ss - 0.5
    py = (ys + 0.5) / ss - 0.5
    dirs_cam = torch.stack([(px - Kt[0, 2]) / Kt[0, 0], (py - Kt[1, 2]) / Kt[1, 1], torch.ones_like(px)], -1)
    dirs = dirs_cam @ Rt  # world direction (not normalised; z_cam component = 1)
    best_t = torch.full(px.shape, float("inf"), dtype=dt, device=dev)
    val = torch.zeros(px.shape, dtype=dt, device=dev)
    nrm = torch.zeros(px.shape + (3,), dtype=dt, device=dev)
    pid = torch.full(px.shape, -1, dtype=torch.int32, device=dev)
    for pi, p in enumerate(prims):
        tex = torch.tensor(p.tex, dtype=dt, device=dev)
        S = p.tex.shape[0]
        if p.kind == "rect":
            n = np.cross(p.u, p.v)
            nt = torch.tensor(n, dtype=dt, device=dev)
            denom = dirs @ nt
            tt_ = ((torch.tensor(p.c, dtype=dt, device=dev) - C) @ nt) / denom
            X = C + dirs * tt_[..., None]
            rel = X - torch.tensor(p.c, dtype=dt, device=dev)
            uu = rel @ torch.tensor(p.u, dtype=dt, device=dev)
            vv = rel @ torch.tensor(p.v, dtype=dt, device=dev)
            hit = (tt_ > 1e-6) & (uu.abs() <= p.a) & (vv.abs() <= p.b) & (tt_ < best_t)
            scale = S / (2.0 * p.tscale)
            g = _sample_tex(tex, uu * scale, vv * scale)
            q = getattr(p, "flat_q", 0.0)
            if q > 0:  # textureless stripes two scene units apart, a share q of the surface
                g = torch.where(torch.remainder(uu, 2.0) < 2.0 * q, torch.full_like(g, 0.5), g)
            g = p.lo + (p.hi - p.lo) * g
            best_t = torch.where(hit, tt_, best_t)
            val = torch.where(hit, g, val)
            pid = torch.where(hit, torch.full_like(pid, pi), pid)
            face_n = nt.expand_as(nrm)
            nrm = torch.where(hit[..., None], face_n, nrm)
        else:  # axis-aligned box, slab test
            c = torch.tensor(p.c, dtype=dt, device=dev)
            h = torch.tensor(p.half, dtype=dt, device=dev)
            inv = 1.0 / torch.where(dirs.abs() < 1e-12, torch.full_like(dirs, 1e-12), dirs)
            t1 = (c - h - C) * inv
            t2 = (c + h - C) * inv
            tmin = torch.minimum(t1, t2)
            tmax = torch.maximum(t1, t2)
            tn, axis = tmin.max(-1)
            tf = tmax.min(-1).values
            hit = (tn <= tf) & (tn > 1e-6) & (tn < best_t)
            X = C + dirs * tn[..., None]
            rel = X - c
            sign = torch.sign(torch.gather(rel, -1, axis[..., None]))[..., 0]
            fn = torch.nn.functional.one_hot(axis, 3).to(dt) * sign[..., None]
            # texture coordinates: the two axes other than the face axis
            a0 = torch.where(axis == 0, rel[..., 1], rel[..., 0])
            a1 = torch.where(axis == 2, rel[..., 1], rel[..., 2])
            scale = S / 2.0
            g = _sample_tex(tex, a0 * scale + 37.0 * axis, a1 * scale + 91.0 * (sign > 0))
            g = p.lo + (p.hi - p.lo) * g
            best_t = torch.where(hit, tn, best_t)
            val = torch.where(hit, g, val)
            pid = torch.where(hit, torch.full_like(pid, pi), pid)
            nrm = torch.where(hit[..., None], fn, nrm)
    if ids_only:
        return pid[ss // 2::ss, ss // 2::ss].cpu().numpy()
    bg = torch.isinf(best_t)
    val = torch.where(bg, torch.full_like(val, 200.0), val)
    # orient normals toward the camera, as PatchMatch hypotheses are
    facing = (nrm * dirs).sum(-1) > 0
    nrm = torch.where(facing[..., None], -nrm, nrm)
    # supersample average
    val = val.reshape(H, ss, W, ss).mean(dim=(1, 3))
    depth_ss = torch.where(bg, torch.zeros_like(best_t), best_t)  # t is the camera-z depth (dirs_cam z = 1)
    depth = depth_ss[ss // 2::ss, ss // 2::ss]
    normal = nrm[ss // 2::ss, ss // 2::ss]
    img = val.cpu().numpy()
    img = img + noise_rng.normal(0.0, 2.0, size=img.shape)
    img = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    return img, depth.cpu().numpy().astype(np.float32), normal.cpu().numpy().astype(np.float32)


def _flatten_to_area(prims, cams, target: float, device) -> float:
    """Makes primitives textureless (std <= 2 grey levels), largest image area first, until they cover about
    `target` of all views' pixels (measured on 160-pixel-wide renders); returns the covered fraction."""
    counts = np.zeros(len(prims))
    total = 0
    for K, R, t, W, H in cams:
        s = 160.0 / W
        Ks = K.copy()
        Ks[:2] *= s
        w, h = 160, max(1, int(round(H * s)))
        ids = render_view(prims, Ks, R, t, w, h, None, device, 1, ids_only=True)
        total += ids.size
        for k in range(len(prims)):
            counts[k] += int((ids == k).sum())
    frac = counts / max(total, 1)
    # the ground plane (primitive 0) in flat stripes of the share that reaches the target, then other
    # surfaces largest first if the whole ground is not enough
    g = float(frac[0])
    q = min(1.0, target / g) if g > 0 else 0.0
    prims[0].flat_q = q
    covered = g * q
    for k in [int(k) for k in np.argsort(-frac) if k != 0]:
        if covered + frac[k] <= target + 0.02 and covered < target - 0.02:
            prims[k].lo, prims[k].hi = 126.0, 130.0
            covered += frac[k]
    return float(covered)


def _saturate(img: np.ndarray, frac: float, rng: np.random.Generator) -> np.ndarray:
    """Specular-like highlights: soft elliptical blobs clipped to 255 over about `frac` of the pixels, placed
    independently in every view (view-dependent, as specular reflections are)."""
    H, W = img.shape
    out = img.astype(np.float32)
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float32)
    target = frac * H * W
    sat = np.zeros((H, W), bool)
    while sat.sum() < target:
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        ax, ay = rng.uniform(0.01, 0.04) * W, rng.uniform(0.01, 0.04) * W
        r2 = ((xs - cx) / ax) ** 2 + ((ys - cy) / ay) ** 2
        blob = r2 < 1.0
        out = np.where(r2 < 1.6, np.maximum(out, 255.0 * (1.6 - r2) / 0.6), out)
        sat |= blob
    return np.clip(np.rint(out), 0, 255).astype(np.uint8)


def make_scene(n_views: int = 5, width: int = 1280, height: int = 960, layout: str = "arc", arc_deg: float = 30.0,
               n_src: int = 4, seed: int = 0, textureless_frac: float = 0.0, device: str = "cpu",
               sizes: Optional[Sequence[tuple]] = None, supersample: int = 2, n_boxes: int = 1,
               textureless_area: float = 0.0, saturated_frac: float = 0.0, box_spread: float = 1.0) -> Scene:
    """Render a seeded scene; `sizes` gives per-view (W, H) for uneven resolutions.  textureless_area: the
    share of image area to make textureless (std <= 2 grey levels); saturated_frac: the share of every view
    covered by saturated specular-like highlights; box_spread: boxes are placed in [-spread, spread]^2."""
    rng = np.random.default_rng(seed)
    prims = _make_primitives(rng, textureless_frac, n_boxes, box_spread)
    centres = _camera_centres(layout, n_views, 4.0, arc_deg)
    target = np.array([0.0, 0.3, 0.0])
    cams = []
    for i, C in enumerate(centres):
        W, H = (sizes[i] if sizes is not None else (width, height))
        R, t = _look_at(C, target)
        f = 0.9 * W
        K = np.array([[f, 0.0, (W - 1) / 2.0], [0.0, f, (H - 1) / 2.0], [0.0, 0.0, 1.0]])
        cams.append((K, R, t, W, H))
    flat_area = _flatten_to_area(prims, cams, textureless_area, device) if textureless_area > 0 else 0.0
    views = []
    for i, (K, R, t, W, H) in enumerate(cams):
        noise_rng = np.random.default_rng(seed * 1000003 + i)
        gray, depth, normal = render_view(prims, K, R, t, W, H, noise_rng, device, supersample)
        if saturated_frac > 0:
            gray = _saturate(gray, saturated_frac, np.random.default_rng(seed * 7919 + i))
        img = np.repeat(gray[..., None], 3, axis=2)
        valid = depth[depth > 0]
        views.append(SceneView(img, K.astype(np.float32), R.astype(np.float32), t.astype(np.float32), depth, normal,
                               float(valid.min()) if valid.size else 1.0, float(valid.max()) if valid.size else 10.0))
    # global depth range from the scene bounds
    dmin = min(v.depth_min for v in views)
    dmax = max(v.depth_max for v in views)
    for v in views:
        v.depth_min, v.depth_max = dmin, dmax
    # pair list: neighbours by viewing-direction angle, score = 1 / (1 + angle in degrees)
    pairs = []
    dirs = [-(v.R.T @ v.t) for v in views]
    for i in range(n_views):
        cand = []
        for j in range(n_views):
            if j == i:
                continue
            ci, cj = dirs[i] - target, dirs[j] - target
            ang = math.degrees(math.acos(np.clip(np.dot(ci, cj) / (np.linalg.norm(ci) * np.linalg.norm(cj)), -1, 1)))
            cand.append((j, 100.0 / (1.0 + ang)))
        cand.sort(key=lambda x: -x[1])
        pairs.append(cand[:n_src])
    return Scene(views, pairs, seed, {"layout": layout, "n_views": n_views, "textureless_frac": textureless_frac,
                                      "textureless_area": flat_area, "saturated_frac": saturated_frac})


# The five workloads of the benchmark, at their full sizes (seeded).
CONFIGS = {
    "c1": "5 views 1280x960 on a 30-degree arc, 4 sources, --initial-image-scale 4",
    "c2": "49 views 1600x1200 on a two-ring hemisphere, 10 sources, --initial-image-scale 1",
    "c3": "49 views 1600x1200 hemisphere, 10 sources, about 40 % of the image area textureless (std <= 2)",
    "c4": "20 views 1024x768 on a two-ring hemisphere, 10 sources, --initial-image-scale 1",
    "c5": "120 views of uneven sizes (40 x 3072x2048, 40 x 1920x1080, 40 x 1024x768), ground plane and 30 boxes, "
          "5 % saturated specular-like patches, 10 sources",
}


def make_config(name: str, seed: int = 2024, device: str = "cpu", n_views: Optional[int] = None) -> Scene:
    """The scene of workload `name` (c1..c5); n_views overrides the view count (c5 keeps its size mix)."""
    if name == "c1":
        return make_scene(n_views=n_views or 5, width=1280, height=960, layout="arc", n_src=4, seed=seed,
                          device=device)
    if name == "c2":
        return make_scene(n_views=n_views or 49, width=1600, height=1200, layout="hemisphere", n_src=10, seed=seed,
                          device=device)
    if name == "c3":
        return make_scene(n_views=n_views or 49, width=1600, height=1200, layout="hemisphere", n_src=10, seed=seed,
                          device=device, textureless_area=0.4)
    if name == "c4":
        return make_scene(n_views=n_views or 20, width=1024, height=768, layout="hemisphere", n_src=10, seed=seed,
                          device=device)
    if name == "c5":
        n = n_views or 120
        mix = [(3072, 2048), (1920, 1080), (1024, 768)]
        sizes = [mix[i % 3] for i in range(n)]
        return make_scene(n_views=n, layout="mixed", n_src=min(10, n - 1), seed=seed, device=device, sizes=sizes,
                          n_boxes=30, box_spread=2.5, saturated_frac=0.05)
    raise ValueError(f"unknown workload {name!r} (c1..c5)")


def write_dense_folder(scene: Scene, folder: str) -> None:
    """images/%08d.jpg (PNG bytes, lossless), cams/%08d_cam.txt, pair.txt (main.cpp:171-200)."""
    import cv2  # only for PNG encoding of the test scene

    os.makedirs(os.path.join(folder, "images"), exist_ok=True)
    os.makedirs(os.path.join(folder, "cams"), exist_ok=True)
    for i, v in enumerate(scene.views):
        ok, buf = cv2.imencode(".png", v.image)
        assert ok
        with open(os.path.join(folder, "images", f"{i:08d}.jpg"), "wb") as fh:
            fh.write(buf.tobytes())
        write_cam(os.path.join(folder, "cams", f"{i:08d}_cam.txt"), v)
    with open(os.path.join(folder, "pair.txt"), "w") as fh:
        fh.write(f"{len(scene.views)}\n")
        for i, pl in enumerate(scene.pairs):
            fh.write(f"{i}\n{len(pl)} " + " ".join(f"{j} {s:.6f}" for j, s in pl) + "\n")


def write_cam(path: str, v: SceneView) -> None:
    with open(path, "w") as fh:
        fh.write("extrinsic\n")
        for r in range(3):
            fh.write(" ".join(f"{v.R[r, c]:.9g}" for c in range(3)) + f" {v.t[r]:.9g}\n")
        fh.write("0 0 0 1\n\nintrinsic\n")
        for r in range(3):
            fh.write(" ".join(f"{v.K[r, c]:.9g}" for c in range(3)) + "\n")
        interval = (v.depth_max - v.depth_min) / 192.0
        fh.write(f"\n{v.depth_min:.9g} {interval:.9g} 192 {v.depth_max:.9g}\n")


def gray_float(img_bgr: np.ndarray) -> np.ndarray:
    """cv::cvtColor(BGR2GRAY) for 8-bit input followed by convertTo(CV_32F) (HPM.cpp:660-661)."""
    b = img_bgr[..., 0].astype(np.int64)
    g = img_bgr[..., 1].astype(np.int64)
    r = img_bgr[..., 2].astype(np.int64)
    return ((b * 1868 + g * 9617 + r * 4899 + (1 << 13)) >> 14).astype(np.float32)
