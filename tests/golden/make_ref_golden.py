"""Generates tests/golden/ref_probe.npz, ref_jbu.npz and ref_init.npz: golden
vectors of the reference's own per-pixel functions, JBU kernels and
RandomInitialization kernel (HPM.cu of HPM-MVS++, compiled from its sources by
oracle/ref_build.mk into oracle/_ref/libhpmref.so) on small seeded synthetic
scenes.

Needs a CUDA device and the reference build; run from the repository root:

    python tests/golden/make_ref_golden.py [--out tests/golden/ref_probe.npz]
                                           [--jbu-out tests/golden/ref_jbu.npz]
                                           [--init-out tests/golden/ref_init.npz]

The functions probed (HPM.cu line ranges):
  ComputeMultiViewCostVector                      490-495  per-source bilateral NCC
  ComputeMultiViewInitialCostandSelectedViews     450-488  top-k cost and view mask
  ComputeDepthfromPlaneHypothesis                 154-157
  ComputeGeomConsistencyCost                      539-564  against each source's depth map
  ComputeTexture                                  349-373
  JBU_cu, JBU_cu_prior (raw kernel output)        3037-3197 upsampling 64x48 -> 128x96
  RandomInitialization, five modes                567-763   a 64x48 view, 4 sources
  + the first one or two half-sweeps              2793-2827 photometric, geometric, mandatory, prior,
                                                            hierarchy

The scene is 5 views of 128x96 (seed 11, 4 sources).  Its grey images are
integers (stored as uint8) and its depth maps are the ground truth rounded to
1/256 (stored as uint16 counts of 1/256), so the stored inputs are exactly
the inputs the reference saw.  Textures use clamp addressing (address_mode 0),
the convention of the CUDA path and the oracle; the reference's host code
selects wrap (HPM.cpp:759-768), which changes only fetches outside the image.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import conftest  # noqa: E402  (registers hpm_b200 and hpm_oracle)

W, H, N_VIEWS, SEED = 128, 96, 5, 11
N_PROBES = 1536


def camera_frame_plane(K, R, n_world, depth, px, py):
    """(n_c, w) with n_c = R n_world and w = -n_c . X, X the camera-frame point at depth."""
    n = R @ n_world
    X = depth * np.array([(px - K[0, 2]) / K[0, 0], (py - K[1, 2]) / K[1, 1], 1.0])
    return np.array([n[0], n[1], n[2], -float(n @ X)])


def _scene():
    """The seeded scene and its views, reference first, then its sources in pair order."""
    from hpm_b200 import synth

    scene = synth.make_scene(n_views=N_VIEWS, width=W, height=H, seed=SEED, n_src=N_VIEWS - 1)
    order = [0] + [j for j, _ in scene.pairs[0]]
    return scene, [scene.views[i] for i in order]


def make_jbu_inputs() -> dict:
    """JBU inputs: the reference view's grey image (128x96) and its ground-truth
    depth (to 1/256) and normals at every second pixel (64x48; the background's
    zero normals replaced by (0, 0, -1)), one coarse depth set to NaN so the NaN
    path is exercised."""
    from hpm_b200 import synth

    _, views = _scene()
    v0 = views[0]
    coarse_d = (np.round(v0.depth[::2, ::2].astype(np.float64) * 256.0) / 256.0).astype(np.float32)
    coarse_d[5, 7] = np.nan
    coarse_n = np.ascontiguousarray(v0.normal[::2, ::2], np.float32)
    coarse_n[np.linalg.norm(coarse_n, axis=2) == 0] = (0.0, 0.0, -1.0)  # background: facing the camera
    return dict(image=synth.gray_float(v0.image).astype(np.uint8), coarse_depth=coarse_d, coarse_normal=coarse_n)


INIT_W, INIT_H, INIT_SEED, INIT_RUN_SEED = 64, 48, 12, 7
INIT_CASES = (("photometric", 0), ("geometric", 1), ("mandatory", 1 | 4 | 32), ("prior", 2), ("hierarchy", 8 | 16))
SWEEP_CASES = (("photometric", 0, 1), ("photometric", 0, 2), ("geometric", 1, 1), ("mandatory", 1 | 4 | 32, 1),
               ("prior", 2, 1), ("hierarchy", 8 | 16, 1))  # (name, mode, half-sweeps)


def make_init_inputs() -> dict:
    """RandomInitialization inputs for a 64x48 view and its four sources.  The
    previous pass's maps are the ground truth (background: depth 0.9 of the far
    limit, normal facing the camera), depths to 1/256; confidences, costs and
    prior masks are seeded random values on a 1/256 grid."""
    import cv2
    import hpm_b200
    from hpm_b200 import synth

    scene = synth.make_scene(n_views=N_VIEWS, width=INIT_W, height=INIT_H, seed=INIT_SEED, n_src=N_VIEWS - 1)
    order = [0] + [j for j, _ in scene.pairs[0]]
    views = [scene.views[i] for i in order]
    cams = [conftest.scene_cams(scene)[i] for i in order]
    dmin, dmax = hpm_b200.widened_range(cams[0])
    depths, normals = [], []
    for v in views:
        d = v.depth.astype(np.float64)
        d = np.where(d > 0, d, 0.9 * float(v.depth_max))
        depths.append((np.round(d * 256.0) / 256.0).astype(np.float32))
        n = v.normal.astype(np.float32).copy()
        n[np.linalg.norm(n, axis=2) == 0] = v.R.T.astype(np.float32) @ np.array([0, 0, -1], np.float32)
        normals.append(n)
    rng = np.random.default_rng(INIT_SEED)
    grid = lambda a: (np.round(a * 256.0) / 256.0).astype(np.float32)  # noqa: E731
    R0 = views[0].R.astype(np.float32)
    cam_normal = np.einsum("ij,hwj->hwi", R0, normals[0]).astype(np.float32)
    sub = normals[0][1::2, 1::2]
    return dict(
        images=np.stack([synth.gray_float(v.image).astype(np.uint8) for v in views]),
        canny=(cv2.Canny(views[0].image, 50, 150) > 0).astype(np.uint8),
        K=np.stack([v.K for v in views]).astype(np.float32), R=np.stack([v.R for v in views]).astype(np.float32),
        t=np.stack([v.t for v in views]).astype(np.float32),
        depth_min=np.array([v.depth_min for v in views], np.float32),
        depth_max=np.array([v.depth_max for v in views], np.float32),
        range=np.array([dmin, dmax], np.float32),
        depths=np.stack(depths), normal=normals[0],
        confidences=grid(rng.uniform(0.0, 0.6, (INIT_H, INIT_W))),
        costs=grid(rng.uniform(0.0, 0.3, (INIT_H, INIT_W))),
        prior_planes=np.concatenate([cam_normal, depths[0][..., None]], axis=2).astype(np.float32),
        plane_masks=(rng.uniform(size=(INIT_H, INIT_W)) < 0.7).astype(np.uint32),
        scaled_planes=np.concatenate([sub, grid(rng.uniform(0.0, 1.0, sub.shape[:2]))[..., None]], axis=2)
        .astype(np.float32))


def init_state(z: dict, mode: int):
    """(images, depth maps, cameras, params, RunState) of one RandomInitialization case."""
    import hpm_b200
    import hpm_oracle as ora

    images = [im.astype(np.float32) for im in z["images"]]
    cams = [hpm_b200.Camera.make(z["K"][i], z["R"][i], z["t"][i], INIT_W, INIT_H, float(z["depth_min"][i]),
                                 float(z["depth_max"][i])) for i in range(len(images))]
    params = hpm_b200.Params.make(len(images), float(z["range"][0]), float(z["range"][1]), mode)
    st = ora.RunState(INIT_W, INIT_H)
    st.canny[:] = z["canny"] * 255
    depths = None
    if mode & 1:
        depths = [d.copy() for d in z["depths"]]
    if mode & (1 | 2):
        st.planes[..., :3] = z["normal"]
        st.planes[..., 3] = z["depths"][0]
        st.costs[:] = z["costs"]
    if mode & (2 | 32):
        st.confidences[:] = z["confidences"]
    if mode & 2:
        st.prior_planes[:] = z["prior_planes"]
        st.plane_masks[:] = z["plane_masks"]
    if mode & 8:
        st.scaled_planes = z["scaled_planes"].copy()
        st.planes[..., 3] = z["depths"][0]
        params.scaled_cols, params.scaled_rows = z["scaled_planes"].shape[1], z["scaled_planes"].shape[0]
    return images, depths, cams, params, st


def make_inputs() -> dict:
    """Scene, probe pixels and planes: one third ground-truth planes, one third
    perturbed ones (normal noise 0.15, depth within 5 %), the rest random planes
    facing the camera (and every probe on the background)."""
    import cv2
    import hpm_b200
    from hpm_b200 import synth

    scene, views = _scene()
    grays = np.stack([synth.gray_float(v.image).astype(np.uint8) for v in views])
    depth_q = np.stack([np.round(v.depth.astype(np.float64) * 256.0).astype(np.uint16) for v in views])
    canny = (cv2.Canny(views[0].image, 50, 150) > 0).astype(np.uint8)
    rng = np.random.default_rng(SEED)
    v0 = views[0]
    K, R = v0.K.astype(np.float64), v0.R.astype(np.float64)
    cam0 = conftest.scene_cams(scene)[0]
    dmin, dmax = hpm_b200.widened_range(cam0)
    pix = np.stack([rng.integers(0, W, N_PROBES), rng.integers(0, H, N_PROBES)], axis=1).astype(np.int32)
    planes = np.zeros((N_PROBES, 4), np.float64)
    kind = np.zeros(N_PROBES, np.int8)  # 0 ground truth, 1 perturbed, 2 random
    for k in range(N_PROBES):
        px, py = int(pix[k, 0]), int(pix[k, 1])
        d = float(v0.depth[py, px])
        kind[k] = k % 3 if d > 0 else 2
        if kind[k] == 0:
            planes[k] = camera_frame_plane(K, R, v0.normal[py, px].astype(np.float64), d, px, py)
        elif kind[k] == 1:
            nw = v0.normal[py, px].astype(np.float64) + rng.normal(0.0, 0.15, 3)
            nw /= np.linalg.norm(nw)
            planes[k] = camera_frame_plane(K, R, nw, d * rng.uniform(0.95, 1.05), px, py)
        else:
            n = rng.normal(0.0, 1.0, 3)
            n[2] = -abs(n[2]) - 0.3
            n /= np.linalg.norm(n)
            X = rng.uniform(dmin, dmax) * np.array([(px - K[0, 2]) / K[0, 0], (py - K[1, 2]) / K[1, 1], 1.0])
            planes[k] = np.array([n[0], n[1], n[2], -float(n @ X)])
    return dict(
        images=grays, depth_q=depth_q, canny=canny,
        K=np.stack([v.K for v in views]).astype(np.float32), R=np.stack([v.R for v in views]).astype(np.float32),
        t=np.stack([v.t for v in views]).astype(np.float32),
        depth_min=np.array([v.depth_min for v in views], np.float32),
        depth_max=np.array([v.depth_max for v in views], np.float32),
        range=np.array([dmin, dmax], np.float32),
        pix=pix, planes=planes.astype(np.float32), kind=kind, address_mode=np.int32(0))


def load(path: str):
    """The stored inputs as the functions take them: (grey float images, depth
    maps, cameras, params) plus the whole archive as a dict."""
    import hpm_b200

    z = dict(np.load(path))
    images = [im.astype(np.float32) for im in z["images"]]
    depths = [(d.astype(np.float64) / 256.0).astype(np.float32) for d in z["depth_q"]]
    cams = [hpm_b200.Camera.make(z["K"][i], z["R"][i], z["t"][i], W, H, float(z["depth_min"][i]),
                                 float(z["depth_max"][i])) for i in range(len(images))]
    params = hpm_b200.Params.make(len(images), float(z["range"][0]), float(z["range"][1]))
    return images, depths, cams, params, z


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_probe.npz"))
    ap.add_argument("--jbu-out", default=os.path.join(HERE, "ref_jbu.npz"))
    ap.add_argument("--init-out", default=os.path.join(HERE, "ref_init.npz"))
    args = ap.parse_args()
    import ref_cuda

    if not ref_cuda.available():
        raise SystemExit("oracle/_ref/libhpmref.so is not built (make -C oracle -f ref_build.mk REF=<reference source tree>)")
    inputs = make_inputs()
    tmp = args.out + ".inputs.npz"
    np.savez_compressed(tmp, **inputs)
    images, depths, cams, params, z = load(tmp)
    os.remove(tmp)
    out = ref_cuda.probe(images, depths, cams, params, z["canny"].astype(np.uint32), z["pix"], z["planes"],
                         address_mode=int(z["address_mode"]))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez_compressed(args.out, **inputs, **{"ref_" + k: v for k, v in out.items()})
    print(f"wrote {args.out}: {len(z['pix'])} probes, {len(images) - 1} sources")
    j = make_jbu_inputs()
    img = j["image"].astype(np.float32)
    jbu_depth = ref_cuda.jbu(img, j["coarse_depth"])
    prior_depth, prior_normal = ref_cuda.jbu(img, j["coarse_depth"], j["coarse_normal"])
    np.savez_compressed(args.jbu_out, **j, ref_jbu_depth=jbu_depth, ref_jbu_prior_depth=prior_depth,
                        ref_jbu_prior_normal=prior_normal)
    print(f"wrote {args.jbu_out}: {img.shape[1]}x{img.shape[0]} from "
          f"{j['coarse_depth'].shape[1]}x{j['coarse_depth'].shape[0]}")
    zi = make_init_inputs()
    outs = {}
    for name, mode in INIT_CASES:
        images, depths, cams, params, st = init_state(zi, mode)
        ref_cuda.random_init(images, depths, cams, params, st, INIT_RUN_SEED, 0)
        outs.update({f"ref_{name}_planes": st.planes, f"ref_{name}_costs": st.costs,
                     f"ref_{name}_selected": st.selected_views})
        if not mode & (2 | 32):
            outs[f"ref_{name}_texture"] = st.texture
        if mode & 32:
            outs[f"ref_{name}_confidences"] = st.confidences
    for name, mode, n_half in SWEEP_CASES:
        images, depths, cams, params, st = init_state(zi, mode)
        ref_cuda.random_init(images, depths, cams, params, st, INIT_RUN_SEED, 0, n_half=n_half)
        outs.update({f"ref_{name}_h{n_half}_planes": st.planes, f"ref_{name}_h{n_half}_costs": st.costs,
                     f"ref_{name}_h{n_half}_selected": st.selected_views})
    np.savez_compressed(args.init_out, **zi, **outs)
    print(f"wrote {args.init_out}: {len(INIT_CASES)} modes at {INIT_W}x{INIT_H}")


if __name__ == "__main__":
    main()
