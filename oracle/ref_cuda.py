"""REFERENCE BUILD wrapper -- test infrastructure only.

ctypes binding of oracle/_ref/libhpmref.so: the reference's own CUDA kernels
(HPM.cu of HPM-MVS++, compiled from its sources for sm_100a by
oracle/ref_build.mk with its own --use_fast_math flags) driven through
HPM::RunPatchMatch (HPM.cu:2987-3035).  Random draws are the shared Philox
stream, so the reference build, the CPU oracle and the CUDA path start from the
same hypotheses.  The library is built in the development container (the
reference sources are read there) and travels prebuilt; where it is absent the
callers skip.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import hpm_oracle as ora

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libhpmref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        _lib.ref_run_patchmatch.restype = ctypes.c_int
        _lib.ref_run_patchmatch.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(ora.Params), vp, vp, vp, vp, vp,
                                            vp, vp, vp, vp, ctypes.c_uint64, ctypes.c_uint32,
                                            ctypes.POINTER(ctypes.c_float)]
        _lib.ref_random_init.restype = ctypes.c_int
        _lib.ref_random_init.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(ora.Params), vp, vp, vp, vp, vp, vp,
                                         vp, vp, vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, vp]
        _lib.ref_jbu.restype = ctypes.c_int
        _lib.ref_jbu.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
        _lib.ref_probe.restype = ctypes.c_int
        _lib.ref_probe.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(ora.Params), vp, vp, vp, ctypes.c_int,
                                   ctypes.c_int, vp, vp, vp, vp, vp, vp]
    return _lib


def _depth_list(depths, imgs):
    """One depth map per view, each of its image's size: the driver uploads
    every entry as a full-size array, so a missing map becomes zeros."""
    out = []
    for i, img in enumerate(imgs):
        d = None if depths is None else depths[i]
        d = np.zeros(img.shape, np.float32) if d is None else np.ascontiguousarray(d, np.float32)
        if d.shape != img.shape:
            raise ValueError(f"depth map {i} has shape {d.shape}, its image {img.shape}")
        out.append(d)
    return out


def _ptrs(arrs):
    return (ctypes.c_void_p * len(arrs))(*[None if a is None else a.ctypes.data for a in arrs])


def run_patchmatch(images, depths, cams, params, st: "ora.RunState", seed: int, view_id: int) -> float:
    """Same arguments and state as hpm_oracle.run_patchmatch; returns the run's device time in ms."""
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    deps = _depth_list(depths, imgs)
    cam_arr = (ora.Camera * len(cams))(*[ora.to_cam(c) for c in cams])
    prm = ora.to_params(params)
    canny = np.ascontiguousarray(st.canny, np.uint32)
    scaled = np.ascontiguousarray(st.scaled_planes, np.float32)
    ms = ctypes.c_float(0.0)
    rc = lib().ref_run_patchmatch(_ptrs(imgs), cam_arr, len(imgs), ctypes.byref(prm), st.planes.ctypes.data,
                                  st.costs.ctypes.data, scaled.ctypes.data, st.prior_planes.ctypes.data,
                                  st.plane_masks.ctypes.data, st.confidences.ctypes.data, canny.ctypes.data,
                                  st.texture.ctypes.data, _ptrs(deps), ctypes.c_uint64(seed), view_id,
                                  ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference build: CUDA error {rc}")
    return float(ms.value)


def random_init(images, depths, cams, params, st: "ora.RunState", seed: int, view_id: int,
                n_half: int = 0) -> None:
    """The reference's RandomInitialization kernel (HPM.cu:567-763), followed by
    its first n_half half-sweeps (Black, Red, ...; HPM.cu:2793-2827), on the
    same arguments and state as hpm_oracle.random_init: fills st.planes (camera
    frame), st.costs, st.selected_views, st.confidences and, outside the prior
    and mandatory modes, st.texture."""
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    deps = _depth_list(depths, imgs)
    cam_arr = (ora.Camera * len(cams))(*[ora.to_cam(c) for c in cams])
    prm = ora.to_params(params)
    canny = np.ascontiguousarray(st.canny, np.uint32)
    scaled = np.ascontiguousarray(st.scaled_planes, np.float32)
    rc = lib().ref_random_init(_ptrs(imgs), cam_arr, len(imgs), ctypes.byref(prm), st.planes.ctypes.data,
                               st.costs.ctypes.data, scaled.ctypes.data, st.prior_planes.ctypes.data,
                               st.plane_masks.ctypes.data, st.confidences.ctypes.data, canny.ctypes.data,
                               st.texture.ctypes.data, _ptrs(deps), ctypes.c_uint64(seed), view_id, n_half,
                               st.selected_views.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference build: RandomInitialization failed ({rc})")


def probe(images, depths, cams, params, canny, pix, planes, address_mode: int = 0) -> dict:
    """The reference's own per-pixel functions at given (pixel, camera-frame plane)
    pairs: ComputeMultiViewCostVector, ComputeMultiViewInitialCostandSelectedViews,
    ComputeDepthfromPlaneHypothesis, ComputeGeomConsistencyCost against every
    source's depth map and ComputeTexture (HPM.cu:154-564).  address_mode 0 =
    clamp, 1 = wrap for the image and depth textures."""
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    deps = [np.ascontiguousarray(d, np.float32) for d in depths]
    cam_arr = (ora.Camera * len(cams))(*[ora.to_cam(c) for c in cams])
    prm = ora.to_params(params)
    can = np.ascontiguousarray(canny, np.uint32)
    px = np.ascontiguousarray(pix, np.int32).reshape(-1, 2)
    pl = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
    n = px.shape[0]
    out = {"cost_vec": np.zeros((n, 32), np.float32), "init_cost": np.zeros(n, np.float32),
           "selected": np.zeros(n, np.uint32), "depth": np.zeros(n, np.float32),
           "geom": np.zeros((n, 32), np.float32), "texture": np.zeros(n, np.float32)}
    rc = lib().ref_probe(_ptrs(imgs), _ptrs(deps), cam_arr, len(imgs), ctypes.byref(prm), can.ctypes.data,
                         px.ctypes.data, pl.ctypes.data, n, address_mode, out["cost_vec"].ctypes.data,
                         out["init_cost"].ctypes.data, out["selected"].ctypes.data, out["depth"].ctypes.data,
                         out["geom"].ctypes.data, out["texture"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference build: probe failed ({rc})")
    S = len(imgs) - 1
    out["cost_vec"] = out["cost_vec"][:, :S].copy()
    out["geom"] = out["geom"][:, :S].copy()
    return out


def jbu(image, src_depth, src_normal=None):
    """Raw output of the reference's JBU_cu (src_normal None) or JBU_cu_prior
    (HPM.cu:3037-3197): the upsampled depth, and for the prior kernel the
    normalised normals (H x W x 3)."""
    img = np.ascontiguousarray(image, np.float32)
    sd = np.ascontiguousarray(src_depth, np.float32)
    sn = None if src_normal is None else np.ascontiguousarray(src_normal, np.float32)
    H, W = img.shape
    sh, sw = sd.shape
    od = np.zeros((H, W), np.float32)
    on = None if sn is None else np.zeros((H, W, 3), np.float32)
    rc = lib().ref_jbu(img.ctypes.data, W, H, sd.ctypes.data, None if sn is None else sn.ctypes.data, sw, sh,
                       od.ctypes.data, None if on is None else on.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference build: JBU probe failed ({rc})")
    return od if on is None else (od, on)
