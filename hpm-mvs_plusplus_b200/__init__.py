"""Python binding of libhpm_cuda.so (the C ABI in include/hpm_capi.h).

This is the test/bench harness view of the B200 HPM-MVS++ hot path.  It mirrors
the C ABI one to one; the product logic lives in the CUDA library.  There is no
CPU fallback: constructing a Context without the built library or without a CUDA
device raises.

The directory name contains a hyphen, so load it with `load_package()` of
__graft_entry__.py or importlib (tests/conftest.py registers it as `hpm_b200`).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Sequence

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "_build", "libhpm_cuda.so")

# ---- ABI mirror of include/hpm_types.h -------------------------------------------------

MODE_GEOM = 1 << 0
MODE_PRIOR = 1 << 1
MODE_MULTIGEOM = 1 << 2
MODE_HIERARCHY = 1 << 3
MODE_UPSAMPLE = 1 << 4
MODE_MAND = 1 << 5

MAP_DEPTH = 0
MAP_DEPTH_GEOM = 1
MAP_NORMAL = 2
MAP_COST = 3
MAP_CONF = 4
MAP_TEXTURE0 = 8

EXPORTED_SYMBOLS = (
    "hpm_create", "hpm_destroy", "hpm_last_error", "hpm_set_view", "hpm_set_map", "hpm_get_map",
    "hpm_set_canny", "hpm_set_prior", "hpm_run_patchmatch", "hpm_eval_costs", "hpm_set_address_mode",
    "hpm_launch_count", "hpm_synchronize", "hpm_sample_view", "hpm_debug_run_partial", "hpm_set_color",
    "hpm_jbu", "hpm_jbu_maps", "hpm_confidence_eval", "hpm_fuse", "hpm_support_points", "hpm_delaunay",
    "hpm_prior_from_triangles", "hpm_build_prior", "hpm_get_prior", "hpm_set_image", "hpm_prepare_level",
    "hpm_get_level", "hpm_reconstruct", "hpm_get_points", "hpm_get_stream", "hpm_profile_enable",
    "hpm_profile_read", "hpm_measure_fp32_peak", "hpm_eval_costs_noalloc", "hpm_eval_cost_grad",
    "hpm_eval_cost_grad_device", "hpm_gn_refine",
    "hpm_set_texture_format", "hpm_run_batch", "hpm_set_batch_options", "hpm_set_ncc_mode", "hpm_measure_tex_peak",
    "hpm_measure_tex_rate",
)

NCC_PLAIN = 0
NCC_SHIFTED = 1

BATCH_AUTOTUNE = 1
BATCH_GRAPH = 2
BATCH_PER_VIEW = 4

RECON_SEQUENTIAL = 0
RECON_BATCH_EXACT = 1
RECON_BATCH_ALL = 2

TEX_F32 = 0
TEX_F16 = 1
TEX_U8 = 2

PROFILE_TIMING = 1
PROFILE_COUNT = 2


class Profile(ctypes.Structure):
    """hpm_profile: PatchMatch launches, their device time and costed (hypothesis, view) pairs."""

    _fields_ = [("init_launches", ctypes.c_int64), ("sweep_launches", ctypes.c_int64),
                ("init_ms", ctypes.c_double), ("sweep_ms", ctypes.c_double),
                ("init_view_evals", ctypes.c_uint64), ("sweep_view_evals", ctypes.c_uint64),
                ("sweep_sampled", ctypes.c_uint64),
                ("confidence_ms", ctypes.c_double), ("prior_ms", ctypes.c_double), ("jbu_ms", ctypes.c_double),
                ("fusion_ms", ctypes.c_double), ("level_ms", ctypes.c_double)]


class ReconOptions(ctypes.Structure):
    """hpm_recon_options: --initial-image-scale, geometric iterations, fusion, seed."""

    _fields_ = [("initial_image_scale", ctypes.c_int32), ("geom_iterations", ctypes.c_int32),
                ("fuse", ctypes.c_int32), ("level_max_side", ctypes.c_int32), ("batch", ctypes.c_int32),
                ("batch_views", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class Point(ctypes.Structure):
    """hpm_point == PointList (main.h:92-96): world xyz, world normal, BGR colour."""

    _fields_ = [("coord", ctypes.c_float * 3), ("normal", ctypes.c_float * 3), ("color", ctypes.c_float * 3)]


class Camera(ctypes.Structure):
    """hpm_camera == struct Camera of the reference (main.h:39-47), 100 bytes."""

    _fields_ = [
        ("K", ctypes.c_float * 9),
        ("R", ctypes.c_float * 9),
        ("t", ctypes.c_float * 3),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("depth_min", ctypes.c_float),
        ("depth_max", ctypes.c_float),
    ]

    @classmethod
    def make(cls, K, R, t, width, height, depth_min, depth_max) -> "Camera":
        c = cls()
        c.K[:] = [float(v) for v in np.asarray(K, np.float32).ravel()]
        c.R[:] = [float(v) for v in np.asarray(R, np.float32).ravel()]
        c.t[:] = [float(v) for v in np.asarray(t, np.float32).ravel()]
        c.width, c.height = int(width), int(height)
        c.depth_min, c.depth_max = float(depth_min), float(depth_max)
        return c

    def copy(self) -> "Camera":
        c = Camera()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(Camera))
        return c

    def scaled(self, width: int, height: int, orig_width: int, orig_height: int) -> "Camera":
        """K rescaled to a resized image (HPM.cpp:669-676, float32 arithmetic)."""
        c = self.copy()
        sx = np.float32(width) / np.float32(orig_width)
        sy = np.float32(height) / np.float32(orig_height)
        c.K[0] = float(np.float32(c.K[0]) * sx)
        c.K[2] = float(np.float32(c.K[2]) * sx)
        c.K[4] = float(np.float32(c.K[4]) * sy)
        c.K[5] = float(np.float32(c.K[5]) * sy)
        c.width, c.height = int(width), int(height)
        return c


class Params(ctypes.Structure):
    """hpm_params (PatchMatchParams, HPM.h:32-55)."""

    _fields_ = [
        ("max_iterations", ctypes.c_int32),
        ("patch_size", ctypes.c_int32),
        ("num_images", ctypes.c_int32),
        ("radius_increment", ctypes.c_int32),
        ("sigma_spatial", ctypes.c_float),
        ("sigma_color", ctypes.c_float),
        ("top_k", ctypes.c_int32),
        ("depth_min", ctypes.c_float),
        ("depth_max", ctypes.c_float),
        ("scaled_cols", ctypes.c_int32),
        ("scaled_rows", ctypes.c_int32),
        ("mode", ctypes.c_uint32),
    ]

    @classmethod
    def make(cls, num_images: int, depth_min: float, depth_max: float, mode: int = 0) -> "Params":
        p = cls()
        p.max_iterations = 3  # RunPatchMatch hard-codes 3 iterations (HPM.cu:3013)
        p.patch_size = 11
        p.num_images = num_images
        p.radius_increment = 2
        p.sigma_spatial = 5.0
        p.sigma_color = 3.0
        p.top_k = 4
        p.depth_min = depth_min
        p.depth_max = depth_max
        p.scaled_cols = 0
        p.scaled_rows = 0
        p.mode = mode
        return p


def widened_range(cam: Camera) -> tuple[float, float]:
    """params.depth_min/max = 0.6 / 1.2 x the camera range (HPM.cpp:685-686)."""
    return float(np.float32(cam.depth_min) * np.float32(0.6)), float(np.float32(cam.depth_max) * np.float32(1.2))


class HPMError(RuntimeError):
    pass


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise HPMError(f"libhpm_cuda.so is not built ({path}); run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    vp, i32, f = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float
    lib.hpm_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    lib.hpm_destroy.argtypes = [vp]
    lib.hpm_destroy.restype = None
    lib.hpm_last_error.argtypes = [vp]
    lib.hpm_last_error.restype = ctypes.c_char_p
    lib.hpm_set_view.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Camera)]
    lib.hpm_set_map.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int]
    lib.hpm_get_map.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_size_t,
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.hpm_set_canny.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int]
    lib.hpm_set_prior.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int]
    lib.hpm_run_patchmatch.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int,
                                       ctypes.c_uint64]
    lib.hpm_eval_costs.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int, vp, vp,
                                   vp]
    lib.hpm_run_batch.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, vp]
    lib.hpm_set_batch_options.argtypes = [vp, ctypes.c_int]
    lib.hpm_set_ncc_mode.argtypes = [vp, ctypes.c_int]
    lib.hpm_eval_costs_noalloc.argtypes = lib.hpm_eval_costs.argtypes
    lib.hpm_eval_cost_grad.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int, vp,
                                       vp, vp, vp]
    lib.hpm_eval_cost_grad_device.argtypes = lib.hpm_eval_cost_grad.argtypes
    lib.hpm_gn_refine.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int,
                                  ctypes.c_int]
    lib.hpm_set_address_mode.argtypes = [vp, ctypes.c_int]
    lib.hpm_set_texture_format.argtypes = [vp, ctypes.c_int]
    lib.hpm_launch_count.argtypes = [vp]
    lib.hpm_launch_count.restype = ctypes.c_int64
    lib.hpm_synchronize.argtypes = [vp]
    lib.hpm_sample_view.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
    lib.hpm_set_color.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.hpm_support_points.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ip, ip, ip]
    lib.hpm_delaunay.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ip]
    lib.hpm_prior_from_triangles.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
    lib.hpm_build_prior.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip]
    lib.hpm_get_prior.argtypes = [vp, ctypes.c_int, vp, vp]
    lib.hpm_set_image.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int]
    lib.hpm_prepare_level.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Camera)]
    lib.hpm_get_level.argtypes = [vp, ctypes.c_int, vp, vp, vp]
    lib.hpm_reconstruct.argtypes = [vp, ctypes.c_int, vp, vp, vp, ctypes.POINTER(ReconOptions),
                                    ctypes.POINTER(ctypes.c_int64)]
    lib.hpm_get_points.argtypes = [vp, vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    lib.hpm_jbu.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.hpm_jbu_maps.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
    lib.hpm_confidence_eval.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.hpm_fuse.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int64,
                             ctypes.POINTER(ctypes.c_int64)]
    lib.hpm_debug_run_partial.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int,
                                          ctypes.c_uint64, ctypes.c_int, vp, vp, vp, vp]
    lib.hpm_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    lib.hpm_profile_enable.argtypes = [vp, ctypes.c_int]
    lib.hpm_profile_read.argtypes = [vp, ctypes.POINTER(Profile)]
    lib.hpm_measure_fp32_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.hpm_measure_tex_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.hpm_measure_tex_rate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_double)]
    for name in EXPORTED_SYMBOLS:
        getattr(lib, name)
    del i32, f
    _lib = lib
    return lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def delaunay(xy: np.ndarray, width: int, height: int) -> np.ndarray:
    """hpm_delaunay: triangles (n, 6) int32 of integer points in [0,w)x[0,h) (host only)."""
    lib = load_library()
    p = np.ascontiguousarray(xy, np.int32).reshape(-1, 2)
    n = ctypes.c_int()
    cap = 2 * p.shape[0] + 8
    out = np.zeros((cap, 6), np.int32)
    rc = lib.hpm_delaunay(_ptr(p) if p.size else None, p.shape[0], width, height, _ptr(out), cap, ctypes.byref(n))
    if rc != 0:
        raise HPMError(f"hpm_delaunay failed ({rc})")
    return out[: n.value].copy()


class Context:
    """One hpm_ctx: resident views and maps on one CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.hpm_create(device, ctypes.byref(h))
        if rc != 0 or not h.value:
            raise HPMError(f"hpm_create(device={device}) failed with status {rc} (no CUDA device?)")
        self.h = h
        self.views: dict[int, tuple[int, int]] = {}

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.hpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            msg = self.lib.hpm_last_error(self.h)
            raise HPMError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def set_texture_format(self, fmt: int) -> None:
        """TEX_F32 or TEX_F16 texels for the source images bound from now on (hpm_set_texture_format)."""
        self._check(self.lib.hpm_set_texture_format(self.h, fmt), "hpm_set_texture_format")

    def set_ncc_mode(self, mode: int) -> None:
        """NCC_PLAIN or NCC_SHIFTED (shifted moments, the precision form) from now on (hpm_set_ncc_mode)."""
        self._check(self.lib.hpm_set_ncc_mode(self.h, mode), "hpm_set_ncc_mode")

    def set_address_mode(self, mode: int) -> None:
        self._check(self.lib.hpm_set_address_mode(self.h, mode), "hpm_set_address_mode")

    def set_view(self, view: int, gray: np.ndarray, cam: Camera) -> None:
        g = np.ascontiguousarray(gray, dtype=np.float32)
        h, w = g.shape
        self._check(self.lib.hpm_set_view(self.h, view, _ptr(g), w, h, ctypes.byref(cam)), "hpm_set_view")
        self.views[view] = (w, h)

    def set_map(self, view: int, kind: int, data: np.ndarray) -> None:
        d = np.ascontiguousarray(data, dtype=np.float32)
        h, w = d.shape[:2]
        self._check(self.lib.hpm_set_map(self.h, view, kind, _ptr(d), w, h), "hpm_set_map")

    def get_map(self, view: int, kind: int, out: np.ndarray | None = None) -> np.ndarray:
        """Download a map; `out` (float32, C-contiguous, e.g. pinned) receives it when given."""
        w, h = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.hpm_get_map(self.h, view, kind, None, 0, ctypes.byref(w), ctypes.byref(h)), "hpm_get_map")
        ch = 3 if kind == MAP_NORMAL else 1
        shape = (h.value, w.value, ch) if ch > 1 else (h.value, w.value)
        if out is None:
            out = np.empty(shape, np.float32)
        elif out.dtype != np.float32 or not out.flags.c_contiguous or out.size < h.value * w.value * ch:
            raise HPMError("get_map: `out` must be C-contiguous float32 with room for the map")
        self._check(self.lib.hpm_get_map(self.h, view, kind, _ptr(out), out.size, None, None), "hpm_get_map")
        return out

    def set_canny(self, view: int, edges: np.ndarray) -> None:
        e = np.ascontiguousarray(edges, dtype=np.uint8)
        h, w = e.shape
        self._check(self.lib.hpm_set_canny(self.h, view, _ptr(e), w, h), "hpm_set_canny")

    def set_prior(self, view: int, planes: np.ndarray, mask: np.ndarray) -> None:
        p = np.ascontiguousarray(planes, dtype=np.float32)
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        h, w = m.shape
        self._check(self.lib.hpm_set_prior(self.h, view, _ptr(p), _ptr(m), w, h), "hpm_set_prior")

    def run_patchmatch(self, ref: int, srcs: Sequence[int], params: Params, texture_level: int = 0,
                       seed: int = 0) -> None:
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        self._check(self.lib.hpm_run_patchmatch(self.h, ref, _ptr(s), len(s), ctypes.byref(params), texture_level,
                                                ctypes.c_uint64(seed)), "hpm_run_patchmatch")

    def run_batch(self, refs: Sequence[int], src_lists, params, seeds: Sequence[int], texture_level: int = 0) -> None:
        """hpm_run_batch: the runs (refs[k], src_lists[k], params[k], seeds[k]) in one launch per stage."""
        n = len(refs)
        r = np.ascontiguousarray(refs, dtype=np.int32)
        off, ids = self._src_lists(src_lists)
        if isinstance(params, Params):
            params = [params] * n
        parr = (Params * n)(*params)
        sd = np.ascontiguousarray(seeds, dtype=np.uint64)
        self._check(self.lib.hpm_run_batch(self.h, n, _ptr(r), _ptr(off), _ptr(ids), parr, texture_level, _ptr(sd)),
                    "hpm_run_batch")

    def set_batch_options(self, flags: int) -> None:
        self._check(self.lib.hpm_set_batch_options(self.h, flags), "hpm_set_batch_options")

    def eval_costs(self, ref: int, srcs: Sequence[int], params: Params, px: np.ndarray,
                   planes: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        p = np.ascontiguousarray(px, dtype=np.int32).reshape(-1, 2)
        pl = np.ascontiguousarray(planes, dtype=np.float32).reshape(-1, 4)
        out = np.empty((p.shape[0], len(s)), np.float32)
        self._check(self.lib.hpm_eval_costs(self.h, ref, _ptr(s), len(s), ctypes.byref(params), p.shape[0], _ptr(p),
                                            _ptr(pl), _ptr(out)), "hpm_eval_costs")
        return out

    def eval_costs_noalloc(self, ref: int, srcs: Sequence[int], params: Params, px: np.ndarray,
                           planes: np.ndarray) -> np.ndarray:
        """eval_costs for callers that cannot have the library allocate device memory while they run
        (hpm_eval_costs_noalloc: fixed 4 MiB of staging per GPU, n * (24 + 4 * len(srcs)) bytes per call)."""
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        p = np.ascontiguousarray(px, dtype=np.int32).reshape(-1, 2)
        pl = np.ascontiguousarray(planes, dtype=np.float32).reshape(-1, 4)
        out = np.empty((p.shape[0], len(s)), np.float32)
        self._check(self.lib.hpm_eval_costs_noalloc(self.h, ref, _ptr(s), len(s), ctypes.byref(params), p.shape[0],
                                                    _ptr(p), _ptr(pl), _ptr(out)), "hpm_eval_costs_noalloc")
        return out

    def eval_cost_grad(self, ref: int, srcs: Sequence[int], params: Params, px: np.ndarray, theta: np.ndarray,
                       with_grad: bool = True):
        """Differentiable costs (n, S) and d cost / d (depth, nx, ny) (n, S, 3) (hpm_eval_cost_grad)."""
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        p = np.ascontiguousarray(px, dtype=np.int32).reshape(-1, 2)
        th = np.ascontiguousarray(theta, dtype=np.float32).reshape(-1, 3)
        cost = np.empty((p.shape[0], len(s)), np.float32)
        grad = np.empty((p.shape[0], len(s), 3), np.float32) if with_grad else None
        self._check(self.lib.hpm_eval_cost_grad(self.h, ref, _ptr(s), len(s), ctypes.byref(params), p.shape[0],
                                                _ptr(p), _ptr(th), _ptr(cost), _ptr(grad) if with_grad else None),
                    "hpm_eval_cost_grad")
        return cost, grad

    def eval_cost_grad_tensors(self, ref: int, srcs: Sequence[int], params: Params, px, theta, with_grad: bool = True):
        """eval_cost_grad on CUDA tensors of the context's GPU (hpm_eval_cost_grad_device): px (n, 2) int32,
        theta (n, 3) float32 -> cost (n, S) and grad (n, S, 3) float32 tensors; no host copies.  The context's
        stream waits for torch's current stream first."""
        import torch
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        p = px.to(torch.int32).reshape(-1, 2).contiguous()
        th = theta.to(torch.float32).reshape(-1, 3).contiguous()
        n = p.shape[0]
        cost = torch.empty((n, len(s)), dtype=torch.float32, device=th.device)
        grad = torch.empty((n, len(s), 3), dtype=torch.float32, device=th.device) if with_grad else None
        stream = torch.cuda.ExternalStream(self.stream_handle(), device=th.device)
        stream.wait_stream(torch.cuda.current_stream(th.device))
        self._check(self.lib.hpm_eval_cost_grad_device(
            self.h, ref, _ptr(s), len(s), ctypes.byref(params), n, ctypes.c_void_p(p.data_ptr()),
            ctypes.c_void_p(th.data_ptr()), ctypes.c_void_p(cost.data_ptr()),
            ctypes.c_void_p(grad.data_ptr()) if with_grad else None), "hpm_eval_cost_grad_device")
        # the call returned after its kernel finished; keep the inputs alive until then
        return cost, grad

    def gn_refine(self, ref: int, srcs: Sequence[int], params: Params, depth_kind: int = MAP_DEPTH_GEOM,
                  steps: int = 3) -> None:
        """Gauss-Newton refinement of the view's resident depth/normal maps (hpm_gn_refine)."""
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        self._check(self.lib.hpm_gn_refine(self.h, ref, _ptr(s), len(s), ctypes.byref(params), depth_kind, steps),
                    "hpm_gn_refine")

    def sample_view(self, view: int, xy: np.ndarray) -> np.ndarray:
        c = np.ascontiguousarray(xy, dtype=np.float32).reshape(-1, 2)
        out = np.empty(c.shape[0], np.float32)
        self._check(self.lib.hpm_sample_view(self.h, view, c.shape[0], _ptr(c), _ptr(out)), "hpm_sample_view")
        return out

    def run_partial(self, ref: int, srcs: Sequence[int], params: Params, n_half_sweeps: int, texture_level: int = 0,
                    seed: int = 0) -> dict:
        """Init + n half-sweeps; returns the raw run state (camera-frame planes)."""
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        w, h = self.views[ref]
        planes = np.empty((h, w, 4), np.float32)
        costs = np.empty((h, w), np.float32)
        sel = np.empty((h, w), np.uint32)
        draws = np.empty((h, w), np.uint32)
        self._check(self.lib.hpm_debug_run_partial(self.h, ref, _ptr(s), len(s), ctypes.byref(params), texture_level,
                                                   ctypes.c_uint64(seed), n_half_sweeps, _ptr(planes), _ptr(costs),
                                                   _ptr(sel), _ptr(draws)), "hpm_debug_run_partial")
        return {"planes": planes, "costs": costs, "selected_views": sel, "rng_draw": draws}

    def set_color(self, view: int, bgr: np.ndarray) -> None:
        c = np.ascontiguousarray(bgr, dtype=np.uint8)
        h, w = c.shape[:2]
        self._check(self.lib.hpm_set_color(self.h, view, _ptr(c), w, h), "hpm_set_color")

    def jbu(self, view: int) -> bool:
        applied = ctypes.c_int()
        self._check(self.lib.hpm_jbu(self.h, view, ctypes.byref(applied)), "hpm_jbu")
        return bool(applied.value)

    def jbu_maps(self, view: int, src_depth: np.ndarray, src_normal: np.ndarray | None = None):
        sd = np.ascontiguousarray(src_depth, np.float32)
        sn = None if src_normal is None else np.ascontiguousarray(src_normal, np.float32)
        w, h = self.views[view]
        od = np.empty((h, w), np.float32)
        on = None if sn is None else np.empty((h, w, 3), np.float32)
        self._check(self.lib.hpm_jbu_maps(self.h, view, _ptr(sd), None if sn is None else _ptr(sn), sd.shape[1],
                                          sd.shape[0], _ptr(od), None if on is None else _ptr(on)), "hpm_jbu_maps")
        return od if on is None else (od, on)

    @staticmethod
    def _src_lists(src_lists):
        off = np.zeros(len(src_lists) + 1, np.int32)
        for i, s in enumerate(src_lists):
            off[i + 1] = off[i] + len(s)
        ids = np.ascontiguousarray(np.concatenate([np.asarray(s, np.int32) for s in src_lists])
                                   if off[-1] else np.zeros(1, np.int32), np.int32)
        return off, ids

    def confidence_eval(self, src_lists, depth_kind: int = MAP_DEPTH) -> int:
        off, ids = self._src_lists(src_lists)
        it = ctypes.c_int()
        self._check(self.lib.hpm_confidence_eval(self.h, len(src_lists), _ptr(off), _ptr(ids), depth_kind,
                                                 ctypes.byref(it)), "hpm_confidence_eval")
        return it.value

    def fuse(self, src_lists, depth_kind: int = MAP_DEPTH_GEOM, sky_masks=None, capacity: int | None = None):
        off, ids = self._src_lists(src_lists)
        if capacity is None:
            capacity = sum(w * h for (w, h) in (self.views[v] for v in range(len(src_lists))))
        out = np.zeros((capacity, 9), np.float32)
        n = ctypes.c_int64()
        sky_arr = None
        keep = []
        if sky_masks is not None:
            sky_arr = (ctypes.c_void_p * len(sky_masks))()
            for i, m in enumerate(sky_masks):
                m = np.ascontiguousarray(m, np.uint8)
                keep.append(m)
                sky_arr[i] = m.ctypes.data
        self._check(self.lib.hpm_fuse(self.h, len(src_lists), _ptr(off), _ptr(ids), depth_kind, sky_arr, _ptr(out),
                                      capacity, ctypes.byref(n)), "hpm_fuse")
        return out[: min(n.value, capacity)], n.value

    def support_points(self, view: int, distance: int = 0):
        n, w, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.hpm_support_points(self.h, view, distance, None, 0, ctypes.byref(n), ctypes.byref(w),
                                                ctypes.byref(h)), "hpm_support_points")
        out = np.zeros((max(n.value, 1), 2), np.int32)
        self._check(self.lib.hpm_support_points(self.h, view, distance, _ptr(out), n.value, None, None, None),
                    "hpm_support_points")
        return out[: n.value], (w.value, h.value)

    def prior_from_triangles(self, view: int, distance: int, tris: np.ndarray) -> None:
        t = np.ascontiguousarray(tris, np.int32).reshape(-1, 6)
        self._check(self.lib.hpm_prior_from_triangles(self.h, view, distance, _ptr(t) if t.size else None,
                                                      t.shape[0]), "hpm_prior_from_triangles")

    def build_prior(self, view: int, distance: int = 0):
        n_p, n_t = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.hpm_build_prior(self.h, view, distance, ctypes.byref(n_p), ctypes.byref(n_t)),
                    "hpm_build_prior")
        return n_p.value, n_t.value

    def get_prior(self, view: int):
        w, h = self.views[view]
        planes = np.empty((h, w, 4), np.float32)
        mask = np.empty((h, w), np.uint8)
        self._check(self.lib.hpm_get_prior(self.h, view, _ptr(planes), _ptr(mask)), "hpm_get_prior")
        return planes, mask

    def set_image(self, view: int, bgr: np.ndarray) -> None:
        c = np.ascontiguousarray(bgr, dtype=np.uint8)
        h, w = c.shape[:2]
        self._check(self.lib.hpm_set_image(self.h, view, _ptr(c), w, h), "hpm_set_image")

    def prepare_level(self, view: int, w: int, h: int, cam: Camera) -> None:
        self._check(self.lib.hpm_prepare_level(self.h, view, w, h, ctypes.byref(cam)), "hpm_prepare_level")
        self.views[view] = (w, h)

    def get_level(self, view: int):
        w, h = self.views[view]
        bgr = np.empty((h, w, 3), np.uint8)
        gray = np.empty((h, w), np.float32)
        edges = np.empty((h, w), np.uint8)
        self._check(self.lib.hpm_get_level(self.h, view, _ptr(bgr), _ptr(gray), _ptr(edges)), "hpm_get_level")
        return bgr, gray, edges

    def reconstruct(self, cams, src_lists, initial_image_scale: int = 4, seed: int = 0, fuse: bool = True,
                    geom_iterations: int = 3, level_max_side: int = 0, batch: int = RECON_SEQUENTIAL,
                    batch_views: int = 0) -> int:
        """hpm_reconstruct; batch = RECON_SEQUENTIAL / RECON_BATCH_EXACT / RECON_BATCH_ALL (batching form)."""
        cam_arr = (Camera * len(cams))(*cams)
        off, ids = self._src_lists(src_lists)
        opt = ReconOptions(initial_image_scale, geom_iterations, 1 if fuse else 0, level_max_side, batch,
                           batch_views, seed)
        n = ctypes.c_int64()
        self._check(self.lib.hpm_reconstruct(self.h, len(cams), cam_arr, _ptr(off), _ptr(ids), ctypes.byref(opt),
                                             ctypes.byref(n)), "hpm_reconstruct")
        return n.value

    def get_points(self, capacity: int | None = None, out: np.ndarray | None = None) -> np.ndarray:
        """Fused points (n, 9): xyz, normal, colour; `out` (float32 (m, 9), e.g. pinned) receives them."""
        n = ctypes.c_int64()
        self._check(self.lib.hpm_get_points(self.h, None, 0, ctypes.byref(n)), "hpm_get_points")
        cap = n.value if capacity is None else min(capacity, n.value)
        if out is None:
            out = np.zeros((max(cap, 1), 9), np.float32)
        elif out.dtype != np.float32 or not out.flags.c_contiguous or out.ndim != 2 or out.shape[1] != 9:
            raise HPMError("get_points: `out` must be C-contiguous float32 of shape (m, 9)")
        cap = min(cap, out.shape[0])
        self._check(self.lib.hpm_get_points(self.h, _ptr(out), cap, None), "hpm_get_points")
        return out[:cap]

    def synchronize(self) -> None:
        self._check(self.lib.hpm_synchronize(self.h), "hpm_synchronize")

    def launch_count(self) -> int:
        return int(self.lib.hpm_launch_count(self.h))

    def stream_handle(self) -> int:
        """The cudaStream_t all of this context's work runs on."""
        s = ctypes.c_void_p()
        self._check(self.lib.hpm_get_stream(self.h, ctypes.byref(s)), "hpm_get_stream")
        return int(s.value or 0)

    def profile_enable(self, flags: int) -> None:
        self._check(self.lib.hpm_profile_enable(self.h, flags), "hpm_profile_enable")

    def profile_read(self) -> Profile:
        p = Profile()
        self._check(self.lib.hpm_profile_read(self.h, ctypes.byref(p)), "hpm_profile_read")
        return p


def measure_fp32_peak(device: int = 0) -> float:
    """FP32 FMA throughput of the device, TFLOP/s (hpm_measure_fp32_peak)."""
    t = ctypes.c_double()
    rc = load_library().hpm_measure_fp32_peak(device, ctypes.byref(t))
    if rc != 0:
        raise HPMError(f"hpm_measure_fp32_peak failed ({rc})")
    return t.value


@dataclass
class View:
    """One view of a scene at some resolution."""

    gray: np.ndarray  # float32 H x W
    cam: Camera


def measure_tex_peak(device: int = 0, fmt: int = TEX_F32) -> float:
    """Linear-filtered texture fetches per second of the device, in 1e9/s (hpm_measure_tex_peak)."""
    lib = load_library()
    out = ctypes.c_double()
    rc = lib.hpm_measure_tex_peak(device, fmt, ctypes.byref(out))
    if rc != 0:
        raise HPMError(f"hpm_measure_tex_peak failed ({rc})")
    return out.value


def measure_tex_rate(device: int = 0, fmt: int = TEX_F32, jitter: float = 0.0) -> float:
    """Filtered fetches per second (1e9/s) with every lane's patch moved by up to +-jitter px
    (hpm_measure_tex_rate)."""
    lib = load_library()
    out = ctypes.c_double()
    rc = lib.hpm_measure_tex_rate(device, fmt, ctypes.c_float(jitter), ctypes.byref(out))
    if rc != 0:
        raise HPMError(f"hpm_measure_tex_rate failed ({rc})")
    return out.value
