"""CPU ORACLE wrapper -- test infrastructure only.

ctypes binding of oracle/_build/libhpm_oracle.so (hpm_oracle.h), the C
restatement of the HPM-MVS++ hot path.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline legs import this module, as the checker; the
product (libhpm_cuda.so and its binding) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhpm_oracle.so")


class Camera(ctypes.Structure):
    _fields_ = [
        ("K", ctypes.c_float * 9), ("R", ctypes.c_float * 9), ("t", ctypes.c_float * 3),
        ("height", ctypes.c_int32), ("width", ctypes.c_int32),
        ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("max_iterations", ctypes.c_int32), ("patch_size", ctypes.c_int32), ("num_images", ctypes.c_int32),
        ("radius_increment", ctypes.c_int32), ("sigma_spatial", ctypes.c_float), ("sigma_color", ctypes.c_float),
        ("top_k", ctypes.c_int32), ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float),
        ("scaled_cols", ctypes.c_int32), ("scaled_rows", ctypes.c_int32), ("mode", ctypes.c_uint32),
    ]


class State(ctypes.Structure):
    _fields_ = [
        ("planes", ctypes.c_void_p), ("costs", ctypes.c_void_p), ("pre_costs", ctypes.c_void_p),
        ("selected_views", ctypes.c_void_p), ("rng_draw", ctypes.c_void_p), ("prior_planes", ctypes.c_void_p),
        ("plane_masks", ctypes.c_void_p), ("confidences", ctypes.c_void_p), ("canny", ctypes.c_void_p),
        ("texture", ctypes.c_void_p), ("scaled_planes", ctypes.c_void_p),
    ]


class Point(ctypes.Structure):
    _fields_ = [("coord", ctypes.c_float * 3), ("normal", ctypes.c_float * 3), ("color", ctypes.c_float * 3)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        L = _lib
        vp = ctypes.c_void_p
        L.ora_tex2d.restype = ctypes.c_float
        L.ora_tex2d.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float]
        L.ora_bilateral_ncc.restype = ctypes.c_float
        L.ora_bilateral_ncc.argtypes = [vp, ctypes.POINTER(Camera), vp, ctypes.POINTER(Camera), ctypes.c_int,
                                        ctypes.c_int, vp, ctypes.POINTER(Params)]
        L.ora_eval_costs.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int, vp, vp, vp]
        L.ora_geom_cost.restype = ctypes.c_float
        L.ora_geom_cost.argtypes = [vp, ctypes.POINTER(Camera), ctypes.POINTER(Camera), vp, ctypes.c_int, ctypes.c_int]
        L.ora_initial_cost.restype = ctypes.c_float
        L.ora_initial_cost.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int, vp,
                                       ctypes.POINTER(ctypes.c_uint32)]
        L.ora_depth_from_plane.restype = ctypes.c_float
        L.ora_depth_from_plane.argtypes = [ctypes.POINTER(Camera), vp, ctypes.c_int, ctypes.c_int]
        L.ora_texture.restype = ctypes.c_float
        L.ora_texture.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ora_set_texture_model.argtypes = [ctypes.c_int]
        L.ora_set_ncc_shift.argtypes = [ctypes.c_int]
        L.ora_bilateral_ncc64.restype = ctypes.c_double
        L.ora_bilateral_ncc64.argtypes = L.ora_bilateral_ncc.argtypes
        for fn in ("ora_random_init",):
            getattr(L, fn).argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(State),
                                       ctypes.c_uint64, ctypes.c_uint32]
        L.ora_half_sweep.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(State),
                                     ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32]
        L.ora_run_patchmatch.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(State),
                                         ctypes.c_uint64, ctypes.c_uint32]
        L.ora_export.argtypes = [ctypes.POINTER(Camera), vp]
        L.ora_jbu.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp]
        L.ora_jbu_prior.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.ora_confidence_eval.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp]
        L.ora_fusion.restype = ctypes.c_int64
        L.ora_fusion.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int64,
                                 ctypes.POINTER(ctypes.c_int64)]
        L.ora_support_points.restype = ctypes.c_int32
        L.ora_support_points.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int32]
        L.ora_planar_prior.restype = ctypes.c_int32
        L.ora_planar_prior.argtypes = [vp, ctypes.c_int32, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Camera),
                                       ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, vp, vp, vp, vp]
        L.ora_resize_linear_f32.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int]
        L.ora_philox.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp]
        L.ora_prior_reload.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Camera), ctypes.c_float,
                                       ctypes.c_float, vp, vp]
        L.ora_cost_grad64.restype = ctypes.c_double
        L.ora_cost_grad64.argtypes = [vp, ctypes.POINTER(Camera), vp, ctypes.POINTER(Camera), ctypes.POINTER(Params),
                                      ctypes.c_int, ctypes.c_int, vp, vp]
        L.ora_uniform.restype = ctypes.c_float
        L.ora_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def to_cam(c) -> Camera:
    out = Camera()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(c), ctypes.sizeof(Camera))
    return out


def to_params(p) -> Params:
    out = Params()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(p), ctypes.sizeof(Params))
    return out


def _ptr_array(arrs: Sequence[Optional[np.ndarray]]):
    arr = (ctypes.c_void_p * max(1, len(arrs)))()
    for i, a in enumerate(arrs):
        arr[i] = None if a is None else a.ctypes.data
    return arr


def philox(ctr, k0: int, k1: int) -> list:
    c = np.ascontiguousarray(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().ora_philox(_p(c), k0, k1, _p(out))
    return [int(v) for v in out]


def uniform(seed: int, view: int, x: int, y: int, draw: int) -> float:
    return float(lib().ora_uniform(ctypes.c_uint64(seed), view, x, y, draw))


def set_texture_model(model: int) -> None:
    lib().ora_set_texture_model(model)


def set_ncc_shift(on: bool) -> None:
    """Shifted-moment NCC of the precision form in every oracle cost (off: the plain arithmetic)."""
    lib().ora_set_ncc_shift(1 if on else 0)


def ncc64(ref, ref_cam, src, src_cam, params, px: int, py: int, plane) -> float:
    """The bilateral NCC of the oracle's own samples (same positions and filter model) with double moments."""
    r = np.ascontiguousarray(ref, np.float32)
    s = np.ascontiguousarray(src, np.float32)
    pl = np.ascontiguousarray(plane, np.float32)
    rc, sc = to_cam(ref_cam), to_cam(src_cam)
    prm = to_params(params)
    return lib().ora_bilateral_ncc64(_p(r), ctypes.byref(rc), _p(s), ctypes.byref(sc), px, py, _p(pl),
                                     ctypes.byref(prm))


def tex2d(img: np.ndarray, x: float, y: float) -> float:
    img = np.ascontiguousarray(img, np.float32)
    return lib().ora_tex2d(_p(img), img.shape[1], img.shape[0], x, y)


def eval_costs(images: Sequence[np.ndarray], cams, params, px: np.ndarray, planes: np.ndarray) -> np.ndarray:
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    px = np.ascontiguousarray(px, np.int32).reshape(-1, 2)
    planes = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
    out = np.empty((px.shape[0], len(imgs) - 1), np.float32)
    prm = to_params(params)
    lib().ora_eval_costs(_ptr_array(imgs), cam_arr, len(imgs), ctypes.byref(prm), px.shape[0], _p(px), _p(planes),
                         _p(out))
    return out


def initial_cost(images: Sequence[np.ndarray], cams, params, px: int, py: int, plane) -> tuple:
    """(cost, selected-view mask) of one hypothesis (ComputeMultiViewInitialCostandSelectedViews)."""
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    pl = np.ascontiguousarray(plane, np.float32)
    sel = ctypes.c_uint32(0)
    prm = to_params(params)
    c = lib().ora_initial_cost(_ptr_array(imgs), cam_arr, len(imgs), ctypes.byref(prm), int(px), int(py), _p(pl),
                               ctypes.byref(sel))
    return float(c), int(sel.value)


def geom_cost(src_depth: np.ndarray, ref_cam, src_cam, plane, px: int, py: int) -> float:
    """Geometric consistency cost of one hypothesis against one source depth map."""
    d = np.ascontiguousarray(src_depth, np.float32)
    pl = np.ascontiguousarray(plane, np.float32)
    rc, sc = to_cam(ref_cam), to_cam(src_cam)
    return float(lib().ora_geom_cost(_p(d), ctypes.byref(rc), ctypes.byref(sc), _p(pl), int(px), int(py)))


def depth_from_plane(cam, plane, px: int, py: int) -> float:
    pl = np.ascontiguousarray(plane, np.float32)
    c = to_cam(cam)
    return float(lib().ora_depth_from_plane(ctypes.byref(c), _p(pl), int(px), int(py)))


def texture(canny: np.ndarray, px: int, py: int) -> float:
    """Edge-density texture term at (px, py) of a 0 / non-zero edge map."""
    e = np.ascontiguousarray(canny, np.uint8)
    return float(lib().ora_texture(_p(e), e.shape[1], e.shape[0], int(px), int(py)))


class RunState:
    """Per-run arrays of one reference view (see ora_state)."""

    def __init__(self, W: int, H: int):
        n = W * H
        self.W, self.H = W, H
        self.planes = np.zeros((H, W, 4), np.float32)
        self.costs = np.zeros((H, W), np.float32)
        self.pre_costs = np.zeros((H, W), np.float32)
        self.selected_views = np.zeros((H, W), np.uint32)
        self.rng_draw = np.zeros((H, W), np.uint32)
        self.prior_planes = np.zeros((H, W, 4), np.float32)
        self.plane_masks = np.zeros((H, W), np.uint32)
        self.confidences = np.zeros((H, W), np.float32)
        self.canny = np.zeros((H, W), np.uint8)
        self.texture = np.zeros((H, W), np.float32)
        self.scaled_planes = np.zeros((1, 1, 4), np.float32)
        del n

    def struct(self) -> State:
        s = State()
        for name, _ in State._fields_:
            setattr(s, name, getattr(self, name).ctypes.data)
        return s


def run_patchmatch(images, depths, cams, params, st: RunState, seed: int, view_id: int) -> None:
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    deps = [None if d is None else np.ascontiguousarray(d, np.float32) for d in (depths or [None] * len(imgs))]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    prm = to_params(params)
    s = st.struct()
    lib().ora_run_patchmatch(_ptr_array(imgs), _ptr_array(deps), cam_arr, len(imgs), ctypes.byref(prm),
                             ctypes.byref(s), ctypes.c_uint64(seed), view_id)


def random_init(images, cams, params, st: RunState, seed: int, view_id: int) -> None:
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    prm = to_params(params)
    s = st.struct()
    lib().ora_random_init(_ptr_array(imgs), cam_arr, len(imgs), ctypes.byref(prm), ctypes.byref(s),
                          ctypes.c_uint64(seed), view_id)


def half_sweep(images, depths, cams, params, st: RunState, color: int, it: int, seed: int, view_id: int) -> None:
    imgs = [np.ascontiguousarray(i, np.float32) for i in images]
    deps = [None if d is None else np.ascontiguousarray(d, np.float32) for d in (depths or [None] * len(imgs))]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    prm = to_params(params)
    s = st.struct()
    lib().ora_half_sweep(_ptr_array(imgs), _ptr_array(deps), cam_arr, len(imgs), ctypes.byref(prm), ctypes.byref(s),
                         color, it, ctypes.c_uint64(seed), view_id)


def export(cam, planes: np.ndarray) -> None:
    c = to_cam(cam)
    lib().ora_export(ctypes.byref(c), _p(planes))


def jbu(image: np.ndarray, src_depth: np.ndarray) -> np.ndarray:
    image = np.ascontiguousarray(image, np.float32)
    src_depth = np.ascontiguousarray(src_depth, np.float32)
    H, W = image.shape
    sh, sw = src_depth.shape
    out = np.empty((H, W), np.float32)
    lib().ora_jbu(_p(image), W, H, _p(src_depth), sw, sh, _p(out))
    return out


def jbu_prior(image: np.ndarray, src_depth: np.ndarray, src_normal: np.ndarray):
    image = np.ascontiguousarray(image, np.float32)
    src_depth = np.ascontiguousarray(src_depth, np.float32)
    src_normal = np.ascontiguousarray(src_normal, np.float32)
    H, W = image.shape
    sh, sw = src_depth.shape
    od = np.empty((H, W), np.float32)
    on = np.empty((H, W, 3), np.float32)
    lib().ora_jbu_prior(_p(image), W, H, _p(src_depth), _p(src_normal), sw, sh, _p(od), _p(on))
    return od, on


def _src_lists(src_lists: Sequence[Sequence[int]]):
    off = np.zeros(len(src_lists) + 1, np.int32)
    for i, s in enumerate(src_lists):
        off[i + 1] = off[i] + len(s)
    ids = np.ascontiguousarray(np.concatenate([np.asarray(s, np.int32) for s in src_lists]) if off[-1] else
                               np.zeros(1, np.int32), np.int32)
    return off, ids


def confidence_eval(cams, depths, normals, src_lists) -> list:
    depths = [np.ascontiguousarray(d, np.float32) for d in depths]
    normals = [np.ascontiguousarray(n, np.float32) for n in normals]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    off, ids = _src_lists(src_lists)
    outs = [np.zeros_like(d) for d in depths]
    lib().ora_confidence_eval(len(cams), cam_arr, _ptr_array(depths), _ptr_array(normals), _p(off), _p(ids),
                              _ptr_array(outs))
    return outs


def fusion(cams, depths, normals, colors, src_lists, sky_masks=None, max_points: Optional[int] = None):
    depths = [np.ascontiguousarray(d, np.float32) for d in depths]
    normals = [np.ascontiguousarray(n, np.float32) for n in normals]
    colors = [np.ascontiguousarray(c, np.uint8) for c in colors]
    sky = None if sky_masks is None else [np.ascontiguousarray(s, np.uint8) for s in sky_masks]
    cam_arr = (Camera * len(cams))(*[to_cam(c) for c in cams])
    off, ids = _src_lists(src_lists)
    if max_points is None:
        max_points = int(sum(d.size for d in depths))
    out = np.zeros((max_points, 9), np.float32)
    total = ctypes.c_int64()
    n = lib().ora_fusion(len(cams), cam_arr, _ptr_array(depths), _ptr_array(normals), _ptr_array(colors),
                         None if sky is None else _ptr_array(sky), _p(off), _p(ids), _p(out), max_points,
                         ctypes.byref(total))
    return out[:n], int(total.value)


def support_points(costs: np.ndarray, conf: np.ndarray, width: int, height: int) -> np.ndarray:
    costs = np.ascontiguousarray(costs, np.float32)
    conf = np.ascontiguousarray(conf, np.float32)
    cap = 2 * ((width + 4) // 5) * ((height + 4) // 5) + 8
    out = np.zeros((cap, 2), np.int32)
    n = lib().ora_support_points(_p(costs), _p(conf), None, 0, width, height, _p(out), cap)
    return out[:n].copy()


def planar_prior(tris: np.ndarray, depths: np.ndarray, cam, factor: float, depth_min: float, depth_max: float,
                 mode: int):
    tris = np.ascontiguousarray(tris, np.int32).reshape(-1, 6)
    depths = np.ascontiguousarray(depths, np.float32)
    H, W = depths.shape
    mask = np.zeros((H, W), np.float32)
    planes = np.zeros((max(1, tris.shape[0]), 4), np.float32)
    pdepth = np.zeros((H, W), np.float32)
    pnormal = np.zeros((H, W, 3), np.float32)
    c = to_cam(cam)
    n = lib().ora_planar_prior(_p(tris), tris.shape[0], _p(depths), W, H, ctypes.byref(c), factor, depth_min,
                               depth_max, mode, _p(mask), _p(planes), _p(pdepth), _p(pnormal))
    return mask, planes[:n].copy(), pdepth, pnormal


def resize_linear(src: np.ndarray, dw: int, dh: int) -> np.ndarray:
    src = np.ascontiguousarray(src, np.float32)
    out = np.empty((dh, dw), np.float32)
    lib().ora_resize_linear_f32(_p(src), src.shape[1], src.shape[0], _p(out), dw, dh)
    return out


def prior_reload(udepth: np.ndarray, unormal: np.ndarray, cam, dmin: float, dmax: float):
    udepth = np.ascontiguousarray(udepth, np.float32)
    unormal = np.ascontiguousarray(unormal, np.float32)
    H, W = udepth.shape
    prior = np.zeros((H, W, 4), np.float32)
    mask = np.zeros((H, W), np.uint8)
    c = to_cam(cam)
    lib().ora_prior_reload(_p(udepth), _p(unormal), W, H, ctypes.byref(c), dmin, dmax, _p(prior), _p(mask))
    return prior, mask


def cost_grad64(ref, ref_cam, src, src_cam, params, px: int, py: int, theta, with_grad: bool = True):
    """FP64 differentiable cost of one (pixel, plane, source view) and d cost / d (depth, nx, ny)."""
    r = np.ascontiguousarray(ref, np.float32)
    s = np.ascontiguousarray(src, np.float32)
    th = np.ascontiguousarray(theta, np.float64)
    g = np.zeros(3, np.float64)
    rc, sc = to_cam(ref_cam), to_cam(src_cam)
    prm = to_params(params)
    c = lib().ora_cost_grad64(_p(r), ctypes.byref(rc), _p(s), ctypes.byref(sc), ctypes.byref(prm), px, py, _p(th),
                              _p(g) if with_grad else None)
    return c, g
