"""The reference's own host stages against the oracle, on the CPU.

oracle/_ref/libhpmref_host.so holds ConfidenceEvaluation and RunFusion /
RunFusion_Sky_Strict of the reference's main.cpp (main.cpp:659-1109), compiled
from its sources with OpenCV stood in (oracle/ref_host.mk).  Each test writes
a dense folder (cams, images, the .dmb maps of a seeded 5-view scene with
perturbed depths and holes), runs the reference stage on it, and compares
what it wrote -- confidence.dmb, fused.ply, HPM_MVS_plusplus(_mask).ply --
with the oracle's restatement (ora_confidence_eval, ora_fusion) on the same
maps.  Both are IEEE host code.  Point sets, order, coordinates, normals and
colours are compared bit for bit, and the library's own PLY writer
(hpm_write_ply) reproduces the reference's files byte for byte.  A confidence value sums float exp terms:
the reference's exp(float) is glibc's expf, accurate to 0.502 ulp, which in
about 0.07 % of evaluations rounds the other way from the correctly rounded
value the oracle and the CUDA path use.  Confidences are therefore required on
exactly the same pixels and to 2 ulp.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

import hpm_oracle as ora
from conftest import scene_cams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libhpmref_host.so")
HOST_LIB = os.path.join(os.path.dirname(HERE), "hpm-mvs_plusplus_b200", "_build", "libhpm_host.so")
if not os.path.exists(LIB):
    pytest.skip("reference host build oracle/_ref/libhpmref_host.so not present", allow_module_level=True)

SKY = (234, 235, 55)  # the sky colour RunFusion_Sky_Strict drops (main.cpp:805)


def _lib():
    lib = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    lib.ref_host_confidence.argtypes = [ctypes.c_char_p, ctypes.c_int, vp, vp, ctypes.c_int]
    lib.ref_host_fusion.argtypes = [ctypes.c_char_p, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int]
    return lib


def _write_dmb(path, a):
    a = np.ascontiguousarray(a, np.float32)
    h, w = a.shape[:2]
    c = 1 if a.ndim == 2 else a.shape[2]
    with open(path, "wb") as fh:
        fh.write(np.array([1, h, w, c], np.int32).tobytes())
        fh.write(a.tobytes())


def _read_dmb(path):
    with open(path, "rb") as fh:
        t, h, w, c = np.frombuffer(fh.read(16), np.int32)
        data = np.frombuffer(fh.read(), np.float32)
    return data.reshape((h, w, c) if c > 1 else (h, w))


def _write_raw(path, img):
    img = np.ascontiguousarray(img, np.uint8)
    c = 1 if img.ndim == 2 else img.shape[2]
    with open(path + ".raw", "wb") as fh:
        fh.write(np.array([img.shape[0], img.shape[1], c], np.int32).tobytes())
        fh.write(img.tobytes())


def _read_ply(path):
    with open(path, "rb") as fh:
        raw = fh.read()
    end = raw.index(b"end_header\n") + len(b"end_header\n")
    header = raw[:end].decode()
    n = int(header.split("element vertex ")[1].split()[0])
    if "property float nx" in header:
        dt = np.dtype([("xyz", "<f4", 3), ("n", "<f4", 3), ("rgb", "u1", 3)])
    else:
        dt = np.dtype([("xyz", "<f4", 3), ("rgb", "u1", 3)])
    return np.frombuffer(raw[end:end + n * dt.itemsize], dt)


@pytest.fixture(scope="module", params=["even", "uneven"])
def folder(request, tmp_path_factory, small_scene):
    """The 5-view 160x120 scene, and a 5-view scene whose views differ in size."""
    if request.param == "even":
        return write_folder(tmp_path_factory.mktemp("dense"), small_scene)
    from hpm_b200 import synth
    scene = synth.make_scene(n_views=5, width=160, height=120, seed=2, n_src=4,
                             sizes=[(160, 120), (144, 108), (176, 132), (160, 100), (120, 120)])
    return write_folder(tmp_path_factory.mktemp("dense_uneven"), scene)


def write_folder(root, small_scene):
    """Dense folder of the 5-view scene: depths with 0.3 % noise, 5 % holes and
    5 % of pixels moved off the surface; normals tilted by noise (sigma 0.02)."""
    from hpm_b200 import synth

    rng = np.random.default_rng(3)
    cams = scene_cams(small_scene)
    os.makedirs(root / "cams")
    os.makedirs(root / "images")
    os.makedirs(root / "masks")
    depths, normals, colors, skies = [], [], [], []
    for i, v in enumerate(small_scene.views):
        synth.write_cam(str(root / "cams" / f"{i:08d}_cam.txt"), v)
        d = v.depth.astype(np.float32) * (1 + rng.normal(0, 0.003, v.depth.shape)).astype(np.float32)
        d[rng.uniform(size=d.shape) < 0.05] = 0.0
        far = rng.uniform(size=d.shape) < 0.05
        d[far] *= np.float32(1.3)
        n = v.normal.astype(np.float32) + rng.normal(0, 0.02, v.normal.shape).astype(np.float32)
        n /= np.maximum(np.linalg.norm(n, axis=2, keepdims=True), 1e-6)
        sky = rng.integers(0, 256, v.image.shape).astype(np.uint8)
        sky[rng.uniform(size=d.shape) < 0.2] = SKY
        sky[rng.uniform(size=d.shape) < 0.05, 0] = SKY[0]  # one channel alone also drops the point
        res = root / "HPM_MVS_plusplus" / f"2333_{i:08d}"
        os.makedirs(res)
        _write_dmb(res / "depths.dmb", d)
        _write_dmb(res / "depths_geom.dmb", d)
        _write_dmb(res / "normals.dmb", n)
        _write_raw(str(root / "images" / f"{i:08d}.jpg"), v.image)
        _write_raw(str(root / "masks" / f"{i:08d}.jpg"), sky)
        depths.append(d); normals.append(n); colors.append(v.image); skies.append(sky)
    srcs = [[j for j, _ in p] for p in small_scene.pairs]
    off = np.zeros(len(srcs) + 1, np.int32)
    for i, s in enumerate(srcs):
        off[i + 1] = off[i] + len(s)
    ids = np.concatenate([np.asarray(s, np.int32) for s in srcs])
    return dict(root=root, cams=cams, depths=depths, normals=normals, colors=colors, skies=skies, srcs=srcs,
                off=off, ids=ids)


@pytest.mark.parametrize("geom", [0, 1])
def test_confidence_evaluation_matches_reference_host_code(folder, geom):
    f = folder
    rc = _lib().ref_host_confidence(str(f["root"]).encode(), len(f["depths"]), f["off"].ctypes.data,
                                    f["ids"].ctypes.data, geom)
    assert rc == 0
    ref = [_read_dmb(f["root"] / "HPM_MVS_plusplus" / f"2333_{i:08d}" / "confidence.dmb")
           for i in range(len(f["depths"]))]
    got = ora.confidence_eval(f["cams"], f["depths"], f["normals"], f["srcs"])
    for i, (a, b) in enumerate(zip(got, ref)):
        assert (b > 0).mean() > 0.05, i  # a good share of the scene is consistent
        assert np.array_equal(a > 0, b > 0), i
        differ = a != b
        assert differ.mean() <= 0.005, (i, int(differ.sum()))
        assert (np.abs(a[differ] - b[differ]) <= 2.4e-7 * b[differ]).all(), i


def _oracle_points(f, sky):
    pts, total = ora.fusion(f["cams"], f["depths"], f["normals"], f["colors"], f["srcs"],
                            sky_masks=f["skies"] if sky else None)
    assert total == len(pts)
    return pts


@pytest.mark.parametrize("sky", [0, 1])
def test_fusion_matches_reference_host_code(folder, sky):
    f = folder
    rc = _lib().ref_host_fusion(str(f["root"]).encode(), len(f["depths"]), f["off"].ctypes.data,
                                f["ids"].ctypes.data, 1, sky)
    assert rc == 0
    pts = _oracle_points(f, sky)
    out = f["root"] / "HPM_MVS_plusplus"
    # HPM_MVS_plusplus(_mask).ply: coordinates and (int) colours, in the reference's order (HPM.cpp:444-498)
    plain = _read_ply(out / ("HPM_MVS_plusplus_mask.ply" if sky else "HPM_MVS_plusplus.ply"))
    assert len(plain) == len(pts) > 1000
    assert np.array_equal(plain["xyz"].view(np.uint32), pts[:, 0:3].view(np.uint32))
    bgr = pts[:, 6:9].astype(np.int32).astype(np.uint8)
    assert np.array_equal(plain["rgb"], bgr[:, ::-1])
    # fused.ply: unit normals normalised in double, colours clamped (HPM.cpp:410-442)
    fused = _read_ply(out / "fused.ply")
    n = pts[:, 3:6].astype(np.float64)
    length = np.sqrt(n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1] + n[:, 2] * n[:, 2])
    keep = np.isfinite(pts[:, 0:3]).all(axis=1) & np.isfinite(length * length) & (length * length > 1e-20)
    assert len(fused) == int(keep.sum())
    assert np.array_equal(fused["xyz"].view(np.uint32), pts[keep, 0:3].view(np.uint32))
    assert np.array_equal(fused["n"], (n[keep] / length[keep, None]).astype(np.float32))
    assert np.array_equal(fused["rgb"], np.clip(pts[keep, 6:9], 0, 255).astype(np.uint8)[:, ::-1])
    # the library's writers (hpm_write_ply, include/hpm_host.h) give the same files byte for byte
    host = ctypes.CDLL(HOST_LIB)
    host.hpm_write_ply.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_size_t)]
    pts = np.ascontiguousarray(pts, np.float32)
    for fused_flag, name in ((0, "HPM_MVS_plusplus_mask.ply" if sky else "HPM_MVS_plusplus.ply"), (1, "fused.ply")):
        mine = f["root"] / f"ours_{sky}_{name}"
        n = ctypes.c_size_t()
        assert host.hpm_write_ply(str(mine).encode(), pts.ctypes.data, len(pts), fused_flag, ctypes.byref(n)) == 0
        assert (out / name).read_bytes() == mine.read_bytes(), name


@pytest.mark.parametrize("factor", [1.0, 0.5, 0.25])
def test_support_points_match_reference_host_code(factor):
    """HPM::GetSupportPoints_Classify_Check (HPM.cpp:1026-1073) on seeded cost
    and confidence maps: the same points in the same order."""
    import hpm_b200

    W, H = 203, 157
    w, h = int(W * np.float32(factor)), int(H * np.float32(factor))
    rng = np.random.default_rng(int(factor * 100))
    costs = rng.uniform(0.0, 0.4, (h, w)).astype(np.float32)
    costs[rng.uniform(size=(h, w)) < 0.2] = 2.0
    costs[rng.uniform(size=(h, w)) < 0.1] = np.float32(0.05)  # ties: the first pixel in scan order wins
    conf = np.where(rng.uniform(size=(h, w)) < 0.5, 0.0, rng.uniform(0.0, 0.3, (h, w))).astype(np.float32)
    texture = rng.uniform(0.4, 1.0, (h, w)).astype(np.float32)
    cam = hpm_b200.Camera.make(np.diag([300.0, 300.0, 1.0]), np.eye(3), np.zeros(3), W, H, 1.0, 5.0)
    lib = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    lib.ref_host_support_points.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, vp,
                                            ctypes.c_int]
    cap = 2 * ((w + 4) // 5) * ((h + 4) // 5) + 8
    out = np.zeros((cap, 2), np.int32)
    n = lib.ref_host_support_points(ctypes.addressof(cam), costs.ctypes.data, conf.ctypes.data, texture.ctypes.data,
                                    w, h, factor, out.ctypes.data, cap)
    assert 0 < n <= cap
    got = ora.support_points(costs, conf, w, h)
    assert np.array_equal(got, out[:n])
