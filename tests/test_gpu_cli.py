"""The HPM-MVS_plusplus command-line driver on a dense folder (B200).

`HPM-MVS_plusplus folder --initial-image-scale 1 --show-medium-result` with a
fixed seed must write the same maps the C ABI's hpm_reconstruct leaves resident
(.dmb layout of HPM.cpp:291-407, bit for bit), and PLY files holding the fused
points (HPM.cpp:410-482).  --fusion-only re-fuses the written maps into the
same cloud; --mask drops the points under the sky colour (main.cpp:805).
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import hpm_b200
from conftest import scene_cams

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "hpm-mvs_plusplus_b200", "_build", "HPM-MVS_plusplus")


def read_dmb(path):
    with open(path, "rb") as fh:
        t, h, w, c = np.frombuffer(fh.read(16), np.int32)
        assert t == 1
        data = np.frombuffer(fh.read(), np.float32)
    assert data.size == h * w * c
    return data.reshape((h, w, c) if c > 1 else (h, w))


def read_ply(path):
    with open(path, "rb") as fh:
        raw = fh.read()
    end = raw.index(b"end_header\n") + len(b"end_header\n")
    header = raw[:end].decode()
    n = int(header.split("element vertex ")[1].split()[0])
    floats = header.count("property float")
    dt = np.dtype([("f", "<f4", (floats,)), ("rgb", "u1", (3,))])
    return n, np.frombuffer(raw[end:], dt, count=n)


def same(a, b):
    return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())


def run_cli(folder, *args, seed=11):
    env = dict(os.environ, HPM_SEED=str(seed))
    r = subprocess.run([CLI, folder, *args], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_cli_matches_c_abi(tmp_path):
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=5, width=160, height=120, seed=1, n_src=4)
    folder = str(tmp_path)
    synth.write_dense_folder(sc, folder)
    out = run_cli(folder, "--initial-image-scale", "1", "--show-medium-result")
    assert "Total execution time" in out

    cams = scene_cams(sc)
    srcs = [[j for j, _ in p] for p in sc.pairs]
    with hpm_b200.Context(0) as ctx:
        for i, v in enumerate(sc.views):
            ctx.set_image(i, v.image)
        n_pts = ctx.reconstruct(cams, srcs, initial_image_scale=1, seed=11, fuse=True)
        pts = ctx.get_points()
        for i in range(len(sc.views)):
            d = os.path.join(folder, "HPM_MVS_plusplus", f"2333_{i:08d}")
            for name, kind in (("depths.dmb", hpm_b200.MAP_DEPTH), ("depths_geom.dmb", hpm_b200.MAP_DEPTH_GEOM),
                               ("normals.dmb", hpm_b200.MAP_NORMAL), ("costs.dmb", hpm_b200.MAP_COST),
                               ("confidence.dmb", hpm_b200.MAP_CONF)):
                assert same(read_dmb(os.path.join(d, name)), ctx.get_map(i, kind)), (i, name)
    n, cloud = read_ply(os.path.join(folder, "HPM_MVS_plusplus", "HPM_MVS_plusplus.ply"))
    assert n == n_pts
    xyz = pts[:, :3].copy()
    xyz[~np.isfinite(xyz).all(1)] = 0
    assert np.array_equal(cloud["f"], xyz)
    assert np.array_equal(cloud["rgb"].astype(np.int64), pts[:, [8, 7, 6]].astype(np.int64) & 0xFF)
    nf, fused = read_ply(os.path.join(folder, "HPM_MVS_plusplus", "fused.ply"))
    assert 0 < nf <= n
    assert np.allclose(np.linalg.norm(fused["f"][:, 3:], axis=1), 1, atol=1e-5)

    # --fusion-only re-reads depths_geom.dmb / normals.dmb and fuses the same points
    run_cli(folder, "--fusion-only")
    n2, cloud2 = read_ply(os.path.join(folder, "HPM_MVS_plusplus", "HPM_MVS_plusplus.ply"))
    assert n2 == n and np.array_equal(cloud2["f"], cloud["f"])

    # --mask: pixels painted in the sky colour (B, G, R) = (234, 235, 55) fuse no point
    import cv2
    os.makedirs(os.path.join(folder, "masks"))
    for i, v in enumerate(sc.views):
        m = np.zeros_like(v.image)
        m[: v.image.shape[0] // 2] = (234, 235, 55)
        ok, png = cv2.imencode(".png", m)  # PNG bytes under the .jpg name, as the scene images
        with open(os.path.join(folder, "masks", f"{i:08d}.jpg"), "wb") as fh:
            fh.write(png.tobytes())
    run_cli(folder, "--fusion-only", "--mask")
    n3, _ = read_ply(os.path.join(folder, "HPM_MVS_plusplus", "HPM_MVS_plusplus.ply"))
    assert 0 < n3 < n


def test_cli_rejects_bad_arguments(tmp_path):
    r = subprocess.run([CLI, str(tmp_path), "--initial-image-scale", "0"], capture_output=True, text=True)
    assert r.returncode != 0 and "positive integer" in r.stderr
    r = subprocess.run([CLI, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode != 0 and "pair.txt" in r.stderr


def test_per_problem_mode_matches_resident_schedule(tmp_path):
    """--per-problem: the reference's main loop through the HPM class with .dmb files between stages,
    two pyramid levels (HPM_LEVEL_MAX_SIDE=100 on 160x120 views), against the default resident run."""
    import shutil
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=5, width=160, height=120, seed=2, n_src=4)
    a, b = str(tmp_path / "resident"), str(tmp_path / "per_problem")
    synth.write_dense_folder(sc, a)
    shutil.copytree(a, b)
    env = dict(os.environ, HPM_SEED="13", HPM_LEVEL_MAX_SIDE="100")
    for folder, extra in ((a, []), (b, ["--per-problem"])):
        r = subprocess.run([CLI, folder, "--initial-image-scale", "1", *extra], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for i in range(5):
        for name in ("depths.dmb", "depths_geom.dmb", "normals.dmb"):
            x = read_dmb(os.path.join(a, "HPM_MVS_plusplus", f"2333_{i:08d}", name))
            y = read_dmb(os.path.join(b, "HPM_MVS_plusplus", f"2333_{i:08d}", name))
            assert x.shape == y.shape and same(x, y), (i, name)
        assert not os.path.exists(os.path.join(b, "HPM_MVS_plusplus", f"2333_{i:08d}", "costs.dmb"))
    na, pa = read_ply(os.path.join(a, "HPM_MVS_plusplus", "HPM_MVS_plusplus.ply"))
    nb, pb = read_ply(os.path.join(b, "HPM_MVS_plusplus", "HPM_MVS_plusplus.ply"))
    assert na == nb and np.array_equal(pa["f"], pb["f"])
