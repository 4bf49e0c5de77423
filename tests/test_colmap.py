"""COLMAP model -> cams/, pair.txt, images/ (hpm-mvs_plusplus_b200/colmap2mvs.py) against
the reference's own colmap2mvsnet_acm.py output on the same model
(tests/golden/colmap, made by tests/golden/make_colmap_golden.py).

pair.txt and every camera file must be byte-identical to the reference's; the
binary model format must give the same output as the text format.
"""
from __future__ import annotations

import importlib.util
import os
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "colmap")


def _converter():
    path = os.path.join(ROOT, "hpm-mvs_plusplus_b200", "colmap2mvs.py")
    spec = importlib.util.spec_from_file_location("colmap2mvs", path)
    mod = importlib.util.module_from_spec(spec)
    import sys
    sys.modules["colmap2mvs"] = mod  # dataclasses resolve their module by name
    spec.loader.exec_module(mod)
    return mod


def _numbers(path):
    with open(path) as fh:
        return np.array([float(t) for t in fh.read().split() if t not in ("extrinsic", "intrinsic")])


def _write_binary_model(conv, sparse_txt: str, out: str) -> None:
    """The text model rewritten in COLMAP's binary layout."""
    cams = conv.read_cameras_text(os.path.join(sparse_txt, "cameras.txt"))
    imgs = conv.read_images_text(os.path.join(sparse_txt, "images.txt"))
    pts = conv.read_points3d_text(os.path.join(sparse_txt, "points3D.txt"))
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(out, "cameras.bin"), "wb") as fh:
        fh.write(struct.pack("<Q", len(cams)))
        for cid, c in cams.items():
            fh.write(struct.pack("<iiQQ", cid, conv.MODEL_BY_NAME[c.model][0], c.width, c.height))
            fh.write(struct.pack("<" + "d" * len(c.params), *c.params))
    with open(os.path.join(out, "images.bin"), "wb") as fh:
        fh.write(struct.pack("<Q", len(imgs)))
        for iid, im in imgs.items():
            fh.write(struct.pack("<idddddddi", iid, *im.qvec, *im.tvec, im.camera_id))
            fh.write(im.name.encode() + b"\x00")
            fh.write(struct.pack("<Q", len(im.point3D_ids)))
            for k, pid in enumerate(im.point3D_ids):
                fh.write(struct.pack("<ddq", float(k), float(k), int(pid)))
    with open(os.path.join(out, "points3D.bin"), "wb") as fh:
        fh.write(struct.pack("<Q", len(pts)))
        for pid, xyz in pts.items():
            fh.write(struct.pack("<QdddBBBd", pid, *xyz, 128, 128, 128, 0.5))
            fh.write(struct.pack("<Q", 2) + struct.pack("<iiii", 1, 0, 2, 0))


@pytest.mark.parametrize("ext", [".txt", ".bin"])
def test_converter_matches_reference_output(tmp_path, ext):
    conv = _converter()
    dense = os.path.join(GOLD, "dense")
    if ext == ".bin":
        import shutil
        dense = str(tmp_path / "dense_bin")
        shutil.copytree(os.path.join(GOLD, "dense", "images"), os.path.join(dense, "images"))
        _write_binary_model(conv, os.path.join(GOLD, "dense", "sparse"), os.path.join(dense, "sparse"))
    out = str(tmp_path / "out")
    assert conv.main(["--dense_folder", dense, "--save_folder", out, "--model_ext", ext]) == 0
    with open(os.path.join(out, "pair.txt")) as a, open(os.path.join(GOLD, "expected", "pair.txt")) as b:
        assert a.read() == b.read()
    names = sorted(os.listdir(os.path.join(GOLD, "expected", "cams")))
    assert sorted(os.listdir(os.path.join(out, "cams"))) == names
    identical = 0
    for n in names:
        mine, ref = os.path.join(out, "cams", n), os.path.join(GOLD, "expected", "cams", n)
        a, b = _numbers(mine), _numbers(ref)
        assert a.shape == b.shape
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)
        assert np.array_equal(a.astype(np.float32), b.astype(np.float32))
        with open(mine) as x, open(ref) as y:
            identical += x.read() == y.read()
    print(f"{identical}/{len(names)} camera files byte-identical to the reference converter's")
    assert identical == len(names)
    # .jpg inputs are copied, others re-encoded
    with open(os.path.join(out, "images", "00000000.jpg"), "rb") as x, \
            open(os.path.join(GOLD, "dense", "images", "view_00.jpg"), "rb") as y:
        assert x.read() == y.read()
    import cv2
    got = cv2.imread(os.path.join(out, "images", "00000001.jpg"))
    src = cv2.imread(os.path.join(GOLD, "dense", "images", "view_01.png"))
    assert got.shape == src.shape and np.abs(got.astype(int) - src.astype(int)).mean() < 3


def test_converter_rejects_an_image_without_points(tmp_path):
    conv = _converter()
    import shutil
    dense = str(tmp_path / "d")
    shutil.copytree(os.path.join(GOLD, "dense"), dense)
    path = os.path.join(dense, "sparse", "images.txt")
    with open(path) as fh:
        lines = fh.readlines()
    lines[2] = "\n"  # the first image's 2D points: none
    with open(path, "w") as fh:
        fh.writelines(lines)
    with pytest.raises(ValueError, match="no 3D point"):
        conv.convert(dense, str(tmp_path / "o"))
