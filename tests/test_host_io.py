"""Host side of the command-line driver (libhpm_host.so and host/formats.cpp), CPU only.

Image decoding is compared with cv2.imdecode(IMREAD_COLOR), what the reference's
cv::imread returns (main.cpp:123-126): PNG bit-exact for every colour type and
depth cv2 writes plus hand-built palette and sub-byte grey files; JPEG within 3
grey levels (mean below 0.5) for 4:4:4, 4:2:2, 4:2:0 and 4:1:1 sampling, with
and without restart markers, because libjpeg's integer IDCT rounds differently.
The .dmb, pair.txt and cam formats are checked against the reference's layout
(HPM.cpp:159-184, 291-407; main.cpp:171-200) as written by the test-scene
generator.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import zlib

import cv2
import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "hpm-mvs_plusplus_b200", "_build")
HOST_LIB = os.path.join(BUILD, "libhpm_host.so")


@pytest.fixture(scope="module")
def host():
    if not os.path.exists(HOST_LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "hpm-mvs_plusplus_b200"), "_build/libhpm_host.so"],
                       check=True)
    lib = ctypes.CDLL(HOST_LIB)
    lib.hpm_decode_image.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.hpm_free_image.argtypes = [ctypes.c_void_p]
    lib.hpm_image_error.restype = ctypes.c_char_p
    return lib


def decode(lib, data: bytes) -> np.ndarray:
    p, w, h = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int()
    buf = np.frombuffer(data, np.uint8)
    rc = lib.hpm_decode_image(buf.ctypes.data, len(data), ctypes.byref(p), ctypes.byref(w), ctypes.byref(h))
    if rc:
        raise ValueError(lib.hpm_image_error().decode())
    out = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), (h.value, w.value, 3)).copy()
    lib.hpm_free_image(p)
    return out


def _image(h=97, w=131, seed=0):
    rng = np.random.default_rng(seed)
    return cv2.GaussianBlur(rng.integers(0, 256, (h, w, 3)).astype(np.uint8), (7, 7), 2)


@pytest.mark.parametrize("kind", ["bgr", "gray", "bgra", "bgr16", "gray16"])
def test_png_matches_cv2(host, kind):
    img = _image()
    im = {"bgr": img, "gray": img[..., 1], "bgra": np.dstack([img, img[..., :1]]),
          "bgr16": img.astype(np.uint16) * 257 + 3, "gray16": img[..., 0].astype(np.uint16) * 250}[kind]
    ok, b = cv2.imencode(".png", im)
    assert ok
    assert np.array_equal(decode(host, b.tobytes()), cv2.imdecode(b, cv2.IMREAD_COLOR))


def _png_chunk(tag: bytes, body: bytes) -> bytes:
    return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)


def _png(width, height, depth, ctype, rows, palette=None) -> bytes:
    raw = b"".join(b"\x00" + r for r in rows)
    out = b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", struct.pack(">IIBBBBB", width, height, depth, ctype, 0, 0, 0))
    if palette is not None:
        out += _png_chunk(b"PLTE", palette)
    return out + _png_chunk(b"IDAT", zlib.compress(raw)) + _png_chunk(b"IEND", b"")


@pytest.mark.parametrize("depth", [1, 2, 4, 8])
def test_png_palette_and_subbyte_grey(host, depth):
    rng = np.random.default_rng(depth)
    w, h = 37, 11
    idx = rng.integers(0, 1 << depth, (h, w))
    pal = rng.integers(0, 256, (1 << depth, 3)).astype(np.uint8)

    def pack(row):
        bits = "".join(format(int(v), f"0{depth}b") for v in row)
        bits += "0" * (-len(bits) % 8)
        return bytes(int(bits[i:i + 8], 2) for i in range(0, len(bits), 8))

    rows = [pack(r) for r in idx]
    for ctype in (3, 0):
        data = _png(w, h, depth, ctype, rows, pal.tobytes() if ctype == 3 else None)
        ref = cv2.imdecode(np.frombuffer(data, np.uint8), cv2.IMREAD_COLOR)
        assert np.array_equal(decode(host, data), ref), (depth, ctype)


@pytest.mark.parametrize("sampling", [0x111111, 0x211111, 0x221111, 0x411111])
@pytest.mark.parametrize("restart", [0, 3])
def test_jpeg_close_to_cv2(host, sampling, restart):
    img = _image(seed=sampling & 0xFF)
    for quality in (75, 95):
        params = [cv2.IMWRITE_JPEG_QUALITY, quality, cv2.IMWRITE_JPEG_SAMPLING_FACTOR, sampling]
        if restart:
            params += [cv2.IMWRITE_JPEG_RST_INTERVAL, restart]
        ok, b = cv2.imencode(".jpg", img, params)
        d = np.abs(decode(host, b.tobytes()).astype(int) - cv2.imdecode(b, cv2.IMREAD_COLOR).astype(int))
        assert d.max() <= 3 and d.mean() < 0.5, (hex(sampling), quality, d.max(), d.mean())


def test_jpeg_grey_and_errors(host):
    g = _image()[..., 0]
    ok, b = cv2.imencode(".jpg", g, [cv2.IMWRITE_JPEG_QUALITY, 90])
    d = np.abs(decode(host, b.tobytes()).astype(int) - cv2.imdecode(b, cv2.IMREAD_COLOR).astype(int))
    assert d.max() <= 1
    ok, b = cv2.imencode(".jpg", _image(), [cv2.IMWRITE_JPEG_PROGRESSIVE, 1])
    with pytest.raises(ValueError, match="progressive"):
        decode(host, b.tobytes())
    with pytest.raises(ValueError, match="unknown image format"):
        decode(host, b"GIF89a........")


def _segment(data: bytearray, marker: int) -> int:
    """Offset of the first segment with the given marker byte (0xFF marker)."""
    return bytes(data).index(bytes([0xFF, marker]))


def _corrupt(data: bytes, marker: int, edit) -> bytes:
    b = bytearray(data)
    edit(b, _segment(b, marker))
    return bytes(b)


def _set_len(b: bytearray, at: int, length: int) -> None:
    b[at + 2], b[at + 3] = length >> 8, length & 0xFF


def test_jpeg_rejects_corrupt_segments(host):
    """Malformed table and scan headers are rejected with an error, never read past their segment."""
    ok, b = cv2.imencode(".jpg", _image(), [cv2.IMWRITE_JPEG_QUALITY, 90])
    good = b.tobytes()
    decode(host, good)
    cases = [
        # SOS: Huffman table selectors 5 / 7 (only 0..3 exist)
        (0xDA, lambda b, at: b.__setitem__(at + 6, 0x57), "Huffman table selector"),
        # SOS: length too short for its component list
        (0xDA, lambda b, at: _set_len(b, at, 2 + 3), "truncated scan header"),
        # DHT: length shorter than the 16 code-length counts
        (0xC4, lambda b, at: _set_len(b, at, 2 + 10), "truncated Huffman table"),
        # DHT: a code-length count whose symbols run past the segment
        (0xC4, lambda b, at: b.__setitem__(at + 5 + 15, 200), "Huffman table"),
        # DQT: precision 2 (only 8- and 16-bit tables exist)
        (0xDB, lambda b, at: b.__setitem__(at + 4, 0x20 | (b[at + 4] & 15)), "precision"),
        # DQT: length shorter than one 64-entry table
        (0xDB, lambda b, at: _set_len(b, at, 2 + 30), "truncated quantisation table"),
        # SOF: length shorter than the component list
        (0xC0, lambda b, at: _set_len(b, at, 2 + 8), "truncated frame header"),
    ]
    for marker, edit, msg in cases:
        with pytest.raises(ValueError, match=msg):
            decode(host, _corrupt(good, marker, edit))
    # a file cut anywhere in its headers or scan decodes or fails cleanly
    sos = _segment(bytearray(good), 0xDA)
    for cut in list(range(2, sos + 16)) + list(range(sos + 16, len(good), 97)):
        try:
            decode(host, good[:cut])
        except ValueError:
            pass


def test_scene_folder_formats(tmp_path):
    """cams, pair.txt and .dmb as the reference reads them, via the command-line driver's own parser."""
    from hpm_b200 import synth

    sc = synth.make_scene(n_views=3, width=64, height=48, seed=2, n_src=2)
    synth.write_dense_folder(sc, str(tmp_path))
    # pair.txt: the reference drops sources with score <= 0
    with open(tmp_path / "pair.txt") as fh:
        tokens = fh.read().split()
    assert int(tokens[0]) == 3
    # cam file: extrinsic, last row, intrinsic, depth line (HPM.cpp:159-184)
    with open(tmp_path / "cams" / "00000001_cam.txt") as fh:
        words = fh.read().split()
    assert words[0] == "extrinsic" and words[17] == "intrinsic"
    R = np.array(words[1:13], float).reshape(3, 4)
    assert np.allclose(R[:, :3], sc.views[1].R, atol=1e-6) and np.allclose(R[:, 3], sc.views[1].t, atol=1e-6)
    K = np.array(words[18:27], float).reshape(3, 3)
    assert np.allclose(K, sc.views[1].K, rtol=1e-6)
    dmin, interval, num, dmax = (float(x) for x in words[27:31])
    assert num == 192 and abs(dmin - sc.views[1].depth_min) < 1e-5 and abs(dmax - sc.views[1].depth_max) < 1e-5
    # images are PNG bytes under .jpg names, which imread sniffs
    with open(tmp_path / "images" / "00000000.jpg", "rb") as fh:
        assert fh.read(8) == b"\x89PNG\r\n\x1a\n"


def _parse_ply(raw: bytes):
    end = raw.index(b"end_header\n") + len(b"end_header\n")
    header = raw[:end].decode()
    n = int(header.split("element vertex ")[1].split()[0])
    fused = "property float nx" in header
    dt = np.dtype([("xyz", "<f4", 3), ("n", "<f4", 3), ("rgb", "u1", 3)]) if fused else \
        np.dtype([("xyz", "<f4", 3), ("rgb", "u1", 3)])
    assert len(raw) == end + n * dt.itemsize
    return np.frombuffer(raw[end:], dt)


def test_write_ply_contracts(host, tmp_path):
    """hpm_write_ply (ExportPointCloud / ExportFusedPointCloud, HPM.cpp:410-498):
    non-finite coordinates become 0 in the plain file; the fused file drops points
    with non-finite coordinates or a zero normal, makes normals unit and clamps
    colours; misuse returns -1."""
    host.hpm_write_ply.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_size_t)]
    pts = np.array([
        [1, 2, 3, 0, 0, 2, 10, 20, 30],              # ordinary point, normal of length 2
        [np.inf, 2, 3, 0, 1, 0, 10, 20, 30],         # non-finite coordinate
        [4, 5, 6, 0, 0, 0, 300, -5, 12.7],           # zero normal, colours out of range
        [7, 8, 9, 3, 4, 0, 255, 128, 0],
    ], np.float32)
    n = ctypes.c_size_t()
    plain = tmp_path / "plain.ply"
    assert host.hpm_write_ply(str(plain).encode(), pts.ctypes.data, len(pts), 0, ctypes.byref(n)) == 0
    p = _parse_ply(plain.read_bytes())
    assert n.value == 4 and len(p) == 4
    assert np.array_equal(p["xyz"][1], [0, 0, 0])
    assert np.array_equal(p["rgb"][0], [30, 20, 10])  # BGR floats stored as R, G, B
    fused = tmp_path / "fused.ply"
    assert host.hpm_write_ply(str(fused).encode(), pts.ctypes.data, len(pts), 1, ctypes.byref(n)) == 0
    f = _parse_ply(fused.read_bytes())
    assert n.value == 2 and len(f) == 2
    assert np.allclose(f["n"], [[0, 0, 1], [0.6, 0.8, 0]])
    assert np.array_equal(f["rgb"][1], [0, 128, 255])
    assert host.hpm_write_ply(None, pts.ctypes.data, len(pts), 0, None) == -1
    assert host.hpm_write_ply(str(tmp_path / "x.ply").encode(), None, 3, 0, None) == -1
    assert host.hpm_write_ply(str(tmp_path / "no_such_dir" / "x.ply").encode(), pts.ctypes.data, 1, 1, None) == -1
