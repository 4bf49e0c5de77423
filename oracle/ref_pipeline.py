"""REFERENCE PIPELINE -- benchmark and test infrastructure only.

The schedule of the reference's main() (main.cpp:1143-1364, restated over
in-memory maps by oracle/pipeline.py) run on the reference's own code wherever
that code was built here, with every stage timed:

  * PatchMatch: HPM::RunPatchMatch of the reference's HPM.cu compiled for
    sm_100a (oracle/_ref/libhpmref.so through ref_cuda.run_patchmatch; its own
    CUDA-event time of the call), plus the per-run host work of ProcessProblem
    and InuputInitialization (grey conversion of the reference and source
    images, Canny of the reference, main.cpp:237-330, HPM.cpp:643-697);
  * JBU between levels: the reference's JBU_cu kernel (ref_cuda.jbu), the maps
    handed on from the C restatement of RunJBU (equal to the kernel's to 2.7e-7);
  * ConfidenceEvaluation (main.cpp:959-1109) and RunFusion (main.cpp:823-957):
    the reference's main.cpp compiled for the CPU (oracle/_ref/libhpmref_host.so),
    single-threaded as the reference runs them, reading the .dmb files of a
    dense folder as the reference does (writing those files is not timed);
  * planar-prior construction (HPM.cpp:1026-1206, main.cpp:384-576): support
    points and the raster, plane fits and prior JBU by the C restatement, the
    Delaunay triangulation by cv2.Subdiv2D, the OpenCV class the reference calls.

Random draws go through the shared Philox stream (ref_cuda).  The runs of one
view (`record_view`) are kept with their exact inputs, so that a benchmark can
replay that view's share of the schedule.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import time

import cv2
import numpy as np

import hpm_oracle as ora
import pipeline as op
import ref_cuda

HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB = os.path.join(HERE, "_ref", "libhpmref_host.so")
MODE_NAMES = {0: "photometric", 2: "prior", 8: "hierarchy", 24: "hierarchy", 1: "geometric", 37: "mandatory"}


def host_available() -> bool:
    return os.path.exists(HOST_LIB)


def _write_dmb(path: str, a: np.ndarray) -> None:
    a = np.ascontiguousarray(a, np.float32)
    with open(path, "wb") as fh:
        fh.write(np.array([1, a.shape[0], a.shape[1], 1 if a.ndim == 2 else a.shape[2]], np.int32).tobytes())
        fh.write(a.tobytes())


def _read_dmb(path: str) -> np.ndarray:
    with open(path, "rb") as fh:
        hdr = np.frombuffer(fh.read(16), np.int32)
        data = np.frombuffer(fh.read(), np.float32)
    h, w, nb = int(hdr[1]), int(hdr[2]), int(hdr[3])
    return data.reshape((h, w) if nb == 1 else (h, w, nb)).copy()


def _write_cam(path: str, c) -> None:
    K = np.array(c.K[:], np.float64).reshape(3, 3)
    R = np.array(c.R[:], np.float64).reshape(3, 3)
    t = np.array(c.t[:], np.float64)
    with open(path, "w") as fh:
        fh.write("extrinsic\n")
        for r in range(3):
            fh.write(" ".join(f"{R[r, k]:.9g}" for k in range(3)) + f" {t[r]:.9g}\n")
        fh.write("0 0 0 1\n\nintrinsic\n")
        for r in range(3):
            fh.write(" ".join(f"{K[r, k]:.9g}" for k in range(3)) + "\n")
        fh.write(f"\n{c.depth_min:.9g} 0.01 192 {c.depth_max:.9g}\n")


class RefPipeline(op.OraclePipeline):
    def __init__(self, images, cams, src_lists, initial_image_scale=1, seed=0, record_view=None, folder=None):
        super().__init__(images, cams, src_lists, initial_image_scale=initial_image_scale, seed=seed)
        self.record_view = record_view
        self.records = []
        self.folder = folder
        self.host = ctypes.CDLL(HOST_LIB) if host_available() else None
        if self.host is not None:
            vp = ctypes.c_void_p
            self.host.ref_host_confidence.argtypes = [ctypes.c_char_p, ctypes.c_int, vp, vp, ctypes.c_int]
            self.host.ref_host_fusion.argtypes = [ctypes.c_char_p, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_int]
        n = len(self.views)
        self.off = np.zeros(n + 1, np.int32)
        for i, s in enumerate(self.srcs):
            self.off[i + 1] = self.off[i] + len(s)
        self.ids = np.concatenate([np.asarray(s, np.int32) for s in self.srcs])
        self.t = {"pm_host_s": 0.0, "prior_s": 0.0, "confidence_s": 0.0, "jbu_s": 0.0, "fusion_s": 0.0}
        self.pm = {}            # (WxH, mode name) -> [reference RunPatchMatch ms, runs]
        self.prior_view_s = {}  # view -> prior construction seconds
        self.written_level = None

    # ---- the reference's dense folder at the current level (not timed) ----
    def _folder_level(self, kind: str) -> None:
        for sub in ("cams", "images"):
            os.makedirs(os.path.join(self.folder, sub), exist_ok=True)
        for i, v in enumerate(self.views):
            if self.written_level != (v.w, v.h):
                _write_cam(os.path.join(self.folder, "cams", f"{i:08d}_cam.txt"), v.cam)
                img = np.ascontiguousarray(v.color, np.uint8)
                with open(os.path.join(self.folder, "images", f"{i:08d}.jpg.raw"), "wb") as fh:
                    fh.write(np.array([img.shape[0], img.shape[1], 3], np.int32).tobytes())
                    fh.write(img.tobytes())
            res = os.path.join(self.folder, "HPM_MVS_plusplus", f"2333_{i:08d}")
            os.makedirs(res, exist_ok=True)
            _write_dmb(os.path.join(res, "depths_geom.dmb" if kind == "depth_geom" else "depths.dmb"), v.maps[kind])
            _write_dmb(os.path.join(res, "normals.dmb"), v.maps["normal"])
        self.written_level = (self.views[0].w, self.views[0].h)

    # ---- stages ----
    def run(self, i: int, mode: int, level: int) -> None:
        v = self.views[i]
        t0 = time.perf_counter()
        for j in [i] + self.srcs[i]:
            cv2.cvtColor(self.views[j].color, cv2.COLOR_BGR2GRAY).astype(np.float32)
        cv2.Canny(v.color, 50, 150)
        self.t["pm_host_s"] += time.perf_counter() - t0

        def runner(images, depths, cams, params, st, seed, view_id):
            if view_id == self.record_view:
                self.records.append({"images": list(images), "depths": None if depths is None else list(depths),
                                     "colors": [self.views[j].color for j in [i] + self.srcs[i]],
                                     "cams": [ora.to_cam(c) for c in cams], "params": ora.to_params(params),
                                     "state": _copy_state(st), "seed": seed, "view": view_id, "level": level,
                                     "mode": int(params.mode)})
            ms = ref_cuda.run_patchmatch(images, depths, cams, params, st, seed, view_id)
            key = (f"{st.W}x{st.H}", MODE_NAMES.get(int(params.mode), str(int(params.mode))))
            acc = self.pm.setdefault(key, [0.0, 0])
            acc[0] += ms
            acc[1] += 1

        saved = ora.run_patchmatch
        ora.run_patchmatch = runner
        try:
            super().run(i, mode, level)
        finally:
            ora.run_patchmatch = saved

    def confidence(self, kind: str) -> None:
        if self.host is None:
            t0 = time.perf_counter()
            super().confidence(kind)
            self.t["confidence_s"] += time.perf_counter() - t0
            return
        self._folder_level(kind)
        t0 = time.perf_counter()
        rc = self.host.ref_host_confidence(self.folder.encode(), len(self.views), self.off.ctypes.data,
                                           self.ids.ctypes.data, 1 if kind == "depth_geom" else 0)
        self.t["confidence_s"] += time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError("reference ConfidenceEvaluation failed")
        for i, v in enumerate(self.views):
            v.maps["conf"] = _read_dmb(os.path.join(self.folder, "HPM_MVS_plusplus", f"2333_{i:08d}",
                                                    "confidence.dmb"))

    def build_prior(self, i: int, distance: int) -> None:
        t0 = time.perf_counter()
        super().build_prior(i, distance)
        dt = time.perf_counter() - t0
        self.t["prior_s"] += dt
        self.prior_view_s[i] = self.prior_view_s.get(i, 0.0) + dt

    def reconstruct(self, fuse: bool = True):
        saved = ora.jbu

        def jbu(image, src_depth):
            t0 = time.perf_counter()
            ref_cuda.jbu(image, src_depth)  # the reference's kernel, timed
            self.t["jbu_s"] += time.perf_counter() - t0
            return saved(image, src_depth)  # the maps handed on (RunJBU's host fallback included)

        ora.jbu = jbu
        try:
            super().reconstruct(fuse=False)
        finally:
            ora.jbu = saved
        if not fuse:
            return None
        if self.host is None:
            t0 = time.perf_counter()
            out = ora.fusion([v.cam for v in self.views], [v.maps["depth_geom"] for v in self.views],
                             [v.maps["normal"] for v in self.views], [v.color for v in self.views], self.srcs)
            self.t["fusion_s"] += time.perf_counter() - t0
            return out
        self._folder_level("depth_geom")
        t0 = time.perf_counter()
        rc = self.host.ref_host_fusion(self.folder.encode(), len(self.views), self.off.ctypes.data,
                                       self.ids.ctypes.data, 1, 0)
        self.t["fusion_s"] += time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError("reference RunFusion failed")
        return None

    def replay(self, view_share: float) -> float:
        """Seconds of the recorded view's share of the schedule: its PatchMatch runs again from their recorded
        inputs (per-run host work and RunPatchMatch), its prior construction time, and `view_share` of the
        whole-scene host stages (confidence, JBU, fusion) measured during reconstruct()."""
        total = 0.0
        for r in self.records:
            st = _copy_state(r["state"])
            t0 = time.perf_counter()
            for color in r["colors"]:
                cv2.cvtColor(color, cv2.COLOR_BGR2GRAY).astype(np.float32)
            cv2.Canny(r["colors"][0], 50, 150)
            ref_cuda.run_patchmatch(r["images"], r["depths"], r["cams"], r["params"], st, r["seed"], r["view"])
            total += time.perf_counter() - t0
        total += self.prior_view_s.get(self.record_view, 0.0)
        total += view_share * (self.t["confidence_s"] + self.t["jbu_s"] + self.t["fusion_s"])
        return total

    def close(self) -> None:
        if self.folder and os.path.isdir(self.folder):
            shutil.rmtree(self.folder, ignore_errors=True)


def _copy_state(st):
    out = ora.RunState(st.W, st.H)
    for name in ("planes", "costs", "pre_costs", "selected_views", "rng_draw", "prior_planes", "plane_masks",
                 "confidences", "canny", "texture"):
        getattr(out, name)[...] = getattr(st, name)
    out.scaled_planes = st.scaled_planes.copy()
    return out
