#!/usr/bin/env python3
"""Throughput of the HPM-MVS++ reconstruction hot path on B200: reference views/s.

One step reconstructs the whole scene the way `./HPM-MVS_plusplus $folder
--initial-image-scale 1` does (main.cpp:1143-1364): every pyramid level's
photometric, planar-prior, hierarchy and geometric PatchMatch passes over all
views, with confidence evaluation, prior construction, JBU and GPU fusion.

Workload (default): the 49-view two-ring hemisphere scene, 1600x1200 8-bit
views, 10 source views each, --initial-image-scale 1, which under the
reference's 1000-pixel pyramid bound (main.cpp:205) gives two levels
(800x600, 1600x1200).  The scene is synthetic (seeded piecewise-planar
geometry with band-limited texture, rendered on the GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device-resident throughput (images already in HBM, CUDA events on
the context's stream); `e2e` is the same through the C ABI with the pinned host
images uploaded and the depth, normal and point results downloaded inside the
timed region.  Each step touches several GB of maps, more than the 126 MB L2,
so no flush is needed between steps.  N > 1 runs independent replicas (one
scene per rank, no collective on the data path) and reports their total.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "hpm-mvs_plusplus_b200")
ORACLE = os.path.join(ROOT, "oracle")

METRIC = "ref-views/s at fixed depth accuracy, plain vs chosen form on 1 B200; HBM GB/s"
UNIT = "ref-views/s"
ALGO_FLOPS_PER_EVAL = 31   # FP32 flops per cost evaluation (1 hypothesis x 1 view x 1 patch sample)
SAMPLES_PER_NCC = 36       # 11x11 window at stride 2 -> 6x6 samples
# Algorithmic HBM bytes per updated pixel of a half-sweep: plane 16 + cost 4 + view mask 4
# read and the same 24 written, plus the grey image of the reference and S sources read once.
STATE_BYTES_PER_PIXEL = 48


def _import_pkg():
    import importlib.util
    if "hpm_b200" in sys.modules:
        return sys.modules["hpm_b200"]
    spec = importlib.util.spec_from_file_location("hpm_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hpm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _import_oracle():
    import importlib.util
    if "hpm_oracle" not in sys.modules:
        spec = importlib.util.spec_from_file_location("hpm_oracle", os.path.join(ORACLE, "oracle.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["hpm_oracle"] = mod
        spec.loader.exec_module(mod)
    if ORACLE not in sys.path:
        sys.path.insert(0, ORACLE)
    return sys.modules["hpm_oracle"]


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", choices=("c1", "c2", "c3", "c4", "c5"), default="c2",
                    help="workload (synth.CONFIGS); c2, the 49-view 1600x1200 scene, is the headline")
    ap.add_argument("--views", type=int, default=None, help="override the workload's view count")
    ap.add_argument("--width", type=int, default=None, help="custom hemisphere scene of this width")
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--n-src", type=int, default=None)
    ap.add_argument("--scale", type=int, default=None, help="--initial-image-scale")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chosen-form", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the precision form (8-bit source textures)")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("gpu_uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9 or (self.uuid and parts[0] != self.uuid):
                    continue
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ workload

def resolve_workload(args):
    """Fills args.views/width/height/n_src/scale from --config unless given (width/height: custom scene)."""
    defaults = {"c1": (5, 1280, 960, 4, 4), "c2": (49, 1600, 1200, 10, 1), "c3": (49, 1600, 1200, 10, 1),
                "c4": (20, 1024, 768, 10, 1), "c5": (120, 3072, 2048, 10, 1)}
    v, w, h, ns, sc = defaults[args.config]
    args.custom = args.width is not None or args.height is not None
    args.views_given = args.views is not None
    args.views = args.views or v
    args.width = args.width or w
    args.height = args.height or h
    args.n_src = args.n_src or ns
    args.scale = args.scale or sc


def make_workload(args, device: str, rank: int):
    """The seeded scene of this rank (rendered on the GPU through torch)."""
    import importlib
    _import_pkg()
    synth = importlib.import_module("hpm_b200.synth")
    if args.custom:
        return synth.make_scene(n_views=args.views, width=args.width, height=args.height, layout="hemisphere",
                                n_src=args.n_src, seed=args.seed + 7919 * rank, device=device)
    return synth.make_config(args.config, seed=args.seed + 7919 * rank, device=device, n_views=args.views)


def workload_text(args, scene=None) -> str:
    if args.custom or args.config in ("c1", "c2", "c4"):
        desc = (f"{args.views} views {args.width}x{args.height} "
                f"{'arc' if args.config == 'c1' and not args.custom else 'hemisphere'}, {args.n_src} sources")
    else:
        import importlib
        _import_pkg()
        desc = importlib.import_module("hpm_b200.synth").CONFIGS[args.config]
        if args.views_given:
            desc += f" ({args.views} views)"
    levels = "/".join(f"{w}x{h}" for w, h in level_sizes(args.width, args.height, args.scale))
    extra = ""
    if scene is not None and scene.meta.get("textureless_area"):
        extra = f", textureless area {scene.meta['textureless_area']:.2f}"
    return (f"{desc}, --initial-image-scale {args.scale}, levels {levels} (largest view), geometric iterations 3, "
            f"fusion{extra}")


def level_sizes(w: int, h: int, scale: int):
    """Pyramid working sizes of ComputeMultiScaleSettings + PrepareScaleImages (main.cpp:107-235)."""
    init = max(1, (max(w, h) + scale // 2) // scale)
    k, side = 0, init
    while side > 1000:
        side //= 2
        k += 1
    out = []
    for lvl in range(k, -1, -1):
        target = int(init / 2 ** lvl)
        if max(w, h) > target:
            f = min(np.float32(target) / np.float32(w), np.float32(target) / np.float32(h))
            out.append((max(1, int(round(w * float(f)))), max(1, int(round(h * float(f))))))
        else:
            out.append((w, h))
    return out


def view_pixel_runs(w: int, h: int, scale: int, geom_iterations: int = 3) -> int:
    """PatchMatch pixel-runs one reference view takes through the whole schedule."""
    sizes = level_sizes(w, h, scale)
    n_levels = len(sizes)
    total = 0
    for li, (lw, lh) in enumerate(sizes):
        level = n_levels - 1 - li                      # max_num_downscale at this level
        prior_passes = (n_levels - 1) - level + 1      # hpm_scale from max down to level
        runs = 1 + prior_passes + geom_iterations      # photometric/hierarchy + priors + geometric
        total += lw * lh * runs
    return total


# ------------------------------------------------------------------ our arm

def depth_accuracy(depths, scene, rel: float = 0.01):
    """Share of the rendered ground truth's valid pixels whose reconstructed depth lies within `rel`
    of it, over all views.  Maps smaller than the truth by an integer factor f (--initial-image-scale f)
    are compared with the truth at full-resolution pixel (f*x, f*y): the level's camera is K scaled by
    1/f (no half-pixel shift), so map pixel x looks along the ray of full-resolution pixel f*x.  None
    when the sizes do not relate that way.  Computed after the timed steps from the maps the
    last step downloaded."""
    try:
        ok = hit = 0
        for d, v in zip(depths, scene.views):
            gt = np.asarray(v.depth, np.float32)
            if gt.shape != d.shape:
                f = gt.shape[0] // d.shape[0]
                if f < 2 or gt.shape[0] != f * d.shape[0] or gt.shape[1] != f * d.shape[1]:
                    return None
                gt = gt[::f, ::f]
            m = gt > 0
            ok += int(m.sum())
            hit += int((np.abs(d[m] - gt[m]) <= rel * gt[m]).sum())
        return hit / ok if ok else None
    except Exception:
        return None


def run_ours(args, scene, rank, world, local_rank):
    import torch
    hb = _import_pkg()
    device = f"cuda:{local_rank}"
    cams = [hb.Camera.make(v.K, v.R, v.t, v.image.shape[1], v.image.shape[0], v.depth_min, v.depth_max)
            for v in scene.views]
    srcs = [[j for j, _ in p] for p in scene.pairs]
    n_views = len(cams)

    ctx = hb.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=device)
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    images = []
    for v in scene.views:
        b = pin(v.image.shape, torch.uint8)
        b[...] = v.image
        images.append(b)
    finals = [level_sizes(v.image.shape[1], v.image.shape[0], args.scale)[-1] for v in scene.views]
    depth_out = [pin((h, w), torch.float32) for w, h in finals]
    normal_out = [pin((h, w, 3), torch.float32) for w, h in finals]
    points_out = [None]  # sized after the first step (the point count repeats: same seed, same work)
    h2d_bytes = int(sum(b.nbytes for b in images))

    def step(**recon):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        for i, b in enumerate(images):
            ctx.set_image(i, b)
        ev[1].record(stream)
        n = ctx.reconstruct(cams, srcs, initial_image_scale=args.scale, seed=args.seed, fuse=True, **recon)
        ev[2].record(stream)
        if points_out[0] is None or points_out[0].shape[0] < n:
            points_out[0] = pin((n + 4096, 9), torch.float32)
        pts = ctx.get_points(out=points_out[0])
        for i in range(n_views):
            ctx.get_map(i, hb.MAP_DEPTH_GEOM, out=depth_out[i])
            ctx.get_map(i, hb.MAP_NORMAL, out=normal_out[i])
        ev[3].record(stream)
        d2h = pts.nbytes + sum(d.nbytes for d in depth_out) + sum(m.nbytes for m in normal_out)
        return ev, n, d2h

    # warm-up: the first step also counts the (hypothesis, view) cost evaluations
    ctx.profile_enable(hb.PROFILE_COUNT)
    for w in range(max(args.warmup, 0)):
        step()
        if w == 0:
            torch.cuda.synchronize()
            counted = ctx.profile_read()
            ctx.profile_enable(0)
    if args.warmup == 0:
        counted = ctx.profile_read()
        ctx.profile_enable(0)
    torch.cuda.synchronize()
    ctx.profile_read()

    uuid = ""
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ctx.profile_enable(hb.PROFILE_TIMING)
    launches0 = ctx.launch_count()
    sampler.start()
    evs = []
    n_pts = 0
    d2h_bytes = 0
    for _ in range(args.steps):
        ev, n_pts, d2h_bytes = step()
        evs.append(ev)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = ctx.launch_count() - launches0
    prof = ctx.profile_read()
    ctx.profile_enable(0)
    if world > 1:
        torch.distributed.barrier()
    dev_ms = sum(e[1].elapsed_time(e[2]) for e in evs)
    e2e_ms = sum(e[0].elapsed_time(e[3]) for e in evs)
    dev_ms, e2e_ms = max_over_ranks([dev_ms, e2e_ms], world, device)
    total_views = n_views * args.steps * world
    value = total_views / (dev_ms / 1e3)
    e2e = total_views / (e2e_ms / 1e3)
    accuracy = depth_accuracy(depth_out, scene)

    # roofline of the dominant kernel: the checkerboard half-sweep
    fp32_peak = hb.measure_fp32_peak(local_rank)
    evals_per_step = counted.sweep_view_evals * SAMPLES_PER_NCC
    flops_per_step = evals_per_step * ALGO_FLOPS_PER_EVAL
    sweep_ms_per_step = prof.sweep_ms / max(args.steps, 1)
    launches_per_step = prof.sweep_launches / max(args.steps, 1)
    achieved = flops_per_step / (sweep_ms_per_step * 1e-3) / 1e12 if sweep_ms_per_step > 0 else None
    traffic = _ncu_traffic()
    # the unit that binds the half-sweep: the texture unit's linear filtering, one fetch per patch sample
    tex_peak = hb.measure_tex_peak(local_rank, hb.TEX_F32)
    # the same fetches with every lane's patch at its own offset (up to +-16 px): the rate when the lanes of
    # a warp sample under unrelated planes, as random refinement candidates do
    tex_divergent = hb.measure_tex_rate(local_rank, hb.TEX_F32, 16.0)
    sampled_per_step = counted.sweep_sampled * SAMPLES_PER_NCC
    tex_achieved = sampled_per_step / (sweep_ms_per_step * 1e-3) / 1e9 if sweep_ms_per_step > 0 else None
    roofline = {
        "kernel": "k_half_sweep", "bound": "fp32", "unit": "TFLOP/s",
        "achieved": achieved, "peak": fp32_peak,
        "peak_source": "FP32 FMA probe on this GPU, hpm_measure_fp32_peak (MEASURED_PEAKS.json has no FP32 figure)",
        "frac": (achieved / fp32_peak) if achieved and fp32_peak else None,
        "traffic": traffic,
        "algorithmic_flops_per_launch": flops_per_step / launches_per_step if launches_per_step else None,
        "launches_per_step": launches_per_step,
        "avg_launch_ms": sweep_ms_per_step / launches_per_step if launches_per_step else None,
        "share_of_step": (sweep_ms_per_step / (dev_ms / args.steps / world)) if dev_ms > 0 else None,
        "cost_evals_per_s": evals_per_step / (sweep_ms_per_step * 1e-3) if sweep_ms_per_step > 0 else None,
        "hbm_peak_gbs": _measured_hbm(),
        "texture": {"unit": "Gfetch/s", "achieved": tex_achieved, "peak": tex_peak,
                    "frac": (tex_achieved / tex_peak) if tex_achieved and tex_peak else None,
                    "peak_source": "hpm_measure_tex_peak: linear-filtered F32 fetches in the half-sweep's access "
                                   "pattern on this GPU",
                    "fetches_per_step": sampled_per_step,
                    "divergent_lanes_rate": tex_divergent,
                    "frac_of_divergent_rate": (tex_achieved / tex_divergent) if tex_achieved and tex_divergent else None,
                    "divergent_source": "hpm_measure_tex_rate(jitter 16 px): the same fetches, each lane's patch moved "
                                        "by its own random offset",
                    "note": "executed work: NCCs that sampled the source (zero-weight views, out-of-image centres "
                            "and flat reference patches skip sampling), 36 fetches each"},
        "fp32_executed": {"achieved": (sampled_per_step * ALGO_FLOPS_PER_EVAL / (sweep_ms_per_step * 1e-3) / 1e12)
                          if sweep_ms_per_step > 0 else None,
                          "frac": (sampled_per_step * ALGO_FLOPS_PER_EVAL / (sweep_ms_per_step * 1e-3) / 1e12
                                   / fp32_peak) if sweep_ms_per_step > 0 and fp32_peak else None},
    }
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_text(args, scene), "name": args.config,
                   "seed": args.seed, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (several GB of maps per step)",
                   "points_per_step": int(n_pts)},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": int(d2h_bytes)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "roofline": roofline,
        "accuracy": {"measure": "share of ground-truth pixels with depth within 1 %, all views, last step",
                     "plain": accuracy},
        "stages": stage_breakdown(prof, dev_ms / max(args.steps, 1), n_views, args.steps),
    }
    if args.chosen_form:
        result["chosen_form"] = chosen_form(args, ctx, step, n_views, world, device, depth_out, scene)
        result["accuracy"]["chosen_form"] = result["chosen_form"].get("accuracy")
    return result, ctx, images


def stage_breakdown(prof, step_ms: float, n_views: int, steps: int) -> dict:
    """Device seconds per reference view of each stage of a step (CUDA events around every stage)."""
    k = 1e-3 / max(steps, 1) / n_views
    sec = {"patchmatch_gpu": (prof.init_ms + prof.sweep_ms) * k, "confidence": prof.confidence_ms * k,
           "prior": prof.prior_ms * k, "jbu": prof.jbu_ms * k, "fusion": prof.fusion_ms * k,
           "level_images": prof.level_ms * k}
    sec["other"] = max(0.0, step_ms * 1e-3 / n_views - sum(sec.values()))
    return {"views": n_views, "seconds_per_view": {a: round(b, 5) for a, b in sec.items()}}


def agreement(depths, ref_depths, rel: float = 0.005):
    """Share of pixels (finite, positive reference depth) whose depth is within `rel` of the reference's."""
    ok = hit = 0
    for d, r in zip(depths, ref_depths):
        m = np.isfinite(r) & (r > 0)
        ok += int(m.sum())
        with np.errstate(invalid="ignore"):
            hit += int((np.abs(d[m] - r[m]) <= rel * r[m]).sum())
    return hit / ok if ok else None


def chosen_form(args, ctx, step, n_views, world, device, depth_out=None, scene=None):
    """The chosen form of the same steps: 8-bit source textures (hpm_set_texture_format(HPM_TEX_U8): the
    grey levels stored exactly in a quarter of the bytes, the filtered sample returned as grey / 255, the
    scale-free NCC only rescaling its flat-source test), every pass batched where that leaves the result
    unchanged (hpm_run_batch: one launch per stage over all views, autotuned launch shape) and the batched
    schedules replayed from CUDA graphs.  Also timed: the same with the multi-geometry passes batched too
    (Jacobi), a change of iteration that is reported with its agreement."""
    import torch
    hb = _import_pkg()
    plain = [d.copy() for d in depth_out] if depth_out is not None else None
    out = {"form": "8-bit source textures + batched passes (exact) + CUDA-graph replay", "unit": UNIT}
    ctx.set_texture_format(hb.TEX_U8)
    ctx.set_batch_options(hb.BATCH_AUTOTUNE | hb.BATCH_GRAPH)
    for name, batch in (("", hb.RECON_BATCH_EXACT), ("jacobi_", hb.RECON_BATCH_ALL)):
        for _ in range(max(1, min(args.warmup, 2))):
            step(batch=batch)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        evs = [step(batch=batch)[0] for _ in range(args.steps)]
        torch.cuda.synchronize()
        dev_ms = sum(e[1].elapsed_time(e[2]) for e in evs)
        e2e_ms = sum(e[0].elapsed_time(e[3]) for e in evs)
        t = max_over_ranks([dev_ms, e2e_ms], world, device)
        total_views = n_views * args.steps * world
        out[name + "value"] = total_views / (float(t[0]) / 1e3)
        out[name + "e2e"] = total_views / (float(t[1]) / 1e3)
        out[name + "ms_per_step"] = float(t[0]) / args.steps
        if depth_out is not None and scene is not None:
            out[name + "accuracy"] = depth_accuracy(depth_out, scene)
            out[name + "agree_with_plain_0p5pct"] = agreement(depth_out, plain)
    ctx.set_texture_format(hb.TEX_F32)
    ctx.set_batch_options(hb.BATCH_AUTOTUNE)
    return out


def max_over_ranks(values, world: int, device):
    """Element-wise maximum of per-rank timings over the process group (the job ends with its slowest replica)."""
    import torch
    if world <= 1:
        return [float(v) for v in values]
    t = torch.tensor(values, dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t]


def _measured_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh).get("hbm_gbs")
    except (OSError, ValueError):
        return None


def _ncu_traffic():
    """dram read+write bytes per k_half_sweep launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "k_half_sweep_800x600_s10.md")
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip().split()[0])
    except (OSError, ValueError):
        pass
    return None


# ------------------------------------------------------------------ CPU baselines

def cpu_port_baseline(args, scene):
    """The oracle (CPU port of the GPU path) on a bounded sample: photometric and geometric PatchMatch runs
    of one reference view at 400x300 with all its sources, scaled to ref-views/s of the workload."""
    ora = _import_oracle()
    hb = _import_pkg()
    import cv2
    sw, sh = 400, 300
    srcs = [j for j, _ in scene.pairs[0]]
    ids = [0] + srcs
    grays, cams = [], []
    for j in ids:
        v = scene.views[j]
        img = cv2.resize(v.image, (sw, sh), interpolation=cv2.INTER_LINEAR)
        grays.append(cv2.cvtColor(img, cv2.COLOR_BGR2GRAY).astype(np.float32))
        c = hb.Camera.make(v.K, v.R, v.t, v.image.shape[1], v.image.shape[0], v.depth_min, v.depth_max)
        oc = ora.to_cam(c)
        sx, sy = sw / v.image.shape[1], sh / v.image.shape[0]
        oc.K[0] *= sx; oc.K[2] *= sx; oc.K[4] *= sy; oc.K[5] *= sy
        oc.width, oc.height = sw, sh
        cams.append(oc)
    p = ora.Params()
    p.max_iterations, p.patch_size, p.num_images, p.radius_increment = 3, 11, len(ids), 2
    p.sigma_spatial, p.sigma_color, p.top_k = 5.0, 3.0, 4
    p.depth_min = float(np.float32(cams[0].depth_min) * np.float32(0.6))
    p.depth_max = float(np.float32(cams[0].depth_max) * np.float32(1.2))
    st = ora.RunState(sw, sh)
    st.canny[:] = cv2.Canny(cv2.resize(scene.views[0].image, (sw, sh)), 50, 150)
    t0 = time.perf_counter()
    p.mode = 0
    ora.run_patchmatch(grays, None, cams, p, st, 1, 0)
    depths = [None] + [np.full((sh, sw), float(np.median(st.planes[..., 3])), np.float32) for _ in srcs]
    st.costs[:] = st.costs
    p.mode = 1
    ora.run_patchmatch(grays, depths, cams, p, st, 2, 0)
    dt = time.perf_counter() - t0
    px_runs = 2 * sw * sh
    rate = px_runs / dt
    per_view = int(np.mean([view_pixel_runs(v.image.shape[1], v.image.shape[0], args.scale) for v in scene.views]))
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": rate / per_view, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"oracle C port (OpenMP), one photometric + one geometric PatchMatch run of one view at "
                      f"{sw}x{sh} with {len(srcs)} sources ({px_runs} pixel-runs in {dt:.1f} s), scaled by the "
                      f"{per_view} pixel-runs one view takes through the workload's schedule; host stages "
                      f"not included"}


# ------------------------------------------------------------------ reference arm

def run_reference(args):
    """The reference's own implementation of the path, like for like: the whole schedule of its main() on
    one reference view and its sources (every view keeping the workload's size and source count), on the
    reference's own code where it was built here (oracle/ref_pipeline.py): HPM::RunPatchMatch of its HPM.cu
    compiled for sm_100a, its JBU kernel, its single-threaded ConfidenceEvaluation and RunFusion compiled
    for the CPU, its prior construction (cv2.Subdiv2D plus the C restatement of its raster and fits).  Each
    pass takes its inputs from the reference's own earlier passes.  That reconstruction is timed stage by
    stage; each step then replays the first view's share of it (its runs from their recorded inputs, its
    prior construction, 1/N of the whole-scene host stages)."""
    _import_oracle()
    import ref_cuda  # noqa: E402  (oracle/ref_cuda.py)
    import ref_pipeline  # noqa: E402  (oracle/ref_pipeline.py)
    if not ref_cuda.available():
        return {"impl": "reference", "unavailable": "reference CUDA build oracle/_ref/libhpmref.so was not built"}
    hb = _import_pkg()
    import torch
    torch.cuda.set_device(0)
    scene = make_workload(args, "cuda:0", 0)
    v0 = 0
    subset = [v0] + [j for j, _ in scene.pairs[v0]]
    score = lambda g, j: dict(scene.pairs[g]).get(j, -1.0)  # noqa: E731
    # every view of the subset keeps its source count: the other subset views by its pair.txt score
    srcs = [sorted([k for k in range(len(subset)) if k != a], key=lambda k: -score(subset[a], subset[k]))
            [:len(scene.pairs[g])] for a, g in enumerate(subset)]
    cams = [hb.Camera.make(scene.views[g].K, scene.views[g].R, scene.views[g].t, scene.views[g].image.shape[1],
                           scene.views[g].image.shape[0], scene.views[g].depth_min, scene.views[g].depth_max)
            for g in subset]
    folder = tempfile.mkdtemp(prefix="hpm_ref_")
    P = ref_pipeline.RefPipeline([scene.views[g].image for g in subset], cams, srcs,
                                 initial_image_scale=args.scale, seed=args.seed, record_view=0, folder=folder)
    try:
        t0 = time.perf_counter()
        P.reconstruct(fuse=True)
        whole_s = time.perf_counter() - t0
        n = len(subset)
        for _ in range(max(args.warmup, 0)):
            P.replay(1.0 / n)
        times = [P.replay(1.0 / n) for _ in range(args.steps)]
    finally:
        P.close()
    total = sum(times)
    value = args.steps / total
    pm_ms = {f"{k[0]} {k[1]}": round(v[0] / v[1], 2) for k, v in P.pm.items()}
    pm_s = sum(v[0] for v in P.pm.values()) / 1e3
    stage_s = {"patchmatch_gpu": pm_s, "patchmatch_host": P.t["pm_host_s"], "prior": P.t["prior_s"],
               "confidence": P.t["confidence_s"], "jbu": P.t["jbu_s"], "fusion": P.t["fusion_s"]}
    host_from = ("the reference's own main.cpp (oracle/_ref/libhpmref_host.so)" if P.host is not None
                 else "their C restatement (the reference's host build is absent)")
    result = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_text(args), "name": args.config, "seed": args.seed,
                   "step": f"view 0's share of the reference's whole schedule over view 0 and its {n - 1} sources"},
        "stages": {"views": n, "seconds": {k: round(v, 3) for k, v in stage_s.items()},
                   "seconds_per_view": {k: round(v / n, 5) for k, v in stage_s.items()},
                   "reconstruct_wall_s": round(whole_s, 2), "views_per_s_whole": n / sum(stage_s.values()),
                   "patchmatch_ms_per_run": pm_ms, "host_cores": 1,
                   "host_stages_from": host_from},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "per step one reference view: its PatchMatch runs on the reference's own CUDA "
                                   "kernels (HPM.cu compiled for sm_100a, fast-math as shipped) from the inputs its "
                                   "own earlier passes produced, its per-run host work (grey conversion, Canny), "
                                   "its prior construction (cv2.Subdiv2D and the C restatement of its raster and "
                                   f"fits), and 1/{n} of the single-threaded ConfidenceEvaluation "
                                   f"({P.t['confidence_s']:.1f} s), RunFusion ({P.t['fusion_s']:.1f} s) and JBU "
                                   f"({P.t['jbu_s']:.2f} s) of that {n}-view reconstruction, timed on {host_from}, "
                                   ".dmb reads included; file writes and image decoding not timed"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return result


# ------------------------------------------------------------------ main

def main():
    args = parse_args()
    resolve_workload(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        # the reference's RunPatchMatch prints "iteration: i" on stdout (HPM.cu:3023); keep stdout for
        # the one JSON line by sending the C-level stdout to stderr while it runs
        sys.stdout.flush()
        saved = os.dup(1)
        os.dup2(2, 1)
        try:
            result = run_reference(args)
        finally:
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)
        print(json.dumps(result), flush=True)
        return 0
    import torch
    if world > 1:
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                             device_id=torch.device(f"cuda:{local_rank}"))
    torch.cuda.set_device(local_rank)
    scene = make_workload(args, f"cuda:{local_rank}", rank)
    result, ctx, _ = run_ours(args, scene, rank, world, local_rank)
    ctx.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_port_baseline(args, scene)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
