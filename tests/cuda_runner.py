"""The CUDA path behind the oracle's run_patchmatch signature (test helper).

`CudaRunner(ctx)(images, depths, cams, params, st, seed, view_id)` loads one
PatchMatch run's inputs -- the reference and source grey images, cameras, the
RunState's planes, costs, confidences, prior, Canny map and the sources' depth
maps -- into a context through the C ABI, runs hpm_run_patchmatch and writes
the results back into `st` the way oracle.run_patchmatch and
ref_cuda.run_patchmatch leave it (world-frame normals and depth in st.planes,
costs, texture).  A pipeline written against the oracle's runner
(oracle/pipeline.py) can therefore drive the CUDA path, the oracle and the
reference's own build on identical inputs.
"""
from __future__ import annotations

import numpy as np

import hpm_b200

MODE_GEOM, MODE_PRIOR, MODE_MULTIGEOM, MODE_HIERARCHY, MODE_UPSAMPLE, MODE_MAND = 1, 2, 4, 8, 16, 32
SRC_SLOT0 = 128  # context slots of the sources: away from any reference view id used by the tests


def copy_state(st):
    import hpm_oracle as ora

    out = ora.RunState(st.W, st.H)
    for name in ("planes", "costs", "pre_costs", "selected_views", "rng_draw", "prior_planes", "plane_masks",
                 "confidences", "canny", "texture"):
        getattr(out, name)[...] = getattr(st, name)
    out.scaled_planes = st.scaled_planes.copy()
    return out


def to_hb_cam(c) -> "hpm_b200.Camera":
    return hpm_b200.Camera.make(np.asarray(c.K[:], np.float32).reshape(3, 3), np.asarray(c.R[:], np.float32).reshape(3, 3),
                                np.asarray(c.t[:], np.float32), c.width, c.height, c.depth_min, c.depth_max)


def to_hb_params(p) -> "hpm_b200.Params":
    q = hpm_b200.Params()
    for name, _ in hpm_b200.Params._fields_:
        setattr(q, name, getattr(p, name))
    return q


class CudaRunner:
    def __init__(self, ctx: "hpm_b200.Context"):
        self.ctx = ctx

    def __call__(self, images, depths, cams, params, st, seed: int, view_id: int) -> None:
        ctx = self.ctx
        if view_id >= SRC_SLOT0:
            raise ValueError("view ids from SRC_SLOT0 on are the runner's source slots")
        S = len(images) - 1
        mode = int(params.mode)
        geom, prior = bool(mode & MODE_GEOM), bool(mode & MODE_PRIOR)
        hier, mand = bool(mode & MODE_HIERARCHY), bool(mode & MODE_MAND)
        dkind = hpm_b200.MAP_DEPTH_GEOM if mode & MODE_MULTIGEOM else hpm_b200.MAP_DEPTH
        ref = view_id
        srcs = [SRC_SLOT0 + j for j in range(S)]
        ctx.set_view(ref, images[0], to_hb_cam(cams[0]))
        for j in range(S):
            ctx.set_view(srcs[j], images[j + 1], to_hb_cam(cams[j + 1]))
        ctx.set_canny(ref, np.asarray(st.canny, np.uint8))
        if geom or prior:
            ctx.set_map(ref, hpm_b200.MAP_NORMAL, st.planes[..., :3])
            ctx.set_map(ref, dkind, st.planes[..., 3])
            ctx.set_map(ref, hpm_b200.MAP_COST, st.costs)
        if geom:
            for j in range(S):
                ctx.set_map(srcs[j], dkind, depths[j + 1])
        if prior or mand:
            ctx.set_map(ref, hpm_b200.MAP_CONF, st.confidences)
        if prior:
            ctx.set_prior(ref, st.prior_planes, np.asarray(st.plane_masks, np.uint8))
        if hier and not geom and not prior:
            sp = st.scaled_planes
            ctx.set_map(ref, hpm_b200.MAP_NORMAL, sp[..., :3])
            ctx.set_map(ref, hpm_b200.MAP_COST, sp[..., 3])
            ctx.set_map(ref, hpm_b200.MAP_DEPTH, st.planes[..., 3])
        ctx.run_patchmatch(ref, srcs, to_hb_params(params), texture_level=0, seed=seed)
        st.planes[..., 3] = ctx.get_map(ref, hpm_b200.MAP_DEPTH_GEOM if geom else hpm_b200.MAP_DEPTH)
        st.planes[..., :3] = ctx.get_map(ref, hpm_b200.MAP_NORMAL)
        st.costs[...] = ctx.get_map(ref, hpm_b200.MAP_COST)
        if not prior and not mand:
            st.texture[...] = ctx.get_map(ref, hpm_b200.MAP_TEXTURE0)
