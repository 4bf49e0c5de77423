"""The CUDA path's bilateral NCC against the golden vectors of the reference's
own ComputeMultiViewCostVector (HPM.cu:490-495, built from its sources with
--use_fast_math; tests/golden/ref_probe.npz, made by
tests/golden/make_ref_golden.py), at the fixture's 1536 fixed hypotheses, under
the same rounding criteria as the oracle (tests/test_golden_ref.py), and against
the oracle on the same inputs; likewise its JBU against the reference's JBU_cu
and JBU_cu_prior kernels (tests/golden/ref_jbu.npz)."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

import hpm_b200

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import hpm_oracle as ora  # noqa: E402
import make_ref_golden as golden  # noqa: E402
from test_golden_ref import FIXTURE, JBU_FIXTURE, check_costs, check_jbu, jbu_fallback, ncc_allowance  # noqa: E402

pytestmark = pytest.mark.gpu


def test_cuda_costs_match_reference_golden_vectors():
    images, depths, cams, params, z = golden.load(FIXTURE)
    srcs = list(range(1, len(images)))
    with hpm_b200.Context(0) as ctx:
        for i, (g, c) in enumerate(zip(images, cams)):
            ctx.set_view(i, g, c)
        got = ctx.eval_costs(0, srcs, params, z["pix"], z["planes"])
    d = np.abs(got - z["ref_cost_vec"])
    print("CUDA vs reference build: median |d| %.3g (%d costs)" % (np.median(d), d.size))
    check_costs(got, z["ref_cost_vec"], *ncc_allowance(images, depths, cams, params, z))
    cpu = ora.eval_costs(images, cams, params, z["pix"], z["planes"])
    assert (np.abs(got - cpu) <= 1e-4).mean() >= 0.999


def test_cuda_jbu_matches_reference_golden_vectors():
    j = dict(np.load(JBU_FIXTURE))
    img = j["image"].astype(np.float32)
    H, W = img.shape
    cam = hpm_b200.Camera.make(np.eye(3), np.eye(3), np.zeros(3), W, H, 1.0, 2.0)
    with hpm_b200.Context(0) as ctx:
        ctx.set_view(0, img, cam)
        depth = ctx.jbu_maps(0, j["coarse_depth"])
        pd, pn = ctx.jbu_maps(0, j["coarse_depth"], j["coarse_normal"])
    check_jbu(depth, jbu_fallback(j["ref_jbu_depth"], j["coarse_depth"]))
    check_jbu(pd, j["ref_jbu_prior_depth"], pn, j["ref_jbu_prior_normal"])
