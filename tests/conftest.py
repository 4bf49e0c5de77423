"""Shared fixtures: registers the package directory (hyphenated) as `hpm_b200`,
the oracle as `hpm_oracle`, and the `gpu` marker."""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hpm-mvs_plusplus_b200")


def _register(name: str, path: str, pkg_dir: str | None = None):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path,
                                                  submodule_search_locations=[pkg_dir] if pkg_dir else None)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


hpm_b200 = _register("hpm_b200", os.path.join(PKG, "__init__.py"), PKG)
hpm_oracle = _register("hpm_oracle", os.path.join(ROOT, "oracle", "oracle.py"))
# the oracle pipeline and the reference-build wrapper import `hpm_oracle` by name
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def small_scene():
    """5 views of 160x120 on a 30-degree arc, 4 sources per view (seed 1)."""
    from hpm_b200 import synth
    return synth.make_scene(n_views=5, width=160, height=120, seed=1, n_src=4)


def scene_cams(scene):
    from hpm_b200 import Camera
    cams = []
    for v in scene.views:
        h, w = v.image.shape[:2]
        cams.append(Camera.make(v.K, v.R, v.t, w, h, v.depth_min, v.depth_max))
    return cams


def scene_grays(scene):
    from hpm_b200 import synth
    return [synth.gray_float(v.image) for v in scene.views]
