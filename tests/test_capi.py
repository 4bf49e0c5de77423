"""CPU tests of the C-ABI library: it loads without a GPU and exports every
function include/*.h declares; without a device the binding refuses to run."""
from __future__ import annotations

import ctypes
import glob
import os
import re

import pytest

import hpm_b200
from conftest import ROOT, gpu_available


HOST_HEADER = "hpm_host.h"  # declared by libhpm_host.so (image decoding of the command-line driver)


def declared_functions(host: bool = False) -> list[str]:
    names = []
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        if (os.path.basename(hdr) == HOST_HEADER) != host:
            continue
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^([A-Za-z_][\w \*]*?)\b(hpm_\w+)\s*\(", text, flags=re.M):
            if m.group(1).strip().startswith(("HPM_HD", "HPM_FP_HD", "static")):
                continue  # header-only inline helpers, not library symbols
            names.append(m.group(2))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(hpm_b200.LIB_PATH), "build libhpm_cuda.so first (__graft_entry__.build())"
    lib = ctypes.CDLL(hpm_b200.LIB_PATH)
    names = declared_functions()
    assert "hpm_run_patchmatch" in names and len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_host_library_exports_its_symbols():
    path = os.path.join(os.path.dirname(hpm_b200.LIB_PATH), "libhpm_host.so")
    assert os.path.exists(path), "build libhpm_host.so first (__graft_entry__.build())"
    lib = ctypes.CDLL(path)
    names = declared_functions(host=True)
    assert "hpm_decode_image" in names
    assert not [n for n in names if not hasattr(lib, n)]


def test_binding_declares_all_symbols():
    assert set(declared_functions()) <= set(hpm_b200.EXPORTED_SYMBOLS) | {"hpm_get_map"}


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    with pytest.raises(hpm_b200.HPMError):
        hpm_b200.Context(0)


def test_struct_layouts():
    assert ctypes.sizeof(hpm_b200.Camera) == 100
    assert ctypes.sizeof(hpm_b200.Params) == 48
