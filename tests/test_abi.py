"""The C ABI library: built for sm_100a, loads without a GPU, and exports every function
include/lrc.h declares (no compute call is made here)."""
import ctypes
import os
import re

import pytest

import little_renderer_b200 as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(lrc_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_headers_declare_functions():
    assert len(declared()) >= 15


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(L.native.LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_open_without_gpu_is_refused_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert L.lib().lrc_open(0, ctypes.byref(h)) == L.native.LRC_E_NODEVICE


def test_build_scratch_bytes_grows_with_n():
    f = L.lib().lrc_build_scratch_bytes
    assert f(1000, 30, 0) < f(100000, 30, 0) < f(100000, 63, 0)
    assert f(100000, 30, 1) > f(100000, 30, 0)
