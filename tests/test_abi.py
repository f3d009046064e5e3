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


def test_binding_constants_match_the_header():
    """Every constant the ctypes binding restates (a name defined in include/lrc.h) has the header's
    value."""
    defs = {}
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            for name, val in re.findall(r"^#define\s+(LRC_[A-Z0-9_]+)\s+(.*)$", txt, flags=re.M):
                val = re.sub(r"/\*.*", "", val).strip()
                val = re.sub(r"(?<=[0-9a-fA-F])u\b", "", val)
                if val and re.fullmatch(r"[0-9a-fA-Fx()<\-\s]+", val):
                    defs[name] = int(eval(val))
    shared = [n for n in defs if hasattr(L.native, n)]
    assert "LRC_WAVEFRONT_DEFAULT_VARIANT" in shared and len(shared) >= 10, shared
    wrong = {n: (getattr(L.native, n), defs[n]) for n in shared if getattr(L.native, n) != defs[n]}
    assert not wrong, wrong
