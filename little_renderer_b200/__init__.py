"""little_renderer's GPU path tracer and BVH builders, as a CUDA backend for B200 (sm_100a).

The product is the C ABI in include/lrc.h, implemented by liblrc.so (built in-tree from
little_renderer_b200/csrc). This package holds the build recipe, a ctypes binding of the ABI
(``native``) and the seeded synthetic workloads (``workloads``).
"""
from . import native, workloads  # noqa: F401
from .native import Context, Scene, LrcError, build, lib, pack_tris  # noqa: F401
