"""lrc_build_static, the build for callers that cannot allocate device memory.

Such callers (a host program whose device memory all comes from its own pool, or a frame loop that
rebuilds a tree every frame and cannot take cudaMalloc's implicit synchronisation) pass device
inputs and outputs; the library keeps its scratch in one fixed device array. This file checks
that entry point through the C ABI against lrc_build (the allocating entry point), bit for bit,
on two calls in a row with different builds (the array keeps the first call's data), and that a
size above the maximum is refused without touching the outputs. It is named to run last.
"""
import ctypes as C

import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _boxes(n, seed):
    quv = W.corners_to_quv(W.soup(n, seed))
    q = quv[:, 0:3]
    b = (q + quv[:, 3:6]).astype(np.float32)
    c = (q + quv[:, 6:9]).astype(np.float32)
    boxes = np.zeros((n, 8), np.float32)
    boxes[:, 0:3] = np.minimum(np.minimum(q, b), c) - np.float32(1e-3)
    boxes[:, 4:7] = np.maximum(np.maximum(q, b), c) + np.float32(1e-3)
    return boxes, boxes[:, 0:3].min(0), boxes[:, 4:7].max(0)


def _static_build(params, boxes):
    """lrc_build_static with device buffers made here (by torch: the test may allocate, the entry
    point does not); returns the host copies of nodes and aux and the status code."""
    import torch
    n = params.n
    d_boxes = torch.from_numpy(boxes.reshape(-1)).cuda()
    d_nodes = torch.full(((params.node0 + 2 * n - 1) * 8,), -1, dtype=torch.int32, device="cuda")
    d_aux = torch.full((params.ref0 + n,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.lib().lrc_build_static(C.byref(params), C.c_void_p(d_boxes.data_ptr()), C.c_void_p(d_nodes.data_ptr()),
                                  C.c_void_p(d_aux.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    nodes = d_nodes.cpu().numpy().view(np.uint32).reshape(-1, 8)
    aux = d_aux.cpu().numpy().view(np.uint32)
    return rc, nodes, aux


def test_static_build_equals_lrc_build_on_two_calls_in_a_row():
    ctx = L.Context(0)
    # first the largest build the array holds (LRC_STATIC_MAX_ITEMS = 65536 items, 63-bit keys,
    # PLOC), then a smaller LBVH with offsets over the first call's leftovers
    cases = [(65536, 63, 1, 11, 0, 0, 0), (40000, 30, 0, 12, 17, 5, 1000)]
    for n, bits, builder, seed, node0, ref0, ref_add in cases:
        boxes, lo, hi = _boxes(n, seed)
        p = ctx.params(n, lo, hi, bits, builder, node0, ref0, ref_add)
        want_nodes, want_aux = ctx.build(p, boxes)
        rc, nodes, aux = _static_build(p, boxes)
        assert rc == L.native.LRC_OK
        assert np.array_equal(nodes[node0:], want_nodes[node0:])
        assert np.array_equal(aux[ref0:], want_aux[ref0:])
    ctx.close()


def test_static_build_tiny_ploc_falls_back_as_lrc_build():
    """PLOC needs three items; with one or two the builder makes the LBVH tree, as lrc_build does."""
    ctx = L.Context(0)
    for n in (1, 2):
        boxes, lo, hi = _boxes(n, 20 + n)
        p = ctx.params(n, lo, hi, 30, 1)
        want_nodes, want_aux = ctx.build(p, boxes)
        rc, nodes, aux = _static_build(p, boxes)
        assert rc == L.native.LRC_OK
        assert np.array_equal(nodes, want_nodes) and np.array_equal(aux, want_aux)
    ctx.close()


def test_static_build_on_a_second_device():
    """The array's address is looked up once per device; a second GPU gets its own."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU visible")
    with torch.cuda.device(1):
        ctx = L.Context(1)
        boxes, lo, hi = _boxes(30000, 31)
        p = ctx.params(30000, lo, hi, 30, 1)
        want_nodes, want_aux = ctx.build(p, boxes)
        rc, nodes, aux = _static_build(p, boxes)
        assert rc == L.native.LRC_OK
        assert np.array_equal(nodes, want_nodes) and np.array_equal(aux, want_aux)
        ctx.close()


def test_static_build_refuses_more_than_its_maximum():
    ctx = L.Context(0)
    n = 65536 + 1
    boxes, lo, hi = _boxes(n, 3)
    p = ctx.params(n, lo, hi, 30, 0)
    rc, nodes, aux = _static_build(p, boxes)
    assert rc == -6                                   # LRC_E_TOO_BIG
    assert (nodes == 0xFFFFFFFF).all() and (aux == 0xFFFFFFFF).all()
    ctx.close()
