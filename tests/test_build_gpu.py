"""GPU parity of the builders: lrc_build (CUDA) against the restated reference builders (oracle),
node for node and bit for bit; triangle boxes against the reference's triangle_bounds."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _inputs(O, n, seed):
    quv = W.corners_to_quv(W.soup(n, seed))
    boxes = O.triangle_bounds(quv)
    blo, bhi = W.mesh_bounds(quv)
    return quv, boxes, blo, bhi


def _check_same(ctx, O, boxes, blo, bhi, bits, builder, node0=0, ref0=0, ref_add=0):
    n = boxes.shape[0]
    p = ctx.params(n, blo, bhi, bits, builder, node0, ref0, ref_add)
    lo, ext = O.params(blo, bhi)
    assert np.array_equal(np.frombuffer(p.lo, np.float32), lo)
    assert np.array_equal(np.frombuffer(p.ext, np.float32), ext)
    use_ploc = builder == 1 and n > 2
    if use_ploc:
        want_n, want_a = O.ploc(boxes, lo, ext, bits, node0, ref0, ref_add)
    else:
        want_n, want_a = O.lbvh(boxes, lo, ext, bits, node0, ref0, ref_add)
    nodes = np.full_like(want_n, 0xDEADBEEF)
    aux = np.full_like(want_a, 0xDEADBEEF)
    if node0:
        nodes[:node0] = want_n[:node0]
    if ref0:
        aux[:ref0] = want_a[:ref0]
    got_n, got_a = ctx.build(p, boxes, nodes, aux)
    bad = np.nonzero((got_n != want_n).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} nodes differ, first {bad[:5]}: got {got_n[bad[:2]]} want {want_n[bad[:2]]}"
    assert np.array_equal(got_a, want_a)
    return got_n


@pytest.mark.parametrize("builder", [0, 1])
@pytest.mark.parametrize("bits", [30, 63])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 64, 1000, 1024, 1025, 4096, 4097, 33333, 262145])
def test_build_matches_oracle(ctx, oracle, n, bits, builder):
    _, boxes, blo, bhi = _inputs(oracle, n, 1000 + n)
    _check_same(ctx, oracle, boxes, blo, bhi, bits, builder)


@pytest.mark.parametrize("builder", [0, 1])
def test_build_offsets(ctx, oracle, builder):
    _, boxes, blo, bhi = _inputs(oracle, 7777, 3)
    _check_same(ctx, oracle, boxes, blo, bhi, 30, builder, node0=1234, ref0=99, ref_add=4321)


@pytest.mark.parametrize("builder", [0, 1])
def test_build_equal_codes(ctx, oracle, builder):
    """Every item at one point: all codes equal, the order and the tree come from positions."""
    n = 20000
    boxes = np.tile(np.array([0.2, 0.3, 0.4, 0, 0.25, 0.35, 0.45, 0], np.float32), (n, 1))
    _check_same(ctx, oracle, boxes, np.zeros(3, np.float32), np.ones(3, np.float32), 30, builder)


@pytest.mark.parametrize("builder", [0, 1])
def test_build_flat_axis_and_outside_bounds(ctx, oracle, builder):
    """A flat axis (ext 0) and boxes outside the bounds (clamped) as the reference clamps them."""
    rng = np.random.default_rng(4)
    n = 50000
    c = rng.random((n, 3)).astype(np.float32) * 3 - 1
    c[:, 1] = 0.5
    boxes = np.zeros((n, 8), np.float32)
    boxes[:, 0:3] = c - 0.001
    boxes[:, 4:7] = c + 0.001
    _check_same(ctx, oracle, boxes, np.array([0, 0.5, 0], np.float32), np.array([1, 0.5, 1], np.float32), 30, builder)


@pytest.mark.parametrize("builder,bits", [(0, 30), (1, 30), (0, 63), (1, 63)])
def test_build_full_size_4m(ctx, oracle, builder, bits):
    """The builder workload at its full size (N = 4M), bit for bit against the oracle."""
    _, boxes, blo, bhi = _inputs(oracle, 4 * 1024 * 1024, 77)
    nodes = _check_same(ctx, oracle, boxes, blo, bhi, bits, builder)
    ok, cost, depth = oracle.check_tree(nodes, boxes.shape[0])
    assert ok


def test_triangle_boxes_match_reference(ctx, oracle):
    quv = W.corners_to_quv(W.soup(100003, 8))
    boxes, bounds = ctx.triangle_boxes(L.pack_tris(quv))
    assert np.array_equal(boxes, oracle.triangle_bounds(quv))
    blo, bhi = W.mesh_bounds(quv)
    assert np.array_equal(bounds, np.concatenate([blo, bhi]))


@pytest.mark.parametrize("builder", [0, 1])
def test_scene_build_matches_oracle(ctx, oracle, builder):
    """lrc_scene_build: boxes and bounds made on the device, the tree as the oracle's."""
    n = 123457
    quv, boxes, blo, bhi = _inputs(oracle, n, 12)
    s = L.Scene(ctx)
    s.set_triangles(L.pack_tris(quv))
    s.build(builder, 30)
    nodes, aux = s.tree()
    lo, ext = oracle.params(blo, bhi)
    want = (oracle.ploc if builder else oracle.lbvh)(boxes, lo, ext, 30)
    assert np.array_equal(nodes, want[0])
    assert np.array_equal(aux, want[1])
