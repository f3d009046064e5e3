"""The oracles themselves, on the CPU: the restated builders against the reference's own code
and against properties the reference's builders guarantee (check_tree, trace_gpu.c:768-805)."""
import numpy as np
import pytest

from little_renderer_b200 import workloads as W


def _boxes(O, n, seed):
    quv = W.corners_to_quv(W.soup(n, seed))
    boxes = O.triangle_bounds(quv)
    lo, ext = O.params(*W.mesh_bounds(quv))
    return quv, boxes, lo, ext


def test_spread_codes_match_naive_interleave(oracle):
    rng = np.random.default_rng(0)
    boxes = rng.random((500, 8)).astype(np.float32)
    boxes[:, 4:7] = boxes[:, 0:3] + 0.01
    lo = np.zeros(3, np.float32)
    ext = np.ones(3, np.float32)
    for bits, per in ((30, 10), (63, 21)):
        keys = oracle.morton(boxes, lo, ext, bits)
        for i in range(0, 500, 37):
            c = (boxes[i, 0:3] + boxes[i, 4:7]) * np.float32(0.5)
            q = (np.clip(c * np.float32(1), 0, np.float32(0.999)) * np.float32(2 ** per)).astype(np.uint32)
            code = 0
            for b in range(per):
                for ax in range(3):
                    code |= ((int(q[ax]) >> b) & 1) << (3 * b + (2 - ax))
            got = int(keys[i, 0]) if bits == 30 else int(keys[i, 0]) | (int(keys[i, 1]) << 32)
            assert got == code
            assert keys[i, -1] == i


@pytest.mark.parametrize("bits", [30, 63])
def test_bitonic_equals_stable_sort(oracle, bits):
    _, boxes, lo, ext = _boxes(oracle, 5000, 3)
    k = oracle.morton(boxes, lo, ext, bits)
    s = oracle.bitonic(k, bits)
    if bits == 30:
        ref = k[np.lexsort((k[:, 1], k[:, 0]))]
    else:
        ref = k[np.lexsort((k[:, 2], k[:, 0], k[:, 1]))]
    assert np.array_equal(s, ref)


@pytest.mark.parametrize("n", [1, 2, 3, 17, 1000, 3001])
@pytest.mark.parametrize("bits", [30, 63])
def test_lbvh_oracle_is_one_tree(oracle, n, bits):
    _, boxes, lo, ext = _boxes(oracle, n, n)
    nodes, aux = oracle.lbvh(boxes, lo, ext, bits)
    ok, cost, depth = oracle.check_tree(nodes, n)
    assert ok
    assert sorted(aux.tolist()) == list(range(n))


@pytest.mark.parametrize("n", [3, 4, 100, 1500, 5000])
def test_ploc_oracle_is_one_tree_and_independent_of_small(oracle, n):
    _, boxes, lo, ext = _boxes(oracle, n, n + 7)
    a = oracle.ploc(boxes, lo, ext, 30, small=1024)
    b = oracle.ploc(boxes, lo, ext, 30, small=8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    ok, cost, depth = oracle.check_tree(a[0], n)
    assert ok


def test_offsets(oracle):
    _, boxes, lo, ext = _boxes(oracle, 300, 5)
    a, aa = oracle.lbvh(boxes, lo, ext, 30)
    b, ab = oracle.lbvh(boxes, lo, ext, 30, node0=10, ref0=7, ref_add=100)
    assert np.array_equal(ab[7:], aa + 100)
    # children and leaf refs shifted, boxes equal
    inner = (a[:, 7] & 0x80000000) == 0
    assert np.array_equal(b[10:][inner, 3], a[inner, 3] + 10)
    assert np.array_equal(b[10:][~inner, 3], a[~inner, 3] + 7)
    assert np.array_equal(b[10:][:, [0, 1, 2, 4, 5, 6]], a[:, [0, 1, 2, 4, 5, 6]])


def test_triangle_bounds_and_params(oracle):
    quv = W.corners_to_quv(W.soup(1000, 9))
    boxes = oracle.triangle_bounds(quv)
    q = quv[:, 0:3]
    c1 = (q + quv[:, 3:6]).astype(np.float32)
    c2 = (q + quv[:, 6:9]).astype(np.float32)
    lo = np.minimum(np.minimum(q, c1), c2) - np.float32(1e-3)
    hi = np.maximum(np.maximum(q, c1), c2) + np.float32(1e-3)
    assert np.array_equal(boxes[:, 0:3], lo.astype(np.float32))
    assert np.array_equal(boxes[:, 4:7], hi.astype(np.float32))
    s = oracle.RefScene()
    m = s.mesh(W.soup(1000, 9), np.zeros(1000, np.int32))
    blo, bhi = W.mesh_bounds(quv)
    assert np.array_equal(s.mesh_box(m), np.concatenate([blo, bhi]))
    lo_, ext = oracle.params(blo, bhi)
    assert np.array_equal(ext, (np.float32(1) / (bhi - blo)).astype(np.float32))


@pytest.mark.parametrize("builder", ["lbvh", "ploc"])
def test_tree_walk_matches_scene_intersect(oracle, builder):
    """Closest hits through the restated builders' trees equal the reference's scene_intersect
    (its own 4-wide SAH tree) on seeded rays: the same triangle and the same t, bit for bit."""
    n = 4000
    cor = W.soup(n, 21)
    quv = W.corners_to_quv(cor)
    boxes = oracle.triangle_bounds(quv)
    lo, ext = oracle.params(*W.mesh_bounds(quv))
    nodes, aux = (oracle.lbvh if builder == "lbvh" else oracle.ploc)(boxes, lo, ext, 30)
    o, d = W.rays_at_cube(20000, 5)
    # aim a quarter of the rays at triangle centroids so that many hit
    pick = np.random.default_rng(1).integers(0, n, 5000)
    tgt = cor[pick].mean(axis=1)
    dd = tgt - o[:5000]
    d[:5000] = (dd / np.linalg.norm(dd, axis=1, keepdims=True)).astype(np.float32)
    s = oracle.RefScene()
    s.material(0, (0.5, 0.5, 0.5))
    s.triangles(cor, np.zeros(n, np.int32))
    s.set_accel()
    pr, _, tr = s.intersect(o, d)
    p2, t2, _ = oracle.trace_tree(nodes, aux, quv, o, d)
    assert (pr >= 0).sum() > 2000
    assert np.array_equal(p2, pr)
    assert np.array_equal(t2[pr >= 0], tr[pr >= 0])


def test_refit_restatement_is_bvh_refit_boxes(oracle):
    """or_refit on the reference's own SAH tree (bvh_build_boxes) gives bvh_refit_boxes' boxes."""
    rng = np.random.default_rng(1)
    n = 3000
    lo = rng.uniform(0, 100, (n, 3)).astype(np.float32)
    boxes = np.zeros((n, 8), np.float32)
    boxes[:, :3] = lo
    boxes[:, 4:7] = lo + rng.uniform(0.1, 5, (n, 3)).astype(np.float32)
    moved = boxes.copy()
    shift = rng.normal(0, 3, (n, 3)).astype(np.float32)
    moved[:, :3] += shift
    moved[:, 4:7] += shift
    nodes, refs, _ = oracle.ref_bvh_refit(boxes, moved)
    assert np.array_equal(oracle.refit(nodes, refs, moved), nodes)



def test_fp64_golden_fixture():
    """The FP64 oracle image (tests/golden/make_fp64_golden.py): its shape and a sane mean."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cornell128_fp64_4096spp.npy"))
    assert g.shape == (128, 128, 3) and g.dtype == np.float32
    assert np.isfinite(g).all() and 0.05 < g.mean() < 0.5
