"""GPU parity of ray queries: closest hits against the reference's own scene_intersect
(engine/rt/accel.c:252) and any hits against scene_occluded (:280), on seeded rays."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _scene(oracle, n, seed):
    cor = W.soup(n, seed)
    ref = oracle.RefScene()
    ref.material(0, (0.5, 0.5, 0.5))
    ref.triangles(cor, np.zeros(n, np.int32))
    ref.set_accel()
    quv, _ = ref.tri_data()
    return cor, quv, ref


def _rays(cor, nrays, seed, aimed=0.5):
    o, d = W.rays_at_cube(nrays, seed)
    k = int(nrays * aimed)
    rng = np.random.default_rng(seed + 1)
    tgt = cor[rng.integers(0, cor.shape[0], k)].mean(axis=1)
    dd = (tgt - o[:k]).astype(np.float64)
    d[:k] = (dd / np.linalg.norm(dd, axis=1, keepdims=True)).astype(np.float32)
    return o, d


def assert_hits_match(prim, t, rprim, rt):
    """Hit ids exactly equal, except ties: where they differ both hit at t within 1e-6 relative."""
    assert np.array_equal(prim >= 0, rprim >= 0)
    diff = prim != rprim
    both = rprim >= 0
    assert np.all(np.abs(t[diff] - rt[diff]) <= 1e-6 * np.abs(rt[diff]))
    same = both & ~diff
    assert np.array_equal(t[same], rt[same])
    return int(diff.sum())


@pytest.mark.parametrize("builder", [0, 1])
@pytest.mark.parametrize("n", [1, 3, 1000, 100000])
def test_closest_hits_match_scene_intersect(ctx, oracle, builder, n):
    cor, quv, ref = _scene(oracle, n, 40 + n)
    o, d = _rays(cor, 200000, 3)
    rp, _, rt = ref.intersect(o, d)
    s = L.Scene(ctx)
    s.set_triangles(L.pack_tris(quv))
    s.build(builder, 30)
    p, t = s.intersect(o, d)
    ties = assert_hits_match(p, t, rp, rt)
    assert ties <= 5
    if n >= 1000:
        assert (rp >= 0).sum() > 50000


def test_closest_hits_full_size(ctx, oracle):
    """The builder workload at N = 4M with 2M of its rays (the CPU reference takes seconds)."""
    n = 4 * 1024 * 1024
    cor, quv, ref = _scene(oracle, n, 77)
    o, d = _rays(cor, 2 * 1024 * 1024, 9, aimed=0.25)
    rp, _, rt = ref.intersect(o, d)
    s = L.Scene(ctx)
    s.set_triangles(L.pack_tris(quv))
    for builder in (0, 1):
        s.build(builder, 30)
        p, t = s.intersect(o, d)
        assert assert_hits_match(p, t, rp, rt) <= 20


@pytest.mark.parametrize("builder", [0, 1])
def test_any_hits_match_scene_occluded(ctx, oracle, builder):
    n = 50000
    cor, quv, ref = _scene(oracle, n, 5)
    o, d = _rays(cor, 100000, 8)
    rp, _, rt = ref.intersect(o, d)
    tmax = np.where(rp >= 0, rt * np.float32(0.999), np.float32(1e30)).astype(np.float32)
    tmax[::3] = 1e30
    want = ref.occluded(o, d, 0.0, 1e30)
    s = L.Scene(ctx)
    s.set_triangles(L.pack_tris(quv))
    s.build(builder, 30)
    got = s.occluded(o, d, np.full(o.shape[0], 1e30, np.float32))
    assert np.array_equal(got.astype(bool), want.astype(bool))
    got2 = s.occluded(o, d, tmax)
    # the blocker before the closest hit cannot exist: blocked only where tmax was left at 1e30
    assert not got2[(rp >= 0) & (np.arange(o.shape[0]) % 3 != 0)].any()
