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


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("builder", [0, 1])
@pytest.mark.parametrize("n", [1, 3, 1000, 100000])
def test_closest_hits_match_scene_intersect(ctx, oracle, builder, n, walk):
    cor, quv, ref = _scene(oracle, n, 40 + n)
    o, d = _rays(cor, 200000, 3)
    rp, _, rt = ref.intersect(o, d)
    s = L.Scene(ctx)
    s.set_triangles(L.pack_tris(quv))
    s.set_walk(walk)
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
        for walk in (1, 2):
            s.set_walk(walk)
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


def _flat_grids(cells=32):
    """Three axis-aligned grids of flat triangles in the unit cube (z = 0.25, x = 0.5, y = 0.75),
    cells x cells squares of 2 triangles each, sharing edges and corners: boxes of no thickness."""
    g = np.linspace(0.0, 1.0, cells + 1, dtype=np.float64)
    tris = []
    for axis, c in ((2, 0.25), (0, 0.5), (1, 0.75)):
        u, v = [k for k in range(3) if k != axis]
        for i in range(cells):
            for j in range(cells):
                p = np.zeros((4, 3))
                p[:, axis] = c
                p[:, u] = [g[i], g[i + 1], g[i + 1], g[i]]
                p[:, v] = [g[j], g[j], g[j + 1], g[j + 1]]
                tris.append(p[[0, 1, 2]])
                tris.append(p[[0, 2, 3]])
    return np.asarray(tris, np.float32)


@pytest.mark.parametrize("builder", [0, 1])
def test_tight_walk_same_hits_on_flat_grids_edges_and_far_rays(ctx, oracle, builder):
    """The walk's tree (lrc_scene_set_walk 1: the triangles' own bounds widened by 2^-17 of the
    scene's size; 2: the same as 8-wide quantised nodes) against the tree as built and against
    scene_intersect, where tight boxes are thinnest: axis-aligned grids of flat triangles, rays aimed at their shared corners and edge
    midpoints from 2 to 40 units away, and rays that graze the grids' planes."""
    cor = _flat_grids()
    ref = oracle.RefScene()
    ref.material(0, (0.5, 0.5, 0.5))
    ref.triangles(cor, np.zeros(cor.shape[0], np.int32))
    ref.set_accel()
    rng = np.random.default_rng(17)
    g = np.linspace(0.0, 1.0, 33)
    targets = []
    for axis, c in ((2, 0.25), (0, 0.5), (1, 0.75)):
        u, v = [k for k in range(3) if k != axis]
        for gu, gv in ((g, g), ((g[:-1] + g[1:]) / 2, g), (g, (g[:-1] + g[1:]) / 2)):
            uu, vv = np.meshgrid(gu, gv, indexing="ij")
            p = np.zeros((uu.size, 3))
            p[:, axis] = c
            p[:, u] = uu.ravel()
            p[:, v] = vv.ravel()
            targets.append(p)
    targets = np.concatenate(targets)
    n = 200000
    tgt = targets[rng.integers(0, targets.shape[0], n)]
    dist = np.exp(rng.uniform(np.log(2.0), np.log(40.0), n))
    dirn = rng.normal(size=(n, 3))
    dirn /= np.linalg.norm(dirn, axis=1, keepdims=True)
    o = tgt + dirn * dist[:, None]
    graze = n // 4                                  # a quarter: origins beside a plane, nearly parallel to it
    ax = rng.integers(0, 3, graze)
    planes = np.array([0.5, 0.75, 0.25])            # the grid at x = 0.5, y = 0.75, z = 0.25
    o[:graze] = rng.uniform(-0.5, 1.5, (graze, 3))
    o[np.arange(graze), ax] = planes[ax] + rng.choice([-1.0, 1.0], graze) * 10.0 ** rng.uniform(-7, -3, graze)
    tg = rng.uniform(0.0, 1.0, (graze, 3))
    tg[np.arange(graze), ax] = planes[ax]
    tgt[:graze] = tg
    d = tgt - o
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    o = o.astype(np.float32)
    rp, _, rt = ref.intersect(o, d)
    s = L.Scene(ctx)
    s.set_triangles(L.pack_tris(W.corners_to_quv(cor)))
    s.build(builder, 30)
    p1, t1 = s.intersect(o, d)
    b1, _ = s.trace_stats(o, d)
    s.set_walk(2)
    p2, t2 = s.intersect(o, d)
    s.set_walk(0)
    p0, t0 = s.intersect(o, d)
    b0, _ = s.trace_stats(o, d)
    print(f"flat grids, builder {builder}: {(rp >= 0).mean():.3f} of rays hit; box tests a ray {b1 / n:.1f} "
          f"(tight) vs {b0 / n:.1f} (as built); differing hits {int((p1 != rp).sum())} / {int((p2 != rp).sum())} / "
          f"{int((p0 != rp).sum())} (tight, 8-wide, as built)")
    assert (rp >= 0).mean() > 0.5
    assert_hits_match(p1, t1, rp, rt)
    assert_hits_match(p2, t2, rp, rt)
    assert_hits_match(p0, t0, rp, rt)
    assert b1 <= b0
    s.close()
