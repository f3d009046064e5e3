"""Seeded synthetic workloads (no public dataset is involved; all inputs are generated here).

Triangles are kept as the reference stores them (engine/scene/scene.h:134-140 ``Triangle``):
corner ``q`` and edges ``u = b - a``, ``v = c - a``, each computed in float32 exactly as
``scene_add_triangle`` (engine/scene/scene.c add_tri) computes them in the float build.
"""
import numpy as np


def corners_to_quv(corners):
    """(n, 3, 3) float32 corners a, b, c -> (n, 9) q, u, v with float32 subtraction."""
    c = np.ascontiguousarray(corners, np.float32).reshape(-1, 3, 3)
    q = c[:, 0]
    u = (c[:, 1] - c[:, 0]).astype(np.float32)
    v = (c[:, 2] - c[:, 0]).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([q, u, v], axis=1), np.float32)


def soup(n, seed=1):
    """The builder workload: n triangles with centroids uniform in the unit cube, edges
    Gaussian with sigma = 0.002 * n^(-1/3), and 2 % of them (a seeded choice) scaled x50 about
    their centroid. Returns (n, 3, 3) float32 corners."""
    rng = np.random.default_rng(seed)
    cen = rng.random((n, 3), dtype=np.float64)
    sigma = 0.002 * n ** (-1.0 / 3.0)
    e1 = rng.normal(0.0, sigma, (n, 3))
    e2 = rng.normal(0.0, sigma, (n, 3))
    big = rng.random(n) < 0.02
    e1[big] *= 50.0
    e2[big] *= 50.0
    a = cen - (e1 + e2) / 3.0
    corners = np.stack([a, a + e1, a + e2], axis=1).astype(np.float32)
    return corners


def rays_at_cube(n, seed=2, radius=2.0, centre=(0.5, 0.5, 0.5)):
    """n rays: origins uniform on the sphere of `radius` about `centre`, unit directions toward
    uniform points of the unit cube. Returns (orig, dir) float32 (n, 3) each."""
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(n, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    o = (np.asarray(centre) + radius * g).astype(np.float32)
    target = rng.random((n, 3), dtype=np.float64).astype(np.float32)
    d = (target - o).astype(np.float32)
    d = (d / np.linalg.norm(d.astype(np.float64), axis=1, keepdims=True)).astype(np.float32)
    return np.ascontiguousarray(o), np.ascontiguousarray(d)


def mesh_bounds(quv):
    """SceneMesh.box (engine/scene/scene.c:638-646 mesh_bounds): the corners' box, unpadded."""
    quv = np.asarray(quv, np.float32).reshape(-1, 9)
    q = quv[:, 0:3]
    b = (q + quv[:, 3:6]).astype(np.float32)
    c = (q + quv[:, 6:9]).astype(np.float32)
    lo = np.minimum(np.minimum(q.min(0), b.min(0)), c.min(0)).astype(np.float32)
    hi = np.maximum(np.maximum(q.max(0), b.max(0)), c.max(0)).astype(np.float32)
    return lo, hi
