"""The builder workload's closest-hit queries through two trees of the same triangles: the
reference's own SAH tree (scene_set_accel, engine/rt/accel.c; handed over in put_nodes' layout by
lrc_scene_set_tree, as the engine's GPU backend hands the Scene's tree over, trace_gpu.c:1103-1112)
and the device-built PLOC tree. Both give scene_intersect's hits; each tree's work per ray (box and
triangle tests of the walk) and the closest-hit kernel's device time over the same rays are
printed, at 1M triangles / 2M rays and at the workload's 4M triangles / 16M rays, each tree walked
as built (its boxes padded by triangle_bounds' 1e-3), as the walk's tree (lrc_scene_set_walk 1:
the triangles' own bounds, widened by 2^-17 of the scene's size) and as that tree's 8-wide
quantised nodes (2; box tests count an 80-byte node as 2.5 records of 32 bytes)."""
import numpy as np
import pytest
import torch

import little_renderer_b200 as L
from little_renderer_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _walk(ctx, s, d_o, d_d, nrays, d_p, d_t, reps=3):
    """(box tests per ray, triangle tests per ray, closest-hit ms per pass) of scene s."""
    boxes, tris = s.trace_stats((nrays, d_o.data_ptr(), d_d.data_ptr()))
    s.intersect_device(d_o.data_ptr(), d_d.data_ptr(), nrays, d_p.data_ptr(), d_t.data_ptr())
    ctx.sync()
    ctx.set_timing(True)
    ctx.timings()
    for _ in range(reps):
        s.intersect_device(d_o.data_ptr(), d_d.data_ptr(), nrays, d_p.data_ptr(), d_t.data_ptr())
    ctx.sync()
    ms = ctx.timings()["trace"][0] / reps
    ctx.set_timing(False)
    return boxes / nrays, tris / nrays, ms


@pytest.mark.parametrize("n,nrays", [(1 << 20, 1 << 21), (4 << 20, 16 << 20)])
def test_sah_and_ploc_trees_give_the_same_hits_and_their_cost(ctx, oracle, n, nrays):
    cor = W.soup(n, 1)
    ref = oracle.RefScene(gpu=True)
    ref.material(0, (0.5, 0.5, 0.5))
    ref.triangles(cor, np.zeros(n, np.int32))
    ref.set_accel()
    nodes, refs = ref.tree()
    orig, dirs = W.rays_at_cube(nrays, 2)
    k = 1 << 18
    rp, _, rt = ref.intersect(orig[:k], dirs[:k])
    ref.close()

    tris = L.pack_tris(W.corners_to_quv(cor))
    sah = L.Scene(ctx)
    sah.set_triangles(tris)
    sah.set_tree(nodes, refs)
    ploc = L.Scene(ctx)
    ploc.set_triangles(tris)
    ploc.build(1, 30)

    dev = torch.device("cuda", 0)
    d_o = torch.from_numpy(orig).to(dev)
    d_d = torch.from_numpy(dirs).to(dev)
    d_p = torch.empty(nrays, dtype=torch.int32, device=dev)
    d_t = torch.empty(nrays, dtype=torch.float32, device=dev)
    out = {}
    for name, s in (("sah", sah), ("ploc", ploc)):
        for tight in (0, 1, 2):
            s.set_walk(tight)
            bpr, tpr, ms = _walk(ctx, s, d_o, d_d, nrays, d_p, d_t)
            out[name, tight] = (d_p.cpu().numpy(), d_t.cpu().numpy(), bpr, tpr, ms)
            print(f"{n} triangles, {nrays} rays, {name.upper()} tree, {('padded', 'tight', '8-wide tight')[tight]} boxes: "
                  f"{bpr:.1f} box and {tpr:.2f} triangle tests a ray ({bpr * 32 + tpr * 48:.0f} B of nodes and "
                  f"triangles), closest-hit pass {ms:.2f} ms = {nrays / ms / 1e3:.1f} Mrays/s")
    sah.close()
    ploc.close()
    for key in out:
        if key != ("sah", 0):
            ps, ts = out["sah", 0][0], out["sah", 0][1]
            pk, tk = out[key][0], out[key][1]
            same = ps == pk
            assert np.array_equal(ps >= 0, pk >= 0)
            assert (~same).sum() <= max(20, nrays // 100000)
            assert np.array_equal(ts[same], tk[same])
            assert np.all(np.abs(ts[~same] - tk[~same]) <= 1e-6 * np.abs(ts[~same]))
    assert out["ploc", 1][2] <= out["ploc", 0][2] and out["sah", 1][2] <= out["sah", 0][2]

    # the SAH tree's walk against scene_intersect on the first 256k rays
    p, t = out["sah", 1][0][:k], out["sah", 1][1][:k]
    same = p == rp
    assert (rp >= 0).sum() > 1000                   # (the soup's tiny triangles: about 1 % of the rays hit)
    assert np.array_equal(p >= 0, rp >= 0)
    assert (~same).sum() <= 20
    assert np.array_equal(t[same], rt[same])
    assert np.all(np.abs(t[~same] - rt[~same]) <= 1e-6 * np.abs(rt[~same]))
