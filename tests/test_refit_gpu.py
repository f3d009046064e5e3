"""GPU refit (lrc_refit, lrc_scene_move_instances): the builders' trees refit on the device for
moved items equal the CPU restatement of bvh_refit_boxes (engine/rt/bvh.c:471-485) to the bit, and
moved instances hit what the reference's scene hits after scene_move_instance and
scene_update_instances (engine/rt/accel.c:197), whichever way the top level is made again."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

pytestmark = pytest.mark.gpu


def boxes_and_moved(n, seed):
    rng = np.random.default_rng(seed)
    lo = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    boxes = np.zeros((n, 8), np.float32)
    boxes[:, :3] = lo
    boxes[:, 4:7] = lo + rng.uniform(1e-4, 0.02, (n, 3)).astype(np.float32)
    moved = boxes.copy()
    shift = rng.normal(0, 0.05, (n, 3)).astype(np.float32)
    moved[:, :3] += shift
    moved[:, 4:7] += shift
    return boxes, moved


@pytest.mark.parametrize("builder", [0, 1])
@pytest.mark.parametrize("n", [3, 1000, 200_000])
def test_refit_is_bvh_refit_boxes(ctx, oracle, builder, n):
    boxes, moved = boxes_and_moved(n, 7 + n)
    p = ctx.params(n, boxes[:, :3].min(0), boxes[:, 4:7].max(0), builder=builder)
    nodes, aux = ctx.build(p, boxes)
    got = ctx.refit(nodes, aux, moved)
    want = oracle.refit(nodes, aux, moved)
    assert np.array_equal(got, want)
    assert np.array_equal(got[:, 3], nodes[:, 3]) and np.array_equal(got[:, 7], nodes[:, 7])   # (topology kept)
    back = ctx.refit(got, aux, boxes)                    # the original boxes give the built boxes back
    assert np.array_equal(back.view(np.float32), nodes.view(np.float32))


def ref_field(O, sc):
    ref = O.RefScene()
    for m in sc["materials"]:
        ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"], m["transmission"])
    g = sc["ground"]
    ref.quad(g["q"], g["u"], g["v"], g["material"])
    for tri, mm in zip(sc["meshes"], sc["mesh_mats"]):
        ref.mesh(tri, np.full(tri.shape[0], mm, np.int32))
    for i in range(sc["xf"].shape[0]):
        ref.instance(int(sc["mesh_of"][i]), sc["xf"][i].reshape(-1), -1)
    ref.set_accel()
    return ref


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_moved_instances_hit_what_the_reference_hits(ctx, oracle, mode):
    sc = W.instanced_field(n_instances=2000, tri_range=(500, 3000), width=32, height=32, sky_w=64, sky_h=32)
    ref = ref_field(oracle, sc)
    s = R.instanced_scene(ctx, sc, 1, sky=False, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    cost0 = s.tlas_cost()
    motion = W.rigid_motion(sc["xf"].shape[0], 11)
    rng = np.random.default_rng(5)
    n = 100_000
    o = np.stack([rng.uniform(-5, 45, n), rng.uniform(0.5, 8, n), rng.uniform(-5, 45, n)], 1).astype(np.float32)
    for t in (1.0, 4.0):
        xf = W.moved_xf(sc["xf"], motion, t)
        moved = dict(sc, xf=xf)
        for i in range(xf.shape[0]):
            ref.move_instance(i, xf[i].reshape(-1))
        ref.update_instances()
        s.move_instances(W.instance_records(moved), mode)
        tgt = xf[rng.integers(0, xf.shape[0], n), :, 3]
        d = (tgt - o).astype(np.float64)
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        rp, ri, rt = ref.intersect(o, d, 2e-3, 1e30)
        p, i, t_ = s.intersect_ex(o, d, 2e-3, 1e30)
        assert (ri >= 0).mean() > 0.3
        same = (p == rp) & (i == ri)
        assert (~same).sum() <= 20
        assert np.all(np.abs(t_[~same] - rt[~same]) <= 1e-6 * np.abs(rt[~same]))
        assert np.array_equal(t_[same], rt[same])
    cost = s.tlas_cost()
    if mode == 0:
        assert cost > cost0                               # (a refit tree loosens as things move apart)
