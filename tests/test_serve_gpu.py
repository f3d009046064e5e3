"""GPU tests of the render server (lrc_server_*): jobs admitted by a byte budget and traced in
waves together - world scenes of several sizes and instanced scenes whose instances move for one
job only (top level refit or built again) - each give the image the job gives alone, to the bit:
through the plain lrc_trace, and through a server holding that job only."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world(ctx, oracle):
    scs = [W.box_scene(20 + i, n, 64, 48, 8) for i, n in enumerate((1500, 12000, 40000))]
    return [(sc, R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())) for sc in scs]


@pytest.fixture(scope="module")
def inst(ctx, oracle):
    sc = W.instanced_box(5, n_instances=2000, width=48, height=40, spp=8)
    return sc, R.instanced_box_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())


def job_params(sc, w, h, seed):
    return L.native.trace_params(W.camera(sc["camera"], w / h), w, h, sc["max_depth"], 1, 1, 0, seed)


def jobs_of(world, inst):
    """(scene dict, scene, params, spp, moved records or None, tlas mode)"""
    out = []
    for k, (sc, s) in enumerate(world):
        for r, (w, h, spp) in enumerate(((64, 48, 8), (40, 30, 32), (96, 72, 4))):
            out.append((sc, s, job_params(sc, w, h, 100 * k + r), spp, None, 0))
    sc, s = inst
    motion = W.rigid_motion(sc["xf"].shape[0], 3)
    for t, mode in ((2.0, 0), (5.0, 1), (9.0, 0)):
        rec = W.instance_records(dict(sc, xf=W.moved_xf(sc["xf"], motion, t)))
        out.append((sc, s, job_params(sc, 48, 40, int(t)), 16, rec, mode))
    out.append((sc, s, job_params(sc, 48, 40, 77), 8, None, 0))
    return out


def alone_plain(job, original):
    sc, s, p, spp, rec, mode = job
    if rec is not None:
        s.move_instances(rec, mode)
    acc, rays = s.trace(p, spp)
    if rec is not None:
        s.move_instances(original, 1)                    # (the scene as built again)
    return acc, rays


def serve_all(ctx, jobs, budget, wave_paths, policy=None):
    sv = L.native.Server(ctx, budget, wave_paths)
    if policy is not None:
        sv.set_policy(policy)
    ids = [sv.submit(s, p, spp, rec, mode) for (_, s, p, spp, rec, mode) in jobs]
    waves, most_active, most_queued = 0, 0, 0
    while sv.state()["finished"] < len(jobs):
        st = sv.state()
        most_queued = max(most_queued, st["queued"])
        sv.step()
        waves += 1
        most_active = max(most_active, sv.state()["active"])
        assert waves < 10_000
    out = []
    for jid in ids:
        res = sv.result(jid)
        out.append((sv.image(jid), res[1]))
        sv.release(jid)
    assert sv.state() == {"queued": 0, "active": 0, "finished": 0, "bytes": 0}
    sv.close()
    return out, waves, most_active, most_queued


@pytest.mark.parametrize("policy", [0, 1, 2])
def test_served_images_are_the_jobs_alone(ctx, world, inst, policy):
    """Whatever the wave policy (even shares, oldest first, fewest paths left first)."""
    sc_i, s_i = inst
    original = W.instance_records(sc_i)
    jobs = jobs_of(world, inst)
    # in the mix: a small wave (bands of a few rows, many waves) and a budget below the jobs' total
    total = sum(p.width * p.height * 16 for (_, _, p, _, _, _) in jobs)
    served, waves, most_active, most_queued = serve_all(ctx, jobs, budget=total // 2 + (4 << 20), wave_paths=20_000,
                                                        policy=policy)
    assert waves > 10 and most_active > 1 and most_queued > 0
    for job, (img, rays) in zip(jobs, served):
        acc, want_rays = alone_plain(job, original)
        assert np.array_equal(img, acc)
        assert rays == want_rays
    # each job alone in a server of its own: the same image
    for job, (img, rays) in zip(jobs[::3], served[::3]):
        alone, _, _, _ = serve_all(ctx, [job], budget=1 << 30, wave_paths=1 << 22)
        assert np.array_equal(alone[0][0], img) and alone[0][1] == rays


def test_budget_refuses_a_job_larger_than_it(ctx, world):
    sc, s = world[0]
    sv = L.native.Server(ctx, 1 << 20, 1 << 20)
    p = job_params(sc, 512, 512, 1)                       # a 4 MB image
    with pytest.raises(L.native.LrcError) as e:
        sv.submit(s, p, 4)
    assert e.value.code == -6
    sv.close()
