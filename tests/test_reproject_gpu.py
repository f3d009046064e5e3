"""GPU checks of the reprojection (lrc_reproject: a new image's samples carried over from the
previous image's, trace_reproject.wgsl `main` without temporal gradients) against its numpy
restatement (oracle/reproject_oracle.py), and its properties: an unmoved camera keeps each pixel's
samples (capped at the history), a moved one keeps what is still seen and makes a converged image
start closer to the truth than a fresh one."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

from test_pathtrace_gpu import cam9, rel_rmse

pytestmark = pytest.mark.gpu


def cam_params(oracle, sc, frm, at, seed):
    c = sc["camera"]
    fau = np.array([*frm, *at, *c["up"]], np.float32)
    return L.native.trace_params(oracle.camera(fau, c["vfov"], 1.0), sc["width"], sc["height"], sc["max_depth"], 1, 1, 0,
                                 seed)


def guided(s, p, spp):
    planes = np.zeros((4, p.height, p.width, 4), np.float32)
    s.guide(p, planes)
    if spp:
        s.trace_guided(p, spp, planes)
    return planes


def cams(p):
    return [list(p.origin), list(p.upper_left), list(p.horizontal), list(p.vertical)]


@pytest.fixture(scope="module")
def scene(ctx):
    sc = W.cornell_spheres(width=128, height=128)
    return sc, R.world_scene(ctx, sc, 1)


def test_unmoved_camera_keeps_the_samples(ctx, oracle, scene):
    sc, s = scene
    c = sc["camera"]
    p = cam_params(oracle, sc, c["from"], c["at"], 1)
    old = guided(s, p, 8)
    new = guided(s, p, 0)
    ctx.reproject(p, p, old, new, 64)
    surf = (old[3][..., 3] % 4) == 0
    kept = new[0][..., 3] > 0
    print(f"unmoved: {kept[surf].mean():.4f} of the surface pixels keep samples")
    assert kept[surf].mean() > 0.99
    both = surf & kept
    assert np.allclose(new[0][both][:, 3], 8, rtol=1e-3)
    assert rel_rmse(new[0][both][:, :3], old[0][both][:, :3]) < 0.05
    new2 = guided(s, p, 0)
    ctx.reproject(p, p, old, new2, 3)
    assert np.all(new2[0][..., 3] <= 3 + 1e-5)


def test_moved_camera_matches_the_restatement(ctx, oracle, scene):
    from oracle import reproject_oracle as RP
    sc, s = scene
    c = sc["camera"]
    p0 = cam_params(oracle, sc, c["from"], c["at"], 1)
    p1 = cam_params(oracle, sc, (c["from"][0] + 25.0, c["from"][1] + 10.0, c["from"][2]), (c["at"][0] + 20.0, c["at"][1], c["at"][2]), 2)
    old = guided(s, p0, 16)
    new = guided(s, p1, 0)
    want = RP.reproject(old, new, cams(p0), cams(p1), 32)
    got = ctx.reproject(p0, p1, old, new.copy(), 32)
    kg, kw = got[0][..., 3] > 0, want[0][..., 3] > 0
    agree = (kg == kw).mean()
    both = kg & kw
    err = rel_rmse(got[0][both], want[0][both])
    print(f"moved: pixels with history {kg.mean():.3f}; the same ones as the restatement's {agree:.4f}; relRMSE {err:.2e}")
    assert kg.mean() > 0.5
    assert agree > 0.995
    assert err < 1e-3
    assert rel_rmse(got[1][both][:, :2], want[1][both][:, :2]) < 1e-3


def test_reprojected_history_helps(ctx, oracle, scene):
    """A moved camera's new image started from the old one's 64 samples and given 4 of its own is
    closer to a converged render than 4 samples alone."""
    sc, s = scene
    c = sc["camera"]
    p0 = cam_params(oracle, sc, c["from"], c["at"], 1)
    p1 = cam_params(oracle, sc, (c["from"][0] + 15.0, c["from"][1], c["from"][2]), (c["at"][0] + 15.0, c["at"][1], c["at"][2]), 3)
    old = guided(s, p0, 64)
    new = guided(s, p1, 0)
    ctx.reproject(p0, p1, old, new, 64)
    s.trace_guided(p1, 4, new)
    fresh = guided(s, p1, 4)
    conv = guided(s, cam_params(oracle, sc, (c["from"][0] + 15.0, c["from"][1], c["from"][2]),
                                (c["at"][0] + 15.0, c["at"][1], c["at"][2]), 99), 512)
    img = lambda q: q[0][..., :3] / np.maximum(q[0][..., 3:4], 1)   # noqa: E731
    e_rep, e_fresh = rel_rmse(img(new), img(conv)), rel_rmse(img(fresh), img(conv))
    print(f"relRMSE to 512 spp: reprojected + 4 spp {e_rep:.4f}, 4 spp alone {e_fresh:.4f}")
    assert e_rep < 0.7 * e_fresh
