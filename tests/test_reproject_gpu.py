"""GPU checks of the reprojection (lrc_reproject: a new image's samples carried over from the
previous image's, trace_reproject.wgsl `main`) and of its temporal gradients
(lrc_reproject_gradients: gmatch, the gradient samples, gfilter, main with each pixel's history)
against their numpy restatement (oracle/reproject_oracle.py), and their properties: an unmoved
camera keeps each pixel's samples (capped at the history), a moved one keeps what is still seen and
makes a converged image start closer to the truth than a fresh one; in a static scene the gradient
samples repeat the old ones and every pixel keeps its history, under a dimmed lamp far less."""
import copy

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


def gradients(s, p0, p1, old, hmax=32, fallback=8, edit=False, nxt=16):
    new = guided(s, p1, 0)
    tiles = s.reproject_gradients(p0, p1, nxt, old, new, hmax, fallback, edit)
    return new, tiles


@pytest.mark.parametrize("edit", [False, True])
def test_gradients_match_the_restatement(ctx, oracle, scene, edit):
    """A moved camera: the tiles' gradient pixels (new and old) are the restated gmatch's; the
    filter over the samples' lambda is the restated gfilter's; the planes are the restated main's
    with each pixel's history from the filtered lambda."""
    from oracle import reproject_oracle as RP
    sc, s = scene
    c = sc["camera"]
    p0 = cam_params(oracle, sc, c["from"], c["at"], 1)
    p1 = cam_params(oracle, sc, (c["from"][0] + 10.0, c["from"][1] + 5.0, c["from"][2]), (c["at"][0] + 8.0, c["at"][1], c["at"][2]), 2)
    old = guided(s, p0, 16)
    new, tiles = gradients(s, p0, p1, old, 32, 8, edit)
    guide = guided(s, p1, 0)
    m = RP.gmatch(old, guide, cams(p0), cams(p1), 16, edit)
    have = tiles[..., 1] >= 0
    same = (tiles[..., 0] == m["k"]) & (tiles[..., 1] == m["o"])
    traced = (tiles[..., 2][have] >= 0).mean()
    filt = RP.gfilter(tiles[..., 2], guide)
    close = np.isclose(filt, tiles[..., 3], rtol=1e-4, atol=1e-6).mean()
    print(f"edit {edit}: tiles with a gradient sample {have.mean():.3f}, the same pixels as the restatement's "
          f"{same.mean():.4f}, traced {traced:.4f}; filtered lambda as restated {close:.4f}; "
          f"median lambda {np.median(tiles[..., 2][have]):.4f}")
    assert have.mean() > 0.5 and same.mean() > 0.98 and traced > 0.95
    assert close > 0.999
    hist = RP.grad_history(tiles[..., 3], guide, 32, 8, edit)
    want = RP.reproject(old, guide, cams(p0), cams(p1), hist, edit)
    kg, kw = new[0][..., 3] > 0, want[0][..., 3] > 0
    both = kg & kw
    print(f"pixels with history {kg.mean():.3f}, the same as the restatement's {(kg == kw).mean():.4f}")
    assert (kg == kw).mean() > 0.995
    assert rel_rmse(new[0][both], want[0][both]) < 1e-3
    assert rel_rmse(new[1][both][:, :2], want[1][both][:, :2]) < 1e-3


def test_static_scene_keeps_its_history(ctx, oracle, scene):
    """Nothing moved: each gradient sample is the old pixel's last sample traced again with its
    random numbers, so lambda is ~0 and every surface pixel keeps all 16 old samples."""
    sc, s = scene
    c = sc["camera"]
    p = cam_params(oracle, sc, c["from"], c["at"], 5)
    old = guided(s, p, 16)
    new, tiles = gradients(s, p, p, old, 32, 8)
    have = tiles[..., 1] >= 0
    lam = tiles[..., 2][have]
    surf = (old[3][..., 3] % 4) == 0
    full = np.isclose(new[0][..., 3], 16, rtol=1e-3)[surf].mean()
    print(f"static: tiles with a sample {have.mean():.3f}; lambda median {np.median(lam):.2e}, "
          f"below 0.05 {(lam < 0.05).mean():.4f}; surface pixels keeping 16 samples {full:.4f}")
    assert have.mean() > 0.8
    assert np.median(lam) < 1e-3 and (lam < 0.05).mean() > 0.9
    assert full > 0.9


def test_dimmed_lamp_drops_the_history(ctx, oracle):
    """The lamp at a third of its power: a gradient sample whose old value had light sees a third
    of it (lambda 2/3; one whose old value was black stays black, lambda 0: in this scene most
    single samples are), and the filtered lambda cuts the history the surfaces keep to under 60 %
    of what they keep when nothing changed (where no tile near had light it stays whole)."""
    sc = W.cornell_spheres(width=128, height=128)
    s = R.world_scene(ctx, sc, 1)
    c = sc["camera"]
    p = cam_params(oracle, sc, c["from"], c["at"], 6)
    old = guided(s, p, 16)
    surf = (old[3][..., 3] % 4) == 0
    still, _ = gradients(s, p, p, old, 32, 8)
    mats = copy.deepcopy(sc["materials"])
    for mt in mats:
        if max(mt["emission"]) > 0:
            mt["emission"] = tuple(e / 3.0 for e in mt["emission"])
    s.set_materials(W.material_records(mats))
    new, tiles = gradients(s, p, p, old, 32, 8)
    have = tiles[..., 1] >= 0
    lit = old[1][..., 2].reshape(-1)[tiles[..., 1][have].astype(np.int64)] > 0
    lam = tiles[..., 2][have]
    k_still, k_dim = still[0][..., 3][surf].mean(), new[0][..., 3][surf].mean()
    print(f"dimmed: tiles whose old sample had light {lit.mean():.3f}, their lambda median {np.median(lam[lit]):.4f}, "
          f"within 0.02 of 2/3 {(np.abs(lam[lit] - 2 / 3) < 0.02).mean():.4f}; the others' lambda 0 "
          f"{(lam[~lit] == 0).mean():.4f}; samples kept a surface pixel: unchanged {k_still:.2f}, dimmed {k_dim:.2f}")
    assert lit.mean() > 0.1
    assert (np.abs(lam[lit] - 2 / 3) < 0.02).mean() > 0.9
    assert (lam[~lit] == 0).mean() > 0.98
    assert k_still > 15 and k_dim < 0.6 * k_still


def test_gradient_arguments(ctx, oracle, scene):
    """An exact-mode old image (its samples cannot be traced alone) and history_max 0 are refused."""
    sc, s = scene
    c = sc["camera"]
    p = cam_params(oracle, sc, c["from"], c["at"], 1)
    old = guided(s, p, 2)
    ex = L.native.trace_params(oracle.camera(np.array([*c["from"], *c["at"], *c["up"]], np.float32), c["vfov"], 1.0),
                               sc["width"], sc["height"], sc["max_depth"], 1, 1, 1, 1)
    for args in ((ex, p, 2, old, guided(s, p, 0), 32, 8), (p, p, 2, old, guided(s, p, 0), 0, 8)):
        with pytest.raises(L.native.LrcError):
            s.reproject_gradients(*args)


def test_gradients_device_arrays(ctx, oracle, scene):
    """The same through device arrays (LRC_DEVICE): planes and tiles equal the host call's."""
    import torch
    sc, s = scene
    c = sc["camera"]
    p0 = cam_params(oracle, sc, c["from"], c["at"], 1)
    p1 = cam_params(oracle, sc, (c["from"][0] + 6.0, c["from"][1], c["from"][2]), c["at"], 2)
    old = guided(s, p0, 4)
    new, tiles = gradients(s, p0, p1, old, 16, 4, nxt=4)
    d_old = torch.from_numpy(old).cuda()
    d_new = torch.from_numpy(guided(s, p1, 0)).cuda()
    d_tiles = torch.zeros(tiles.shape, device="cuda")
    torch.cuda.synchronize()
    s.reproject_gradients_device(p0, p1, 4, d_old.data_ptr(), d_new.data_ptr(), 16, 4, d_tiles.data_ptr())
    ctx.sync()
    assert np.array_equal(d_new.cpu().numpy(), new)
    assert np.array_equal(d_tiles.cpu().numpy(), tiles)


@pytest.mark.parametrize("hmax,edit", [(32, False), (32, True), (0, False)])
def test_frame_is_the_separate_calls(ctx, oracle, scene, hmax, edit):
    """lrc_trace_frame gives the planes of lrc_guide + lrc_reproject_gradients (or lrc_reproject
    with history_max 0) + lrc_trace with LRC_TRACE_GUIDED, to the bit, from host or device arrays;
    the first frame (no old planes) those of lrc_guide + lrc_trace."""
    import torch
    sc, s = scene
    c = sc["camera"]
    p0 = cam_params(oracle, sc, c["from"], c["at"], 3)
    p1 = cam_params(oracle, sc, (c["from"][0] + 8.0, c["from"][1] - 4.0, c["from"][2]), (c["at"][0] + 6.0, c["at"][1], c["at"][2]), 3)
    first = s.trace_frame(None, p0, 0, 4, None, hmax, 8, edit)
    want0 = guided(s, p0, 0)
    s.trace_guided(p0, 4, want0)
    assert np.array_equal(first, want0)
    got = s.trace_frame(p0, p1, 4, 2, first, hmax, 8, edit)
    want = guided(s, p1, 0)
    if hmax:
        s.reproject_gradients(p0, p1, 4, first, want, hmax, 8, edit)
    else:
        ctx.reproject(p0, p1, first, want, 8)
    s.trace_guided(p1, 2, want, spp0=4)
    print(f"hmax {hmax} edit {edit}: pixels with history {(want[0][..., 3] > 2).mean():.3f}; "
          f"planes equal {[bool(np.array_equal(got[i], want[i])) for i in range(4)]}")
    assert np.array_equal(got, want)
    d_old = torch.from_numpy(first).cuda()
    d_new = torch.zeros(4, p1.height, p1.width, 4, device="cuda")
    torch.cuda.synchronize()
    s.trace_frame_device(p0, p1, 4, 2, d_old.data_ptr(), d_new.data_ptr(), hmax, 8, edit)
    ctx.sync()
    assert np.array_equal(d_new.cpu().numpy(), want)
