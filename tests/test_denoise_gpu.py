"""GPU checks of the denoiser (lrc_guide, lrc_trace with LRC_TRACE_GUIDED, lrc_denoise): the guide
against its restatement on the reference's own CPU scene (oracle/ref_bridge.c rb_guide, following
trace.wgsl guide()), the a-trous filter against its numpy restatement (oracle/denoise_oracle.py,
following denoise.wgsl), the moments against the samples, and the denoised image against the FP64
oracle. The reference's WGSL cannot run here, so the restatements are the parity targets."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

from test_pathtrace_gpu import GOLDEN, cam9, ref_scene, rel_rmse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell128():
    return W.cornell_spheres(width=128, height=128)


def params(oracle, sc, exact=0, seed=1):
    cam = oracle.camera(cam9(sc), sc["camera"]["vfov"], 1.0)
    return L.native.trace_params(cam, sc["width"], sc["height"], sc["max_depth"], 1, 1, exact, seed)


def guided(ctx, s, p, spp):
    planes = np.zeros((4, p.height, p.width, 4), np.float32)
    s.guide(p, planes)
    s.trace_guided(p, spp, planes)
    return planes


def test_guide_is_the_restated_guide(ctx, oracle, cornell128):
    """Kind, albedo and instance equal on all but a few pixels (a ray through glass that grazes an
    edge); normal and distance equal to float rounding where they agree."""
    sc = cornell128
    ref = ref_scene(oracle, sc)
    n_cpu, a_cpu = ref.guide(cam9(sc), sc["camera"]["vfov"], 128, 128)
    s = R.world_scene(ctx, sc, 1)
    planes = s.guide(params(oracle, sc))
    n_gpu, a_gpu = planes[2], planes[3]
    same = np.all(a_gpu == a_cpu, axis=2)
    print(f"guide: kind + albedo equal on {same.mean():.4f} of the pixels; "
          f"surfaces {(a_cpu[..., 3] == 0).mean():.3f}")
    assert same.mean() > 0.995
    assert np.allclose(n_gpu[same][:, :3], n_cpu[same][:, :3], atol=1e-5)
    z_ok = n_cpu[same][:, 3] < 1e29
    assert np.allclose(n_gpu[same][z_ok, 3], n_cpu[same][z_ok, 3], rtol=1e-5)
    assert np.array_equal(planes[0], np.zeros_like(planes[0]))       # planes 0 and 1 untouched


def test_guided_trace_keeps_the_image_and_adds_moments(ctx, oracle, cornell128):
    """Plane 0 equals the unguided image to the bit; with one sample per pixel the moments are
    (l, l^2) of that sample's luminance over the guide's albedo."""
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc)
    planes = guided(ctx, s, p, 1)
    plain, _ = s.trace(p, 1)
    assert np.array_equal(planes[0], plain)
    c = planes[0][..., :3]
    surf = (planes[3][..., 3] % 4) == 0
    irr = np.where(surf[..., None], c / np.maximum(planes[3][..., :3], np.float32(1e-3)), c)
    l = 0.2126 * irr[..., 0] + 0.7152 * irr[..., 1] + 0.0722 * irr[..., 2]
    assert np.allclose(planes[1][..., 0], l, rtol=1e-5, atol=1e-6)
    assert np.allclose(planes[1][..., 1], l * l, rtol=1e-4, atol=1e-6)
    # z, w: the last sample's l and its number + 1 (trace.wgsl keeps them for the temporal gradients)
    assert np.array_equal(planes[1][..., 2], planes[1][..., 0]) and np.all(planes[1][..., 3] == 1)
    s.trace_guided(p, 3, planes, spp0=1)
    assert np.all(planes[1][..., 3] == 4)
    ex = guided(ctx, s, params(oracle, sc, exact=1), 4)
    acc, _ = s.trace(params(oracle, sc, exact=1), 4)
    assert np.array_equal(ex[0], acc)
    assert np.all(ex[1][..., 1] >= ex[1][..., 0] ** 2 / 4 * (1 - 1e-5) - 1e-6)   # sum l^2 >= (sum l)^2 / n


@pytest.mark.parametrize("spp", [2, 16])
def test_denoise_matches_the_restatement(ctx, oracle, cornell128, spp):
    """The CUDA passes against denoise.wgsl restated in numpy on the same planes (2 spp: the
    variance from the neighbours; 16: from the pixel's moments). Values pass between passes as
    halves in both, so a weight that rounds differently can move a pixel by a half's ulp."""
    from oracle import denoise_oracle as D
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    planes = guided(ctx, s, params(oracle, sc, seed=spp), spp)
    gpu = ctx.denoise(planes)
    cpu = D.denoise(planes)
    err = rel_rmse(gpu[..., :3], cpu[..., :3])
    close = np.isclose(gpu[..., :3], cpu[..., :3], rtol=1e-2, atol=1e-4).all(axis=2).mean()
    print(f"{spp} spp: relRMSE to the restatement {err:.2e}, pixels within 1 %: {close:.4f}")
    assert np.array_equal(gpu[..., 3], cpu[..., 3])
    assert err < 2e-3
    assert close > 0.99
    one = ctx.denoise(planes, passes=1)
    assert rel_rmse(one[..., :3], D.denoise(planes, passes=1)[..., :3]) < 2e-3


def test_denoised_image_is_closer_to_the_fp64_oracle(ctx, oracle, cornell128):
    """At 16 spp the denoised image is closer to the FP64 oracle (the reference's double build at
    4096 spp) than the noisy one and keeps its mean within 2 %. Measured away from the lamp and
    its rim (3 pixels): there the guide sees the ceiling through the pixel's centre while the lamp
    covers part of the pixel, and the reference's filter spreads that coverage like noise."""
    golden = np.load(GOLDEN).astype(np.float64)
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    planes = guided(ctx, s, params(oracle, sc, seed=7), 16)
    noisy = (planes[0][..., :3] / planes[0][..., 3:4]).astype(np.float64)
    den = ctx.denoise(planes)[..., :3].astype(np.float64)
    bright = golden.mean(axis=2) > 2.0
    near = np.zeros_like(bright)
    for dy in range(-3, 4):
        for dx in range(-3, 4):
            near |= np.roll(np.roll(bright, dy, 0), dx, 1)
    keep = ~near

    def rr(x):
        return float(np.sqrt(((x - golden) ** 2)[keep].sum() / (golden ** 2)[keep].sum()))

    def mrae(x):
        return float(np.mean((np.abs(x - golden).sum(axis=2) / (golden.sum(axis=2) + 0.03))[keep]))
    print(f"16 spp, {keep.mean():.3f} of the pixels: relRMSE to the FP64 oracle noisy {rr(noisy):.4f} denoised "
          f"{rr(den):.4f}; relative mean absolute error noisy {mrae(noisy):.4f} denoised {mrae(den):.4f}")
    assert rr(den) < 0.8 * rr(noisy)
    assert mrae(den) < 0.85 * mrae(noisy)
    assert abs(den.mean() - golden.mean()) / golden.mean() < 0.02


def test_denoise_device_arrays(ctx, oracle, cornell128):
    """The same through device arrays (LRC_DEVICE), twice in a row (scratch reused)."""
    import torch
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc, seed=3)
    d_planes = torch.zeros(4, 128, 128, 4, device="cuda")
    d_out = torch.zeros(128, 128, 4, device="cuda")
    torch.cuda.synchronize()
    s.guide_device(p, d_planes.data_ptr())
    s.trace_guided_device(p, 8, d_planes.data_ptr())
    ctx.denoise_device(128, 128, d_planes.data_ptr(), d_out.data_ptr())
    ctx.sync()
    first = d_out.cpu().numpy()
    ctx.denoise_device(128, 128, d_planes.data_ptr(), d_out.data_ptr())
    ctx.sync()
    assert np.array_equal(d_out.cpu().numpy(), first)
    host = ctx.denoise(d_planes.cpu().numpy())
    assert np.array_equal(host, first)


@pytest.mark.parametrize("engine", [1, 0])
def test_batched_guided_equals_plain(ctx, oracle, cornell128, engine):
    """A guided batch job (lrc_batch_add_guided) beside an unguided one: its samples and moments
    equal lrc_trace's with LRC_TRACE_GUIDED to the bit (the moments summed in the same tree order),
    in both engines."""
    import torch
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc, seed=11)
    want = guided(ctx, s, p, 8)
    d_planes = torch.zeros(4, 128, 128, 4, device="cuda")
    img = torch.zeros(128, 128, 4, device="cuda")
    torch.cuda.synchronize()
    s.guide_device(p, d_planes.data_ptr())
    b = L.native.Batch(ctx)
    b.set_engine(engine)
    b.add(s, p, 8, d_planes.data_ptr(), guided=True)
    b.add(s, params(oracle, sc, seed=12), 4, img.data_ptr())
    b.run(zero=True)
    ctx.sync()
    got = d_planes.cpu().numpy()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    assert np.array_equal(got[2:], want[2:])
    plain, _ = s.trace(params(oracle, sc, seed=12), 4)
    assert np.array_equal(img.cpu().numpy(), plain)
    b.close()


def test_served_denoised_job_is_the_plain_denoise(ctx, oracle, cornell128):
    """A denoised server job among plain ones: its image is lrc_denoise of the plain guided planes,
    to the bit (admission's guide, the waves' moments, the passes at its end); the plain jobs keep
    their lrc_trace images."""
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    sv = L.native.Server(ctx, 1 << 30, 200_000)
    jobs = [(params(oracle, sc, seed=21), 8, True), (params(oracle, sc, seed=22), 4, False),
            (params(oracle, sc, seed=23), 16, True)]
    ids = [sv.submit(s, p, spp, denoise=d) for p, spp, d in jobs]
    while sv.state()["finished"] < len(jobs):
        sv.step()
    for jid, (p, spp, d) in zip(ids, jobs):
        got = sv.image(jid)
        if d:
            want = ctx.denoise(guided(ctx, s, p, spp))
        else:
            want, _ = s.trace(p, spp)
        assert np.array_equal(got, want), (jid, d)
        sv.release(jid)
    assert sv.state()["bytes"] == 0
    sv.close()
