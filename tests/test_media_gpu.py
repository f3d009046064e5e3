"""GPU parity of participating media (lrc_scene_set_volumes; delta and ratio tracking over majorant
bricks, engine/rt/medium.c, in the path tracer of engine/rt/tracer.c:384-420) against the
reference's own CPU path tracer on the same Volume (scene_add_volume), and of light tracing
through media against light_trace_caustics."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

from test_pathtrace_gpu import cam9, ref_scene, rel_rmse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def foggy():
    return W.foggy_cornell(width=96, height=96)


def ref_foggy(oracle, sc):
    ref = ref_scene(oracle, sc)
    for den, lo, hi, st, al, g in sc["volumes"]:
        assert ref.volume(den, lo, hi, st, al, g) >= 0
    return ref


def params(oracle, sc, exact, seed):
    cam = oracle.camera(cam9(sc), sc["camera"]["vfov"], 1.0)
    return L.native.trace_params(cam, sc["width"], sc["height"], sc["max_depth"], 1, 1, exact, seed)


def test_exact_mode_is_the_cpu_image_with_media(ctx, oracle, foggy):
    """Exact mode: the CPU's random streams through delta tracking, ratio tracking and the phase
    function; equal up to the paths where CUDA's and the C library's logf / sinf / cosf round
    differently (a tentative collision moves by an ulp and can change a decision)."""
    sc = foggy
    spp, seed = 4, 3
    ref = ref_foggy(oracle, sc)
    cpu, (closest, shadow) = ref.trace_image(cam9(sc), sc["camera"]["vfov"], 96, 96, spp, seed, sc["max_depth"])
    s = R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    acc, rays = s.trace(params(oracle, sc, 1, seed), spp)
    gpu = acc[..., :3] * (np.float32(1) / np.float32(spp))
    plain = R.world_scene(ctx, dict(sc, volumes=[]), 1)
    clear, _ = plain.trace(params(oracle, sc, 1, seed), spp)
    exact = np.all(gpu == cpu, axis=2).mean()
    err = rel_rmse(gpu, cpu)
    print(f"media: pixels equal to the bit {exact:.4f}; relRMSE {err:.2e}; rays GPU {rays} CPU {closest + shadow}; "
          f"the medium changes {np.any(acc != clear, axis=2).mean():.3f} of the pixels")
    assert np.any(acc != clear, axis=2).mean() > 0.5
    # measured: 74 % of the pixels equal to the bit, relRMSE 3e-8
    assert exact >= 0.65
    assert err <= 1e-5
    assert abs(gpu.mean() - cpu.mean()) / cpu.mean() < 1e-4
    assert abs(rays - (closest + shadow)) / (closest + shadow) < 1e-3


def test_fast_mode_mean_matches_cpu_with_media(ctx, oracle, foggy):
    sc = foggy
    ref = ref_foggy(oracle, sc)
    cpu, _ = ref.trace_image(cam9(sc), sc["camera"]["vfov"], 96, 96, 64, 5, sc["max_depth"])
    s = R.world_scene(ctx, sc, 1)
    acc, _ = s.trace(params(oracle, sc, 0, 9), 64)
    gpu = acc[..., :3] / acc[..., 3:4]
    print(f"64 spp means: GPU {gpu.mean():.5f} CPU {cpu.mean():.5f}")
    assert abs(gpu.mean() - cpu.mean()) / cpu.mean() < 0.02


def test_clear_medium_changes_nothing(ctx, oracle, foggy):
    """A volume with no extinction: no collision, transmittance 1, the image of the scene without
    it to the bit (MIS already normalises the rays)."""
    sc = foggy
    den, lo, hi, _, al, g = sc["volumes"][0]
    a = R.world_scene(ctx, dict(sc, volumes=[(den, lo, hi, 0.0, al, g)]), 1)
    b = R.world_scene(ctx, dict(sc, volumes=[]), 1)
    for exact in (1, 0):
        p = params(oracle, sc, exact, 4)
        assert np.array_equal(a.trace(p, 4)[0], b.trace(p, 4)[0])


def test_megakernel_batch_equals_plain_with_media(ctx, oracle, foggy):
    """The batch's engine 0 traces media (shadow rays in place): its image is lrc_trace's to the bit;
    the wavefront engine refuses the job."""
    import torch
    sc = foggy
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc, 0, 6)
    want, _ = s.trace(p, 8)
    img = torch.zeros(96, 96, 4, device="cuda")
    torch.cuda.synchronize()
    b = L.native.Batch(ctx)
    b.add(s, p, 8, img.data_ptr())
    with pytest.raises(L.native.LrcError):
        b.run()
    b.set_engine(0)
    b.run(zero=True)
    ctx.sync()
    assert np.array_equal(img.cpu().numpy(), want)
    b.close()


def test_light_tracing_through_media_is_the_cpu_one(ctx, oracle, foggy):
    """Light paths that scatter in the medium stop; camera connections are dimmed by ratio
    tracking: exact mode against light_trace_caustics."""
    sc = foggy
    photons, seed = 96 * 96 * 16, 31
    ref = ref_foggy(oracle, sc)
    cpu, (closest, shadow) = ref.light_trace_caustics(cam9(sc), sc["camera"]["vfov"], 96, 96, photons,
                                                      sc["max_depth"], seed)
    s = R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    gpu, rays = s.caustics(params(oracle, sc, 1, 0), photons, seed)
    err = rel_rmse(gpu, cpu)
    print(f"caustics through media: relRMSE {err:.2e}; rays GPU {rays} CPU {closest + shadow}")
    assert err <= 1e-2                              # (measured 2.7e-3)
    assert abs(rays - (closest + shadow)) / (closest + shadow) < 2e-3
