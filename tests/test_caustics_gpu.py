"""GPU parity of light-traced caustics (lrc_caustics, lrc_caustics_sums) against the reference's own
CPU light tracer (light_trace_caustics, engine/rt/tracer.c:553-665), and of the path tracer's
skip_caustics (tracer.c:371-500) against trace_image with skip_caustics set: the two together give
the full image, checked against the FP64 oracle."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

from test_pathtrace_gpu import GOLDEN, cam9, ref_scene, rel_rmse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell128():
    return W.cornell_spheres(width=128, height=128)


def params(oracle, sc, exact, seed=0, skip=0):
    cam = oracle.camera(cam9(sc), sc["camera"]["vfov"], 1.0)
    return L.native.trace_params(cam, sc["width"], sc["height"], sc["max_depth"], 1, 1, exact, seed, 0.0, skip)


def test_exact_mode_is_the_cpu_light_tracer(ctx, oracle, cornell128):
    """Exact mode: the CPU's batches of 4096 light paths on their random streams. Equal images up
    to the paths where CUDA's and the C library's sinf/cosf round differently; the rays counted
    (scene_intersect and scene_occluded calls) equal within 1 %."""
    sc = cornell128
    photons, seed = 128 * 128 * 16, 77
    ref = ref_scene(oracle, sc)
    cpu, (closest, shadow) = ref.light_trace_caustics(cam9(sc), sc["camera"]["vfov"], 128, 128, photons,
                                                      sc["max_depth"], seed)
    s = R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    gpu, rays = s.caustics(params(oracle, sc, 1), photons, seed)
    lit = np.any(cpu > 0, axis=2)
    equal = np.all(gpu == cpu, axis=2)[lit].mean()
    err = rel_rmse(gpu, cpu)
    print(f"lit pixels {lit.mean():.3f}, of them equal to the bit {equal:.4f}; relRMSE {err:.2e}; "
          f"rays GPU {rays} CPU {closest + shadow}")
    # measured: 63 % of the lit pixels equal to the bit, relRMSE 2e-3 (a light path whose sinf / cosf
    # rounds differently lands a whole splat elsewhere)
    assert lit.mean() > 0.3
    assert equal >= 0.55
    assert err <= 5e-3
    assert abs(gpu.mean() - cpu.mean()) / cpu.mean() < 2e-3
    assert abs(rays - (closest + shadow)) / (closest + shadow) < 1e-3


def test_sums_are_the_image_and_order_free(ctx, oracle, cornell128):
    """The 32.32 sums: the same for the same arguments, whatever the scheduling; the image is the
    sums / 2^32 converted as the float build converts them; two passes add up."""
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc, 0)
    a, ra = s.caustics_sums(p, 500_000, 3)
    b, rb = s.caustics_sums(p, 500_000, 3)
    assert np.array_equal(a, b) and ra == rb and a.any()
    img, _ = s.caustics(p, 500_000, 3)
    want = a.astype(np.float32) * np.float32(2.0 ** -32)
    assert np.array_equal(img, want)
    two, _ = s.caustics_sums(p, 500_000, 5, a.copy())
    c, _ = s.caustics_sums(p, 500_000, 5)
    assert np.array_equal(two, a + c)


def test_fast_mode_matches_exact_mode(ctx, oracle, cornell128):
    """Per-path streams: the same estimator, so the mean within 3 % of the exact mode's and as far
    from a converged caustic image as the exact mode at the same count. Four seeds each, and the
    mean absolute error: a caustic image's mean and squared error are ruled by a few rare bright
    paths (one run's mean spreads by about 3 % at 1M paths)."""
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    n = 128 * 128 * 256
    conv, _ = s.caustics(params(oracle, sc, 0), 16 * n, 9)

    def err(x):
        return float(np.abs(x.astype(np.float64) - conv).sum() / conv.sum())
    ex = [s.caustics(params(oracle, sc, 1), n, seed)[0] for seed in (1, 3, 5, 7)]
    fa = [s.caustics(params(oracle, sc, 0), n, seed)[0] for seed in (2, 4, 6, 8)]
    e_ex, e_fa = np.mean([err(x) for x in ex]), np.mean([err(x) for x in fa])
    m_ex, m_fa = np.mean([x.mean() for x in ex]), np.mean([x.mean() for x in fa])
    print(f"means: exact {m_ex:.6f} fast {m_fa:.6f} 16x {conv.mean():.6f}; relative mean absolute error to "
          f"16x the paths: exact {e_ex:.4f} fast {e_fa:.4f}")
    assert abs(m_fa - m_ex) / m_ex < 0.03
    assert e_fa < 1.15 * e_ex and e_ex < 1.15 * e_fa


def test_skip_caustics_is_the_cpu_image(ctx, oracle, cornell128):
    """trace_image with skip_caustics: the exact-mode GPU image against the CPU's, as the plain
    path tracer's parity test; dropping the caustic paths makes the image darker."""
    sc = cornell128
    spp, seed = 8, 5
    ref = ref_scene(oracle, sc)
    cpu, (closest, shadow) = ref.trace_image(cam9(sc), sc["camera"]["vfov"], 128, 128, spp, seed, sc["max_depth"],
                                             skip_caustics=1)
    s = R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    acc, rays = s.trace(params(oracle, sc, 1, seed, 1), spp)
    gpu = acc[..., :3] * (np.float32(1) / np.float32(spp))
    full, _ = s.trace(params(oracle, sc, 1, seed, 0), spp)
    exact = np.all(gpu == cpu, axis=2).mean()
    err = rel_rmse(gpu, cpu)
    print(f"pixels equal to the bit: {exact:.4f}; relRMSE {err:.2e}; rays GPU {rays} CPU {closest + shadow}")
    # measured: 85 % of the pixels equal to the bit, relRMSE 3.1e-6
    assert exact >= 0.7 and err <= 1e-4
    assert abs(rays - (closest + shadow)) / (closest + shadow) < 1e-3
    assert gpu.sum() < (full[..., :3] / spp).sum()


def test_path_plus_light_tracing_is_the_full_image(ctx, oracle, cornell128):
    """skip_caustics + lrc_caustics estimate the same image as the plain path tracer: against the
    FP64 oracle (the reference's double build, 4096 spp) the mean within 1 %, and the sum at least
    as close to it as the plain path tracer at the same spp (the caustics converge faster)."""
    golden = np.load(GOLDEN)
    sc = cornell128
    spp = 256
    s = R.world_scene(ctx, sc, 1)
    plain, _ = s.trace(params(oracle, sc, 0, 3, 0), spp)
    plain = plain[..., :3] / np.float32(spp)
    skip, _ = s.trace(params(oracle, sc, 0, 3, 1), spp)
    both = skip[..., :3] / np.float32(spp)
    both, _ = s.caustics(params(oracle, sc, 0), 128 * 128 * spp, 4, both)
    e_plain, e_both = rel_rmse(plain, golden), rel_rmse(both, golden)
    print(f"relRMSE to the FP64 oracle at {spp} spp: path tracing {e_plain:.4f}, "
          f"path tracing without caustics + light tracing {e_both:.4f}")
    assert abs(both.mean() - golden.mean()) / golden.mean() < 0.01
    assert e_both < 1.05 * e_plain


def test_batched_skip_caustics_equals_plain(ctx, oracle, cornell128):
    """The batch's wavefront carries the caustic chain state: with skip_caustics its image is the
    plain lrc_trace image to the bit."""
    import torch
    sc = cornell128
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc, 0, 6, 1)
    want, _ = s.trace(p, 8)
    img = torch.zeros(128, 128, 4, device="cuda")
    torch.cuda.synchronize()
    b = L.native.Batch(ctx)
    b.add(s, p, 8, img.data_ptr())
    b.run()
    ctx.sync()
    assert np.array_equal(img.cpu().numpy(), want)
    b.close()


def test_nothing_without_a_smooth_material(ctx, oracle):
    """No mirror / glass material (scene_has_specular false): no light paths, nothing added."""
    sc = W.cornell_spheres(n_spheres=4, width=32, height=32)
    for m in sc["materials"]:
        if m["type"] != 3:
            m.update(type=0, roughness=1.0, metallic=0.0, transmission=0.0)
    s = R.world_scene(ctx, sc, 1)
    img = np.full((32, 32, 3), 0.25, np.float32)
    out, rays = s.caustics(params(oracle, sc, 0), 100_000, 1, img.copy())
    assert rays == 0 and np.array_equal(out, img)
