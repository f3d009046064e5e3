"""GPU parity of the materials' textures (lrc_scene_set_texmaps, lrc_scene_set_texcoords: base colour,
metal-rough and normal maps, bilinear at level 0, sRGB decoding, wrap modes) against the reference's
own CPU path tracer and light tracer on the same TexMaps, Material.tex_* and Triangle.t
(hit_shading, engine/rt/tracer.c:241-255; material_at / material_normal, scene.c:259-301)."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

from test_pathtrace_gpu import cam9, ref_scene, rel_rmse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def textured():
    return W.textured_cornell(width=128, height=128)


def ref_textured(oracle, sc):
    ref = ref_scene(oracle, sc)
    for px, srgb, wu, wv in sc["texmaps"]:
        assert ref.texmap(px, srgb, wu, wv) > 0
    for i, m in enumerate(sc["materials"]):
        t = m.get("tex")
        if t:
            ref.material_textures(i, t.get("base", 0), t.get("mr", 0), t.get("normal", 0), t.get("emissive", 0),
                                  t.get("occlusion", 0), t.get("uv_scale", 0.0), t.get("normal_scale", 0.0))
    ref.texcoords(*sc["texcoords"])
    return ref


def params(oracle, sc, exact, seed):
    cam = oracle.camera(cam9(sc), sc["camera"]["vfov"], 1.0)
    return L.native.trace_params(cam, sc["width"], sc["height"], sc["max_depth"], 1, 1, exact, seed)


def test_exact_mode_is_the_cpu_image_with_textures(ctx, oracle, textured):
    sc = textured
    spp, seed = 4, 3
    ref = ref_textured(oracle, sc)
    cpu, (closest, shadow) = ref.trace_image(cam9(sc), sc["camera"]["vfov"], 128, 128, spp, seed, sc["max_depth"])
    s = R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    acc, rays = s.trace(params(oracle, sc, 1, seed), spp)
    gpu = acc[..., :3] * (np.float32(1) / np.float32(spp))
    bare = R.world_scene(ctx, dict(sc, texmaps=[], texcoords=None, materials=[dict(m, tex=None) for m in sc["materials"]]), 1)
    plain, _ = bare.trace(params(oracle, sc, 1, seed), spp)
    exact = np.all(gpu == cpu, axis=2).mean()
    err = rel_rmse(gpu, cpu)
    print(f"textures: pixels equal to the bit {exact:.4f}; relRMSE {err:.2e}; rays GPU {rays} CPU {closest + shadow}; "
          f"the textures change {np.any(acc != plain, axis=2).mean():.3f} of the pixels")
    assert np.any(acc != plain, axis=2).mean() > 0.3
    # measured: 70 % of the pixels equal to the bit, relRMSE 5e-6 (the rest differ in the last bits)
    assert exact >= 0.6
    assert err <= 1e-4
    assert abs(rays - (closest + shadow)) / (closest + shadow) < 1e-3


def test_light_tracing_with_textures_is_the_cpu_one(ctx, oracle, textured):
    """The metal-rough texture makes its materials possibly smooth (scene_has_specular), and the
    light tracer shades with the textures too: exact mode against light_trace_caustics."""
    sc = textured
    photons, seed = 128 * 128 * 8, 5
    ref = ref_textured(oracle, sc)
    cpu, (closest, shadow) = ref.light_trace_caustics(cam9(sc), sc["camera"]["vfov"], 128, 128, photons,
                                                      sc["max_depth"], seed)
    s = R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    gpu, rays = s.caustics(params(oracle, sc, 1, 0), photons, seed)
    err = rel_rmse(gpu, cpu)
    print(f"caustics with textures: relRMSE {err:.2e}; rays GPU {rays} CPU {closest + shadow}")
    assert err <= 2e-3                              # (measured 2.4e-4)
    assert abs(rays - (closest + shadow)) / (closest + shadow) < 2e-3


@pytest.mark.parametrize("engine", [1, 0])
def test_batched_textured_equals_plain(ctx, oracle, textured, engine):
    import torch
    sc = textured
    s = R.world_scene(ctx, sc, 1)
    p = params(oracle, sc, 0, 6)
    want, _ = s.trace(p, 8)
    img = torch.zeros(128, 128, 4, device="cuda")
    torch.cuda.synchronize()
    b = L.native.Batch(ctx)
    b.set_engine(engine)
    b.add(s, p, 8, img.data_ptr())
    b.run(zero=True)
    ctx.sync()
    assert np.array_equal(img.cpu().numpy(), want)
    b.close()


def test_fast_mode_mean_matches_cpu_with_textures(ctx, oracle, textured):
    sc = textured
    ref = ref_textured(oracle, sc)
    cpu, _ = ref.trace_image(cam9(sc), sc["camera"]["vfov"], 128, 128, 64, 5, sc["max_depth"])
    s = R.world_scene(ctx, sc, 1)
    acc, _ = s.trace(params(oracle, sc, 0, 9), 64)
    gpu = acc[..., :3] / acc[..., 3:4]
    print(f"64 spp means: GPU {gpu.mean():.5f} CPU {cpu.mean():.5f}")
    assert abs(gpu.mean() - cpu.mean()) / cpu.mean() < 0.02
