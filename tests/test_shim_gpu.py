"""The drop-in backend: the reference engine's own offline GPU entry point, gpu_frame_trace
(engine/app/gpu_frame.c:49, compiled unmodified from the reference's sources), running on the CUDA
backend (little_renderer_b200/shim/gpu_cuda.c: the engine's gpu.h / view_gpu.h on liblrc) in place
of the reference's WebGPU one. It traces the scene's OWN tree (scene_bvh), as the reference's GPU
path tracer does, and its image equals lrc_trace's of the same scene, tree and samples to the bit."""
import os

import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GPU_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_gpu.so")


def engine_scene(O, sc, gpu=True):
    ref = O.RefScene(gpu=gpu)
    for m in sc["materials"]:
        ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"], m["transmission"])
    ref.triangles(sc["corners"], sc["tri_mats"])
    lamp = sc["lamp"]
    ref.quad(lamp["q"], lamp["u"], lamp["v"], lamp["material"], light=True)
    ref.set_accel()
    return ref


def cam9(sc):
    c = sc["camera"]
    return np.array([*c["from"], *c["at"], *c["up"]], np.float32)


@pytest.fixture(scope="module")
def plain_render():
    if not os.path.exists(GPU_LIB):
        pytest.fail(f"{GPU_LIB} is not built (make -C oracle REF=<the reference's checkout>)")
    return W.cornell_spheres(width=256, height=256)


def lrc_image_by_passes(s, p, spp):
    """lrc_trace one sample per pixel at a time, in sample order (as the backend's passes add them)."""
    acc = np.zeros((p.height, p.width, 4), np.float32)
    rays = 0
    for k in range(spp):
        acc, r = s.trace(p, 1, accum=acc, spp0=k)
        rays += r
    return acc, rays


def test_gpu_frame_trace_on_the_cuda_backend_is_lrc_trace(ctx, oracle, plain_render):
    """The plain render as configured (256 x 256, 16 spp, depth 8, NEE + MIS, Owen-Sobol) through the
    engine's gpu_frame_open / gpu_frame_trace / gpu_frame_close on the CUDA backend: its image (the
    sums read back by gpu_view_trace_read, divided by the counts in gpu_frame.c) equals, to the bit,
    the mean of lrc_trace's passes on the same scene, the same tree (the engine's SAH tree given by
    lrc_scene_set_tree) and the same samples (image seed 0)."""
    sc = plain_render
    ref = engine_scene(oracle, sc)
    rc, img = ref.gpu_frame_trace(cam9(sc), sc["camera"]["vfov"], 256, 256, 16, sc["max_depth"])
    assert rc == 0
    s = R.world_scene(ctx, sc, 1)
    nodes, refs = ref.tree()
    assert nodes.shape[0] < 2 * refs.shape[0] - 1            # (leaves of up to 4 shapes: a smaller tree)
    s.set_tree(nodes, refs)
    p = L.native.trace_params(oracle.camera(cam9(sc), sc["camera"]["vfov"], 1.0), 256, 256, sc["max_depth"], 1, 1, 0, 0)
    acc, _ = lrc_image_by_passes(s, p, 16)
    assert (acc[..., 3] == 16).all()
    want = acc[..., :3] / acc[..., 3:4]
    print(f"gpu_frame_trace image mean {img.mean():.5f}; equal to lrc_trace's passes: {np.array_equal(img, want)}")
    assert np.array_equal(img, want)


def test_the_engines_tree_gives_the_built_trees_image(ctx, oracle, plain_render):
    """The scene's own SAH tree (lrc_scene_set_tree) and the device-built PLOC tree trace the same
    image in exact mode, but for the rare pixels where two triangles tie in t and the trees find them
    in another order; the tree given is checked (a child out of range is refused)."""
    sc = plain_render
    ref = engine_scene(oracle, sc)
    nodes, refs = ref.tree()
    a = R.world_scene(ctx, sc, 1)
    b = R.world_scene(ctx, sc, 1)
    b.set_tree(nodes, refs)
    p = L.native.trace_params(oracle.camera(cam9(sc), sc["camera"]["vfov"], 1.0), 256, 256, sc["max_depth"], 1, 1, 1, 4)
    ia, ra = a.trace(p, 4)
    ib, rb = b.trace(p, 4)
    equal = np.all(ia == ib, axis=2).mean()
    print(f"PLOC tree vs the engine's SAH tree: pixels equal {equal:.5f}, rays {ra} vs {rb}")
    assert equal >= 0.999
    assert abs(ra - rb) <= 1e-4 * ra
    bad = nodes.copy()
    inner = np.nonzero((bad[:, 7] & 0x80000000) == 0)[0][0]
    bad[inner, 3] = nodes.shape[0] + 5
    with pytest.raises(L.native.LrcError):
        b.set_tree(bad, refs)
