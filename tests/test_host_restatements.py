"""What the library makes on the host by the reference's published methods, pinned against the
reference's own code on the CPU: the blue-noise mask (sampler.c bn_make), the BSDF tables
(scene/brdf_tables.h), the sky's sampling tables (env.c make_weights/prepare_base), and the scene
generators' float32 restatements of make_quad, camera_make, xform_inverse and xform_box."""
import ctypes

import numpy as np

import little_renderer_b200 as L
from little_renderer_b200 import workloads as W


def test_default_blue_noise_is_the_reference_mask(oracle):
    mine = np.zeros(4096, np.uint16)
    L.lib().lrc_default_blue_noise(mine.ctypes.data_as(ctypes.c_void_p))
    assert np.array_equal(mine, oracle.blue_noise())


def test_default_bsdf_tables_are_the_reference_tables(oracle):
    mine = np.zeros(2112, np.float32)
    L.lib().lrc_default_bsdf_tables(mine.ctypes.data_as(ctypes.c_void_p))
    assert np.array_equal(mine, oracle.bsdf_tables())


def test_sky_tables_are_env_prepare_s(oracle):
    rgb = W.sky(256, 128, seed=9)
    ref = oracle.RefScene()
    ref.env(rgb)
    want = ref.env_tables(256, 128)
    got = L.native.sky_tables(rgb)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_quad_and_camera_restatements(oracle):
    sc = W.cornell_spheres()
    ref = oracle.RefScene()
    ref.material(3, (0, 0, 0), (15, 15, 15))
    lamp = sc["lamp"]
    ref.quad(lamp["q"], lamp["u"], lamp["v"], 0, light=True)
    assert np.array_equal(ref.prim_data()[0], W.make_quad(lamp["q"], lamp["u"], lamp["v"], 0))
    c = sc["camera"]
    fau = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
    for aspect in (1.0, 16 / 9):
        assert np.array_equal(oracle.camera(fau, c["vfov"], aspect), W.camera(c, aspect))


def test_instance_transforms_and_boxes(oracle):
    sc = W.instanced_field(n_instances=200, tri_range=(500, 2000), sky_w=64, sky_h=32)
    ref = oracle.RefScene()
    ref.material(0, (0.5, 0.5, 0.5))
    for tri in sc["meshes"]:
        ref.mesh(tri, np.zeros(tri.shape[0], np.int32))
    for i in range(sc["xf"].shape[0]):
        ref.instance(int(sc["mesh_of"][i]), sc["xf"][i].reshape(-1), -1)
    rec = W.instance_records(sc)
    for i in range(sc["xf"].shape[0]):
        box, inv = ref.instance_data(i)
        assert np.array_equal(inv, rec[i, 12:24])
        assert np.array_equal(box[:3], rec[i, 24:27]) and np.array_equal(box[3:], rec[i, 28:31])
