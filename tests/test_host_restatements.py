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


def test_volume_majorants_are_volume_update_s(oracle):
    """The majorants lrc_scene_set_volumes derives on the host (largest density, active box, brick
    maxima) equal the reference's volume_update to the bit, for the workloads' cloud and for grids
    whose sides are not multiples of the 8-voxel brick (delta tracking draws its random numbers per
    majorant segment, so these must be the reference's)."""
    lib = oracle.ref_lib()
    rng = np.random.default_rng(4)
    grids = [(W.cloud_grid(3), (80.0, 60.0, 80.0), (480.0, 380.0, 480.0)),
             (np.clip(rng.normal(0.2, 0.5, (13, 21, 10)), 0, None).astype(np.float32), (-1.5, 0.25, 2.0), (3.5, 2.0, 7.25)),
             (np.zeros((9, 9, 9), np.float32), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))]
    for den, lo, hi in grids:
        mx, act, bricks = L.native.volume_majorants(den, lo, hi)
        nz, ny, nx = den.shape
        rmx = np.zeros(1, np.float32)
        ract = np.zeros(6, np.float32)
        rbr = np.zeros(bricks.size, np.float32)
        lib.rb_volume_majorants(nx, ny, nz, np.array([*lo, *hi], np.float32), np.ascontiguousarray(den).reshape(-1), rmx,
                                ract, rbr)
        assert mx == rmx[0]
        assert np.array_equal(act, ract)
        assert np.array_equal(bricks.reshape(-1), rbr)


def test_srgb_table_is_texmap_srgb_table_s(oracle):
    want = np.zeros(256, np.float32)
    oracle.ref_lib().rb_srgb_table(want)
    assert np.array_equal(L.native.srgb_table(), want)
