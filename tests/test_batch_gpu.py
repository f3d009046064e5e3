"""GPU tests of the batch (lrc_batch_*): many jobs over many scenes through one persistent
megakernel (engine 0) or the wavefront loop (engine 1). Each job's image must equal the plain
lrc_trace image of the same arguments to the bit (fast and exact mode), and its ray count must be
the plain count; building the scenes inside the run, replaying the run as a CUDA graph, bands,
sample offsets, wavefront sizes and the autotuner must change nothing."""
import numpy as np
import pytest

import little_renderer_b200 as L
from little_renderer_b200 import render as R, workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def params(sc, exact=0, seed=5):
    return L.native.trace_params(R.camera12(sc), sc["width"], sc["height"], sc["max_depth"], 1, 1, exact, seed)


@pytest.fixture(scope="module")
def scenes():
    return W.batch_scenes(6, seed=4, tri_range=(1_000, 30_000), resolutions=(24, 40, 64), spps=(1, 4, 8, 32))


@pytest.fixture(scope="module")
def built(ctx, oracle, scenes):
    return [R.world_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables()) for sc in scenes]


def device_images(scenes):
    imgs = [torch.zeros(sc["height"], sc["width"], 4, device="cuda") for sc in scenes]
    torch.cuda.synchronize()
    return imgs


def plain(built, scenes, exact=0):
    out = []
    for s, sc in zip(built, scenes):
        acc, rays = s.trace(params(sc, exact), sc["spp"])
        out.append((acc, rays))
    return out


def host(ctx, imgs):
    ctx.sync()
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in imgs]


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("exact", [0, 1])
def test_batched_images_are_the_plain_ones(ctx, scenes, built, exact, engine):
    want = plain(built, scenes, exact)
    imgs = device_images(scenes)
    b = L.native.Batch(ctx)
    b.set_engine(engine)
    for s, sc, t in zip(built, scenes, imgs):
        b.add(s, params(sc, exact), sc["spp"], t.data_ptr())
    b.run()
    got = host(ctx, imgs)
    per, total = b.rays()
    for i, ((acc, rays), g) in enumerate(zip(want, got)):
        assert np.array_equal(g, acc), f"job {i}: pixels differ {np.sum(np.any(g != acc, axis=2))}"
        assert int(per[i]) == rays
    assert total == sum(r for _, r in want)
    info = b.info()
    assert info["pixels"] == sum(sc["width"] * sc["height"] for sc in scenes)


@pytest.mark.parametrize("engine", [0, 1])
def test_graph_replay_with_builds(ctx, oracle, scenes, engine):
    """Builds (LBVH, PLOC, both) inside the run, the run replayed as one CUDA graph: every replay
    gives the plain image of a scene built by the same builder."""
    own = [R.world_scene(ctx, sc, 0, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables()) for sc in scenes]
    builders = [i % 3 for i in range(len(scenes))]
    imgs = device_images(scenes)
    b = L.native.Batch(ctx)
    b.set_engine(engine)
    for s, sc, t, bl in zip(own, scenes, imgs, builders):
        b.add(s, params(sc), sc["spp"], t.data_ptr(), builder=bl, key_bits=30)
    refs = []
    for sc, bl in zip(scenes, builders):
        ref = R.world_scene(ctx, sc, min(bl, 1), blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
        refs.append(ref.trace(params(sc), sc["spp"])[0])
        ref.close()
    used = []
    for i in range(4):
        if i == 3:      # every scene's triangles set again (as a host copy would): the replay builds them
            for s, sc in zip(own, scenes):
                s.set_triangles(L.pack_tris(W.corners_to_quv(sc["corners"]), sc["tri_mats"]))
        b.run(build=True, graph=True, zero=True)
        got = host(ctx, imgs)
        used.append(b.info()["graph_used"])
        for g, acc in zip(got, refs):
            assert np.array_equal(g, acc)
    assert used == [0, 1, 1, 1]


def test_bands_and_sample_offsets_add_up(ctx, scenes, built):
    """Two jobs on one image - the top band, then all rows at later samples - equal the two plain
    calls made in the same order."""
    sc, s = scenes[1], built[1]
    p = params(sc)
    h = sc["height"]
    acc = np.zeros((h, sc["width"], 4), np.float32)
    s.trace(p, 4, accum=acc, y0=0, rows=h // 2)
    s.trace(p, 8, accum=acc, y0=0, rows=h, spp0=4)
    img = device_images([sc])[0]
    b = L.native.Batch(ctx)
    b.add(s, p, 4, img.data_ptr(), y0=0, rows=h // 2)
    b.run()
    b.clear()
    b.add(s, p, 8, img.data_ptr(), y0=0, rows=h, spp0=4)
    b.run()
    got = host(ctx, [img])[0]
    assert np.array_equal(got, acc)


def test_tuner_changes_no_image(ctx, scenes, built):
    want = plain(built, scenes)
    imgs = device_images(scenes)
    b = L.native.Batch(ctx)
    b.set_engine(0)
    for s, sc, t in zip(built, scenes, imgs):
        b.add(s, params(sc), sc["spp"], t.data_ptr())
    v, grid, ns = b.tune(sample_tasks=20000)
    shapes = L.native.batch_shapes()
    assert 0 <= v < len(shapes) and grid == shapes[v][2] * ctx.num_sms() and ns > 0
    got_before = host(ctx, imgs)
    assert all(not g.any() for g in got_before)          # tuning wrote no image
    b.run()
    got = host(ctx, imgs)
    for (acc, _), g in zip(want, got):
        assert np.array_equal(g, acc)
    for v in range(len(shapes)):                         # every shape gives the same images
        b.set_shape(v)
        b.run(zero=True)
        got = host(ctx, imgs)
        for (acc, _), g in zip(want, got):
            assert np.array_equal(g, acc)


def test_wavefront_tuner_and_sizes_change_no_image(ctx, scenes, built):
    want = plain(built, scenes)
    imgs = device_images(scenes)
    b = L.native.Batch(ctx)
    for s, sc, t in zip(built, scenes, imgs):
        b.add(s, params(sc), sc["spp"], t.data_ptr())
    assert b.engine()["engine"] == 1
    v, slots, ns = b.tune(sample_tasks=50000)
    shapes = L.native.wavefront_shapes()
    assert 0 <= v < len(shapes) and slots % 256 == 0 and ns > 0
    assert b.engine() == {"engine": 1, "slots": slots, "wf_variant": v}
    assert all(not g.any() for g in host(ctx, imgs))     # tuning wrote no image
    b.run()
    for (acc, _), g in zip(want, host(ctx, imgs)):
        assert np.array_equal(g, acc)
    b.run(zero=True, stepped=True)                       # the host-looped passes (for profilers)
    for (acc, _), g in zip(want, host(ctx, imgs)):
        assert np.array_equal(g, acc)
    # tiny pools (paths regenerate in every pass) and every launch shape
    for slots, v in [(256, 0), (4096, 1), (65536, 2)] + [(1 << 16, k) for k in range(len(shapes))]:
        b.set_wavefront(slots, v)
        b.run(zero=True)
        got = host(ctx, imgs)
        per, _ = b.rays()
        for i, ((acc, rays), g) in enumerate(zip(want, got)):
            assert np.array_equal(g, acc), (slots, v, i)
            assert int(per[i]) == rays


def test_wavefront_instanced_scene_with_sky(ctx, oracle):
    """The two-level scene (instances, sky, no lamp) through the wavefront, exact and fast mode."""
    sc = W.instanced_field(n_instances=300, tri_range=(500, 3000), width=40, height=24, sky_w=128, sky_h=64, spp=4,
                           max_depth=12)
    s = R.instanced_scene(ctx, sc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    for exact in (0, 1):
        p = L.native.trace_params(R.camera12(sc), sc["width"], sc["height"], sc["max_depth"], 1, 1, exact, 9)
        acc, rays = s.trace(p, sc["spp"])
        img = device_images([sc])[0]
        b = L.native.Batch(ctx)
        b.add(s, p, sc["spp"], img.data_ptr())
        b.run()
        got = host(ctx, [img])[0]
        assert np.array_equal(got, acc)
        assert int(b.rays()[0][0]) == rays
        b.close()


def test_wavefront_runs_alternating_with_and_without_instances(ctx, oracle, scenes, built):
    """Runs of one batch that alternate between jobs without instances and jobs with an instanced
    scene (a server's waves do): each key's graph is captured once, then kept and replayed when
    the key comes back, and every run's images are the plain ones."""
    isc = W.instanced_box(5, n_instances=2000, width=48, height=40, spp=8)
    inst = R.instanced_box_scene(ctx, isc, 1, blue_noise=oracle.blue_noise(), bsdf_tables=oracle.bsdf_tables())
    sets = [list(zip(built[:3], scenes[:3])), list(zip(built[:2], scenes[:2])) + [(inst, isc)]]
    want = [[s.trace(params(sc), sc["spp"])[0] for s, sc in js] for js in sets]
    b = L.native.Batch(ctx)
    b.set_engine(1)
    used = []
    for r in range(4):
        js = sets[r % 2]
        imgs = device_images([sc for _, sc in js])
        b.clear()
        for (s, sc), t in zip(js, imgs):
            b.add(s, params(sc), sc["spp"], t.data_ptr())
        b.run(graph=True)
        got = host(ctx, imgs)
        used.append(b.info()["graph_used"])
        for g, acc in zip(got, want[r % 2]):
            assert np.array_equal(g, acc)
    assert used == [0, 0, 1, 1]
    inst.close()
