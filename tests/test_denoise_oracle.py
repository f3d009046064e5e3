"""CPU checks of the denoiser's restatement (oracle/denoise_oracle.py): properties the reference's
a-trous filter has by construction (denoise.wgsl), since no golden output of it exists."""
import numpy as np

from oracle import denoise_oracle as D


def flat_planes(h=24, w=32, spp=8, value=(0.3, 0.5, 0.7), albedo=(0.5, 0.5, 0.5)):
    px = np.zeros((4, h, w, 4), np.float32)
    px[0, ..., :3] = np.asarray(value, np.float32) * spp
    px[0, ..., 3] = spp
    l = D.luma(np.asarray(value, np.float32) / np.asarray(albedo, np.float32))
    px[1, ..., 0] = l * spp
    px[1, ..., 1] = l * l * spp
    px[2, ..., :3] = (0.0, 0.0, 1.0)
    px[2, ..., 3] = 10.0 + np.arange(w, dtype=np.float32)[None, :] * 0.01
    px[3, ..., :3] = albedo
    px[3, ..., 3] = 0.0
    return px


def test_flat_image_is_kept():
    """A noise-free flat surface: every pass averages equal values, so the image stays (up to the
    halves the passes store)."""
    px = flat_planes()
    out = D.denoise(px)
    want = px[0, ..., :3] / px[0, ..., 3:4]
    assert np.allclose(out[..., :3], want, rtol=2e-3)
    assert np.all(out[..., 3] == 1)


def test_lamp_and_empty_pixels_pass_through():
    px = flat_planes()
    px[3, 5:8, 5:8, 3] = 1.0                 # a lamp: kind 1, not filtered
    px[0, 5:8, 5:8, :3] = 50.0 * 8
    px[0, 0, 0] = 0                          # no sample yet
    out = D.denoise(px)
    assert np.allclose(out[5:8, 5:8, :3], 50.0, rtol=1e-3)
    assert np.all(out[0, 0] == 0)
    assert np.allclose(out[12:, 12:, :3], px[0, 12:, 12:, :3] / 8, rtol=2e-3)


def test_noise_is_reduced_and_edges_kept():
    """Noisy halves of two surfaces (normals apart): the filter lowers the noise within each half
    and does not mix the halves."""
    rng = np.random.default_rng(1)
    h, w, spp = 32, 32, 4
    px = flat_planes(h, w, spp)
    px[2, :, 16:, :3] = (1.0, 0.0, 0.0)      # the right half faces another way
    px[0, :, 16:, :3] = np.asarray((0.9, 0.1, 0.1), np.float32) * spp
    noise = rng.gamma(2.0, 0.5, (h, w)).astype(np.float32)
    px[0, ..., :3] *= noise[..., None]
    l = D.luma(px[0, ..., :3] / spp / px[3, ..., :3])
    px[1, ..., 0] = l * spp
    px[1, ..., 1] = l * l * spp * 1.5
    out = D.denoise(px)
    noisy = px[0, ..., :3] / spp
    assert out[:, 2:14, :3].std() < 0.5 * noisy[:, 2:14].std()
    assert out[:, :14, 0].mean() < 0.5 and out[:, 18:, 0].mean() > 0.6     # the halves stay apart


def test_reprojection_restatement_keeps_an_unmoved_image():
    """oracle/reproject_oracle.py: with the camera unmoved every pixel keeps its samples (capped at
    the history), and a pixel whose surface changed (another kind) keeps none."""
    from oracle import reproject_oracle as RP
    h = w = 16
    old = np.zeros((4, h, w, 4), np.float32)
    old[0, ..., :3], old[0, ..., 3] = 4.0, 8.0
    old[1, ..., 0], old[1, ..., 1] = 2.0, 1.0
    old[2, ..., 2], old[2, ..., 3] = -1.0, 100.0
    old[3, ..., :3] = 0.5
    cam = [[0, 0, 0], [-0.5, 0.5, 1], [1, 0, 0], [0, 1, 0]]
    new = old.copy()
    new[0] = new[1] = 0
    new[3, 5, 5, 3] = 1.0                        # a lamp now
    out = RP.reproject(old, new, cam, cam, 64)
    keep = np.ones((h, w), bool)
    keep[5, 5] = False
    assert np.allclose(out[0][keep], old[0][keep]) and np.allclose(out[1][keep][:, :2], old[1][keep][:, :2])
    assert np.all(out[0][5, 5] == 0)
    capped = RP.reproject(old, new, cam, cam, 3)
    assert np.allclose(capped[0][keep][:, 3], 3.0) and np.allclose(capped[0][keep][:, :3], 4.0 * 3 / 8)
