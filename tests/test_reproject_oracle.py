"""CPU checks of the temporal gradients' restatement (oracle/reproject_oracle.py: gmatch, gfilter
and main's history, trace_reproject.wgsl) on synthetic planes: the history formula's values, the
filter's normalisation and reach, gmatch on an unmoved camera (each tile's gradient pixel is its
own old pixel) and its sample number across the 24-bit wrap. The GPU kernels are checked against
the same restatement in test_reproject_gpu.py."""
import numpy as np
import pytest

from oracle import reproject_oracle as RP

F = np.float32


def camera():
    """(origin, upper_left, horizontal, vertical): the eye at 0 looking down -z, a 90-degree view."""
    return [[0, 0, 0], [-1, 1, -1], [2, 0, 0], [0, 2, 0]]


def wall_planes(W, H, depth=5.0, samples=4.0, last_tag=16.0):
    """4 planes of a wall at z = -depth seen from camera(): plane 0 samples, plane 1 moments and the
    last sample (its value 0.5, its number tag), plane 2 the normal (+z) and distance, plane 3 a
    grey albedo and kind 0 of object 0."""
    o, ul, h, v = (np.asarray(a, np.float32) for a in camera())
    y, x = np.mgrid[0:H, 0:W].astype(np.float32)
    d = ul + h * ((x + F(0.5)) / F(W))[..., None] - v * ((y + F(0.5)) / F(H))[..., None] - o
    d = d / np.sqrt((d * d).sum(-1, keepdims=True))
    t = F(depth) / np.abs(d[..., 2])
    pl = np.zeros((4, H, W, 4), np.float32)
    pl[0] = (1.0, 1.0, 1.0, samples)
    pl[1] = (2.0, 1.5, 0.5, last_tag)
    pl[2][..., 2] = 1.0
    pl[2][..., 3] = t
    pl[3] = (0.5, 0.5, 0.5, 4.0)
    return pl


def test_history_from_lambda():
    """floor((1 - lambda) / lambda + 1/2) samples' worth, at most history_max; the fallback without
    a lambda; an edit's lambda counts 4 times and what is not a surface keeps the fallback."""
    cur = np.zeros((4, 8, 8, 4), np.float32)
    cur[3][..., 3] = 4.0                                  # kind 0 (a surface) of object 0
    cur[3][4:, 4:, 3] = 5.0                               # kind 1 (a lamp) in the last tile
    lam = np.array([[0.0, 1.0], [0.5, -1.0]], np.float32)
    h = RP.grad_history(lam, cur, 32, 8)
    assert h[0, 0] == 32 and h[0, 4] == 0 and h[4, 0] == 1 and h[4, 4] == 8
    lam_e = np.array([[0.05, 0.5], [0.0, 0.0]], np.float32)
    he = RP.grad_history(lam_e, cur, 32, 8, edit=True)
    assert he[0, 0] == 4 and he[0, 4] == 0 and he[4, 0] == 32 and he[4, 4] == 8


def test_filter_normalises_and_reaches_seven_tiles():
    W = H = 64
    cur = wall_planes(W, H)
    th, tw = H // 4, W // 4
    const = np.full((th, tw), 0.3, np.float32)
    assert np.allclose(RP.gfilter(const, cur), 0.3, rtol=1e-6)
    assert np.all(RP.gfilter(np.full((th, tw), -1, np.float32), cur) == -1)
    one = np.full((th, tw), -1, np.float32)
    one[8, 8] = 0.5
    out = RP.gfilter(one, cur)
    reach = np.argwhere(out >= 0)
    # passes 1, 2 and 4 tiles apart: a lambda reaches up to 7 tiles away in each direction
    assert np.abs(reach - 8).max() == 7
    assert np.allclose(out[out >= 0], 0.5, rtol=1e-6)


def test_gmatch_unmoved_picks_the_same_pixel():
    W = H = 16
    pl = wall_planes(W, H)
    m = RP.gmatch(pl, pl, camera(), camera(), 16)
    assert np.all(m["o"] >= 0) and np.array_equal(m["k"], m["o"])
    assert np.all(m["kk"] == 15) and np.all(m["l"] == 0.5)
    assert np.abs(m["d"]).max() < 1e-3
    # the tiles' pixels start from a point that moves with the next sample number
    m2 = RP.gmatch(pl, pl, camera(), camera(), 17)
    assert not np.array_equal(m["k"], m2["k"])


def test_gmatch_sample_number_across_the_24_bit_wrap():
    """The old sample's number from its low 24 bits and the next number's high bits: 0xFFFFFF
    (kept as 2^24) before 0x1000001 is 0xFFFFFF, not 0x1FFFFFF."""
    W = H = 8
    pl = wall_planes(W, H, last_tag=float(0xFFFFFF + 1))
    m = RP.gmatch(pl, pl, camera(), camera(), 0x1000001)
    assert np.all(m["kk"] == 0xFFFFFF)


@pytest.mark.parametrize("what", ["no_samples", "other_object", "far"])
def test_gmatch_needs_the_same_surface(what):
    W = H = 8
    old = wall_planes(W, H)
    new = wall_planes(W, H)
    if what == "no_samples":
        old[1][..., 3] = 0.0                              # no last sample recorded
    elif what == "other_object":
        old[3][..., 3] = 8.0                              # kind 0 of object 1
    else:
        new = wall_planes(W, H, depth=6.0)                # the surface moved back 20 %
    m = RP.gmatch(old, new, camera(), camera(), 16)
    assert np.all(m["o"] == -1)
