"""The multi-GPU sample split of one image (render.trace_split): the ranks' sample ranges cover
[0, spp) once each, and after the sum all-reduce every rank holds the image of all samples. Run as
gloo ranks on the CPU with a stand-in scene whose samples are known values; on GPUs the same code
runs lrc_trace on each rank's range and the all-reduce over NCCL."""
import os
import socket
import types

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from little_renderer_b200.render import sample_range, trace_split


def test_ranges_cover_every_sample_once():
    for world in (1, 2, 3, 4, 8):
        for spp in (0, 1, 2, 7, 16, 33):
            got = []
            for r in range(world):
                s0, n = sample_range(r, world, spp)
                got.extend(range(s0, s0 + n))
            assert got == list(range(spp)), (world, spp)
    with pytest.raises(ValueError):
        sample_range(2, 2, 4)


class FakeScene:
    """trace_device adds sample s's value (s + 1) x (pixel index + 1) to every pixel of the tensor."""

    def __init__(self, t):
        self.t = t

    def trace_device(self, params, n, ptr, spp0=0):
        assert ptr == self.t.data_ptr()
        pix = torch.arange(self.t.shape[0] * self.t.shape[1], dtype=torch.float32).reshape(self.t.shape[:2]) + 1
        for s in range(spp0, spp0 + n):
            self.t[..., 0] += (s + 1) * pix
            self.t[..., 3] += 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, spp, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = torch.zeros(3, 5, 4)
        share = trace_split(FakeScene(t), types.SimpleNamespace(exact=0), spp, t, dist)
        out[rank] = (share, t.clone())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spp", [7, 1])
def test_split_image_is_every_sample(spp):
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), spp, out), nprocs=world, join=True)
    pix = torch.arange(15, dtype=torch.float32).reshape(3, 5) + 1
    want0 = sum(s + 1 for s in range(spp)) * pix
    for r in range(world):
        share, t = out[r]
        assert share == sample_range(r, world, spp)
        assert torch.equal(t[..., 0], want0) and torch.all(t[..., 3] == spp)
    assert torch.equal(out[0][1], out[1][1])


def test_exact_mode_is_not_split():
    class OneRank:
        def get_world_size(self, group=None):
            return 2

        def get_rank(self, group=None):
            return 0
    with pytest.raises(ValueError):
        trace_split(FakeScene(torch.zeros(1, 1, 4)), types.SimpleNamespace(exact=1), 4, torch.zeros(1, 1, 4),
                    OneRank())
