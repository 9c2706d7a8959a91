"""Host logic of one view split across GPUs, on CPU ranks (gloo).

Each rank renders a contiguous range of every pixel's samples
(`sample_range`) and the ranks' films are summed in place (`sum_films`, an
all-reduce; NCCL over NVLink for device films).  Here the films are CPU
tensors standing in for the device films; the GPU side (ranges adding up to
the full frame) is tested in test_gpu_split.py.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from crystalgraphics_b200 import backend as B  # noqa: E402


def test_sample_ranges_partition_every_pixel_s_samples():
    for spp in (1, 2, 3, 7, 16, 64, 1000):
        for world in range(1, 10):
            ranges = [B.sample_range(spp, r, world) for r in range(world)]
            assert ranges[0][0] == 0
            for (b0, c0), (b1, _) in zip(ranges, ranges[1:]):
                assert b0 + c0 == b1
            assert sum(c for _, c in ranges) == spp
            assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from crystalgraphics_b200 import backend as Bk
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    spp, H, W = 7, 5, 6
    begin, count = Bk.sample_range(spp, rank, world)
    # this rank's share: per pixel, the sum of its samples' terms / spp, with
    # sample s of pixel p contributing (p + 1) * (s + 1)
    pix = torch.arange(H * W, dtype=torch.float32).reshape(H, W, 1) + 1.0
    share = sum((s + 1.0) for s in range(begin, begin + count)) / spp
    film = torch.cat([pix * share, pix * share * 2.0, pix * share * 3.0,
                      torch.zeros(H, W, 1)], dim=2).contiguous()
    Bk.sum_films(film)
    out[rank] = film.numpy().tolist()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
@pytest.mark.parametrize("world", [2, 3])
def test_ranks_sum_their_shares_into_the_full_film(world):
    import numpy as np
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    spp, H, W = 7, 5, 6
    pix = np.arange(H * W, dtype=np.float32).reshape(H, W) + 1.0
    full = pix * sum(s + 1.0 for s in range(spp)) / spp
    for rank in range(world):
        film = np.array(res[rank], dtype=np.float32)
        np.testing.assert_allclose(film[..., 0], full, rtol=1e-6)
        np.testing.assert_allclose(film[..., 1], 2 * full, rtol=1e-6)
        np.testing.assert_allclose(film[..., 2], 3 * full, rtol=1e-6)
        assert not film[..., 3].any()
