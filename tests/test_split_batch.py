"""Host logic of batches and request streams spread over GPUs, on CPU ranks
(gloo): every rank computes the same assignment of views (partition_views)
and of requests (RequestRouter) from the same inputs, with no communication,
and the shares cover every view or request exactly once with balanced work.
The GPU side (a view's or request's film does not depend on its share) is in
test_gpu_split.py."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from crystalgraphics_b200 import backend as B  # noqa: E402
from crystalgraphics_b200 import scenes  # noqa: E402


def _samples(v):
    return v[2] * v[3] * v[4]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_views_covers_every_view_once_with_balanced_work(world):
    views = scenes.batch_views(256)
    parts = B.partition_views(views, world)
    assert len(parts) == world
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(views)))
    loads = [sum(_samples(views[k]) for k in p) for p in parts]
    # longest first to the least-loaded rank: within one view of each other
    assert max(loads) - min(loads) <= max(_samples(v) for v in views)
    assert B.partition_views(views, world) == parts   # deterministic


def test_request_router_balances_the_stream():
    stream = scenes.request_stream(200, 100.0)
    for world in (1, 2, 4):
        r = B.RequestRouter(world)
        owners = [r.route(w, h, spp) for _, _, _, _, w, h, spp, _ in stream]
        assert set(owners) <= set(range(world))
        biggest = max(w * h * spp for _, _, _, _, w, h, spp, _ in stream)
        assert max(r.load) - min(r.load) <= biggest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from crystalgraphics_b200 import backend as Bk
    from crystalgraphics_b200 import scenes as S
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    views = S.batch_views(64, seed=9)
    mine = Bk.partition_views(views, world)[rank]
    router = Bk.RequestRouter(world)
    stream = S.request_stream(64, 50.0, seed=10)
    routed = [k for k, (_, _, _, _, w, h, spp, _) in enumerate(stream)
              if router.route(w, h, spp) == rank]
    got = [None] * world
    dist.all_gather_object(got, (mine, routed))
    out[rank] = got
    dist.destroy_process_group()


@pytest.mark.timeout(120)
@pytest.mark.parametrize("world", [2, 3])
def test_ranks_agree_on_shares_without_communication(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    # each rank's own share, as every rank saw it
    for rank in range(world):
        assert res[rank] == res[0]
    views = sorted(k for mine, _ in res[0] for k in mine)
    reqs = sorted(k for _, routed in res[0] for k in routed)
    assert views == list(range(64))
    assert reqs == list(range(64))
