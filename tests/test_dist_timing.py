"""The multi-rank timing logic of bench.py on CPU ranks (gloo, world size 2).

Every rank renders its own frames (replicas, no collective on the render
data); the only collectives are the barriers around the timed region and the
reductions that turn per-rank times into the whole-job figure: the units all
ranks processed over the slowest rank's time.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, local = bench.dist_env()
    d = bench.Dist(ws, r, local, backend="gloo")
    d.barrier()
    # rank k "rendered" 100 * (k + 1) samples in (k + 1) seconds
    units, secs = 100.0 * (rank + 1), float(rank + 1)
    out[rank] = (d.max(secs), d.sum(units), d.job_rate(units, secs))
    d.barrier()
    d.close()


@pytest.mark.timeout(120)
def test_two_rank_job_rate_is_sum_over_max():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        mx, total, rate = res[rank]
        assert mx == 2.0
        assert total == 300.0
        assert rate == 150.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(1, 0, 0, backend="gloo")
    assert d.pg is None
    assert d.job_rate(10.0, 4.0) == 2.5
    d.close()
