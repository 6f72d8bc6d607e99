"""The multi-GPU form of bench.py is replicas only: every rank runs its own
mesh and the job time is the maximum over ranks. This checks that reduction
and the rank environment with two gloo processes on the CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, l = bench.dist_env()
        ms = 10.0 + 5.0 * rank  # per-rank timed-region milliseconds
        out[rank] = (r, w, l, bench.reduce_max(ms, w, torch.device("cpu")))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank, (r, w, l, mx) in res.items():
        assert (r, w, l) == (rank, world, rank)
        assert mx == 15.0


def test_reduce_max_single_rank():
    import bench
    assert bench.reduce_max(3.5, 1) == 3.5
