"""The multi-GPU mode of bench.py runs independent replicas (no collective on the data path); the
only cross-rank operations are the barrier and the max over ranks of the device time.  Checked here
as two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 10.0 + 5.0 * rank          # per-rank device time of K steps
    ms_max = bench.reduce_max(ms, dist, "cpu")
    rate = bench.whole_job_rate(world, 1000, 4, ms_max)
    dist.barrier()
    out.put((rank, ms_max, rate))
    dist.destroy_process_group()


def test_replica_reduction_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms_max, rate in res:
        assert ms_max == 15.0                       # max over ranks, on every rank
        assert rate == pytest.approx(2 * 1000 * 4 / 0.015)


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.reduce_max(3.5, None, "cpu") == 3.5
