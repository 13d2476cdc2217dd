"""The replica path of bench.py (N > 1 processes, one per GPU, "replicas
only"): the cross-rank reductions, run as two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out):
    import datetime
    import sys
    from pathlib import Path
    import torch.distributed as dist
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = [10.0, 25.0][rank]          # rank 1 is the slow one
    units = [300.0, 100.0][rank]
    out[rank] = (bench.max_over_ranks(ms, dist, "cpu"),
                 bench.replica_throughput(units, ms / 1e3, dist, "cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reductions_two_gloo_ranks():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        mx, thr = out[r]
        assert mx == 25.0                     # the slowest rank's time
        assert thr == pytest.approx(400.0 / 0.025)  # all ranks' work / that time


def test_single_process_reductions_are_identity():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_throughput(10.0, 2.0) == 5.0
