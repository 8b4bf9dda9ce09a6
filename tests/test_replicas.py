"""The multi-GPU form is replicas only (no exchange step): each rank runs the whole path on
its own GPU and the bench reports the units all ranks processed over the slowest rank's
device time.  These CPU tests run that reduction on a world-size-2 gloo process group."""
import os
import socket
from datetime import timedelta

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    import bench
    slowest = bench.max_over_ranks(10.0 * (rank + 1), ws)      # rank r timed 10 (r+1) ms
    value = bench.replica_value(1_000_000, 5, slowest, ws)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, slowest, value))


def test_max_over_ranks_single_rank():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_value(2_000_000, 10, 20.0, 1) == pytest.approx(1000.0)


def test_replicas_gloo_world_size_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get() for _ in range(2))
    # both ranks see the slowest rank's 20 ms; the job value counts both ranks' units
    assert [r[1] for r in res] == [20.0, 20.0]
    assert res[0][2] == pytest.approx(2 * 1_000_000 * 5 / 20e-3 / 1e6)
    assert res[0][2] == res[1][2]
