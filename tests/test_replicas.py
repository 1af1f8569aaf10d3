"""bench.py's multi-GPU path is replicas only: per-rank counts are summed and
per-rank device times maxed.  Checked with two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    counts, times = bench.aggregate_replicas([10.0 * (rank + 1), 1.0], [5.0 + rank, 2.0 - rank], dist, "cpu")
    out[rank] = (list(counts), list(times))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_with_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        counts, times = out[r]
        assert np.allclose(counts, [30.0, 2.0])
        assert np.allclose(times, [6.0, 2.0])


def test_single_process_passthrough():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    c, t = bench.aggregate_replicas([1, 2], [3, 4])
    assert list(c) == [1, 2] and list(t) == [3, 4]
