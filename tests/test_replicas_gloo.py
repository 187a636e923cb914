"""Multi-GPU is replicas only: every rank advances an independent copy of the
grid and bench.py reports the slowest rank's time and the summed work.  The
reduction runs here as two gloo ranks on the CPU."""
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


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    # rank r: 100 + 10 r ms for (r + 1) * 1000 zone-updates
    t, w = bench.replica_totals(100.0 + 10.0 * rank, (rank + 1) * 1000, world, "cpu")
    t1, w1 = bench.replica_totals(5.0, 7, 1, "cpu")          # world size 1: unchanged
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t, w, t1, w1))


def test_replica_totals_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, w, t1, w1 in out:
        assert t == pytest.approx(110.0)      # the slowest rank's time
        assert w == pytest.approx(3000.0)     # the sum of the work
        assert (t1, w1) == (5.0, 7)
