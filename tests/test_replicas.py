"""More than one GPU runs independent replicas of the Fock build (no data exchange): the
only multi-rank step is the bench's timing, the max over ranks of each rank's device time.
Checked here with two gloo ranks on the CPU."""
import os
import socket
import sys
from datetime import timedelta

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=ws,
                            timeout=timedelta(seconds=60))
    try:
        q.put((rank, bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert got == [(0, 20.0), (1, 20.0)]
    assert all(p.exitcode == 0 for p in procs)


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
