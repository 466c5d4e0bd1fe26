"""Replica scaling of bench.py on CPU: world_size 2 over gloo (127.0.0.1).

A sweep is a sequential chain of dependent site solves, so N GPUs run N
independent replicas with no data-path collective; the only collective is the
max-over-ranks of the timed region.  Each rank reports a different time; every
rank must see the slowest, the whole-job rate counts all ranks' sweeps over it,
and the replicas start from different seeds.
"""
import importlib.util
import os
import socket

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        seconds = 2.0 + rank            # rank 1 is the slowest
        t = b.max_over_ranks(seconds, True, "cpu")
        q.put((rank, t, b.replica_throughput(3, world, t), b.replica_seed(2024, rank)))
    finally:
        td.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [3.0, 3.0]
    assert [r[2] for r in res] == [2.0, 2.0]          # 3 sweeps x 2 ranks / 3 s
    assert res[0][3] != res[1][3]


def test_single_rank_needs_no_collective():
    b = _bench()
    assert b.max_over_ranks(1.5, False, "cpu") == 1.5
    assert b.replica_throughput(2, 1, 4.0) == 0.5
