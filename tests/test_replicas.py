"""Replica timing of bench.py --gpus N on CPU: two gloo ranks report
different times; every rank gets the slowest, and the throughput counts the
work of all ranks over that time."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.max_over_ranks(dist, 10.0 * (rank + 1), "cpu")
    out.put((rank, t, bench.replica_throughput(4, world, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    assert all(abs(r[2] - 4 * 2 / 0.02) < 1e-9 for r in res)
