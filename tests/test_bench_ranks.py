"""bench.py's multi-rank plumbing (one process per GPU under torchrun, replica
runs, time reduced as the max over ranks) exercised with two gloo ranks on
the CPU: the same functions, a CPU backend."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.init_ranks(world, rank, backend="gloo", timeout_s=30)
    times = [3.0, 5.0]
    result = (bench.reduce_over_ranks(dist, times[rank], "max", "cpu"),
              bench.reduce_over_ranks(dist, times[rank], "min", "cpu"),
              bench.reduce_over_ranks(dist, times[rank], "sum", "cpu"))
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, result))


def test_two_gloo_ranks_reduce_like_the_bench():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0] == results[1] == (5.0, 3.0, 8.0)


def test_one_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.init_ranks(1, 0) is None
    assert bench.reduce_over_ranks(None, 2.5, "max") == 2.5
