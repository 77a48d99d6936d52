"""The multi-GPU plumbing with two gloo ranks on CPU: timings reported as the slowest rank's,
whole-job throughput over all ranks' units, and the ensemble partition balanced by size."""
import os
import socket

import torch.multiprocessing as mp

from meeuuw_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    n = replicas.init("gloo", timeout_s=60)
    assert n == world
    ms = 100.0 + 50.0 * rank                  # rank 1 is the slowest
    replicas.barrier()
    mx = replicas.max_over_ranks(ms)
    units = 8 * (rank + 1)                    # ranks processed 8 and 16 units
    thr = replicas.throughput(units, mx)
    out[rank] = (mx, thr)
    replicas.finalize()


def test_two_gloo_ranks_timing_and_throughput():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        mx, thr = out[r]
        assert mx == 150.0                    # the slowest rank's time on every rank
        assert abs(thr - 24 / 0.150) < 1e-9   # all ranks' units over that time


def test_partition_balances_element_counts():
    sizes = [64 * 64, 192 * 192, 100 * 100, 150 * 150, 80 * 80, 180 * 180, 120 * 120, 70 * 70]
    parts = replicas.partition(sizes, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)      # LPT bound
    assert replicas.partition(sizes, 1) == [list(range(len(sizes)))]
    assert replicas.partition([5], 2) == [[0], []]
