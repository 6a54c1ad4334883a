"""bench.py's multi-rank bookkeeping on two gloo ranks (CPU, 127.0.0.1): the max over ranks of
each timed interval, the whole-job throughput, and the size-balanced split of independent
instances that --batched uses under torchrun."""

import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mx = bench.max_over_ranks(1.5 + rank)
        thr = bench.whole_job_throughput(3, 100.0 * (rank + 1))  # ms: rank 1 is the slowest
        dist.barrier()
        out.put((rank, mx, thr))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, thr in res:
        assert mx == 2.5                      # max over ranks, seen by every rank
        assert abs(thr - 2 * 3 / 0.2) < 1e-12  # 2 ranks x 3 units in the slowest rank's 200 ms


def test_single_process_needs_no_group():
    assert not dist.is_initialized()
    assert bench.max_over_ranks(4.0) == 4.0
    assert bench.whole_job_throughput(5, 500.0) == 10.0


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_by_size_covers_and_balances(world):
    import numpy as np

    sizes = np.random.default_rng(1).uniform(30e3, 600e3, 128)
    parts = bench.partition_by_size(list(sizes), world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(128))
    loads = [sizes[p].sum() for p in parts]
    # greedy largest-first stays within one largest instance of the mean
    assert max(loads) - min(loads) <= sizes.max() + 1e-6
