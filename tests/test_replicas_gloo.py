# SPDX-License-Identifier: Apache-2.0
"""The multi-GPU harness of bench.py on CPU: two gloo ranks.

With N GPUs every rank compresses its own permutation (the compress path does
not shard), the job time is the slowest rank's, and the whole-job value is
all ranks' entries over that time.  These tests run the same helpers bench.py
uses, with gloo on CPU tensors instead of NCCL on CUDA ones.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, seconds, out):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        job = bench.max_over_ranks(seconds[rank], dist, "cpu")
        value = bench.replica_throughput(1 << 20, 3, world, job)
        out.put((rank, job, value, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("seconds", [(1.5, 2.5), (3.0, 0.5)])
def test_job_time_is_the_slowest_rank(seconds):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, seconds, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    slowest = max(seconds)
    assert [r[1] for r in results] == [slowest, slowest]
    assert all(r[2] == (1 << 20) * 3 * 2 / slowest for r in results)
    assert results[0][3] != results[1][3]  # replicas compress different permutations


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(1.25, None, "cpu") == 1.25
    assert bench.replica_throughput(1 << 30, 5, 1, 5.0) == float(1 << 30)
