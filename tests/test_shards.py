# SPDX-License-Identifier: Apache-2.0
"""Subtree sharding (bpb200_compress_device_shard): with 2^k shards every
shard runs routing levels 0..k-1 in full and only its own subtree below, and
the byte-wise sum of the shards' blobs must be the whole blob.

On one GPU the shards of a permutation run one after another (they never
wait on each other), each into its own blob; the sum must equal the plain
call's bytes and the shards must set disjoint bits.  The combination step
of a multi-GPU run (combine_shards, a SUM reduce) is checked with two gloo
ranks on the CPU against the oracle's blob split into two disjoint parts.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from helpers import b200_format


@pytest.mark.gpu
@pytest.mark.parametrize("n,dtype,kind,kw", [
    (1 << 18, np.uint32, 0, dict()),
    (100_003, np.uint64, 1, dict(middle_group_log2=4, middle_placement=2)),
    ((1 << 20) + 5, np.uint32, 0, dict(middle_group_log2=3, middle_placement=1,
                                       input_clusters=[2, 9, 7], output_clusters=[18])),
    ((1 << 23) + 4097, np.uint64, 0, dict(middle_group_log2=5, middle_placement=2)),
])
def test_shards_sum_to_the_plain_blob(gpu, n, dtype, kind, kw):
    perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0x5A + n, n, dtype)
    fmt = b200_format(gpu, kw)
    want = gpu.compress(perm, gpu.CompressOptions(format=fmt))
    size = len(want)
    width = perm.dtype.itemsize
    d_in = torch.from_numpy(perm.view(np.int64 if width == 8 else np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for shards in (2, 4, 8):
        total = torch.zeros(size, dtype=torch.int32, device="cuda")
        seen = torch.zeros(size, dtype=torch.uint8, device="cuda")
        for shard in range(shards):
            d_blob = torch.full(((size + 3) // 4 * 4,), 0xC3, dtype=torch.uint8, device="cuda")
            gpu.compress_device_shard(d_in.data_ptr(), n, width, d_blob.data_ptr(), size, shard,
                                      shards, fmt, stream)
            part = d_blob[:size]
            assert int((seen & part).count_nonzero()) == 0, (shards, shard)  # disjoint bits
            seen |= part
            total += part.to(torch.int32)
        torch.cuda.synchronize()
        assert int(total.max()) <= 255
        assert total.to(torch.uint8).cpu().numpy().tobytes() == want, shards


@pytest.mark.gpu
def test_shard_arguments_are_checked(gpu):
    n = 1 << 16
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 3, n)
    size = gpu.encoded_size(n)
    d_in = torch.from_numpy(perm.view(np.int32)).cuda()
    d_blob = torch.zeros((size + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError, match="power of two"):
        gpu.compress_device_shard(d_in.data_ptr(), n, 4, d_blob.data_ptr(), size, 0, 3)
    with pytest.raises(ValueError, match="power of two"):
        gpu.compress_device_shard(d_in.data_ptr(), n, 4, d_blob.data_ptr(), size, 4, 4)
    with pytest.raises(ValueError, match="too small"):
        gpu.compress_device_shard(d_in.data_ptr(), n, 4, d_blob.data_ptr(), size, 0, 64)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _combine_rank(rank, world, port, parts, want, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import benes_perm_b200 as bp
        blob = torch.from_numpy(np.frombuffer(parts[rank], dtype=np.uint8).copy())
        bp.combine_shards(blob)
        if rank == 0:
            out.put(blob.numpy().tobytes() == want)
    finally:
        dist.destroy_process_group()


def test_combine_shards_gloo(oracle):
    # the oracle's blob split into two byte-disjoint-bit halves, summed back
    perm = np.random.default_rng(5).permutation(20000).astype(np.uint32)
    want = oracle.compress(perm)
    full = np.frombuffer(want, dtype=np.uint8)
    mask = np.random.default_rng(6).integers(0, 256, full.size).astype(np.uint8)
    parts = [(full & mask).tobytes(), (full & ~mask).tobytes()]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_combine_rank, args=(r, 2, port, parts, want, out))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out.get(timeout=10) is True
