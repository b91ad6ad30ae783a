# SPDX-License-Identifier: Apache-2.0
"""Batched and serving forms: every blob must be byte-identical to the plain
per-request call on the same input, whether the request ran alone or mixed
with others (sizes, widths and formats drawn like the mixed-stream
configuration, scaled down), and the replayed 240-request stream must give
the reference's own bytes (digests made by tests/golden/make_digests.py with
the reference's portable encoder)."""
import concurrent.futures as cf
import hashlib

import numpy as np
import pytest

import bench
from helpers import b200_format, load_digests, oracle_format

pytestmark = pytest.mark.gpu


def _mixed(gpu, count, max_log2, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(2 ** rng.uniform(4, max_log2)))
        kind = int(rng.integers(0, 2))
        dtype = np.uint32 if rng.integers(0, 2) == 0 else np.uint64
        kw = dict(middle_group_log2=int(rng.choice([4, 5])),
                  middle_placement=int(rng.integers(0, 3)))
        perm = gpu.fill_permutation(gpu.PermutationKind(kind), seed * 100003 + i, n, dtype)
        out.append((perm, kw))
    return out


def test_batch_device_matches_plain(gpu):
    torch = pytest.importorskip("torch")
    reqs = _mixed(gpu, 60, 17, 1)
    items, keep, expected = [], [], []
    for perm, kw in reqs:
        fmt = b200_format(gpu, kw)
        n = perm.size
        size = gpu.encoded_size(n, fmt)
        width = perm.dtype.itemsize
        d_in = torch.from_numpy(perm.view(np.int64 if width == 8 else np.int32)).cuda()
        d_blob = torch.full(((size + 3) // 4 * 4,), 0x5A, dtype=torch.uint8, device="cuda")
        keep.append((d_in, d_blob, size))
        items.append((d_in.data_ptr(), n, width, fmt, d_blob.data_ptr(), size))
        expected.append(gpu.compress(perm, gpu.CompressOptions(format=fmt)))
    statuses, launches = gpu.compress_batch_device(items)
    assert all(s == 0 for s in statuses)
    assert launches > 0
    torch.cuda.synchronize()
    for (d_in, d_blob, size), want in zip(keep, expected):
        assert d_blob[:size].cpu().numpy().tobytes() == want


def test_batch_small_only_single_launch(gpu, oracle):
    torch = pytest.importorskip("torch")
    items, keep, perms = [], [], []
    for i in range(200):
        n = 1 + (i * 37) % 8192
        perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 900 + i, n)
        fmt = gpu.FormatOptions()
        size = gpu.encoded_size(n, fmt)
        d_in = torch.from_numpy(perm.view(np.int32)).cuda()
        d_blob = torch.empty(((size + 3) // 4 * 4,), dtype=torch.uint8, device="cuda")
        keep.append((d_blob, size))
        perms.append(perm)
        items.append((d_in.data_ptr(), n, 4, fmt, d_blob.data_ptr(), size))
        keep.append(d_in)
    statuses, launches = gpu.compress_batch_device(items)
    assert launches == 1  # every single-tile permutation in one launch
    blobs = [k for k in keep if isinstance(k, tuple)]
    for (d_blob, size), perm in zip(blobs, perms):
        assert d_blob[:size].cpu().numpy().tobytes() == oracle.compress(perm)


def test_server_mixed_equals_alone(gpu):
    reqs = _mixed(gpu, 120, 19, 2)
    alone = [hashlib.sha256(gpu.compress(p, gpu.CompressOptions(format=b200_format(gpu, kw))))
             .hexdigest() for p, kw in reqs]
    with gpu.Server(hbm_budget_bytes=2 * 10**9, max_batch=64, workers=3) as server:
        # submit from several threads at once so requests overlap on the device
        def submit(item):
            perm, kw = item
            return server.submit(perm, gpu.CompressOptions(format=b200_format(gpu, kw)))
        with cf.ThreadPoolExecutor(4) as pool:
            tickets = list(pool.map(submit, reqs))
        results = [server.wait(t) for t in tickets]
        stats = server.stats()
    for (blob, latency), want in zip(results, alone):
        assert hashlib.sha256(blob).hexdigest() == want
        assert latency > 0
    assert stats["completed"] == len(reqs)
    assert stats["p99_seconds"] >= stats["p50_seconds"] > 0


def test_server_rejects_bad_request_without_harming_others(gpu, oracle):
    good = gpu.fill_permutation(gpu.PermutationKind.uniform, 3, 5000)
    bad = good.copy()
    bad[10] = bad[11]
    big = gpu.fill_permutation(gpu.PermutationKind.single_cycle, 4, 70000)
    with gpu.Server(hbm_budget_bytes=10**9) as server:
        t1 = server.submit(good)
        t2 = server.submit(bad)
        t3 = server.submit(big)
        assert server.wait(t1)[0] == oracle.compress(good)
        with pytest.raises(ValueError):
            server.wait(t2)
        assert server.wait(t3)[0] == oracle.compress(big)


@pytest.mark.gpu
def test_concurrent_host_calls_are_independent(gpu):
    """The reference's compress is reentrant (one stream per call,
    src/cuda/benes_cuda.cu:1192); calls from several host threads at once,
    with inputs of different sizes and widths, give the bytes of the same
    calls made one at a time."""
    sizes = [(1 << 22) + 3, 70001, (1 << 20) + 17, 5000, (1 << 21), 3 * (1 << 19) + 1]
    perms = [gpu.fill_permutation(gpu.PermutationKind.uniform, 40 + i, n,
                                  np.uint64 if i % 2 else np.uint32)
             for i, n in enumerate(sizes)]
    alone = [gpu.compress(p) for p in perms]
    with cf.ThreadPoolExecutor(len(perms)) as pool:
        for _ in range(2):
            assert list(pool.map(gpu.compress, perms)) == alone


@pytest.mark.gpu
def test_shrinking_then_growing_sizes(gpu, oracle):
    """Workspaces grow geometrically and are reused: a large call, then small
    ones, then a larger one must all stay byte-exact."""
    for i, n in enumerate([1 << 21, 777, 40000, (1 << 22) + 5, 12345]):
        perm = np.random.default_rng(200 + i).permutation(n)
        if n <= 40000:
            assert gpu.compress(perm.astype(np.uint64)) == oracle.compress(perm.astype(np.uint64))
        else:
            assert gpu.compress(perm.astype(np.uint32)) == gpu.compress(perm.astype(np.uint64))


def _stream240(gpu):
    d = load_digests()["stream240"]
    specs = bench.serving_specs(d["requests"], d["max_log2"], d["seed"])
    assert len(specs) == len(d["sha256_128"]) >= 200
    reqs = []
    for i, (n, kind, dtype, m, placement) in enumerate(specs):
        perm = gpu.fill_permutation(gpu.PermutationKind(kind), d["seed"] + i, n, dtype)
        fmt = gpu.FormatOptions(middle_group_log2=m, middle_placement=gpu.MiddlePlacement(placement))
        reqs.append((perm, fmt))
    return reqs, d["sha256_128"]


def _digest(blob):
    return hashlib.sha256(blob).hexdigest()[:32]


def test_stream240_plain_batch_and_server_match_reference(gpu):
    """The 240-request mixed stream (sizes up to 2^21, uint32 and uint64,
    m in {4, 5}, every placement, Fisher-Yates and Sattolo) through the plain
    host call, the batched device call and the serving loop: every blob
    equals the reference's."""
    torch = pytest.importorskip("torch")
    reqs, want = _stream240(gpu)
    kinds = {(p.dtype.itemsize, f.middle_group_log2, int(f.middle_placement)) for p, f in reqs}
    assert len(kinds) == 12  # both widths x both m x three placements
    assert max(p.size for p, _ in reqs) > (1 << 20)
    for (perm, fmt), w in zip(reqs, want):
        assert _digest(gpu.compress(perm, gpu.CompressOptions(format=fmt))) == w
    items, keep = [], []
    for perm, fmt in reqs:
        n, width = perm.size, perm.dtype.itemsize
        size = gpu.encoded_size(n, fmt)
        d_in = torch.from_numpy(perm.view(np.int64 if width == 8 else np.int32)).cuda()
        d_blob = torch.full(((size + 3) // 4 * 4,), 0xA5, dtype=torch.uint8, device="cuda")
        keep.append((d_in, d_blob, size))
        items.append((d_in.data_ptr(), n, width, fmt, d_blob.data_ptr(), size))
    statuses, _ = gpu.compress_batch_device(items)
    assert all(s == 0 for s in statuses)
    torch.cuda.synchronize()
    for (_, d_blob, size), w in zip(keep, want):
        assert _digest(d_blob[:size].cpu().numpy().tobytes()) == w
    del keep, items
    with gpu.Server(hbm_budget_bytes=8 * 10**9, max_batch=64, workers=4) as server:
        tickets = [server.submit(p, gpu.CompressOptions(format=f)) for p, f in reqs]
        for t, w in zip(tickets, want):
            blob, latency = server.wait(t)
            assert _digest(blob) == w and latency > 0


def _device_items(gpu, torch, reqs):
    items, keep = [], []
    for perm, fmt in reqs:
        n, width = perm.size, perm.dtype.itemsize
        size = gpu.encoded_size(n, fmt)
        d_in = torch.from_numpy(perm.view(np.int64 if width == 8 else np.int32)).cuda()
        d_blob = torch.full(((size + 3) // 4 * 4,), 0x3C, dtype=torch.uint8, device="cuda")
        keep.append((d_in, d_blob, size))
        items.append((d_in.data_ptr(), n, width, fmt, d_blob.data_ptr(), size))
    return items, keep


def test_batch_groups_few_launches_and_union_find(gpu):
    """Mid-size requests (above one tile, up to the walk limit) are encoded
    together, level by level, by the batched level kernels: far fewer
    launches than one level chain per request, and the same bytes as the
    plain call, with the orbit walks and with union-find forced."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(77)
    reqs = []
    for i in range(48):
        n = int(rng.integers(8193, 1 << 18))
        dtype = np.uint64 if i % 3 == 0 else np.uint32
        perm = gpu.fill_permutation(gpu.PermutationKind(i % 2), 500 + i, n, dtype)
        fmt = gpu.FormatOptions(middle_group_log2=4 + i % 2,
                                middle_placement=gpu.MiddlePlacement(i % 3))
        reqs.append((perm, fmt))
    for uf in (False, True):
        gpu.set_union_find_only(uf)
        try:
            want = [gpu.compress(p, gpu.CompressOptions(format=f)) for p, f in reqs]
            items, keep = _device_items(gpu, torch, reqs)
            statuses, launches = gpu.compress_batch_device(items)
            torch.cuda.synchronize()
        finally:
            gpu.set_union_find_only(False)
        assert statuses == [0] * len(reqs)
        assert launches < 4 * len(reqs), launches  # a level chain alone is ~50-100
        for (_, d_blob, size), w in zip(keep, want):
            assert d_blob[:size].cpu().numpy().tobytes() == w


def test_batch_group_member_with_duplicate(gpu, oracle):
    """A non-permutation inside a group fails alone: it reports
    invalid_argument and every other member keeps its exact bytes."""
    torch = pytest.importorskip("torch")
    reqs = []
    for i, n in enumerate((20000, 70001, 150000, 9000, 33333)):
        perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 900 + i, n)
        reqs.append((perm, gpu.FormatOptions()))
    bad = reqs[2][0].copy()
    bad[5] = bad[77]
    reqs[2] = (bad, reqs[2][1])
    items, keep = _device_items(gpu, torch, reqs)
    statuses, _ = gpu.compress_batch_device(items, raise_errors=False)
    torch.cuda.synchronize()
    assert statuses == [0, 0, 1, 0, 0]
    for k, ((_, d_blob, size), (perm, _)) in enumerate(zip(keep, reqs)):
        if k != 2:
            assert d_blob[:size].cpu().numpy().tobytes() == oracle.compress(perm)
