# SPDX-License-Identifier: Apache-2.0
"""Parity of the B200 backend with the reference's canonical bytes.

Every check calls the CUDA path through the C ABI (``bpb200_compress`` /
``bpb200_compress_device``) and compares against the committed golden
fixtures or the CPU oracle on the same seeded inputs; the bar is byte
equality.  Mirrors the reference's accelerated-backend tests
(tests/test_benes.cpp:141-266, 598-677).
"""
import hashlib
import itertools

import numpy as np
import pytest

from helpers import (b200_format, corpus_permutation, load_corpus, load_digests, load_goldens,
                     oracle_format, routing_depth)

pytestmark = pytest.mark.gpu


def test_reference_goldens(gpu):
    for g in load_goldens():
        perm = np.array(g["permutation"], dtype=np.uint32)
        assert gpu.compress(perm).hex() == g["blob_hex"], g["name"]
        assert gpu.compress(perm.astype(np.uint64)).hex() == g["blob_hex"], g["name"]


def test_corpus(gpu):
    for e in load_corpus():
        perm = corpus_permutation(gpu, e)
        opts = gpu.CompressOptions(format=b200_format(gpu, e["format"]))
        blob = gpu.compress(perm, opts)
        assert len(blob) == e["size"], (e["n"], e["name"])
        assert hashlib.sha256(blob).hexdigest() == e["sha256"], (e["n"], e["name"], e["kind"])


def test_exhaustive_small(gpu, oracle):
    # all permutations of up to 7 entries and a sample of 8 (test_benes.cpp:141-176)
    for n in range(1, 8):
        for p in itertools.permutations(range(n)):
            perm = np.array(p, dtype=np.uint32)
            assert gpu.compress(perm) == oracle.compress(perm), p
    rng = np.random.default_rng(8)
    for _ in range(300):
        perm = rng.permutation(8).astype(np.uint32)
        for m in (1, 2):
            for pl in (0, 1, 2):
                kw = dict(middle_group_log2=m, middle_placement=pl)
                assert gpu.compress(perm, gpu.CompressOptions(format=b200_format(gpu, kw))) == \
                    oracle.compress(perm, oracle_format(kw))


@pytest.mark.parametrize("n", [9, 15, 17, 30, 31, 33, 34, 47, 62, 63, 65, 66, 95, 96, 97, 126,
                               127, 129, 130, 255, 257, 511, 513, 1023, 1025, 4095, 4097, 8191,
                               8192, 8193, 16385, 40000, 131073])
def test_boundary_sizes(gpu, oracle, n):
    for kind in (0, 1, 3):
        perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0xC04FAC70 + n + kind, n)
        assert gpu.compress(perm) == oracle.compress(perm), (n, kind)


def test_uint64_canonical_parity(gpu, oracle):
    for n in (1, 2, 3, 31, 32, 33, 63, 65, 127, 129, 4097, 70001):
        perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 0x640000 + n, n)
        d = routing_depth(n, 4)
        kw = dict(middle_group_log2=4, input_clusters=[1] * d, output_clusters=[d] if d else [],
                  middle_placement=1 if n % 2 == 0 else 2)
        opts = gpu.CompressOptions(format=b200_format(gpu, kw))
        want = oracle.compress(perm, oracle_format(kw))
        assert gpu.compress(perm, opts) == want
        assert gpu.compress(perm.astype(np.uint64), opts) == want


def test_format_options(gpu, oracle):
    rng = np.random.default_rng(11)
    for n in (3, 7, 15, 17, 31, 33, 63, 65, 127, 129, 257, 4097, 9000, 70000):
        perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 0xF04A7000 + n, n)
        for m in (1, 2, 3, 4, 5):
            d = routing_depth(n, m)
            comp = []
            r = d
            while r:
                x = int(rng.integers(1, r + 1))
                comp.append(x)
                r -= x
            for pl in (0, 1, 2):
                for kw in (dict(middle_group_log2=m, middle_placement=pl),
                           dict(middle_group_log2=m, middle_placement=pl,
                                input_clusters=[1] * d, output_clusters=[d] if d else []),
                           dict(middle_group_log2=m, middle_placement=pl,
                                input_clusters=comp, output_clusters=comp[::-1])):
                    got = gpu.compress(perm, gpu.CompressOptions(format=b200_format(gpu, kw)))
                    assert got == oracle.compress(perm, oracle_format(kw)), (n, kw)


@pytest.mark.parametrize("union_find_only", [False, True, "fallback"])
def test_global_levels_both_colourings(gpu, oracle, union_find_only):
    # sizes that run several global levels (nodes above 8192 entries);
    # "fallback": the walks run, then every walk level is coloured by the
    # union-find fallback, whose roots that level sets up itself
    gpu.set_union_find_only(union_find_only)
    try:
        for n, kind in ((40000, 0), (65537, 1), (131072, 4), (100003, 2), (99999, 3)):
            perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0x600D + n, n)
            for kw in (dict(), dict(middle_group_log2=3, middle_placement=1)):
                got = gpu.compress(perm, gpu.CompressOptions(format=b200_format(gpu, kw)))
                assert got == oracle.compress(perm, oracle_format(kw)), (n, kind, kw)
    finally:
        gpu.set_union_find_only(False)


def test_partitioned_inverse_levels(gpu, oracle):
    # Nodes above 2^23 entries (the walk limit) take the partitioned inverse
    # (level_bucket + level_place, profile kind "place") and union-find
    # colouring (no "walk" launch on that level); smaller global nodes take
    # the orbit walks, with the inverse written by the parent's output pass
    # (no inverse launch at all below level 0).  n = 2^23 + 4097 puts level 0
    # above the limit and level 1 below it.
    n = (1 << 23) + 4097
    kw = dict(middle_group_log2=4, middle_placement=2)
    opts = gpu.CompressOptions(format=b200_format(gpu, kw))
    gpu.set_profiling(True)
    try:
        for kind, dtype in ((0, np.uint32), (1, np.uint64), (0, np.uint64), (1, np.uint32)):
            perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0xB1C + kind, n, dtype)
            got = gpu.compress(perm, opts)
            launches = gpu.last_profile_launches()
            place = {lvl for k, lvl, _ in launches if k == "place"}
            walk = {lvl for k, lvl, _ in launches if k == "walk"}
            plain = {lvl for k, lvl, _ in launches if k == "inverse"}
            assert place == {0} and 0 not in walk and 0 not in plain, (kind, launches[:8])
            assert 1 in walk and not plain and 1 not in place
            assert got == oracle.compress(perm, oracle_format(kw)), (kind, dtype)
    finally:
        gpu.set_profiling(False)
    # a repeated value at that size overfills one destination window of
    # level_bucket or leaves an inverse slot unwritten: invalid_argument
    for dtype in (np.uint32, np.uint64):
        bad = gpu.fill_permutation(gpu.PermutationKind.uniform, 5, n, dtype)
        bad[n // 3] = bad[n // 2]
        with pytest.raises(ValueError, match="every value"):
            gpu.compress(bad)
        clash = np.zeros(n, dtype=dtype)  # n > 2^23 records for window 0: it overfills
        with pytest.raises(ValueError, match="every value"):
            gpu.compress(clash)
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 6, n)
    assert gpu.compress(perm, opts) == oracle.compress(perm, oracle_format(kw))


def test_host_path_early_download(gpu, oracle):
    # On inputs whose first cluster groups end above the tile levels (here
    # 2^23 + 12345 entries: 20 or 19 routing levels, tiles from level 11),
    # the host entry point downloads the header and those groups' packets
    # while the lower levels run: on a copy stream into a pinned blob, through
    # the staging ring on a helper thread into a pageable one.  Both must
    # equal the device-resident path, and one format the oracle.
    import torch
    cases = [dict(middle_group_log2=4, middle_placement=0),
             dict(middle_group_log2=5, middle_placement=2),
             dict(middle_group_log2=4, middle_placement=1, input_clusters=[4, 7, 9],
                  output_clusters=[10, 10]),
             dict(middle_group_log2=5, middle_placement=0, input_clusters=[4, 7, 8],
                  output_clusters=[10, 9])]
    # 2^27 + 12345 entries: 16384 or 32768 tiles, launched in 8 parts, the blob's
    # finished clusters downloaded after each part
    cases.append(dict(middle_group_log2=5, middle_placement=2, n=(1 << 27) + 12345))
    cases.append(dict(middle_group_log2=4, middle_placement=0, n=(1 << 27) + 12345))
    for i, kw in enumerate(cases):
        kw = dict(kw)
        n = kw.pop("n", (1 << 23) + 12345)
        dtype = np.uint64 if i % 2 else np.uint32
        perm = gpu.fill_permutation(gpu.PermutationKind(i % 2), 0xE4 + i, n, dtype)
        fmt = b200_format(gpu, kw)
        size = gpu.encoded_size(n, fmt)
        w = np.dtype(dtype).itemsize
        d_in = torch.from_numpy(perm.view(np.int64 if w == 8 else np.int32)).cuda()
        d_blob = torch.empty((size + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        gpu.compress_device(d_in.data_ptr(), n, w, d_blob.data_ptr(), size, fmt, stream)
        torch.cuda.synchronize()
        want = d_blob[:size].cpu().numpy().tobytes()
        opts = gpu.CompressOptions(format=fmt)
        assert gpu.compress(perm, opts) == want, kw
        pinned = torch.zeros(size + 64, dtype=torch.uint8, pin_memory=True)
        pinned[size:] = 0xA5
        got = gpu.compress(perm, opts, out=pinned.numpy())
        assert bytes(got) == want, kw
        # bytes past the encoded size are left as they were
        assert bool((pinned[size:] == 0xA5).all()), kw
        if n > (1 << 25):
            # inputs above 2^25 entries are uploaded in parts that level 0
            # buckets as they arrive: from pageable memory (above), and from
            # pinned memory straight to the device
            held = torch.empty(n, dtype=torch.int64 if w == 8 else torch.int32,
                               pin_memory=True).numpy().view(dtype)
            held[:] = perm
            assert gpu.compress(held, opts) == want, kw
        if i == 2:
            assert want == oracle.compress(perm, oracle_format(kw)), kw


def test_host_path_narrowed_upload(gpu, oracle):
    # 64-bit host inputs of 4 MB and more cross PCIe as 32-bit values; a
    # value of 2^32 or more must still be reported as a non-permutation, and
    # a narrowed input must give the bytes of the 32-bit input.
    import torch
    n = (1 << 20) + 3
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 0x4A, n, np.uint64)
    kw = dict(middle_group_log2=4, middle_placement=2)
    opts = gpu.CompressOptions(format=b200_format(gpu, kw))
    want = oracle.compress(perm, oracle_format(kw))
    assert gpu.compress(perm, opts) == want
    assert gpu.compress(perm.astype(np.uint32), opts) == want
    pinned = torch.empty(n, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    pinned[:] = perm
    assert gpu.compress(pinned, opts) == want
    for bad_value in (1 << 32, (1 << 63) + 5, n):
        bad = perm.copy()
        bad[n // 2] = bad_value
        with pytest.raises(ValueError, match="every value"):
            gpu.compress(bad, opts)
    assert gpu.compress(perm, opts) == want
    # from 2^25 entries the narrowed upload overlaps level 0: a wide value
    # found while the encode already runs still fails the call
    big = (1 << 25) + 7
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 0x4B, big, np.uint64)
    good = gpu.compress(perm, opts)
    assert good == gpu.compress(perm.astype(np.uint32), opts)
    for at in (0, big // 3, big - 1):
        bad = perm.copy()
        bad[at] = 1 << 40
        with pytest.raises(ValueError, match="every value"):
            gpu.compress(bad, opts)
    assert gpu.compress(perm, opts) == good


def test_invalid_inputs_then_recovery(gpu, oracle):
    for bad in ([0, 1, 1], [0, 1, 3], [5, 0, 1, 2, 3, 4, 4]):
        for dt in (np.uint32, np.uint64):
            with pytest.raises(ValueError):
                gpu.compress(np.array(bad, dtype=dt))
    big = np.arange(100000, dtype=np.uint32)
    big[500] = 7  # duplicate in a large input: caught by the level kernels
    with pytest.raises(ValueError):
        gpu.compress(big)
    big = np.arange(100000, dtype=np.uint64)
    big[99999] = 100000  # out of range
    with pytest.raises(ValueError):
        gpu.compress(big)
    with pytest.raises(ValueError):
        gpu.compress(np.array([], dtype=np.uint32))
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 1, 5000)
    assert gpu.compress(perm) == oracle.compress(perm)


def test_device_entry_point(gpu, oracle):
    torch = pytest.importorskip("torch")
    n = 300001
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 77, n, np.uint64)
    fmt = gpu.FormatOptions(4, [], [], gpu.MiddlePlacement.embedded_output)
    size = gpu.encoded_size(n, fmt)
    d_in = torch.from_numpy(perm.view(np.int64)).cuda()
    d_blob = torch.empty((size + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        gpu.compress_device(d_in.data_ptr(), n, 8, d_blob.data_ptr(), size, fmt,
                            torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = d_blob[:size].cpu().numpy().tobytes()
        assert got == oracle.compress(perm, oracle_format(dict(middle_group_log2=4,
                                                                middle_placement=2)))


def test_misaligned_device_buffers_are_rejected(gpu):
    # rejected on the host before any device work; a valid call still works
    import torch
    n = 1000
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 1, n, np.uint64)
    size = gpu.encoded_size(n)
    d_in = torch.from_numpy(perm.view(np.int64)).cuda()
    raw = torch.zeros(size + 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError, match="entry width"):
        gpu.compress_device(d_in.data_ptr() + 4, n, 8, raw.data_ptr(), size)
    with pytest.raises(ValueError, match="4-byte aligned"):
        gpu.compress_device(d_in.data_ptr(), n, 8, raw.data_ptr() + 1, size)
    with pytest.raises(ValueError, match="entry width"):
        gpu.compress_batch_device([(d_in.data_ptr() + 4, n, 8, None, raw.data_ptr(), size)])
    gpu.compress_device(d_in.data_ptr(), n, 8, raw.data_ptr(), size)
    assert raw[:size].cpu().numpy().tobytes() == gpu.compress(perm)


def _spot_check(oracle, blob, perm, count=1024, seed=0):
    oracle.validate(blob)
    rng = np.random.default_rng(seed)
    n = len(perm)
    for i in rng.integers(0, n, count):
        i = int(i)
        assert oracle.lookup(blob, i) == int(perm[i])
        assert oracle.lookup(blob, int(perm[i]), inverse=True) == i


def test_config_1_uniform_65536(gpu, oracle):
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 1, 1 << 16)
    blob = gpu.compress(perm)
    assert blob == oracle.compress(perm)
    _spot_check(oracle, blob, perm)


def test_config_2_one_mebi(gpu, oracle):
    fmt_kw = dict(middle_group_log2=5, input_clusters=[8, 7], output_clusters=[7, 8],
                  middle_placement=1)
    opts = gpu.CompressOptions(format=b200_format(gpu, fmt_kw))
    for kind in (gpu.PermutationKind.uniform, gpu.PermutationKind.bit_reversal,
                 gpu.PermutationKind.identity):
        perm = gpu.fill_permutation(kind, 2, 1 << 20)
        assert gpu.compress(perm, opts) == oracle.compress(perm, oracle_format(fmt_kw)), kind


@pytest.mark.slow
def test_config_4_sattolo_100m(gpu):
    # bytes pinned to the reference's own blob (its SHA-256, made by
    # tests/golden/make_digests.py with the reference's portable encoder)
    d = load_digests()["config4"]
    n = d["n"]
    assert n == 100_000_007
    perm = gpu.fill_permutation(gpu.PermutationKind.single_cycle, d["seed"], n, np.uint64)
    kw = dict(middle_group_log2=4, input_clusters=[12, 11], output_clusters=[11, 12],
              middle_placement=0)
    assert d["format"] == kw
    blob = gpu.compress(perm, gpu.CompressOptions(format=b200_format(gpu, kw)))
    assert len(blob) == d["size"] == 317326221
    assert hashlib.sha256(blob).hexdigest() == d["sha256"]


def _device_round_trip(gpu, blob, perm, fmt):
    """Every forward and inverse lookup of `blob` through the device verifier
    (bpb200_lookup_device): p[i] for all i, then p^-1[p[i]] == i."""
    import torch
    n = len(perm)
    d_blob = torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda()
    d_perm = torch.from_numpy(np.ascontiguousarray(perm, dtype=np.uint64).view(np.int64)).cuda()
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    gpu.lookup_device(d_blob.data_ptr(), len(blob), n, fmt, out.data_ptr(), n, stream=stream)
    assert torch.equal(out, d_perm)
    gpu.lookup_device(d_blob.data_ptr(), len(blob), n, fmt, out.data_ptr(), n,
                      d_queries=d_perm.data_ptr(), inverse=True, stream=stream)
    assert torch.equal(out, torch.arange(n, dtype=torch.int64, device="cuda"))


def test_lookup_verifier_round_trips(gpu, oracle):
    cases = [(1 << 16, {}, gpu.PermutationKind.uniform),
             (1 << 20, dict(middle_group_log2=5, input_clusters=[8, 7], output_clusters=[7, 8],
                            middle_placement=1), gpu.PermutationKind.bit_reversal),
             (1_000_003, dict(middle_group_log2=4, middle_placement=2),
              gpu.PermutationKind.single_cycle),
             (4097, dict(middle_group_log2=1, middle_placement=0), gpu.PermutationKind.identity)]
    for n, kw, kind in cases:
        perm = gpu.fill_permutation(kind, 6, n)
        fmt = b200_format(gpu, kw)
        blob = gpu.compress(perm, gpu.CompressOptions(format=fmt))
        _device_round_trip(gpu, blob, perm, fmt)


def test_lookup_verifier_agrees_with_oracle_and_errors(gpu, oracle):
    import torch
    n = 50_000
    kw = dict(middle_group_log2=3, middle_placement=1, input_clusters=[4, 9])
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, 8, n)
    blob = oracle.compress(perm, oracle_format(kw))
    fmt = b200_format(gpu, kw)
    queries = np.random.default_rng(2).integers(0, n, 512).astype(np.int64)
    d_blob = torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda()
    d_q = torch.from_numpy(queries).cuda()
    out = torch.empty(512, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for inverse in (False, True):
        gpu.lookup_device(d_blob.data_ptr(), len(blob), n, fmt, out.data_ptr(), 512,
                          d_queries=d_q.data_ptr(), inverse=inverse, stream=stream)
        want = [oracle.lookup(blob, int(q), inverse=inverse) for q in queries]
        assert out.cpu().tolist() == want
    d_q[7] = n
    with pytest.raises(IndexError):
        gpu.lookup_device(d_blob.data_ptr(), len(blob), n, fmt, out.data_ptr(), 512,
                          d_queries=d_q.data_ptr(), stream=stream)
    assert int(out[7]) == -1 and int(out[6]) == int(perm[int(queries[6])])
    with pytest.raises(ValueError):
        gpu.lookup_device(d_blob.data_ptr(), len(blob) - 1, n, fmt, out.data_ptr(), 512,
                          stream=stream)


@pytest.mark.slow
def test_config_3_uniform_2p30(gpu, oracle):
    # the headline workload: 2^30 uint64 entries, m = 5, default clusters,
    # embedded_output.  The blob must be the reference's canonical bytes (its
    # SHA-256 from the reference's portable encoder, tests/golden/
    # make_digests.py); a decodable blob with another valid colouring would
    # pass lookups but not this.
    d = load_digests()["config3"]
    n = d["n"]
    assert n == 1 << 30 and d["format"] == dict(middle_group_log2=5, middle_placement=2)
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, d["seed"], n, np.uint64)
    fmt = gpu.FormatOptions(5, [], [], gpu.MiddlePlacement.embedded_output)
    blob = gpu.compress(perm, gpu.CompressOptions(format=fmt))
    assert len(blob) == d["size"] == 3850371096
    assert hashlib.sha256(blob).hexdigest() == d["sha256"]
    _spot_check(oracle, blob, perm, count=256, seed=3)
    # every entry, both directions, on the device
    _device_round_trip(gpu, blob, perm, fmt)
