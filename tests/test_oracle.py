# SPDX-License-Identifier: Apache-2.0
"""Pins the CPU oracle (oracle/benes_oracle.c) before anything trusts it.

Checked against the reference's golden blobs, the reference-encoded corpus
(tests/golden/corpus.json), the exact payload sizes the reference tests
assert (tests/test_benes.cpp:116-125, BENCHMARKS.md:40-53), exhaustive small
permutations and, when it is built here, the reference library itself.
"""
import hashlib
import itertools

import numpy as np
import pytest

from helpers import corpus_permutation, load_corpus, load_goldens, oracle_format, routing_depth


def test_reference_goldens(oracle):
    for g in load_goldens():
        perm = np.array(g["permutation"], dtype=np.uint32)
        blob = oracle.compress(perm)
        assert blob.hex() == g["blob_hex"], g["name"]
        oracle.validate(blob)
        for i in range(len(perm)):
            assert oracle.lookup(blob, i) == perm[i]
            assert oracle.lookup(blob, int(perm[i]), inverse=True) == i


def test_corpus(oracle, b200):
    for e in load_corpus():
        if e["n"] > 5000:
            continue
        perm = corpus_permutation(b200, e)
        blob = oracle.compress(perm, oracle_format(e["format"]))
        assert len(blob) == e["size"]
        assert hashlib.sha256(blob).hexdigest() == e["sha256"], (e["n"], e["name"], e["kind"])
        if "blob_hex" in e:
            assert blob.hex() == e["blob_hex"]


@pytest.mark.parametrize("n,payload", [(31, 15), (32, 15), (33, 16), (63, 37), (64, 38),
                                       (65, 39), (96, 64), (127, 91), (128, 91), (129, 92),
                                       (1048575, 2449406), (1048576, 2449408)])
def test_payload_sizes(oracle, n, payload):
    lay = oracle.layout(n)
    header = 20 + lay.format.input_cluster_count + lay.format.output_cluster_count
    assert lay.end_offset - header == payload


def test_exhaustive_small(oracle):
    # every permutation up to 7 entries, default format (tests/test_benes.cpp:141-176)
    for n in range(1, 8):
        for p in itertools.permutations(range(n)):
            perm = np.array(p, dtype=np.uint32)
            blob = oracle.compress(perm)
            for i in range(n):
                assert oracle.lookup(blob, i) == p[i]


def test_uint64_matches_uint32(oracle, b200):
    for n in (1, 2, 3, 31, 32, 33, 63, 65, 127, 129, 4097):
        perm = b200.fill_permutation(b200.PermutationKind.uniform, 0x640000 + n, n)
        d = routing_depth(n, 4)
        kw = dict(middle_group_log2=4, input_clusters=[1] * d, output_clusters=[d] if d else [],
                  middle_placement=1 if n % 2 == 0 else 2)
        f = oracle_format(kw)
        assert oracle.compress(perm, f) == oracle.compress(perm.astype(np.uint64), f)


def test_placement_keeps_size(oracle, b200):
    for n in (3, 7, 15, 17, 31, 33, 63, 65, 127, 129, 257):
        for m in (2, 3, 4, 5):
            sizes = {len(oracle.compress(np.arange(n, dtype=np.uint32),
                                         oracle_format(dict(middle_group_log2=m,
                                                            middle_placement=pl))))
                     for pl in (0, 1, 2)}
            assert len(sizes) == 1


def test_invalid_inputs(oracle):
    from oracle.oracle import CheckerError
    for bad in ([0, 1, 1], [0, 1, 3]):
        for dt in (np.uint32, np.uint64):
            with pytest.raises(CheckerError) as ei:
                oracle.compress(np.array(bad, dtype=dt))
            assert ei.value.code == 1
    with pytest.raises(CheckerError) as ei:
        oracle.compress(np.array([], dtype=np.uint32))
    assert ei.value.code == 1
    perm = np.arange(4097, dtype=np.uint32)
    for kw in (dict(input_clusters=[1, 1]), dict(middle_group_log2=6),
               dict(middle_group_log2=0), dict(middle_placement=3)):
        with pytest.raises(CheckerError):
            oracle.compress(perm, oracle_format(kw))


def test_oracle_matches_reference_library(oracle, reference, b200):
    rng = np.random.default_rng(7)
    for n in (5, 33, 65, 200, 1000, 4097, 20000):
        for kind in (0, 1, 3):
            perm = b200.fill_permutation(b200.PermutationKind(kind), n + kind, n)
            for m in (1, 3, 5):
                d = routing_depth(n, m)
                comp = []
                r = d
                while r:
                    x = int(rng.integers(1, r + 1))
                    comp.append(x)
                    r -= x
                for pl in (0, 1, 2):
                    kw = dict(middle_group_log2=m, middle_placement=pl, input_clusters=comp,
                              output_clusters=comp[::-1])
                    f = oracle_format(kw)
                    assert oracle.compress(perm, f) == reference.compress(perm, f, threads=4)


def test_workload_generator_matches_library(oracle, b200):
    # the oracle's restatement of the seeded generator (used by the CPU
    # baseline and the digest fixtures) gives the library's permutations
    for kind in range(5):
        for n in (1, 2, 3, 5, 64, 1000, 4096, 100003, 1 << 18):
            if kind == 4 and n & (n - 1):
                continue
            for dt in (np.uint32, np.uint64):
                a = oracle.fill_permutation(kind, 0x5EED + 31 * n + kind, n, dt)
                b = b200.fill_permutation(b200.PermutationKind(kind), 0x5EED + 31 * n + kind, n, dt)
                assert a.dtype == b.dtype and a.tobytes() == b.tobytes(), (kind, n, dt)
    single = oracle.fill_permutation(1, 9, 4099, np.uint64)
    seen, v = set(), 0
    for _ in range(4099):  # Sattolo: one cycle through every value
        seen.add(v)
        v = int(single[v])
    assert len(seen) == 4099 and v == 0
