# SPDX-License-Identifier: Apache-2.0
"""Host-side checks of the B200 library that need no GPU: the C ABI loads
and exports every symbol include/benes_b200.h declares, the layout matches
the oracle, the closed-form switch and rank addresses match the oracle's
SectionAddress walk, and argument errors map to the reference's kinds."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import b200_format, oracle_format, routing_depth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "benes_b200.h")).read()
    return sorted(set(re.findall(r"\b(bpb200_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(b200):
    lib = b200.library()
    names = declared_symbols()
    assert "bpb200_compress" in names and len(names) >= 8
    for name in names:
        assert hasattr(lib, name), name


def test_backend_name(b200):
    assert b200.backend_name() == "b200"


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 4097, 65536, 1048575, 1048576,
                               100_000_007, 1 << 30, (1 << 32) - 1, 1 << 32, (1 << 33)])
def test_encoded_size_matches_oracle(b200, oracle, n):
    for kw in (dict(), dict(middle_group_log2=4, middle_placement=1),
               dict(middle_group_log2=3, middle_placement=2)):
        assert b200.encoded_size(n, b200_format(b200, kw)) == oracle.layout(n, oracle_format(kw)).end_offset


def test_configured_sizes(b200):
    # blob sizes of the benchmark configurations
    assert b200.encoded_size(65536) == 120344
    assert b200.encoded_size(1 << 20, b200.FormatOptions(5, [8, 7], [7, 8],
                                                          b200.MiddlePlacement.embedded_input)) == 2449432
    assert b200.encoded_size(1 << 30, b200.FormatOptions(
        5, [], [], b200.MiddlePlacement.embedded_output)) == 3850371096
    assert b200.encoded_size(100_000_007, b200.FormatOptions(4, [12, 11], [11, 12])) == 317326221


def test_format_errors(b200):
    with pytest.raises(ValueError):
        b200.encoded_size(4097, b200.FormatOptions(input_clusters=[1, 1]))
    with pytest.raises(ValueError):
        b200.encoded_size(4097, b200.FormatOptions(middle_group_log2=6))
    with pytest.raises(ValueError):
        b200.encoded_size(4097, b200.FormatOptions(middle_group_log2=0))
    with pytest.raises(OverflowError):
        b200.encoded_size((1 << 64) - 1)


def _cases():
    out = []
    rng = np.random.default_rng(3)
    for n in (17, 33, 65, 100, 257, 1000, 4097, 10007):
        for m in (1, 3, 4, 5):
            d = routing_depth(n, m)
            comp = []
            r = d
            while r:
                x = int(rng.integers(1, r + 1))
                comp.append(x)
                r -= x
            for pl in (0, 1, 2):
                out.append((n, dict(middle_group_log2=m, middle_placement=pl,
                                    input_clusters=comp, output_clusters=[d] if d else [])))
    return out


@pytest.mark.parametrize("n,kw", _cases()[::3])
def test_closed_form_addresses_match_oracle(b200, oracle, n, kw):
    rng = np.random.default_rng(n)
    bf = b200_format(b200, kw)
    of = oracle_format(kw)
    m = kw["middle_group_log2"]
    d = routing_depth(n, m)
    leaf = 1 << m

    def size_of(level, node):
        c = n
        for t in range(level):
            right = (node >> (level - 1 - t)) & 1
            c = c // 2 if right else c - c // 2
        return c

    for level in range(d + 1):
        nodes = 1 << level
        picks = range(nodes) if nodes <= 8 else rng.integers(0, nodes, 8)
        for node in picks:
            node = int(node)
            turns = [(node >> (level - 1 - t)) & 1 for t in range(level)]
            if level and size_of(level - 1, node >> 1) <= leaf:
                continue
            s = size_of(level, node)
            if s > leaf:
                for side in (0, 1):
                    for pair in sorted({0, s // 2 - 1, int(rng.integers(0, s // 2))}):
                        assert b200.probe_switch_bit(n, bf, side, level, node, pair) == \
                            oracle.switch_bit(n, of, side, turns, pair)
            else:
                _, bit = b200.probe_rank_bit(n, bf, level, node)
                assert bit == oracle.middle_bit(n, of, turns)


def test_fill_permutation_is_a_seeded_permutation(b200):
    for kind in (0, 1, 2, 3):
        a = b200.fill_permutation(b200.PermutationKind(kind), 99, 1000)
        b = b200.fill_permutation(b200.PermutationKind(kind), 99, 1000, np.uint64)
        assert np.array_equal(np.sort(a), np.arange(1000))
        assert np.array_equal(a, b.astype(np.uint32))
    cyc = b200.fill_permutation(b200.PermutationKind.single_cycle, 5, 999)
    x, length = 0, 0
    while True:
        x = int(cyc[x])
        length += 1
        if x == 0:
            break
    assert length == 999
    br = b200.fill_permutation(b200.PermutationKind.bit_reversal, 0, 8)
    assert br.tolist() == [0, 4, 2, 6, 1, 5, 3, 7]


def test_compress_without_gpu_reports_unavailable(b200):
    if b200.backend_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        b200.compress(np.arange(10, dtype=np.uint32))


def test_python_argument_errors_come_before_device_work(b200):
    # the reference takes a span of uint32 or uint64; an empty one is
    # "permutation size is out of range" (src/benes.cpp:153-156)
    with pytest.raises(TypeError):
        b200.compress(np.arange(10, dtype=np.int64))
    with pytest.raises(ValueError, match="one-dimensional"):
        b200.compress(np.arange(16, dtype=np.uint32).reshape(4, 4))
    with pytest.raises(ValueError, match="out of range"):
        b200.compress(np.zeros(0, dtype=np.uint64))
    with pytest.raises(ValueError, match="middle_group_log2"):
        b200.compress(np.arange(10, dtype=np.uint32),
                      b200.CompressOptions(format=b200.FormatOptions(middle_group_log2=9)))
