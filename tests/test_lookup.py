# SPDX-License-Identifier: Apache-2.0
"""The batch lookup verifier's per-query walk (benes_perm_b200/csrc/lookup.hpp),
evaluated on the host through the probe hook: every forward and inverse
lookup of oracle-encoded blobs over all formats, the reference's golden
blobs, and the out-of-range error.  The device kernel runs the same walk;
tests/test_parity_gpu.py checks it on the GPU."""
import numpy as np
import pytest

from helpers import b200_format, load_goldens, oracle_format, routing_depth


def _formats():
    out = []
    rng = np.random.default_rng(11)
    for n in (1, 2, 3, 17, 32, 33, 65, 100, 257, 1000, 4097):
        for m in (1, 2, 3, 4, 5):
            d = routing_depth(n, m)
            comp, r = [], d
            while r:
                x = int(rng.integers(1, r + 1))
                comp.append(x)
                r -= x
            for pl in (0, 1, 2):
                kw = dict(middle_group_log2=m, middle_placement=pl)
                if d and (n + m + pl) % 2:
                    kw.update(input_clusters=comp, output_clusters=[d])
                out.append((n, kw))
    return out


@pytest.mark.parametrize("n,kw", _formats()[::2])
def test_probe_lookup_inverts_every_entry(b200, oracle, n, kw):
    rng = np.random.default_rng(n * 7 + kw["middle_group_log2"])
    perm = rng.permutation(n).astype(np.uint32)
    blob = oracle.compress(perm, oracle_format(kw))
    bf = b200_format(b200, kw)
    for i in range(n):
        assert b200.probe_lookup(n, bf, blob, i) == int(perm[i])
        assert b200.probe_lookup(n, bf, blob, int(perm[i]), inverse=True) == i


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_probe_lookup_structured_inputs(b200, oracle, kind):
    n = 3000
    perm = b200.fill_permutation(b200.PermutationKind(kind), 5, n)
    kw = dict(middle_group_log2=4, middle_placement=2, input_clusters=[3, 5],
              output_clusters=[8])
    blob = oracle.compress(perm, oracle_format(kw))
    bf = b200_format(b200, kw)
    for i in range(0, n, 7):
        assert b200.probe_lookup(n, bf, blob, i) == int(perm[i])
        assert b200.probe_lookup(n, bf, blob, int(perm[i]), inverse=True) == i


def test_probe_lookup_reference_goldens(b200):
    for g in load_goldens():
        perm = g["permutation"]
        blob = bytes.fromhex(g["blob_hex"])
        n = len(perm)
        for i in range(n):
            assert b200.probe_lookup(n, None, blob, i) == perm[i], g["name"]
            assert b200.probe_lookup(n, None, blob, perm[i], inverse=True) == i, g["name"]


def test_probe_lookup_agrees_with_oracle_lookup(b200, oracle):
    n = 100_003
    perm = b200.fill_permutation(b200.PermutationKind.single_cycle, 9, n)
    kw = dict(middle_group_log2=3, middle_placement=1)
    blob = oracle.compress(perm, oracle_format(kw))
    bf = b200_format(b200, kw)
    for i in np.random.default_rng(1).integers(0, n, 300):
        i = int(i)
        assert b200.probe_lookup(n, bf, blob, i) == oracle.lookup(blob, i)
        assert b200.probe_lookup(n, bf, blob, i, inverse=True) == \
            oracle.lookup(blob, i, inverse=True)


def test_probe_lookup_errors(b200, oracle):
    perm = np.arange(100, dtype=np.uint32)
    blob = oracle.compress(perm)
    with pytest.raises(IndexError):
        b200.probe_lookup(100, None, blob, 100)
    with pytest.raises(ValueError):
        b200.probe_lookup(100, None, blob[:-1], 0)
