# SPDX-License-Identifier: Apache-2.0
"""Shared helpers for the tests: format conversion and corpus loading."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def routing_depth(n, m):
    d = 0
    while n > (1 << m):
        n = (n + 1) // 2
        d += 1
    return d


def b200_format(bp, kw):
    return bp.FormatOptions(middle_group_log2=kw.get("middle_group_log2", 5),
                            input_clusters=list(kw.get("input_clusters", [])),
                            output_clusters=list(kw.get("output_clusters", [])),
                            middle_placement=bp.MiddlePlacement(kw.get("middle_placement", 0)))


def oracle_format(kw):
    from oracle.oracle import make_format
    return make_format(**kw)


def load_goldens():
    with open(os.path.join(GOLDEN, "reference_goldens.json")) as f:
        return json.load(f)


def load_corpus():
    with open(os.path.join(GOLDEN, "corpus.json")) as f:
        return json.load(f)


def corpus_permutation(bp, entry, dtype=np.uint32):
    return bp.fill_permutation(bp.PermutationKind(entry["kind"]), entry["seed"], entry["n"], dtype)


def load_digests():
    """SHA-256 digests of blobs the reference encoded (make_digests.py)."""
    with open(os.path.join(GOLDEN, "reference_digests.json")) as f:
        return json.load(f)
