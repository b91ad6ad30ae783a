# SPDX-License-Identifier: Apache-2.0
"""Regenerates the golden fixtures in this directory (run in a container that
has the reference sources; the fixtures are committed and nothing at test
time reads the reference).

1. ``reference_goldens.json``: the reference's three golden blobs
   (tests/golden/{identity-32,reverse-33,random-47}.benes of the reference).
   Each permutation is recovered by decoding the blob with the reference's own
   CompressedPermutationView (its random-47 permutation comes from a libc++
   std::shuffle, which libstdc++ does not reproduce), then re-encoded with the
   reference's portable encoder (threads = 1); the script asserts the
   re-encoding is byte-identical before writing it.
2. ``corpus.json``: reference-encoded blobs for seeded permutations over the
   reference test suite's sizes and format options
   (tests/test_benes.cpp:101-354), small ones stored in full, larger ones as
   SHA-256 digests.

Usage: python tests/golden/make_golden.py  (needs oracle/_ref built).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import REF_DIR, Oracle, Reference, make_format  # noqa: E402

# the reference's golden blobs (BENES_REFERENCE_DIR names its checkout)
REFERENCE_GOLDEN_DIR = os.path.join(REF_DIR, "tests", "golden")


def routing_depth(n: int, m: int) -> int:
    d = 0
    while n > (1 << m):
        n = (n + 1) // 2
        d += 1
    return d


def seeded_permutation(kind: int, seed: int, n: int) -> np.ndarray:
    # the oracle's restatement of the workload generator (pinned against the
    # library's by tests/test_oracle.py)
    return Oracle().fill_permutation(kind, seed, n, np.uint32)


def format_cases(n: int):
    """(name, format kwargs) covering the reference's format tests."""
    out = [("default", dict())]
    for m in (1, 2, 3, 4, 5):
        d = routing_depth(n, m)
        for pl in (0, 1, 2):
            out.append((f"m{m}-p{pl}", dict(middle_group_log2=m, middle_placement=pl)))
            if d > 0:
                out.append((f"m{m}-p{pl}-ones", dict(middle_group_log2=m, middle_placement=pl,
                                                     input_clusters=[1] * d,
                                                     output_clusters=[d])))
    return out


def main() -> None:
    ref = Reference()
    goldens = []
    for name in ("identity-32.benes", "reverse-33.benes", "random-47.benes"):
        blob = open(os.path.join(REFERENCE_GOLDEN_DIR, name), "rb").read()
        n = int.from_bytes(blob[8:16], "little")
        perm = np.array([ref.lookup(blob, i) for i in range(n)], dtype=np.uint32)
        again = ref.compress(perm, make_format(), threads=1)
        assert again == blob, f"{name}: re-encoding differs"
        goldens.append({"name": name, "permutation": perm.tolist(), "blob_hex": blob.hex()})
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as f:
        json.dump(goldens, f, indent=1)

    corpus = []
    sizes = [1, 2, 3, 7, 9, 15, 16, 17, 30, 31, 32, 33, 34, 47, 62, 63, 64, 65, 66, 95, 96, 97,
             126, 127, 128, 129, 130, 255, 257, 511, 513, 1023, 1025, 4095, 4097]
    for n in sizes:
        for kind in (0, 1, 2, 3):
            seed = 0xB200_0000 + n * 16 + kind
            perm = seeded_permutation(kind, seed, n)
            cases = format_cases(n) if kind == 0 else [("default", dict())]
            for fname, kw in cases:
                blob = ref.compress(perm, make_format(**kw), threads=1)
                entry = {"n": n, "kind": kind, "seed": seed, "format": kw, "name": fname,
                         "size": len(blob), "sha256": hashlib.sha256(blob).hexdigest()}
                if len(blob) <= 512:
                    entry["blob_hex"] = blob.hex()
                corpus.append(entry)
    for n in (32767, 32768, 32769, 43690, 65535, 65536, 65537, 100003):
        for kind in (0, 1):
            seed = 0xB200_0000 + n * 16 + kind
            perm = seeded_permutation(kind, seed, n)
            for fname, kw in (("default", dict()),
                              ("m4-p1", dict(middle_group_log2=4, middle_placement=1)),
                              ("m5-p2", dict(middle_group_log2=5, middle_placement=2))):
                blob = ref.compress(perm, make_format(**kw), threads=8)
                corpus.append({"n": n, "kind": kind, "seed": seed, "format": kw, "name": fname,
                               "size": len(blob), "sha256": hashlib.sha256(blob).hexdigest()})
    with open(os.path.join(HERE, "corpus.json"), "w") as f:
        json.dump(corpus, f, indent=0)
    print(f"wrote {len(goldens)} goldens and {len(corpus)} corpus entries")


if __name__ == "__main__":
    main()
