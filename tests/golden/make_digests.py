# SPDX-License-Identifier: Apache-2.0
"""Regenerates ``reference_digests.json``: SHA-256 digests of blobs that the
reference itself produced, for workloads too large to re-encode at test time.

Every blob here comes from the reference's portable encoder built from its
own sources (oracle/_ref, ``benes::compress`` with Backend::portable_cpu and
all host threads; thread count does not change bytes,
tests/test_benes.cpp:197-228 of the reference).  Inputs come from the
oracle's workload generator (oracle_fill_permutation), so nothing here runs
the B200 library.  Sets:

- ``config3``: N = 2^30 uint64, Fisher-Yates seed 0x5EED2030, m = 5, default
  clusters, embedded_output (the benchmark's headline workload).
- ``config4``: N = 100,000,007 uint64, Sattolo seed 4, m = 4, clusters
  {12,11}/{11,12}, separate placement.
- ``stream240``: the 240-request mixed stream the GPU tests replay (sizes up
  to 2^21, both widths, m in {4,5}, all placements).
- ``stream4096``: the benchmark's 4096-request mixed serving stream (sizes
  up to 2^24).

The stream specifications come from ``bench.serving_specs`` (numpy only).
Usage: python tests/golden/make_digests.py [--out FILE] [set ...]
(needs oracle/_ref).  The 2^30 set needs about 70 GB of host memory and
several minutes; ``--out`` writes the sets made by this run to FILE instead
(to merge into this directory's file afterwards).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle, Reference, make_format  # noqa: E402

import bench  # noqa: E402

OUT = os.path.join(HERE, "reference_digests.json")

SINGLE = {
    "config3": dict(n=1 << 30, kind=0, seed=bench.SEED, entry_bytes=8,
                    format=dict(middle_group_log2=5, middle_placement=2)),
    "config4": dict(n=100_000_007, kind=1, seed=4, entry_bytes=8,
                    format=dict(middle_group_log2=4, input_clusters=[12, 11],
                                output_clusters=[11, 12], middle_placement=0)),
}
STREAMS = {
    "stream240": dict(requests=240, max_log2=21, seed=bench.STREAM_TEST_SEED),
    "stream4096": dict(requests=4096, max_log2=24, seed=bench.SEED),
}


def load(path: str) -> dict:
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def save(d: dict, path: str) -> None:
    with open(path + ".tmp", "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
        f.write("\n")
    os.replace(path + ".tmp", path)


def single(name: str, ref: Reference, oracle: Oracle, threads: int) -> dict:
    spec = SINGLE[name]
    dtype = np.uint64 if spec["entry_bytes"] == 8 else np.uint32
    perm = oracle.fill_permutation(spec["kind"], spec["seed"], spec["n"], dtype)
    fmt = make_format(**spec["format"])
    t0 = time.perf_counter()
    blob = ref.compress(perm, fmt, threads=threads)
    secs = time.perf_counter() - t0
    return dict(spec, size=len(blob), sha256=hashlib.sha256(blob).hexdigest(),
                reference_seconds=round(secs, 1), threads=threads)


def stream(name: str, ref: Reference, oracle: Oracle, threads: int) -> dict:
    spec = STREAMS[name]
    specs = bench.serving_specs(spec["requests"], spec["max_log2"], spec["seed"])
    digests = []
    t0 = time.perf_counter()
    for i, (n, kind, dtype, m, placement) in enumerate(specs):
        perm = oracle.fill_permutation(kind, spec["seed"] + i, n, dtype)
        blob = ref.compress(perm, make_format(m, [], [], placement), threads=threads)
        digests.append(hashlib.sha256(blob).hexdigest()[:32])
    return dict(spec, sha256_128=digests, entries=int(sum(s[0] for s in specs)),
                reference_seconds=round(time.perf_counter() - t0, 1), threads=threads)


def main(argv) -> None:
    out = OUT
    if argv[:1] == ["--out"]:
        out, argv = argv[1], argv[2:]
    names = argv or list(SINGLE) + list(STREAMS)
    ref, oracle = Reference(), Oracle()
    threads = ref.hardware_threads()
    for name in names:
        if name in SINGLE:
            made = single(name, ref, oracle, threads)
        elif name in STREAMS:
            made = stream(name, ref, oracle, threads)
        else:
            raise SystemExit(f"unknown set {name}")
        d = load(out)  # read just before writing: other sets may have landed meanwhile
        d[name] = made
        save(d, out)
        print(name, "done", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
