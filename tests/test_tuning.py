# SPDX-License-Identifier: Apache-2.0
"""The per-size-class tuning table (tuning.json, made by
benes_perm_b200/tune.py): the library reads it at load, takes the nearest
class for classes it lacks, clamps values to their ranges, and a forced
setting overrides it.  On a B200 every setting gives the same bytes."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _query(env, counts):
    code = ("import sys, json; sys.path.insert(0, %r); import benes_perm_b200 as bp; "
            "print(json.dumps([bp.get_tuning(c) for c in %r]))" % (ROOT, counts))
    run = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=120)
    assert run.returncode == 0, run.stderr[-2000:]
    return json.loads(run.stdout.strip().splitlines()[-1])


def test_table_is_read_with_nearest_class_and_clamping(tmp_path, b200):
    b200.library()  # built before the subprocesses load it
    table = {"device": "test", "classes": {
        "16": {"walk_blocks_per_sm": 2, "walk_max_log2": 18, "jump_block_log2": 10,
               "tile_max_log2": 12},
        "24": {"walk_blocks_per_sm": 99, "walk_max_log2": 40, "jump_block_log2": 1,
               "tile_max_log2": 3}}}
    path = tmp_path / "tuning.json"
    path.write_text(json.dumps(table))
    env = dict(os.environ, BPB200_TUNING_FILE=str(path))
    got = _query(env, [1 << 16, 40000, 1 << 19, 1 << 23, 1 << 30])
    want16 = table["classes"]["16"]
    assert got[0] == want16 and got[1] == want16 and got[2] == want16  # 2^16, class 16, nearest
    clamped = {"walk_blocks_per_sm": 8, "walk_max_log2": 23, "jump_block_log2": 4,
               "tile_max_log2": 9}
    assert got[3]["tile_max_log2"] == 9
    assert got[3] == clamped and got[4] == clamped
    off = _query(dict(os.environ, BPB200_TUNING_FILE="none"), [1 << 20])[0]
    assert off == {"walk_blocks_per_sm": 4, "walk_max_log2": 23, "jump_block_log2": 14,
                   "tile_max_log2": 13}


def test_forced_setting_and_describe(b200):
    try:
        b200.set_tuning({"tile_max_log2": 11})
        assert b200.get_tuning(12345)["tile_max_log2"] == 11
        assert b200.describe(1 << 20)[1] == 9   # tile level of 2^11-entry nodes
    finally:
        b200.set_tuning(None)


@pytest.mark.gpu
def test_every_setting_gives_the_same_bytes(gpu, oracle):
    settings = [None,
                {"walk_blocks_per_sm": 2, "walk_max_log2": 16, "jump_block_log2": 10,
                 "tile_max_log2": 11},
                {"walk_blocks_per_sm": 6, "walk_max_log2": 23, "jump_block_log2": 16,
                 "tile_max_log2": 12},
                {"tile_max_log2": 14}]
    cases = [(70001, np.uint32, 0), (1 << 18, np.uint64, 1), (3 * (1 << 19) + 5, np.uint32, 0)]
    for n, dtype, kind in cases:
        perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0x7A + n, n, dtype)
        blobs = []
        for s in settings:
            gpu.set_tuning(s)
            try:
                blobs.append(gpu.compress(perm))
            finally:
                gpu.set_tuning(None)
        assert blobs[0] == blobs[1] == blobs[2] == blobs[3], n
        if n <= 1 << 18:
            assert blobs[0] == oracle.compress(perm)


@pytest.mark.gpu
def test_wide_tiles_of_16384_entries(gpu, oracle):
    """tile_max_log2 = 14 hands nodes of up to 16384 entries to the
    shared-memory tile (one 1024-thread CTA per SM); bytes stay the
    reference's, including a permutation that is a single such tile."""
    try:
        gpu.set_tuning({"tile_max_log2": 14})
        assert gpu.describe(1 << 20)[1] == 6
        for n, dtype, kind in ((16384, np.uint32, 0), (16383, np.uint64, 1), (1 << 17, np.uint32, 0),
                               (100003, np.uint64, 1)):
            perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0x1D + n, n, dtype)
            for kw in (dict(), dict(middle_group_log2=2, middle_placement=1)):
                fmt = gpu.FormatOptions(middle_group_log2=kw.get("middle_group_log2", 5),
                                        middle_placement=gpu.MiddlePlacement(
                                            kw.get("middle_placement", 0)))
                from helpers import oracle_format
                assert gpu.compress(perm, gpu.CompressOptions(format=fmt)) == \
                    oracle.compress(perm, oracle_format(kw)), (n, kw)
    finally:
        gpu.set_tuning(None)
