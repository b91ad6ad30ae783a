# SPDX-License-Identifier: Apache-2.0
"""Host-side arithmetic behind bench.py's roofline figures: the section bit
counts it derives match the oracle's layout, and the pipeline's algorithmic
bytes for the 2^30 workload equal the closed form stated for it
(w_in*N + (8L - 4)*N + 2*switch_bits/8 + 4N + middle_bytes)."""
import pytest

from helpers import oracle_format


@pytest.mark.parametrize("n", [1, 33, 1000, 65536, 1 << 20, 100_000_007, 1 << 30])
@pytest.mark.parametrize("m", [4, 5])
def test_section_bits_match_oracle_layout(b200, oracle, n, m):
    import bench
    switch_bits, middle_bits = bench._section_bits(n, b200.FormatOptions(middle_group_log2=m))
    lay = oracle.layout(n, oracle_format(dict(middle_group_log2=m)))
    assert switch_bits == lay.switch_bits
    assert middle_bits == lay.middle_bits


def test_pipeline_bytes_of_the_2p30_workload(b200):
    import bench
    n, fmt = bench.workload(30)
    depth, tile = b200.describe(n, fmt)
    switch_bits, middle_bits = bench._section_bits(n, fmt)
    per, pipeline = bench.algorithmic_bytes(n, depth, tile, 8, switch_bits, middle_bits,
                                            set(range(7, tile)))
    assert depth == 25
    closed_form = 8 * n + (8 * depth - 4) * n + 2 * switch_bits / 8 + 4 * n + middle_bits / 8
    assert pipeline == closed_form
    assert abs(pipeline / 227.2e9 - 1) < 1e-3          # about 227.2 GB per compress
    # every level's kernels are charged: kinds sum to more than one pass per level
    assert sum(per.values()) > 8 * n * tile


def test_reference_arm_loads_nothing_of_the_b200_library(tmp_path):
    """bench.py --impl reference times the reference library alone: its
    input comes from the oracle's generator, and neither the package nor
    libbenes_b200.so is loaded in that process."""
    import json
    import os
    import subprocess
    import sys
    from oracle.oracle import REF_SO
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref is not built")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', "
            "'--warmup', '1', '--cpu-log2n', '14']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print('LOADED' if ('libbenes_b200' in maps or 'benes_perm_b200' in sys.modules) "
            "else 'CLEAN')")
    run = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True,
                         timeout=300)
    assert run.returncode == 0, run.stderr[-2000:]
    lines = run.stdout.strip().splitlines()
    assert lines[-1] == "CLEAN"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["config"]["n"] == 1 << 14
    assert line["value"] > 0 and line["cpu_baseline"]["cores"] >= 1
