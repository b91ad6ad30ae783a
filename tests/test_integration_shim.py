# SPDX-License-Identifier: Apache-2.0
"""The reference-side shim of INTEGRATION.md, compiled as written.

``oracle.oracle.build_shim`` compiles the backend unit and declarations of
its section 2 and the dispatch fragment of its section 3 with
``oracle/shim_driver.cpp`` against the reference's own headers, the
reference library built from its unmodified sources (oracle/_ref) and
libbenes_b200.so.  The driver feeds the same arguments to the shim and to
the reference's portable_cpu path (benes::compress / benes::compress_file,
src/benes.cpp:422-553) and prints the exception type and message each
raised; they must agree.  Without a GPU the valid calls must fail with
"b200 backend is unavailable"; on a B200 (the ``gpu`` tests) the shim's
bytes must equal the reference's, including a 2^20-entry uint64 call and
one through the dispatch branch.  The driver is built where the reference
sources are present (``build()``) and travels prebuilt; without either the
tests skip.
"""
import os
import subprocess

import pytest

from oracle.oracle import REF_DIR, SHIM_DRIVER, build_shim


@pytest.fixture(scope="module")
def shim_results(tmp_path_factory, reference, b200):
    if os.path.exists(os.path.join(REF_DIR, "src", "internal.hpp")):
        build_shim()  # rebuild from the current integration notes
    elif not os.path.exists(SHIM_DRIVER):
        pytest.skip("neither the reference sources nor a prebuilt shim driver are present")
    b200.library()  # builds libbenes_b200.so if it is stale
    work = tmp_path_factory.mktemp("shim")
    run = subprocess.run([SHIM_DRIVER, str(work)], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr[-2000:]
    rows = {}
    for line in run.stdout.splitlines():
        name, *rest = line.split("\t")
        rows[name] = rest
    return rows


ERROR_CASES = ["group_log2_zero", "group_log2_six", "clusters_short", "clusters_long",
               "bad_placement", "empty", "file_missing", "file_ragged", "file_directory",
               "file_bad_width"]
VALID_CASES = ["valid_u32", "valid_u64_embedded", "valid_u64_2p20", "dispatch_u64_2p20"]


@pytest.mark.parametrize("case", ERROR_CASES)
def test_shim_errors_match_reference(shim_results, case):
    shim, ref = shim_results[case]
    assert not ref.startswith("ok|"), ref
    assert shim == ref


@pytest.mark.parametrize("case", VALID_CASES)
def test_shim_valid_call_without_gpu(shim_results, case):
    if shim_results["available"][0] == "1":
        pytest.skip("a B200 is present: the gpu test checks the bytes")
    shim, ref = shim_results[case]
    assert ref == "ok|"
    assert shim == "runtime_error|b200 backend is unavailable"


@pytest.mark.gpu
@pytest.mark.parametrize("case", VALID_CASES)
def test_shim_valid_call_same_bytes(shim_results, case):
    assert shim_results["available"][0] == "1", "the gpu tests need a B200"
    shim, ref = shim_results[case]
    assert ref == "ok|"
    assert shim == "ok|"
    assert shim_results[case + "_bytes"][0] == "same"
