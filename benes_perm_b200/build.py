# SPDX-License-Identifier: Apache-2.0
"""Build recipe for the in-tree B200 library (sm_100a only).

Produces ``benes_perm_b200/libbenes_b200.so`` next to this file with one nvcc
invocation.  nvcc cross-compiles, so this runs on machines without a GPU.
``defines`` (e.g. ``["BPB200_RULER_LOG2=5"]``) and ``out`` build a variant
library elsewhere, for tuning the compile-time knobs of the walk colouring.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbenes_b200.so")
SOURCES = ["encode.cu", "layout.cpp", "permgen.cpp"]
HEADERS = ["plan.hpp", "layout.hpp", "device.cuh", "kernels.cuh", "tile.cuh", "walk.cuh",
           "batch_levels.cuh", "group.inc", "serve.inc", "file.inc", "staging.inc", "lookup.hpp",
           "lookup.inc", "probe.inc"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "-shared", "-lcudart",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the B200 library cannot be built")


def _stale(lib: str) -> bool:
    if not os.path.exists(lib):
        return True
    built = os.path.getmtime(lib)
    inputs = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    inputs.append(os.path.join(HERE, "..", "include", "benes_b200.h"))
    inputs.append(os.path.abspath(__file__))
    return any(os.path.getmtime(p) > built for p in inputs if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, defines=(), out: str | None = None) -> str:
    lib = out or LIB
    if not force and not defines and not _stale(lib):
        return lib
    cmd = [_nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-o", lib + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    proc = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
    if verbose:
        sys.stderr.write(proc.stdout + proc.stderr)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
