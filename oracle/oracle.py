# SPDX-License-Identifier: Apache-2.0
"""ctypes bindings of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps ``oracle/liboracle.so`` (the plain-C restatement of the
reference's portable encoder); ``Reference`` wraps ``oracle/_ref/libbenes_ref.so``
(the reference itself, compiled from its own sources by ``oracle/Makefile``).
Only tests, the smoke check and the benchmark's CPU-baseline leg use these.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbenes_ref.so")
SHIM_DRIVER = os.path.join(HERE, "_ref", "shim", "driver")
# where the reference sources lie (only the build recipes read them)
REF_DIR = os.environ.get("BENES_REFERENCE_DIR", "/root/reference")


class CFormat(ctypes.Structure):
    _fields_ = [
        ("middle_group_log2", ctypes.c_uint8),
        ("middle_placement", ctypes.c_uint8),
        ("input_cluster_count", ctypes.c_uint8),
        ("output_cluster_count", ctypes.c_uint8),
        ("input_clusters", ctypes.c_uint8 * 64),
        ("output_clusters", ctypes.c_uint8 * 64),
    ]


def make_format(middle_group_log2: int = 5, input_clusters: Sequence[int] = (),
                output_clusters: Sequence[int] = (), middle_placement: int = 0) -> CFormat:
    f = CFormat()
    f.middle_group_log2 = middle_group_log2
    f.middle_placement = int(middle_placement)
    f.input_cluster_count = len(input_clusters)
    f.output_cluster_count = len(output_clusters)
    for i, v in enumerate(input_clusters):
        f.input_clusters[i] = v
    for i, v in enumerate(output_clusters):
        f.output_clusters[i] = v
    return f


class CheckerError(Exception):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


def build() -> None:
    """Builds liboracle.so and, when the reference sources exist, the
    reference library and the integration-shim driver."""
    subprocess.run(["make", "-s", "liboracle.so"], cwd=HERE, check=True)
    if os.path.exists(os.path.join(REF_DIR, "src", "benes.cpp")):
        subprocess.run(["make", "-s", "ref", f"REF={REF_DIR}"], cwd=HERE, check=True)
        build_shim()


def integration_blocks():
    """The C++ of the integration notes: the backend unit and its
    declarations (section 2) and the dispatch fragment (section 3)."""
    import re
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section2 = text.split("## 2.", 1)[1].split("\n## 3.", 1)[0]
    section3 = text.split("## 3.", 1)[1].split("\n## 4.", 1)[0]
    blocks = re.findall(r"```cpp\n(.*?)```", section2, re.S)
    if len(blocks) != 2:
        raise ValueError("section 2 must hold the backend unit and its declarations")
    unit = next(b for b in blocks if "#include <benes_b200.h>" in b)
    decls = next(b for b in blocks if b is not unit)
    dispatch = re.findall(r"```cpp\n(.*?)```", section3, re.S)[0]
    return unit, decls, dispatch


def build_shim() -> str:
    """Compiles the integration notes' shim, as written there, with
    oracle/shim_driver.cpp against the reference's headers, the reference
    library (oracle/_ref) and libbenes_b200.so, into oracle/_ref/shim/driver.
    The reference headers lack the appended Backend::b200 enumerator, so the
    dispatch fragment names it as the driver's kB200 constant."""
    work = os.path.dirname(SHIM_DRIVER)
    os.makedirs(work, exist_ok=True)
    unit, decls, dispatch = integration_blocks()
    with open(os.path.join(work, "b200_decls.hpp"), "w") as f:
        f.write('#pragma once\n#include "internal.hpp"\n' + decls)
    with open(os.path.join(work, "benes_b200_backend.cpp"), "w") as f:
        f.write('#include "b200_decls.hpp"\n' + unit)
    with open(os.path.join(work, "dispatch_fragment.inc"), "w") as f:
        f.write(dispatch.replace("Backend::b200", "kB200"))
    ref_dir = os.path.join(HERE, "_ref")
    lib_dir = os.path.join(ROOT, "benes_perm_b200")
    cmd = ["g++", "-std=c++20", "-O1", "-pthread",
           "-I", work, "-I", os.path.join(REF_DIR, "src"), "-I", os.path.join(REF_DIR, "include"),
           "-I", os.path.join(ROOT, "include"),
           os.path.join(work, "benes_b200_backend.cpp"), os.path.join(HERE, "shim_driver.cpp"),
           "-L", ref_dir, "-lbenes_ref", "-L", lib_dir, "-lbenes_b200",
           "-Wl,-rpath,$ORIGIN/..:$ORIGIN/../../../benes_perm_b200", "-o", SHIM_DRIVER + ".tmp"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("shim build failed:\n" + proc.stderr[-4000:])
    os.replace(SHIM_DRIVER + ".tmp", SHIM_DRIVER)
    return SHIM_DRIVER


class _Checker:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)

    def _err(self):
        return ctypes.create_string_buffer(256)


class Oracle(_Checker):
    """The plain-C restatement (single-threaded, canonical bytes)."""

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        L = self.lib
        fp = ctypes.POINTER(CFormat)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.oracle_compress.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, fp,
                                      ctypes.c_void_p, ctypes.c_uint64, u64p, ctypes.c_char_p,
                                      ctypes.c_size_t]
        L.oracle_validate.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p,
                                      ctypes.c_size_t]
        L.oracle_lookup.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                    u64p, ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_switch_bit.argtypes = [ctypes.c_uint64, fp, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_uint64, u64p]
        L.oracle_middle_bit.argtypes = [ctypes.c_uint64, fp, ctypes.c_int, ctypes.c_void_p, u64p]
        L.oracle_factoradic_bits.argtypes = [ctypes.c_uint32]
        L.oracle_factoradic_bits.restype = ctypes.c_uint32
        L.oracle_fill_permutation.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                              ctypes.c_uint32, ctypes.c_void_p]

        class _Layout(ctypes.Structure):
            _fields_ = [(n, ctypes.c_uint64) for n in (
                "size", "network_size", "switch_bits", "middle_bits", "input_offset",
                "output_offset", "middle_offset", "end_offset")] + [("format", CFormat)]
        self._Layout = _Layout
        L.oracle_make_layout.argtypes = [ctypes.c_uint64, fp, ctypes.POINTER(_Layout),
                                         ctypes.c_char_p, ctypes.c_size_t]

    def layout(self, n: int, fmt: Optional[CFormat] = None):
        fmt = fmt or make_format()
        out = self._Layout()
        err = self._err()
        rc = self.lib.oracle_make_layout(n, ctypes.byref(fmt), ctypes.byref(out), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())
        return out

    def compress(self, perm: np.ndarray, fmt: Optional[CFormat] = None) -> bytes:
        fmt = fmt or make_format()
        perm = np.ascontiguousarray(perm)
        n = int(perm.size)
        err = self._err()
        cap = self.layout(n, fmt).end_offset if n else 0
        out = np.zeros(max(cap, 1), dtype=np.uint8)
        got = ctypes.c_uint64(0)
        rc = self.lib.oracle_compress(perm.ctypes.data, n, perm.dtype.itemsize, ctypes.byref(fmt),
                                      out.ctypes.data, cap, ctypes.byref(got), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())
        return out[:got.value].tobytes()

    def validate(self, blob: bytes) -> None:
        buf = np.frombuffer(blob, dtype=np.uint8)
        err = self._err()
        rc = self.lib.oracle_validate(buf.ctypes.data, len(blob), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())

    def lookup(self, blob: bytes, value: int, inverse: bool = False) -> int:
        buf = np.frombuffer(blob, dtype=np.uint8)
        err = self._err()
        out = ctypes.c_uint64(0)
        rc = self.lib.oracle_lookup(buf.ctypes.data, len(blob), value, int(inverse),
                                    ctypes.byref(out), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())
        return out.value

    def switch_bit(self, n: int, fmt: CFormat, side: int, turns: Sequence[int], pair: int) -> int:
        arr = (ctypes.c_uint8 * max(1, len(turns)))(*turns)
        out = ctypes.c_uint64(0)
        rc = self.lib.oracle_switch_bit(n, ctypes.byref(fmt), side, len(turns), arr, pair,
                                        ctypes.byref(out))
        if rc:
            raise CheckerError(rc, "switch probe")
        return out.value

    def middle_bit(self, n: int, fmt: CFormat, turns: Sequence[int]) -> int:
        arr = (ctypes.c_uint8 * max(1, len(turns)))(*turns)
        out = ctypes.c_uint64(0)
        rc = self.lib.oracle_middle_bit(n, ctypes.byref(fmt), len(turns), arr, ctypes.byref(out))
        if rc:
            raise CheckerError(rc, "middle probe")
        return out.value

    def factoradic_bits(self, c: int) -> int:
        return int(self.lib.oracle_factoradic_bits(c))

    def fill_permutation(self, kind: int, seed: int, n: int, dtype=np.uint32,
                         out: Optional[np.ndarray] = None) -> np.ndarray:
        """The configs' seeded workload permutation (kind 0 Fisher-Yates,
        1 Sattolo, 2 identity, 3 reverse, 4 bit reversal)."""
        dtype = np.dtype(dtype)
        if out is None:
            out = np.empty(n, dtype=dtype)
        if out.dtype != dtype or out.size != n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous array of n values of dtype")
        rc = self.lib.oracle_fill_permutation(int(kind), seed & (2**64 - 1), n, dtype.itemsize,
                                              out.ctypes.data)
        if rc:
            raise CheckerError(rc, "invalid workload arguments")
        return out


class Reference(_Checker):
    """The reference's own portable encoder, compiled from its sources."""

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        fp = ctypes.POINTER(CFormat)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.ref_hardware_threads.restype = ctypes.c_uint
        L.ref_encoded_size.argtypes = [ctypes.c_uint64, fp, u64p, ctypes.c_char_p, ctypes.c_size_t]
        L.ref_compress.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, fp,
                                   ctypes.c_size_t, ctypes.c_void_p, ctypes.c_uint64, u64p,
                                   ctypes.c_char_p, ctypes.c_size_t]
        L.ref_validate.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p,
                                   ctypes.c_size_t]
        L.ref_lookup.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                 u64p, ctypes.c_char_p, ctypes.c_size_t]

    def hardware_threads(self) -> int:
        return int(self.lib.ref_hardware_threads())

    def encoded_size(self, n: int, fmt: Optional[CFormat] = None) -> int:
        fmt = fmt or make_format()
        out = ctypes.c_uint64(0)
        err = self._err()
        rc = self.lib.ref_encoded_size(n, ctypes.byref(fmt), ctypes.byref(out), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())
        return out.value

    def compress(self, perm: np.ndarray, fmt: Optional[CFormat] = None, threads: int = 1,
                 out: Optional[np.ndarray] = None) -> bytes:
        fmt = fmt or make_format()
        perm = np.ascontiguousarray(perm)
        n = int(perm.size)
        err = self._err()
        cap = self.encoded_size(n, fmt) if n else 0
        if out is None or out.size < cap:
            out = np.zeros(max(cap, 1), dtype=np.uint8)
        got = ctypes.c_uint64(0)
        rc = self.lib.ref_compress(perm.ctypes.data, n, perm.dtype.itemsize, ctypes.byref(fmt),
                                   threads, out.ctypes.data, cap, ctypes.byref(got), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())
        return out[:got.value].tobytes()

    def validate(self, blob: bytes) -> None:
        buf = np.frombuffer(blob, dtype=np.uint8)
        err = self._err()
        rc = self.lib.ref_validate(buf.ctypes.data, len(blob), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())

    def lookup(self, blob: bytes, value: int, inverse: bool = False) -> int:
        buf = np.frombuffer(blob, dtype=np.uint8)
        err = self._err()
        out = ctypes.c_uint64(0)
        rc = self.lib.ref_lookup(buf.ctypes.data, len(blob), value, int(inverse),
                                 ctypes.byref(out), err, 256)
        if rc:
            raise CheckerError(rc, err.value.decode())
        return out.value
