# SPDX-License-Identifier: Apache-2.0
"""B200 compression backend for benes-perm: Python host mirror.

Mirrors the reference's public compression API (include/benes/benes.hpp:
``FormatOptions``, ``CompressOptions``, ``compress``, ``backend_available``,
``backend_name``) for the one backend this package provides.  Every call goes
through the C ABI in ``include/benes_b200.h`` into ``libbenes_b200.so``; there
is no CPU fallback.  Errors raise the Python counterparts of the reference's
exception types: ``ValueError`` for std::invalid_argument, ``OverflowError``
for std::overflow_error, ``LengthError`` (a ``ValueError`` subclass, as
std::length_error derives from std::logic_error) for std::length_error and
``RuntimeError`` for std::runtime_error and ``IndexError`` for
std::out_of_range (lookup verifier).
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libbenes_b200.so")


class LengthError(ValueError):
    """std::length_error counterpart."""


class MiddlePlacement(enum.IntEnum):
    """benes::MiddlePlacement (include/benes/benes.hpp:21-25)."""

    separate = 0
    embedded_input = 1
    embedded_output = 2


class InputValueWidth(enum.IntEnum):
    """benes::InputValueWidth (include/benes/benes.hpp:27-30)."""

    bits32 = 4
    bits64 = 8


class PermutationKind(enum.IntEnum):
    """Synthetic permutation generators (workload inputs)."""

    uniform = 0       # Fisher-Yates
    single_cycle = 1  # Sattolo
    identity = 2
    reverse = 3
    bit_reversal = 4


@dataclass
class FormatOptions:
    """benes::FormatOptions (include/benes/benes.hpp:32-39)."""

    middle_group_log2: int = 5
    input_clusters: Sequence[int] = field(default_factory=list)
    output_clusters: Sequence[int] = field(default_factory=list)
    middle_placement: MiddlePlacement = MiddlePlacement.separate


@dataclass
class CompressOptions:
    """benes::CompressOptions (include/benes/benes.hpp:41-45); ``threads`` is
    accepted and ignored, like the reference's GPU backends."""

    threads: int = 0
    format: FormatOptions = field(default_factory=FormatOptions)


class _Format(ctypes.Structure):
    _fields_ = [
        ("middle_group_log2", ctypes.c_uint8),
        ("middle_placement", ctypes.c_uint8),
        ("input_cluster_count", ctypes.c_uint8),
        ("output_cluster_count", ctypes.c_uint8),
        ("input_clusters", ctypes.c_uint8 * 64),
        ("output_clusters", ctypes.c_uint8 * 64),
    ]


def to_c_format(fmt: Optional[FormatOptions]) -> _Format:
    fmt = fmt or FormatOptions()
    if len(fmt.input_clusters) > 64 or len(fmt.output_clusters) > 64:
        raise ValueError("cluster depths do not span every routing level")
    c = _Format()
    c.middle_group_log2 = int(fmt.middle_group_log2) & 0xFF
    c.middle_placement = int(fmt.middle_placement) & 0xFF
    c.input_cluster_count = len(fmt.input_clusters)
    c.output_cluster_count = len(fmt.output_clusters)
    for i, v in enumerate(fmt.input_clusters):
        c.input_clusters[i] = int(v) & 0xFF
    for i, v in enumerate(fmt.output_clusters):
        c.output_clusters[i] = int(v) & 0xFF
    return c


_lib = None


def library() -> ctypes.CDLL:
    """Loads libbenes_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `python benes_perm_b200/build.py`"
            )
        lib = ctypes.CDLL(LIBRARY_PATH)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        fp = ctypes.POINTER(_Format)
        lib.bpb200_available.restype = ctypes.c_int
        lib.bpb200_backend_name.restype = ctypes.c_char_p
        lib.bpb200_encoded_size.argtypes = [ctypes.c_uint64, fp, ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.c_char_p, ctypes.c_size_t]
        lib.bpb200_compress.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, fp,
                                        u8p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_char_p, ctypes.c_size_t]
        lib.bpb200_compress_device.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                               fp, ctypes.c_void_p, ctypes.c_uint64,
                                               ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                               ctypes.c_char_p, ctypes.c_size_t]
        lib.bpb200_compress_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32,
                                             fp, ctypes.POINTER(ctypes.c_double),
                                             ctypes.c_char_p, ctypes.c_size_t]
        lib.bpb200_fill_permutation.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                                ctypes.c_uint32, ctypes.c_void_p]
        lib.bpb200_probe_switch_bit.argtypes = [ctypes.c_uint64, fp, ctypes.c_int, ctypes.c_uint32,
                                                ctypes.c_uint64, ctypes.c_uint64,
                                                ctypes.POINTER(ctypes.c_uint64)]
        lib.bpb200_probe_rank_bit.argtypes = [ctypes.c_uint64, fp, ctypes.c_uint32, ctypes.c_uint64,
                                              ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_uint64)]
        lib.bpb200_lookup_device.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                             fp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                             ctypes.c_size_t]
        lib.bpb200_probe_lookup.argtypes = [ctypes.c_uint64, fp, ctypes.c_char_p,
                                            ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_uint64)]
        lib.bpb200_shutdown.restype = None
        lib.bpb200_set_profiling.argtypes = [ctypes.c_int]
        lib.bpb200_set_profiling.restype = None
        lib.bpb200_last_profile.argtypes = [ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_uint32), ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_uint32)]
        lib.bpb200_describe.argtypes = [ctypes.c_uint64, fp, ctypes.POINTER(ctypes.c_uint32),
                                        ctypes.POINTER(ctypes.c_uint32)]
        lib.bpb200_last_profile_launches.argtypes = [ctypes.POINTER(ctypes.c_int),
                                                     ctypes.POINTER(ctypes.c_int),
                                                     ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        _lib = lib
    return _lib


def raise_for(code: int, message: str) -> None:
    if code == 0:
        return
    if code == 1:
        raise ValueError(message)
    if code == 2:
        raise OverflowError(message)
    if code == 3:
        raise LengthError(message)
    if code == 5:
        raise IndexError(message)
    raise RuntimeError(message or f"b200 backend error {code}")


def backend_available() -> bool:
    """backend_available(Backend::b200)."""
    try:
        return bool(library().bpb200_available())
    except OSError:
        return False


def backend_name() -> str:
    return library().bpb200_backend_name().decode()


def encoded_size(count: int, fmt: Optional[FormatOptions] = None) -> int:
    err = ctypes.create_string_buffer(256)
    out = ctypes.c_uint64(0)
    cf = to_c_format(fmt)
    raise_for(library().bpb200_encoded_size(count, ctypes.byref(cf), ctypes.byref(out), err, 256),
              err.value.decode())
    return out.value


_last_device_seconds = 0.0

_bytes_new = ctypes.pythonapi.PyBytes_FromStringAndSize
_bytes_new.restype = ctypes.py_object
_bytes_new.argtypes = [ctypes.c_void_p, ctypes.c_ssize_t]
_bytes_data = ctypes.pythonapi.PyBytes_AsString
_bytes_data.restype = ctypes.c_void_p
_bytes_data.argtypes = [ctypes.py_object]


def _fresh_bytes(size: int):
    """A new, not yet shared ``bytes`` object of ``size`` bytes and the address
    of its contents, for the library to write the blob into: the C-API idiom
    for building a bytes object in place, so the blob is not copied again
    (fresh host pages are expensive to fault in, once is enough)."""
    blob = _bytes_new(None, size)
    return blob, _bytes_data(blob)


def last_device_seconds() -> float:
    """detail::last_device_seconds() of the most recent compress call."""
    return _last_device_seconds


def compress(permutation, options: Optional[CompressOptions] = None,
             out: Optional[np.ndarray] = None):
    """benes::compress(span<const uint32_t|uint64_t>, {.backend = b200, ...}).

    ``permutation`` is a 1-D numpy array of uint32 or uint64 values.  Returns
    the canonical version-1 blob as ``bytes``; when ``out`` (a uint8 array of
    at least the encoded size, e.g. a view of pinned memory) is given, the
    blob is written there and the used slice of ``out`` is returned instead.
    """
    global _last_device_seconds
    options = options or CompressOptions()
    arr = np.ascontiguousarray(permutation)
    if arr.dtype not in (np.uint32, np.uint64):
        raise TypeError("permutation must be uint32 or uint64")
    if arr.ndim != 1:
        raise ValueError("permutation must be a one-dimensional array")
    n = int(arr.size)
    cf = to_c_format(options.format)
    err = ctypes.create_string_buffer(512)
    size = ctypes.c_uint64(0)
    if n == 0:
        raise ValueError("permutation size is out of range")
    raise_for(library().bpb200_encoded_size(n, ctypes.byref(cf), ctypes.byref(size), err, 512),
              err.value.decode())
    if out is not None:
        if out.dtype != np.uint8 or out.size < size.value or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous uint8 array of the encoded size")
        blob = out[:size.value]
        address = blob.ctypes.data
    else:
        blob, address = _fresh_bytes(size.value)
    secs = ctypes.c_double(0)
    rc = library().bpb200_compress(
        arr.ctypes.data, n, arr.dtype.itemsize, ctypes.byref(cf),
        ctypes.cast(address, ctypes.POINTER(ctypes.c_uint8)), size.value,
        ctypes.byref(secs), err, 512)
    raise_for(rc, err.value.decode())
    _last_device_seconds = secs.value
    return blob


def compress_file(input, output, input_width: InputValueWidth = InputValueWidth.bits64,
                  options: Optional[CompressOptions] = None) -> None:
    """benes::compress_file(input, output, input_width, {.backend = b200, ...})
    (src/benes.cpp:498-553): encodes a raw little-endian permutation file and
    writes the blob to ``output``.  The file is streamed to the device through
    pinned chunks; the output is created only after the encode succeeded."""
    global _last_device_seconds
    options = options or CompressOptions()
    cf = to_c_format(options.format)
    err = ctypes.create_string_buffer(512)
    secs = ctypes.c_double(0)
    rc = library().bpb200_compress_file(os.fsencode(input), os.fsencode(output),
                                        int(input_width), ctypes.byref(cf), ctypes.byref(secs),
                                        err, 512)
    raise_for(rc, err.value.decode())
    _last_device_seconds = secs.value


KERNEL_KINDS = ("prologue", "inverse", "descriptors", "union", "orient", "resolve",
                "output_bits", "tile", "emit", "walk", "jump", "place")


def set_profiling(enabled: bool) -> None:
    """Bracket every kernel launch of later calls with CUDA events."""
    library().bpb200_set_profiling(1 if enabled else 0)


def set_union_find_only(enabled) -> None:
    """Test hook: colour global levels with union-find instead of orbit walks
    (True), or run the walks and colour their levels with the union-find
    fallback anyway ("fallback"); False restores the default."""
    library().bpb200_set_colouring(2 if enabled == "fallback" else (1 if enabled else 0))


def last_profile():
    """(seconds by kernel kind, launches by kernel kind, total launches) of
    the calling thread's last compress call."""
    k = len(KERNEL_KINDS)
    secs = (ctypes.c_double * k)()
    counts = (ctypes.c_uint32 * k)()
    total = ctypes.c_uint32(0)
    library().bpb200_last_profile(secs, counts, k, ctypes.byref(total))
    return ({KERNEL_KINDS[i]: secs[i] for i in range(k)},
            {KERNEL_KINDS[i]: counts[i] for i in range(k)}, total.value)


def last_profile_launches():
    """[(kind name, routing level, seconds)] of every timed launch of the
    calling thread's last compress call (profiling must be enabled)."""
    lib = library()
    n = lib.bpb200_last_profile_launches(None, None, None, 0)
    kinds = (ctypes.c_int * max(n, 1))()
    levels = (ctypes.c_int * max(n, 1))()
    secs = (ctypes.c_double * max(n, 1))()
    lib.bpb200_last_profile_launches(kinds, levels, secs, n)
    return [(KERNEL_KINDS[kinds[i]], levels[i], secs[i]) for i in range(n)]


class Tuning(ctypes.Structure):
    """Launch choices of one size class (bpb200_tuning); none changes bytes."""
    _fields_ = [("walk_blocks_per_sm", ctypes.c_uint32), ("walk_max_log2", ctypes.c_uint32),
                ("jump_block_log2", ctypes.c_uint32), ("tile_max_log2", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


def get_tuning(count: int) -> dict:
    """The setting calls with ``count`` entries use (table or forced)."""
    lib = library()
    lib.bpb200_get_tuning.argtypes = [ctypes.c_uint64, ctypes.POINTER(Tuning)]
    t = Tuning()
    raise_for(lib.bpb200_get_tuning(count, ctypes.byref(t)), "invalid tuning query")
    return t.as_dict()


def set_tuning(setting: Optional[dict]) -> None:
    """Forces ``setting`` (a dict of Tuning fields; missing ones take the
    current table's value for 2^20 entries) for every later call, or returns
    to the table with None."""
    lib = library()
    lib.bpb200_set_tuning.argtypes = [ctypes.POINTER(Tuning)]
    if setting is None:
        lib.bpb200_set_tuning(None)
        return
    base = get_tuning(1 << 20)
    base.update(setting)
    t = Tuning(**base)
    lib.bpb200_set_tuning(ctypes.byref(t))


def probe_random_access(log2_words: int) -> dict:
    """Random 4-byte access rates (per second) of the GPU over an array of
    2^log2_words words: reads, writes and dependent chain steps."""
    lib = library()
    d = ctypes.c_double
    lib.bpb200_probe_random_access.argtypes = [ctypes.c_uint32, ctypes.POINTER(d),
                                               ctypes.POINTER(d), ctypes.POINTER(d)]
    r, w, c = d(0), d(0), d(0)
    raise_for(lib.bpb200_probe_random_access(log2_words, ctypes.byref(r), ctypes.byref(w),
                                             ctypes.byref(c)), "random-access probe failed")
    return {"reads_per_s": r.value, "writes_per_s": w.value, "chain_steps_per_s": c.value}


def describe(count: int, fmt: Optional[FormatOptions] = None):
    """(routing depth, first tile level) of the encode for (count, fmt)."""
    cf = to_c_format(fmt)
    d = ctypes.c_uint32(0)
    t = ctypes.c_uint32(0)
    raise_for(library().bpb200_describe(count, ctypes.byref(cf), ctypes.byref(d),
                                        ctypes.byref(t)), "invalid format")
    return d.value, t.value


def compress_device(d_entries: int, count: int, entry_bytes: int, d_blob: int, blob_len: int,
                    fmt: Optional[FormatOptions] = None, stream: int = 0) -> float:
    """Device-resident compress: device pointers in, device blob out.
    Returns device seconds."""
    cf = to_c_format(fmt)
    err = ctypes.create_string_buffer(512)
    secs = ctypes.c_double(0)
    rc = library().bpb200_compress_device(d_entries, count, entry_bytes, ctypes.byref(cf),
                                          d_blob, blob_len, stream, ctypes.byref(secs), err, 512)
    raise_for(rc, err.value.decode())
    return secs.value


def compress_device_shard(d_entries: int, count: int, entry_bytes: int, d_blob: int,
                          blob_len: int, shard: int, shards: int,
                          fmt: Optional[FormatOptions] = None, stream: int = 0) -> float:
    """One shard of a subtree-sharded compress (bpb200_compress_device_shard):
    the blob receives shard `shard`'s bits only; the byte-wise sum of all
    `shards` shards' blobs is the whole blob.  Returns device seconds."""
    lib = library()
    fp = ctypes.POINTER(_Format)
    lib.bpb200_compress_device_shard.argtypes = [
        ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, fp, ctypes.c_void_p, ctypes.c_uint64,
        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
        ctypes.c_char_p, ctypes.c_size_t]
    cf = to_c_format(fmt)
    err = ctypes.create_string_buffer(512)
    secs = ctypes.c_double(0)
    rc = lib.bpb200_compress_device_shard(d_entries, count, entry_bytes, ctypes.byref(cf), d_blob,
                                          blob_len, shard, shards, stream, ctypes.byref(secs),
                                          err, 512)
    raise_for(rc, err.value.decode())
    return secs.value


def combine_shards(blob, group=None, dst: int = 0):
    """Sums the shards' blobs (a uint8 tensor per rank, the same length on
    every rank) into rank `dst` over torch.distributed.  Every bit of the
    blob is set by at most one shard, so the byte-wise sum carries nothing
    and equals the OR of the shards: `dst` ends up with the whole blob.
    Works with the NCCL and the gloo backends."""
    import torch.distributed as dist
    dist.reduce(blob, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return blob


def compress_sharded(permutation, options: Optional[CompressOptions] = None, group=None):
    """Subtree-sharded compress of one host permutation over the ranks of a
    torch.distributed process group (one GPU each, the current device of
    every rank): each rank encodes its shard and the shards are combined on
    rank 0, which returns the blob bytes; the other ranks return None.  The
    world size must be a power of two."""
    import numpy as _np
    import torch
    import torch.distributed as dist
    options = options or CompressOptions()
    arr = _np.ascontiguousarray(permutation)
    if arr.dtype not in (_np.uint32, _np.uint64):
        raise TypeError("permutation must be uint32 or uint64")
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n = int(arr.size)
    size = encoded_size(n, options.format)
    width = arr.dtype.itemsize
    d_in = torch.from_numpy(arr.view(_np.int64 if width == 8 else _np.int32)).cuda()
    d_blob = torch.zeros((size + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    compress_device_shard(d_in.data_ptr(), n, width, d_blob.data_ptr(), size, rank, world,
                          options.format, stream)
    combine_shards(d_blob, group)
    return d_blob[:size].cpu().numpy().tobytes() if rank == 0 else None


class _Request(ctypes.Structure):
    _fields_ = [
        ("d_entries", ctypes.c_void_p),
        ("count", ctypes.c_uint64),
        ("entry_bytes", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("format", _Format),
        ("d_blob", ctypes.c_void_p),
        ("blob_len", ctypes.c_uint64),
        ("status", ctypes.c_int),
        ("error", ctypes.c_char * 124),
    ]


def compress_batch_device(items, stream: int = 0, raise_errors: bool = True):
    """Batched form: ``items`` is a list of
    (d_entries, count, entry_bytes, FormatOptions, d_blob, blob_len) with
    device pointers.  Returns (statuses, kernel launches); raises for the
    first failing request unless ``raise_errors`` is false."""
    lib = library()
    arr = (_Request * len(items))()
    for i, (d_in, n, width, fmt, d_blob, blob_len) in enumerate(items):
        arr[i].d_entries = d_in
        arr[i].count = n
        arr[i].entry_bytes = width
        arr[i].format = to_c_format(fmt)
        arr[i].d_blob = d_blob
        arr[i].blob_len = blob_len
    launches = ctypes.c_uint32(0)
    lib.bpb200_compress_batch.argtypes = [ctypes.POINTER(_Request), ctypes.c_uint32,
                                          ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]
    rc = lib.bpb200_compress_batch(arr, len(items), stream, ctypes.byref(launches))
    statuses = [arr[i].status for i in range(len(items))]
    if rc != 0 and raise_errors:
        bad = next(i for i, s in enumerate(statuses) if s != 0)
        raise_for(statuses[bad], arr[bad].error.decode())
    return statuses, launches.value


class _ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("submitted", "completed", "failed", "entries", "kernel_launches")] + \
               [(n, ctypes.c_double) for n in ("p50_seconds", "p99_seconds", "mean_seconds")]


class Server:
    """Serving form: a request loop with HBM-budget admission and continuous
    batching (bpb200_server_*).  ``submit`` returns a ticket; ``wait`` returns
    (blob bytes, latency seconds) and raises like ``compress`` on failure."""

    def __init__(self, hbm_budget_bytes: int = 120 * 10**9, max_batch: int = 256,
                 workers: int = 4):
        lib = library()
        lib.bpb200_server_create.restype = ctypes.c_void_p
        lib.bpb200_server_create.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_char_p, ctypes.c_size_t]
        lib.bpb200_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.POINTER(_Format),
                                             ctypes.c_void_p, ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_uint64)]
        lib.bpb200_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_double), ctypes.c_char_p,
                                           ctypes.c_size_t]
        lib.bpb200_server_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(_ServerStats)]
        lib.bpb200_server_destroy.argtypes = [ctypes.c_void_p]
        lib.bpb200_server_destroy.restype = None
        err = ctypes.create_string_buffer(256)
        self._lib = lib
        self._handle = lib.bpb200_server_create(int(hbm_budget_bytes), max_batch, workers, err, 256)
        if not self._handle:
            raise RuntimeError(err.value.decode() or "server creation failed")
        self._held = {}

    def submit(self, permutation, options: Optional[CompressOptions] = None) -> int:
        options = options or CompressOptions()
        arr = np.ascontiguousarray(permutation)
        if arr.dtype not in (np.uint32, np.uint64):
            raise TypeError("permutation must be uint32 or uint64")
        if arr.ndim != 1:
            raise ValueError("permutation must be a one-dimensional array")
        n = int(arr.size)
        if n == 0:
            raise ValueError("permutation size is out of range")
        size = encoded_size(n, options.format)
        blob, address = _fresh_bytes(size)
        cf = to_c_format(options.format)
        ticket = ctypes.c_uint64(0)
        rc = self._lib.bpb200_server_submit(self._handle, arr.ctypes.data, n, arr.dtype.itemsize,
                                            ctypes.byref(cf), address, size,
                                            ctypes.byref(ticket))
        raise_for(rc, "submit failed")
        self._held[ticket.value] = (arr, blob, cf)
        return ticket.value

    def wait(self, ticket: int):
        err = ctypes.create_string_buffer(256)
        latency = ctypes.c_double(0)
        rc = self._lib.bpb200_server_wait(self._handle, ticket, ctypes.byref(latency), err, 256)
        _, blob, _ = self._held.pop(ticket, (None, None, None))
        raise_for(rc, err.value.decode())
        return blob, latency.value

    def stats(self) -> dict:
        s = _ServerStats()
        self._lib.bpb200_server_get_stats(self._handle, ctypes.byref(s))
        return {n: getattr(s, n) for n, _ in _ServerStats._fields_}

    def close(self) -> None:
        if self._handle:
            self._lib.bpb200_server_destroy(self._handle)
            self._handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def fill_permutation(kind: PermutationKind, seed: int, count: int,
                     dtype=np.uint32, out: Optional[np.ndarray] = None) -> np.ndarray:
    """Seeded synthetic permutation (xoshiro256** from splitmix64(seed))."""
    dtype = np.dtype(dtype)
    if out is None:
        out = np.empty(count, dtype=dtype)
    rc = library().bpb200_fill_permutation(int(kind), seed & 0xFFFFFFFFFFFFFFFF, count,
                                           out.dtype.itemsize, out.ctypes.data)
    raise_for(rc, "invalid permutation request")
    return out


def probe_switch_bit(count: int, fmt: FormatOptions, side: int, level: int, node: int,
                     pair: int) -> int:
    cf = to_c_format(fmt)
    out = ctypes.c_uint64(0)
    rc = library().bpb200_probe_switch_bit(count, ctypes.byref(cf), side, level, node, pair,
                                           ctypes.byref(out))
    raise_for(rc, "no such switch")
    return out.value


def probe_rank_bit(count: int, fmt: FormatOptions, level: int, node: int):
    cf = to_c_format(fmt)
    sec = ctypes.c_int(0)
    out = ctypes.c_uint64(0)
    rc = library().bpb200_probe_rank_bit(count, ctypes.byref(cf), level, node, ctypes.byref(sec),
                                         ctypes.byref(out))
    raise_for(rc, "not a leaf")
    return sec.value, out.value


def lookup_device(d_blob: int, blob_len: int, count: int, fmt: Optional[FormatOptions],
                  d_out: int, query_count: int, d_queries: Optional[int] = None,
                  inverse: bool = False, stream: int = 0) -> None:
    """Batch lookup verifier on a device blob: d_out[i] (uint64) = p[q] or,
    with ``inverse``, p^-1[q], for q = d_queries[i] (uint64) or q = i when
    ``d_queries`` is None.  Raises IndexError for a query >= count."""
    cf = to_c_format(fmt)
    err = ctypes.create_string_buffer(512)
    rc = library().bpb200_lookup_device(d_blob, blob_len, count, ctypes.byref(cf), d_queries,
                                        query_count, 1 if inverse else 0, d_out, stream, err, 512)
    raise_for(rc, err.value.decode())


def probe_lookup(count: int, fmt: Optional[FormatOptions], blob: bytes, value: int,
                 inverse: bool = False) -> int:
    """Host evaluation of the verifier's per-query walk (test hook)."""
    cf = to_c_format(fmt)
    out = ctypes.c_uint64(0)
    rc = library().bpb200_probe_lookup(count, ctypes.byref(cf), blob, len(blob), value,
                                       1 if inverse else 0, ctypes.byref(out))
    raise_for(rc, "lookup failed")
    return out.value


def shutdown() -> None:
    library().bpb200_shutdown()
