# SPDX-License-Identifier: Apache-2.0
"""The allocation-free entry point, bpb200_compress_device_noalloc.

It exists for callers that cannot call cudaMalloc (device memory owned by a
pooling allocator, latency-critical paths that cannot pay for an
allocation's synchronisation): its scratch is a fixed device array inside
the library.  This test calls it through the C ABI and checks that two
calls in a row produce exactly the bytes of the allocating entry point,
bpb200_compress_device (the bar is byte equality: the encoding is integer
work), that a non-permutation is still rejected when the shared scratch
holds an earlier call's data, and that sizes above its 2^18-entry limit are
rejected.  The file sorts last so a failing run that
stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ENTRIES = 1 << 18


def _entry(lib):
    fn = lib.bpb200_compress_device_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_char_p,
                   ctypes.c_size_t]
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.parametrize("n,kind,dtype,fmt_kw", [
    (MAX_ENTRIES, 0, np.uint64, dict(middle_group_log2=5, middle_placement=2)),
    (200_003, 1, np.uint32, dict(middle_group_log2=4, middle_placement=0)),
    (70_001, 0, np.uint32, dict(middle_group_log2=3, middle_placement=1)),
    (5_000, 0, np.uint64, dict()),
    (31, 3, np.uint32, dict()),
])
def test_noalloc_matches_allocating_entry_point(gpu, n, kind, dtype, fmt_kw):
    torch = pytest.importorskip("torch")
    fn = _entry(gpu.library())
    fmt = gpu.FormatOptions(middle_group_log2=fmt_kw.get("middle_group_log2", 5),
                            middle_placement=gpu.MiddlePlacement(fmt_kw.get("middle_placement", 0)))
    perm = gpu.fill_permutation(gpu.PermutationKind(kind), 0xA110C + n, n, dtype)
    size = gpu.encoded_size(n, fmt)
    width = np.dtype(dtype).itemsize
    d_in = torch.from_numpy(perm.view(np.int64 if width == 8 else np.int32)).cuda()
    padded = (size + 3) // 4 * 4
    expected = torch.empty(padded, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    gpu.compress_device(d_in.data_ptr(), n, width, expected.data_ptr(), size, fmt, stream)
    want = expected[:size].cpu().numpy().tobytes()

    cfmt = gpu.to_c_format(fmt)
    err = ctypes.create_string_buffer(256)
    for _ in range(2):  # two calls in a row reuse the same scratch array
        out = torch.full((padded,), 0xAB, dtype=torch.uint8, device="cuda")
        rc = fn(d_in.data_ptr(), n, width, ctypes.byref(cfmt), out.data_ptr(), size, stream,
                err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        assert out[:size].cpu().numpy().tobytes() == want


def test_noalloc_rejects_duplicate_after_valid_call(gpu):
    # the scratch keeps the previous call's inverse and status word: the
    # per-call reset of both must still catch a repeated value
    torch = pytest.importorskip("torch")
    fn = _entry(gpu.library())
    stream = torch.cuda.current_stream().cuda_stream
    err = ctypes.create_string_buffer(256)
    for n, dtype in ((100_003, np.uint32), (MAX_ENTRIES, np.uint64), (4_000, np.uint32)):
        fmt = gpu.FormatOptions()
        cfmt = gpu.to_c_format(fmt)
        size = gpu.encoded_size(n, fmt)
        width = np.dtype(dtype).itemsize
        view = np.int64 if width == 8 else np.int32
        good = gpu.fill_permutation(gpu.PermutationKind.uniform, 0xD0B + n, n, dtype)
        bad = good.copy()
        bad[n // 3] = bad[n // 2]
        want = torch.empty((size + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
        d_good = torch.from_numpy(good.view(view)).cuda()
        gpu.compress_device(d_good.data_ptr(), n, width, want.data_ptr(), size, fmt, stream)
        out = torch.empty_like(want)
        for d_in, rc_want in ((d_good, 0), (torch.from_numpy(bad.view(view)).cuda(), 1),
                              (d_good, 0)):
            rc = fn(d_in.data_ptr(), n, width, ctypes.byref(cfmt), out.data_ptr(), size, stream,
                    err, 256)
            assert rc == rc_want, (n, err.value.decode())  # 1 = BPB200_INVALID_ARGUMENT
            if rc == 0:
                torch.cuda.synchronize()
                assert torch.equal(out[:size], want[:size])


def test_noalloc_rejects_oversized_input(gpu):
    torch = pytest.importorskip("torch")
    fn = _entry(gpu.library())
    n = MAX_ENTRIES + 1
    fmt = gpu.FormatOptions()
    size = gpu.encoded_size(n, fmt)
    d_in = torch.arange(n, dtype=torch.int32, device="cuda")
    out = torch.empty((size + 3) // 4 * 4, dtype=torch.uint8, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = fn(d_in.data_ptr(), n, 4, ctypes.byref(gpu.to_c_format(fmt)), out.data_ptr(), size,
            torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 3  # BPB200_LENGTH
    assert b"262144" in err.value
