# SPDX-License-Identifier: Apache-2.0
"""compress_file: the file form of the encoder.

Mirrors the reference's raw-file round trip (tests/test_benes.cpp:533-565):
a permutation written as little-endian u32 or u64 values and encoded from the
file must give the same bytes as the in-memory encode, and the error cases of
benes::compress_file (src/benes.cpp:503-552) keep their exception types and
messages.  The file-level checks (open, width, size) run before any device
work, so they are tested on the CPU too.
"""
import numpy as np
import pytest

from helpers import oracle_format


def _write(path, values, dtype):
    np.asarray(values).astype(dtype).tofile(path)
    return path


def test_missing_input_file(b200, tmp_path):
    with pytest.raises(RuntimeError, match="cannot open permutation input file"):
        b200.compress_file(tmp_path / "absent.bin", tmp_path / "out.benes")
    assert not (tmp_path / "out.benes").exists()


@pytest.mark.parametrize("raw,width", [(b"", 8), (b"\x00" * 5, 4), (b"\x00" * 12, 8),
                                       (b"\x00" * 8, 3), (b"\x00" * 8, 0)])
def test_invalid_width_or_size(b200, tmp_path, raw, width):
    src = tmp_path / "in.bin"
    src.write_bytes(raw)
    with pytest.raises(ValueError, match="invalid element width or size"):
        b200.compress_file(src, tmp_path / "out.benes", width)
    assert not (tmp_path / "out.benes").exists()


def test_file_without_gpu_reports_unavailable(b200, tmp_path):
    if b200.backend_available():
        pytest.skip("a GPU is present")
    src = _write(tmp_path / "in.bin", np.arange(16), "<u4")
    with pytest.raises(RuntimeError, match="unavailable"):
        b200.compress_file(src, tmp_path / "out.benes", b200.InputValueWidth.bits32)
    assert not (tmp_path / "out.benes").exists()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 33, 1000, 65536])
@pytest.mark.parametrize("width", [4, 8])
def test_file_matches_oracle(gpu, oracle, tmp_path, n, width):
    rng = np.random.default_rng(n * 7 + width)
    perm = rng.permutation(n)
    src = _write(tmp_path / "in.bin", perm, "<u4" if width == 4 else "<u8")
    out = tmp_path / "out.benes"
    gpu.compress_file(src, out, width)
    assert out.read_bytes() == oracle.compress(perm.astype(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("n,width,m,placement", [
    ((1 << 23) + 5, 8, 5, 2),        # 64 MB: several pinned chunks, ragged tail
    (5_000_011, 4, 4, 0),
    ((1 << 22), 4, 5, 1),
])
def test_file_matches_memory_encode(gpu, oracle, tmp_path, n, width, m, placement):
    """Multi-chunk files: the streamed upload and download give the bytes of
    the in-memory encode of the same values, and (one size) of the oracle."""
    dtype = np.uint32 if width == 4 else np.uint64
    perm = gpu.fill_permutation(gpu.PermutationKind.uniform, n, n, dtype)
    src = tmp_path / "in.bin"
    perm.astype("<u4" if width == 4 else "<u8").tofile(src)
    opts = gpu.CompressOptions(format=gpu.FormatOptions(
        middle_group_log2=m, middle_placement=gpu.MiddlePlacement(placement)))
    out = tmp_path / "out.benes"
    out.write_bytes(b"\xff" * 64)  # a longer stale file must be truncated
    gpu.compress_file(src, out, width, opts)
    assert out.read_bytes() == gpu.compress(perm, opts)
    assert gpu.last_device_seconds() > 0
    if n == 5_000_011:
        assert out.read_bytes() == oracle.compress(
            perm, oracle_format(dict(middle_group_log2=m, middle_placement=placement)))


@pytest.mark.gpu
def test_file_non_permutation_leaves_no_output(gpu, tmp_path):
    perm = np.arange(5000, dtype=np.uint64)
    perm[17] = perm[4000]
    src = _write(tmp_path / "in.bin", perm, "<u8")
    out = tmp_path / "out.benes"
    with pytest.raises(ValueError, match="every value from zero"):
        gpu.compress_file(src, out, gpu.InputValueWidth.bits64)
    assert not out.exists()


@pytest.mark.gpu
def test_file_u32_u64_identical(gpu, oracle, tmp_path):
    """A u32 file and a u64 file of the same values give the same blob
    (tests/test_benes.cpp:230-266 for the in-memory spans)."""
    perm = np.random.default_rng(5).permutation(70001)
    a = tmp_path / "a.benes"
    b = tmp_path / "b.benes"
    gpu.compress_file(_write(tmp_path / "u32.bin", perm, "<u4"), a, 4)
    gpu.compress_file(_write(tmp_path / "u64.bin", perm, "<u8"), b, 8)
    assert a.read_bytes() == b.read_bytes() == oracle.compress(perm.astype(np.uint64))
