"""jfx_sort_static, the sort entry point that allocates nothing, against
jfx_sort, both called through the C ABI.

Some callers of this library cannot allocate device memory: code that runs
inside an allocator or memory-pool callback (allocating there re-enters the
allocator), loops that must not take cudaMalloc's device-wide
synchronisation, and plugins whose host framework owns all device memory and
hands them only input and output buffers.  jfx_sort_static serves them from a
fixed 16 MiB device array inside the library, up to
JFX_SORT_STATIC_MAX_ROWS rows.  Its results must equal jfx_sort's bit for bit
(an order and the sorted keys: no tolerance), on consecutive calls that find
the previous call's data in the shared array.

The file name puts it last in collection, so a run that stops at the first
failure has already run every other test."""

import ctypes

import numpy as np
import pytest
import torch

from jaxframes_b200 import _lib

MAX_ROWS = _lib.SORT_STATIC_MAX_ROWS
SCRATCH_BYTES = 16 << 20


def _library():
    from jaxframes_b200 import build
    build.build()
    return _lib.load_library()


def test_rejects_more_rows_than_the_scratch_holds():
    """Host-side size check: no GPU work is started."""
    lib = _library()
    col = _lib.Column(None, _lib.I64, 0)
    st = lib.jfx_sort_static(ctypes.byref(col), MAX_ROWS + 1, 1, ctypes.c_void_p(8), None, None)
    assert st == -5 and b"at most" in lib.jfx_last_error()
    assert lib.jfx_sort_static(ctypes.byref(col), 0, 1, ctypes.c_void_p(8), None, None) == 0


def test_scratch_holds_the_largest_sort():
    """The sort buffers of MAX_ROWS rows fit the array (the sort workspace size
    also counts the lexsort's 4-byte row buffer, which this sort does not use)."""
    lib = _library()
    lexsort_extra = (4 * MAX_ROWS + 255) // 256 * 256
    assert lib.jfx_workspace_size(_lib.WS_SORT, MAX_ROWS, 0) - lexsort_extra <= SCRATCH_BYTES


def _run(lib, static, key, ascending):
    n = key.numel()
    perm = torch.full((n,), -1, dtype=torch.int32, device=key.device)
    out = torch.empty_like(key)
    col = _lib.column(key)
    stream = _lib.stream_handle()
    if static:
        st = lib.jfx_sort_static(ctypes.byref(col), n, int(ascending), perm.data_ptr(), out.data_ptr(), stream)
    else:
        ws = _lib.workspace(_lib.WS_SORT, n)
        st = lib.jfx_sort(ctypes.byref(col), n, int(ascending), perm.data_ptr(), out.data_ptr(),
                          ws.data_ptr(), ws.numel(), stream)
    _lib.check(st)
    torch.cuda.synchronize()
    return perm.cpu().numpy(), out.cpu().numpy()


def _cases():
    rng = np.random.default_rng(71)
    # largest size, 64-bit keys with many duplicates, ascending
    k1 = rng.integers(-(1 << 40), 1 << 40, MAX_ROWS, dtype=np.int64)
    k1[::5] = k1[7]
    # ragged size, float keys with NaN, -0.0 and +0.0, descending
    k2 = rng.standard_normal(300_001).astype(np.float32)
    k2[::97] = np.nan
    k2[1::89] = -0.0
    k2[2::89] = 0.0
    # small int32 call after the large ones (stale data in the array)
    k3 = rng.integers(-1000, 1000, 1003, dtype=np.int64).astype(np.int32)
    # descending integer keys (the whole order reversed, ties included)
    k4 = rng.integers(-(1 << 50), 1 << 50, 200_003, dtype=np.int64)
    k4[::3] = k4[11]
    k5 = rng.integers(-50_000, 50_000, MAX_ROWS, dtype=np.int64).astype(np.int32)
    return [(k1, True), (k2, False), (k3, True), (k4, False), (k5, False)]


@pytest.mark.gpu
def test_static_sort_matches_workspace_sort_on_consecutive_calls():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    lib = _library()
    for key_np, ascending in _cases():
        key = torch.from_numpy(key_np).cuda()
        want_perm, want_keys = _run(lib, False, key, ascending)
        for _ in range(2):  # two calls in a row on the same shared array
            perm, keys = _run(lib, True, key, ascending)
            np.testing.assert_array_equal(perm, want_perm)
            # bit patterns, so NaN and the sign of zero compare exactly
            np.testing.assert_array_equal(keys.view(np.uint8), want_keys.view(np.uint8))
        assert np.array_equal(np.sort(perm), np.arange(len(key_np)))  # a permutation


@pytest.mark.gpu
def test_static_sort_matches_the_oracle():
    """One case straight against the oracle's restatement of
    ParallelRadixSort.sort (parallel_algorithms.py:463-581)."""
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from oracle import jfx_oracle as O
    lib = _library()
    rng = np.random.default_rng(72)
    for ascending in (True, False):
        key_np = rng.integers(-(1 << 33), 1 << 33, 250_007, dtype=np.int64)
        key_np[::4] = key_np[5]
        perm, keys = _run(lib, True, torch.from_numpy(key_np).cuda(), ascending)
        want_keys, want_perm = O.radix_sort(key_np, np.arange(len(key_np)), ascending=ascending)
        np.testing.assert_array_equal(perm, want_perm)
        np.testing.assert_array_equal(keys, want_keys)
