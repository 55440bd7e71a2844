"""Error paths of the C ABI, exercised without faulting a GPU.

Failures are injected on the host (jfx_set_fault) or by a bounded device-side
wait that is made to run out: a look-back tile that never publishes its
counts, with a short wait limit, so the later tiles give up, the kernel
returns and the call reports JFX_ERR_TIMEOUT; the context stays usable and
the next call is correct.  The reference's own error convention (ValueError
for an unknown aggregation, parallel_algorithms.py:660 and :1228) is covered
by the known-answer tests."""

import contextlib
import ctypes

import numpy as np
import pytest
import torch

from jaxframes_b200 import _lib

ALLOC, TIMEOUT, CAPACITY, ARG = -3, -4, -5, -1


@pytest.fixture(scope="module")
def lib():
    from jaxframes_b200 import build
    build.build()
    return _lib.load_library()


@contextlib.contextmanager
def fault(lib, withhold_tile=0, learned_fallback=0, fail_workspace=0, withhold_order=0):
    f = _lib.Fault(withhold_tile, learned_fallback, fail_workspace, withhold_order)
    _lib.check(lib.jfx_set_fault(ctypes.byref(f)))
    try:
        yield
    finally:
        _lib.check(lib.jfx_set_fault(None))


@contextlib.contextmanager
def spin_limit(lib, us):
    old = _lib.Tuning()
    _lib.check(lib.jfx_get_tuning(ctypes.byref(old)))
    new = _lib.Tuning(old.max_digit_bits, old.two_phase, us, 0)
    _lib.check(lib.jfx_set_tuning(ctypes.byref(new)))
    try:
        yield
    finally:
        _lib.check(lib.jfx_set_tuning(ctypes.byref(old)))


# ------------------------------------------------------------ host only ---
def test_fault_and_tuning_arguments_are_checked(lib):
    assert lib.jfx_set_fault(ctypes.byref(_lib.Fault(-1, 0, 0, 0))) == ARG
    assert lib.jfx_set_fault(ctypes.byref(_lib.Fault(0, -7, 0, 0))) == ARG
    assert lib.jfx_set_fault(ctypes.byref(_lib.Fault(0, -2, 0, 0))) == ARG
    assert lib.jfx_set_fault(ctypes.byref(_lib.Fault(0, 0, 2, 0))) == ARG
    assert lib.jfx_set_fault(ctypes.byref(_lib.Fault(0, 0, 0, 2))) == ARG
    assert lib.jfx_set_fault(None) == 0
    t = _lib.Tuning()
    assert lib.jfx_get_tuning(ctypes.byref(t)) == 0
    assert t.spin_limit_us == 1_000_000  # 1 s by default
    for bad in (0, 10_000_001):
        assert lib.jfx_set_tuning(ctypes.byref(_lib.Tuning(t.max_digit_bits, t.two_phase, bad, 0))) == ARG
    assert lib.jfx_set_tuning(None) == 0


def test_injected_workspace_failure_stops_before_any_launch(lib):
    """Every workspace-taking entry point checks the workspace on the host,
    before it touches the device, so this runs without a GPU."""
    fake = ctypes.c_void_p(1 << 40)  # never dereferenced: the check comes first
    col = _lib.Column(fake, _lib.I64, 0)
    launches = lib.jfx_launch_count()
    with fault(lib, fail_workspace=1):
        st = lib.jfx_sort(ctypes.byref(col), 1000, 1, fake, None, fake, 1 << 30, None)
        assert st == ALLOC and b"injected" in lib.jfx_last_error()
        assert lib.jfx_lexsort(ctypes.byref(col), 1, 1000, fake, fake, 1 << 30, None) == ALLOC
        g = ctypes.c_int64(0)
        assert lib.jfx_groupby(ctypes.byref(col), 1, 1000, 0, None, 0, None, ctypes.byref(g), fake, 1 << 30,
                               None) == ALLOC
        assert lib.jfx_hash_partition(ctypes.byref(col), 1, 1000, 16, fake, fake, fake, fake, 1 << 30, None) == ALLOC
        assert lib.jfx_learned_sort(fake, 1000, fake, fake, 0, None, fake, 1 << 30, None) == ALLOC
    assert lib.jfx_launch_count() == launches


def test_misaligned_workspace_is_rejected_before_any_launch(lib):
    """The workspace carve hands out 256-byte offsets and kernels load 16-byte
    vectors from them: a base that is not 256-byte aligned is an argument
    error, found on the host before the device is touched."""
    fake = ctypes.c_void_p(1 << 40)
    bad = ctypes.c_void_p((1 << 40) + 16)
    col = _lib.Column(fake, _lib.I64, 0)
    launches = lib.jfx_launch_count()
    assert lib.jfx_sort(ctypes.byref(col), 1000, 1, fake, None, bad, 1 << 30, None) == ARG
    assert b"aligned" in lib.jfx_last_error()
    assert lib.jfx_learned_sort(fake, 1000, fake, fake, 0, None, bad, 1 << 30, None) == ARG
    assert lib.jfx_launch_count() == launches


# ------------------------------------------------------------------ GPU ---
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")


def _sort(lib, key, ascending=True):
    n = key.numel()
    perm = torch.full((n,), -1, dtype=torch.int32, device=key.device)
    ws = _lib.workspace(_lib.WS_SORT, n)
    col = _lib.column(key)
    st = lib.jfx_sort(ctypes.byref(col), n, int(ascending), perm.data_ptr(), None, ws.data_ptr(), ws.numel(),
                      _lib.stream_handle())
    torch.cuda.synchronize()
    return st, perm


@pytest.mark.gpu
def test_look_back_wait_runs_out_and_the_call_reports_a_timeout(lib):
    """A float key's first radix pass resolves its tile offsets by decoupled
    look-back.  Tile 5 withholds its counts; the later tiles wait 2 ms at most,
    record the timeout and exit, and jfx_sort returns JFX_ERR_TIMEOUT."""
    _need_gpu()
    from oracle import jfx_oracle as O
    rng = np.random.default_rng(81)
    key_np = rng.standard_normal(400_000).astype(np.float32)
    key = torch.from_numpy(key_np).cuda()
    with spin_limit(lib, 2000), fault(lib, withhold_tile=5):
        st, _ = _sort(lib, key)
    assert st == TIMEOUT, (st, lib.jfx_last_error())
    assert b"wait" in lib.jfx_last_error()
    # the context is usable and the next call is correct
    st, perm = _sort(lib, key)
    assert st == 0
    np.testing.assert_array_equal(perm.cpu().numpy(), O.radix_sort(key_np, np.arange(len(key_np)))[1])


@pytest.mark.gpu
def test_timeout_surfaces_as_a_python_error(lib):
    _need_gpu()
    import jaxframes_b200.parallel_algorithms as P
    key = torch.from_numpy(np.random.default_rng(82).standard_normal(300_000).astype(np.float32)).cuda()
    with spin_limit(lib, 2000), fault(lib, withhold_tile=3):
        with pytest.raises(_lib.JfxError) as e:
            P.ParallelRadixSort().sort(key)
    assert e.value.status == TIMEOUT
    sk, _ = P.ParallelRadixSort().sort(key)
    assert bool((sk[1:] >= sk[:-1]).all())


@pytest.mark.gpu
def test_withheld_publication_with_a_generous_limit_still_times_out_not_hangs(lib):
    """An integer key with two_phase off: every pass uses the look-back."""
    _need_gpu()
    key = torch.from_numpy(np.random.default_rng(83).integers(0, 1 << 40, 300_000)).cuda()
    old = _lib.Tuning()
    _lib.check(lib.jfx_get_tuning(ctypes.byref(old)))
    _lib.check(lib.jfx_set_tuning(ctypes.byref(_lib.Tuning(old.max_digit_bits, 0, 20_000, 0))))
    try:
        with fault(lib, withhold_tile=1):
            st, _ = _sort(lib, key)
        assert st == TIMEOUT
        st, perm = _sort(lib, key)
        assert st == 0
    finally:
        _lib.check(lib.jfx_set_tuning(ctypes.byref(old)))
    want = np.argsort(key.cpu().numpy(), kind="stable")
    np.testing.assert_array_equal(perm.cpu().numpy(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("why", [-1, -3])
def test_forced_learned_fallback_gives_the_plain_sort(lib, why):
    _need_gpu()
    import jaxframes_b200.parallel_algorithms as P
    rng = np.random.default_rng(84)
    keys = torch.from_numpy(rng.lognormal(20, 2, 1 << 20).astype(np.uint64)).cuda()
    plain_k, plain_p, used0 = P.learned_sort(keys, mode="plain")
    assert used0 == 0
    with fault(lib, learned_fallback=why):
        k, p, used = P.learned_sort(keys)
    assert used == why
    assert torch.equal(k, plain_k) and torch.equal(p, plain_p)


@pytest.mark.gpu
def test_injected_workspace_failure_on_the_device_path(lib):
    _need_gpu()
    import jaxframes_b200.parallel_algorithms as P
    k = torch.arange(1000, dtype=torch.int32, device="cuda")
    with fault(lib, fail_workspace=1):
        with pytest.raises(_lib.JfxError) as e:
            P.groupby_aggregate(k, {"v": k.float()}, {"v": "sum"})
    assert e.value.status == ALLOC
    uk, out = P.groupby_aggregate(k, {"v": k.float()}, {"v": "sum"})
    assert uk.numel() == 1000


@pytest.mark.gpu
def test_short_output_capacity_is_reported(lib):
    """jfx_join_unmatched checks the caller's capacity against the count."""
    _need_gpu()
    import jaxframes_b200.parallel_algorithms as P
    lk = torch.arange(100, dtype=torch.int64, device="cuda")
    rk = torch.arange(50, 80, dtype=torch.int64, device="cuda")
    plan, m, ws = P._join_prepare([lk], [rk], "outer")
    out = torch.empty(100, dtype=torch.int32, device="cuda")
    cnt = ctypes.c_int64(0)
    st = lib.jfx_join_unmatched(ctypes.byref(plan), 0, out.data_ptr(), 10, ctypes.byref(cnt), _lib.stream_handle())
    assert st == CAPACITY and cnt.value == 70
    st = lib.jfx_join_unmatched(ctypes.byref(plan), 0, out.data_ptr(), 100, ctypes.byref(cnt), _lib.stream_handle())
    assert st == 0 and cnt.value == 70
    want = np.r_[np.arange(50), np.arange(80, 100)]
    np.testing.assert_array_equal(out[:70].cpu().numpy(), want)
    del ws


@pytest.mark.gpu
def test_withheld_batch_order_times_out_and_the_next_batch_is_correct(lib):
    """Every CTA of the batch kernel waits for the query order CTA 0
    publishes; when it is withheld, their bounded waits run out, the kernel
    exits and the status reports JFX_ERR_TIMEOUT.  The next batch on the same
    buffers is correct."""
    _need_gpu()
    from jaxframes_b200.batch import BatchedGroupBy
    from oracle import jfx_oracle as O
    rng = np.random.default_rng(91)
    nq = 16
    off = np.zeros(nq + 1, dtype=np.int64)
    off[1:] = np.cumsum(rng.integers(100, 5000, nq))
    n = int(off[-1])
    keys = rng.integers(0, 1000, n).astype(np.int32)
    vals = rng.standard_normal(n).astype(np.float32)
    b = BatchedGroupBy(n, nq, 64, 10)
    b.keys[:n].copy_(torch.from_numpy(keys))
    b.values[:n].copy_(torch.from_numpy(vals))
    b.query_offsets.copy_(torch.from_numpy(off))
    with spin_limit(lib, 2000), fault(lib, withhold_order=1):
        b.run()
        with pytest.raises(_lib.JfxError) as e:
            b.status()
    assert e.value.status == TIMEOUT
    b.run()
    b.status()
    for q in range(nq):
        k, v = keys[off[q]:off[q + 1]], vals[off[q]:off[q + 1]]
        po, pk, pv, gk, gs, gc = (t.cpu().numpy() for t in b.query(q))
        _, perm, eoffs = O.hash_partition([k], 64)
        assert np.array_equal(po, eoffs) and np.array_equal(pk, k[perm]) and np.array_equal(pv, v[perm])
        ek, eo = O.groupby_aggregate(k, {"s": v, "c": v}, {"s": "sum", "c": "count"})
        assert np.array_equal(gk, ek) and np.array_equal(gc, eo["c"])
        np.testing.assert_allclose(gs, eo["s"], rtol=1e-5, atol=1e-4)
