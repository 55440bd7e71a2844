"""The oracle against the reference tests' known answers (CPU only)."""

import numpy as np
import pytest

from oracle import jfx_oracle as O
from _kat import check_kat, load_kats

KATS = load_kats()


class OracleImpl:
    @staticmethod
    def parallel_sort(keys, values, ascending):
        return O.radix_sort(keys, values, ascending)

    @staticmethod
    def lexsort(keys, ascending):
        return O.multi_column_lexsort(keys, ascending)

    @staticmethod
    def groupby(keys, values, aggs):
        return O.groupby_aggregate(keys, values, aggs)

    @staticmethod
    def groupby_multi(keys, names, values, aggs):
        return O.groupby_aggregate_multi_column(keys, names, values, aggs)

    @staticmethod
    def join(lk, lv, rk, rv, how):
        mk, out, _, _ = O.sort_merge_join(lk, lv, rk, rv, how)
        return mk, out

    @staticmethod
    def join_multi(lk, rk, how):
        return O.join_multi_column(lk, rk, how)

    @staticmethod
    def hash(keys):
        return O.hash_multi_columns(keys)

    @staticmethod
    def partition(keys, p):
        return O.hash_partition(keys, p)


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_oracle_kat(kat):
    check_kat(kat, OracleImpl)


def test_inner_join_matches_broadcast_matrix():
    """The run-expansion restatement equals the reference's nL x nR matrix form
    (parallel_algorithms.py:987-994) on random small inputs with duplicates."""
    rng = np.random.default_rng(3)
    for trial in range(20):
        lk = rng.integers(0, 12, rng.integers(0, 40)).astype(np.int32)
        rk = rng.integers(0, 12, rng.integers(0, 40)).astype(np.int32)
        li, ri, sl, pl, sr, pr = O.inner_join_pairs(lk, rk)
        m = sl[:, None] == sr[None, :]
        a, b = np.nonzero(m)
        np.testing.assert_array_equal(li, a)
        np.testing.assert_array_equal(ri, b)


def test_radix_order_matches_lsd_passes():
    """The restated order equals literally running 8-bit stable LSD passes on
    the sign-flipped key (parallel_algorithms.py:495-549)."""
    rng = np.random.default_rng(5)
    for dt in (np.int32, np.int64, np.uint32):
        info = np.iinfo(dt)
        k = rng.integers(info.min, info.max, 500, dtype=dt, endpoint=True)
        k[::7] = k[3]
        t = O._radix_order_key(k).astype(np.uint64)
        perm = np.arange(len(k))
        bits = np.dtype(dt).itemsize * 8
        for p in range(bits // 8):
            d = (t[perm] >> np.uint64(8 * p)) & np.uint64(255)
            perm = perm[np.argsort(d, kind="stable")]
        sk, sv = O.radix_sort(k, np.arange(len(k)))
        np.testing.assert_array_equal(sv, perm)


def test_narrow_signed_keys_order_as_unsigned_pattern():
    """int16 keys are not sign-flipped by the reference (line 495-501), so
    negatives sort after non-negatives."""
    k = np.array([-1, 3, -5, 0], dtype=np.int16)
    sk, _ = O.radix_sort(k)
    np.testing.assert_array_equal(sk, [0, 3, -5, -1])


def test_float_keys_nan_last_and_signed_zero_equal():
    k = np.array([np.nan, 1.0, -0.0, 0.0, -np.inf, np.nan, -0.0], dtype=np.float32)
    sk, sv = O.radix_sort(k, np.arange(len(k)))
    np.testing.assert_array_equal(sv, [4, 2, 3, 6, 1, 0, 5])
    sk, sv = O.radix_sort(k, np.arange(len(k)), ascending=False)
    np.testing.assert_array_equal(sv, [5, 0, 1, 6, 3, 2, 4])


def test_groupby_nan_keys_are_singletons():
    k = np.array([np.nan, 1.0, np.nan, 1.0], dtype=np.float32)
    uk, out = O.groupby_aggregate(k, {"v": np.arange(4, dtype=np.int32)}, {"v": "count"})
    assert len(uk) == 3
    np.testing.assert_array_equal(out["v"], [2, 1, 1])


def test_empty_inputs():
    uk, out = O.groupby_aggregate(np.zeros(0, np.int32), {"v": np.zeros(0, np.float32)}, {"v": "sum"})
    assert len(uk) == 0 and len(out["v"]) == 0
    mk, out, li, ri = O.sort_merge_join(np.zeros(0, np.int32), {}, np.arange(3, dtype=np.int32), {})
    assert len(mk) == 0


def test_unknown_agg_raises():
    with pytest.raises(ValueError):
        O.groupby_aggregate(np.arange(3), {"v": np.arange(3)}, {"v": "median"})
