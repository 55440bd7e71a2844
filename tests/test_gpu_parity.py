"""GPU parity: the product API (through libjfx.so) against the oracle and the
reference tests' known answers.  Bit-exact for orders, keys, counts, min/max,
index pairs and partition assignments; float sums within 2^-16 * sum(|x|)
per group (the tolerance stated for float32 sums and means)."""

import numpy as np
import pytest
import torch

from oracle import jfx_oracle as O
from _kat import check_kat, load_kats

pytestmark = pytest.mark.gpu

KATS = load_kats()


def _np(t):
    if isinstance(t, torch.Tensor):
        t = t.cpu()
        if t.dtype in (torch.uint16, torch.uint32, torch.uint64):
            return t.numpy()
        return t.numpy()
    return np.asarray(t)


@pytest.fixture(scope="module")
def P():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jaxframes_b200 import build
    build.build()
    import jaxframes_b200.parallel_algorithms as P
    return P


class ProductImpl:
    def __init__(self, P):
        self.P = P

    def parallel_sort(self, keys, values, ascending):
        if values is None:
            return _np(self.P.parallel_sort(keys, ascending=ascending)), None
        sk, sv = self.P.parallel_sort(keys, values=values, ascending=ascending)
        return _np(sk), _np(sv)

    def lexsort(self, keys, ascending):
        return _np(self.P.multi_column_lexsort(keys, ascending))

    def groupby(self, keys, values, aggs):
        uk, out = self.P.groupby_aggregate(keys, values, aggs)
        return _np(uk), {c: _np(v) for c, v in out.items()}

    def groupby_multi(self, keys, names, values, aggs):
        uk, out = self.P.groupby_aggregate_multi_column(keys, names, values, aggs)
        return {n: _np(v) for n, v in uk.items()}, {c: _np(v) for c, v in out.items()}

    def join(self, lk, lv, rk, rv, how):
        mk, out = self.P.sort_merge_join(lk, lv, rk, rv, how)
        return _np(mk), {c: _np(v) for c, v in out.items()}

    def join_multi(self, lk, rk, how):
        j = self.P.ParallelSortMergeJoin()
        li, ri = j.join_multi_indices(lk, rk, how)
        return _np(li), _np(ri)

    def hash(self, keys):
        return _np(self.P.hash_multi_columns(keys))

    def partition(self, keys, p):
        t, perm, offs = self.P.hash_partition(keys, p)
        return _np(t), _np(perm), _np(offs)


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_product_kat(P, kat):
    check_kat(kat, ProductImpl(P))


# ----------------------------------------------------------------- sorting ---
SIZES = [1, 2, 31, 32, 33, 255, 4095, 4096, 4097, 8191, 8192, 8193, 100_000, 1_000_003]


def _keys(rng, dt, n, kind):
    info = np.iinfo(dt) if np.issubdtype(dt, np.integer) else None
    if kind == "full":
        if info is not None:
            return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
        x = rng.standard_normal(n).astype(dt) * 1e3
        x[rng.integers(0, n, max(1, n // 50))] = np.nan
        x[rng.integers(0, n, max(1, n // 50))] = -0.0
        x[rng.integers(0, n, max(1, n // 50))] = 0.0
        x[rng.integers(0, n, max(1, n // 100))] = np.inf
        return x
    if kind == "small":
        return rng.integers(0, 7, n).astype(dt)
    if kind == "equal":
        return np.full(n, 5, dtype=dt)
    if kind == "desc":
        return np.arange(n, 0, -1).astype(dt)
    if kind == "heavy":
        x = rng.integers(0, 1 << 20, n).astype(dt)
        x[rng.random(n) < 0.6] = 12345
        return x
    raise ValueError(kind)


@pytest.mark.parametrize("dt", [np.int32, np.int64, np.uint32, np.uint64, np.float32, np.float64, np.int16])
@pytest.mark.parametrize("kind", ["full", "small", "equal", "desc", "heavy"])
def test_radix_sort_matches_oracle(P, dt, kind):
    rng = np.random.default_rng(hash((np.dtype(dt).name, kind)) & 0xffff)
    for n in SIZES:
        k = _keys(rng, dt, n, kind)
        for asc in (True, False):
            sk, perm = P.ParallelRadixSort().sort(k, np.arange(n, dtype=np.int32), asc)
            ek, ep = O.radix_sort(k, np.arange(n), asc)
            np.testing.assert_array_equal(_np(perm), ep, err_msg=f"n={n} asc={asc}")
            np.testing.assert_array_equal(_np(sk).view(np.uint8), ek.view(np.uint8), err_msg=f"n={n}")


@pytest.mark.parametrize("two_phase", [0, 1])
@pytest.mark.parametrize("dt", [np.int64, np.uint64, np.float32])
def test_later_pass_modes_match_oracle(P, two_phase, dt):
    """The passes after the first run either with a decoupled look-back or in
    two phases (tile counts + scan, then the pass); both give the oracle's
    order, including ragged last tiles, heavy digits and carried payloads."""
    from jaxframes_b200.autotune import tuning
    rng = np.random.default_rng(5 + two_phase)
    with tuning(two_phase=bool(two_phase)):
        for n in [4095, 4097, 8193, 250_001, 1_000_003]:
            for kind in ("full", "heavy"):
                k = _keys(rng, dt, n, kind)
                sk, perm = P.ParallelRadixSort().sort(k, np.arange(n, dtype=np.int32), True)
                ek, ep = O.radix_sort(k, np.arange(n), True)
                np.testing.assert_array_equal(_np(perm), ep, err_msg=f"n={n} {kind}")
                np.testing.assert_array_equal(_np(sk).view(np.uint8), ek.view(np.uint8), err_msg=f"n={n}")
        n = 300_007
        k1 = rng.integers(0, 50_000, n).astype(np.int32)
        k2 = rng.integers(0, 64, n).astype(np.int32)
        v = rng.integers(-1000, 1000, n).astype(np.int64)
        uk, out = P.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], {"v": v, "w": v}, {"v": "sum", "w": "min"})
        ek, eout = O.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], {"v": v, "w": v}, {"v": "sum", "w": "min"})
        np.testing.assert_array_equal(_np(uk["k1"]), ek["k1"])
        np.testing.assert_array_equal(_np(out["v"]), eout["v"])
        np.testing.assert_array_equal(_np(out["w"]), eout["w"])


@pytest.mark.parametrize("ncols", [2, 3])
def test_lexsort_matches_oracle(P, ncols):
    rng = np.random.default_rng(11 + ncols)
    for n in [1, 33, 4097, 50_000]:
        cols = [rng.integers(-5, 5, n).astype(np.int32), rng.standard_normal(n).round(1).astype(np.float32),
                rng.integers(0, 3, n).astype(np.int64)][:ncols]
        for asc in [True, [True, False, True][:ncols], [False] * ncols]:
            got = _np(P.multi_column_lexsort(cols, asc))
            exp = O.multi_column_lexsort(cols, asc)
            np.testing.assert_array_equal(got, exp, err_msg=f"n={n} asc={asc}")


def test_lexsort_wide_keys_multi_round(P):
    """Packed width above 64 bits: LSD rounds over column groups."""
    rng = np.random.default_rng(4)
    n = 20_000
    cols = [rng.integers(-2**62, 2**62, n), rng.integers(-2**62, 2**62, n), rng.integers(0, 4, n)]
    cols[0][::3] = cols[0][1]
    cols[1][::5] = cols[1][2]
    got = _np(P.multi_column_lexsort(cols, [True, False, True]))
    exp = O.multi_column_lexsort(cols, [True, False, True])
    np.testing.assert_array_equal(got, exp)


# ----------------------------------------------------------------- groupby ---
def _abs_sums_single(keys, v):
    uk, a = O.groupby_aggregate(keys, {"v": np.abs(v.astype(np.float64))}, {"v": "sum"})
    return a["v"]


@pytest.mark.parametrize("n", [1, 5, 512, 513, 8192, 100_000, 1_000_000])
def test_groupby_single_key(P, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, max(1, n // 7), n).astype(np.int32)
    v32 = rng.standard_normal(n).astype(np.float32)
    vi = rng.integers(-1000, 1000, n).astype(np.int32)
    vals = {"a": v32, "b": vi, "c": v32, "d": v32, "e": vi, "f": vi, "g": v32}
    aggs = {"a": "sum", "b": "sum", "c": "mean", "d": "max", "e": "min", "f": "count", "g": "count"}
    uk, out = P.groupby_aggregate(keys, vals, aggs)
    ek, eout = O.groupby_aggregate(keys, vals, aggs)
    np.testing.assert_array_equal(_np(uk), ek)
    got = {c: _np(t) for c, t in out.items()}
    asum = _abs_sums_single(keys, v32)
    cnt = np.bincount(np.unique(keys, return_inverse=True)[1])
    for c in aggs:
        g, e = got[c], eout[c]
        assert g.dtype == e.dtype, (c, g.dtype, e.dtype)
        if c == "a":
            assert (np.abs(g.astype(np.float64) - e) <= asum * 2.0 ** -16 + 1e-30).all()
        elif c == "c":
            assert (np.abs(g.astype(np.float64) - e) <= asum / cnt * 2.0 ** -16 + 1e-30).all()
        else:
            np.testing.assert_array_equal(g, e, err_msg=c)


def test_groupby_multi_key_c3_like(P):
    """Shapes of the 100M-row multi-key config, at 2M rows."""
    rng = np.random.default_rng(42 + 2)
    n = 2_000_000
    ranks = np.arange(1, 1_000_001, dtype=np.float64)
    cdf = np.cumsum(ranks ** -1.1)
    cdf /= cdf[-1]
    perm = rng.permutation(1_000_000)
    k1 = perm[np.searchsorted(cdf, rng.random(n))].astype(np.int32)
    k2 = rng.integers(0, 64, n).astype(np.int32)
    v1 = rng.standard_normal(n).astype(np.float32)
    v2 = rng.integers(-1_000_000, 1_000_001, n).astype(np.int64)
    vals = {f"v1_{a}": v1 for a in ("sum", "mean", "min", "max", "count")}
    vals.update({f"v2_{a}": v2 for a in ("sum", "mean", "min", "max", "count")})
    aggs = {c: c.split("_")[1] for c in vals}
    uk, out = P.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], vals, aggs)
    ek, eout = O.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], vals, aggs)
    np.testing.assert_array_equal(_np(uk["k1"]), ek["k1"])
    np.testing.assert_array_equal(_np(uk["k2"]), ek["k2"])
    _, asum = O.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], {"x": np.abs(v1).astype(np.float64)},
                                               {"x": "sum"})
    asum = asum["x"]
    cnt = eout["v1_count"]
    for c in aggs:
        g = _np(out[c])
        e = eout[c]
        assert g.dtype == e.dtype, (c, g.dtype, e.dtype)
        if c == "v1_sum":
            assert (np.abs(g.astype(np.float64) - e) <= asum * 2.0 ** -16 + 1e-30).all()
        elif c == "v1_mean":
            assert (np.abs(g.astype(np.float64) - e) <= asum / cnt * 2.0 ** -16 + 1e-30).all()
        else:
            np.testing.assert_array_equal(g, e, err_msg=c)


def test_groupby_float_keys_nan_groups(P):
    rng = np.random.default_rng(9)
    n = 10_000
    k = rng.integers(0, 20, n).astype(np.float32)
    k[rng.integers(0, n, 50)] = np.nan
    k[rng.integers(0, n, 50)] = -0.0
    v = rng.integers(0, 100, n).astype(np.int32)
    uk, out = P.groupby_aggregate(k, {"v": v}, {"v": "sum"})
    ek, eout = O.groupby_aggregate(k, {"v": v}, {"v": "sum"})
    np.testing.assert_array_equal(_np(uk).view(np.uint32), ek.view(np.uint32))
    np.testing.assert_array_equal(_np(out["v"]), eout["v"])


def test_groupby_all_equal_and_heavy(P):
    n = 300_000
    k = np.full(n, 7, dtype=np.int64)
    v = np.ones(n, dtype=np.float64)
    uk, out = P.groupby_aggregate(k, {"v": v}, {"v": "sum"})
    assert _np(uk).tolist() == [7] and _np(out["v"]).tolist() == [float(n)]
    rng = np.random.default_rng(1)
    k = rng.integers(0, 1000, n).astype(np.int32)
    k[rng.random(n) < 0.7] = 3
    v = rng.integers(-5, 5, n).astype(np.int64)
    uk, out = P.groupby_aggregate(k, {"v": v}, {"v": "max"})
    ek, eout = O.groupby_aggregate(k, {"v": v}, {"v": "max"})
    np.testing.assert_array_equal(_np(uk), ek)
    np.testing.assert_array_equal(_np(out["v"]), eout["v"])


# -------------------------------------------------------------------- join ---
@pytest.mark.parametrize("nl,nr,kr", [(1, 1, 2), (100, 50, 20), (10_000, 5_000, 3000), (200_000, 100_000, 50_000),
                                      (5_000, 7, 3)])
def test_inner_join_pairs(P, nl, nr, kr):
    rng = np.random.default_rng(nl + nr)
    lk = rng.integers(0, kr, nl).astype(np.int64)
    rk = rng.integers(0, kr, nr).astype(np.int64)
    j = P.ParallelSortMergeJoin()
    mk, li, ri = j.join_indices(lk, rk, "inner")
    eli, eri, sl, pl, sr, pr = O.inner_join_pairs(lk, rk)
    np.testing.assert_array_equal(_np(li), pl[eli])
    np.testing.assert_array_equal(_np(ri), pr[eri])
    np.testing.assert_array_equal(_np(mk), sl[eli])


def test_join_c2_like_payloads(P):
    rng = np.random.default_rng(42 + 1)
    nl, nr = 1_000_000, 500_000
    lk = rng.integers(0, nr, nl).astype(np.int64)
    lv = rng.standard_normal(nl).astype(np.float32)
    rk = rng.permutation(nr).astype(np.int64)
    rv = rng.integers(-2**31, 2**31, nr).astype(np.int32)
    mk, out = P.sort_merge_join(lk, {"lv": lv}, rk, {"rv": rv}, "inner")
    emk, eout, _, _ = O.sort_merge_join(lk, {"lv": lv}, rk, {"rv": rv}, "inner")
    np.testing.assert_array_equal(_np(mk), emk)
    for c in eout:
        g = _np(out[c])
        assert g.dtype == eout[c].dtype
        np.testing.assert_array_equal(g, eout[c])


@pytest.mark.parametrize("kdt", [np.int32, np.int64, np.uint32, np.uint64])
def test_join_every_row_matches_once_payload_kinds(P, kdt):
    """Every left row matches exactly one right row (the expand that writes
    output i from sorted left row i), all payloads carried through the sorts,
    one integer key column of each width and signedness: each payload
    conversion (4- and 8-byte copies, int32/uint32/int64/uint64 to float32)."""
    rng = np.random.default_rng(19 + np.dtype(kdt).itemsize)
    nl, nr = 300_001, 120_000
    lk = rng.integers(0, nr, nl).astype(kdt)
    rk = rng.permutation(nr).astype(kdt)
    lv = {"a": rng.standard_normal(nl), "b": rng.integers(0, 2**32, nl, dtype=np.uint64).astype(np.uint32),
          "c": rng.integers(-2**31, 2**31, nl).astype(np.int32)}
    rv = {"d": rng.integers(-2**62, 2**62, nr), "e": rng.integers(0, 2**63, nr, dtype=np.uint64)}
    mk, out = P.sort_merge_join(lk, lv, rk, rv, "inner")
    emk, eout, _, _ = O.sort_merge_join(lk, lv, rk, rv, "inner")
    np.testing.assert_array_equal(_np(mk), emk)
    assert _np(mk).dtype == emk.dtype
    assert set(out) == set(eout)
    for c in eout:
        g = _np(out[c])
        assert g.dtype == eout[c].dtype, c
        np.testing.assert_array_equal(g, eout[c], err_msg=c)


@pytest.mark.parametrize("how", ["inner", "left", "right"])
def test_join_many_payloads_partial_matches(P, how):
    """Unique right keys with half the left keys unmatched (the general expand,
    not the every-row-matches one), ten payload columns of mixed dtypes (two
    expand calls of at most 8 gathers)."""
    rng = np.random.default_rng(11 + len(how))
    nl, nr = 30_000, 12_000
    lk = rng.integers(0, 2 * nr, nl).astype(np.int64)
    rk = rng.permutation(nr).astype(np.int64)
    dts = [np.float32, np.float64, np.int32, np.int64, np.uint8, np.int16, np.uint32, np.float32, np.int64, np.bool_]
    mk_cols = lambda n: {f"c{i}": (rng.integers(0, 2, n).astype(dt) if dt == np.bool_ else
                                   (rng.standard_normal(n) * 1000).astype(dt)) for i, dt in enumerate(dts)}
    lv, rv = mk_cols(nl), mk_cols(nr)
    mk, out = P.sort_merge_join(lk, lv, rk, rv, how)
    emk, eout, _, _ = O.sort_merge_join(lk, lv, rk, rv, how)
    np.testing.assert_array_equal(_np(mk), emk)
    assert set(out) == set(eout)
    for c in eout:
        g = _np(out[c])
        assert g.dtype == eout[c].dtype, c
        np.testing.assert_array_equal(g, eout[c], err_msg=f"{how} {c}")


@pytest.mark.parametrize("how", ["inner", "left", "right"])
@pytest.mark.parametrize("layout", ["both_carried", "right_too_wide", "float_key"])
def test_join_carried_payloads(P, how, layout):
    """Payload columns carried through the sorts (4- and 8-byte words, at most
    4 per side) or gathered when a side does not fit or the key is float;
    duplicate keys on both sides, unmatched rows on both sides."""
    rng = np.random.default_rng(3 + len(how) + len(layout))
    nl, nr = 40_000, 25_000
    kdt = np.float32 if layout == "float_key" else np.int64
    lk = rng.integers(0, 20_000, nl).astype(kdt)
    rk = rng.integers(5_000, 30_000, nr).astype(kdt)
    lv = {"a": rng.standard_normal(nl), "b": rng.integers(-9, 9, nl).astype(np.int32)}
    rv = {"c": rng.integers(-2**40, 2**40, nr), "d": rng.standard_normal(nr).astype(np.float32)}
    if layout == "right_too_wide":
        rv["e"] = rng.integers(0, 99, nr).astype(np.int64)
        rv["f"] = rng.integers(0, 99, nr).astype(np.uint64)
    mk, out = P.sort_merge_join(lk, lv, rk, rv, how)
    emk, eout, _, _ = O.sort_merge_join(lk, lv, rk, rv, how)
    np.testing.assert_array_equal(_np(mk), emk)
    assert set(out) == set(eout)
    for c in eout:
        g = _np(out[c])
        assert g.dtype == eout[c].dtype, c
        np.testing.assert_array_equal(g, eout[c], err_msg=f"{how} {layout} {c}")


@pytest.mark.parametrize("how", ["left", "right", "outer"])
def test_non_inner_joins(P, how):
    rng = np.random.default_rng(len(how))
    for nl, nr in [(1, 1), (50, 80), (20_000, 9_000)]:
        lk = rng.integers(0, 60, nl).astype(np.int32)
        rk = rng.integers(20, 90, nr).astype(np.int32)
        lv = rng.integers(0, 100, nl).astype(np.int32)
        rv = rng.standard_normal(nr).astype(np.float32)
        mk, out = P.sort_merge_join(lk, {"a": lv}, rk, {"b": rv}, how)
        emk, eout, _, _ = O.sort_merge_join(lk, {"a": lv}, rk, {"b": rv}, how)
        np.testing.assert_array_equal(_np(mk), emk)
        for c in eout:
            np.testing.assert_array_equal(_np(out[c]), eout[c], err_msg=f"{how} {c}")


@pytest.mark.parametrize("how", ["inner", "left", "right", "outer"])
def test_join_multi_column_original_order(P, how):
    """join_multi_column pairs in original row-major order plus unmatched rows
    (parallel_algorithms.py:868-917), against the broadcast-matrix oracle."""
    rng = np.random.default_rng(7 + len(how))
    for nl, nr in [(1, 1), (40, 30), (3000, 2000)]:
        lk = [rng.integers(0, 6, nl).astype(np.int32), rng.integers(0, 5, nl).astype(np.int64)]
        rk = [rng.integers(2, 8, nr).astype(np.int32), rng.integers(0, 5, nr).astype(np.int64)]
        li, ri = P.ParallelSortMergeJoin().join_multi_indices(lk, rk, how)
        eli, eri = O.join_multi_column(lk, rk, how)
        np.testing.assert_array_equal(_np(li), eli, err_msg=f"{how} {nl}x{nr}")
        np.testing.assert_array_equal(_np(ri), eri, err_msg=f"{how} {nl}x{nr}")


def test_join_multi_column_values(P):
    lk = [np.array([1, 1, 2], np.int32), np.array([10, 20, 30], np.int32)]
    rk = [np.array([1, 2], np.int32), np.array([10, 40], np.int32)]
    keys, vals = P.ParallelSortMergeJoin().join_multi_column(
        lk, ["a", "b"], {"v": np.array([1, 2, 3], np.int32)}, rk, ["a", "b"], {"w": np.array([4, 5], np.int32)},
        "left")
    assert _np(keys["a"]).tolist() == [1, 1, 2] and _np(keys["b"]).tolist() == [10, 20, 30]
    assert _np(vals["left_v"]).dtype == np.int32  # every left index valid: no promotion
    w = _np(vals["right_w"])
    assert w.dtype == np.float32 and w[0] == 4 and np.isnan(w[1:]).all()
    keys, vals = P.ParallelSortMergeJoin().join_multi_column(
        lk, ["a", "b"], {}, rk, ["a", "b"], {}, "outer")
    assert _np(keys["a"]).tolist() == [1, 1, 2, 2] and _np(keys["b"]).tolist() == [10, 20, 30, 40]


# --------------------------------------------------------------- partition ---
@pytest.mark.parametrize("p", [1, 7, 256, 2048])
def test_hash_partition(P, p):
    rng = np.random.default_rng(p)
    for n in [1, 1000, 300_001]:
        k1 = rng.integers(-2**31, 2**31, n).astype(np.int32)
        k2 = rng.integers(0, 100, n).astype(np.int64)
        for keys in ([k1], [k1, k2]):
            t, perm, offs = P.hash_partition(keys, p)
            et, ep, eo = O.hash_partition(keys, p)
            np.testing.assert_array_equal(_np(t), et)
            np.testing.assert_array_equal(_np(perm), ep)
            np.testing.assert_array_equal(_np(offs), eo)


def test_hash_values_all_dtypes(P):
    rng = np.random.default_rng(3)
    n = 5000
    cols = [rng.integers(-100, 100, n).astype(np.int8), rng.integers(-2**15, 2**15, n).astype(np.int16),
            rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32), rng.integers(-2**40, 2**40, n),
            rng.standard_normal(n).astype(np.float32), rng.standard_normal(n)]
    for c in cols:
        if c.dtype == np.float64:
            continue  # single float64 key: 2 words per row (covered below)
        np.testing.assert_array_equal(_np(P.hash_multi_columns([c])), O.hash_multi_columns([c]))
    np.testing.assert_array_equal(_np(P.hash_multi_columns(cols)), O.hash_multi_columns(cols))
    np.testing.assert_array_equal(_np(P.hash_multi_columns([cols[-1]])), O.hash_multi_columns([cols[-1]]))


# ----------------------------------------------------------- learned sort ---
def _c4_like(n):
    import bench
    return bench.c4_keys(nblocks=max(1, n // 4096))


def test_every_visible_device(P):
    """Kernels that need more than 48 KB of shared memory (the bucket sorts,
    the batch kernel) get that attribute on each device they run on: the
    learned sort and a small batch on every visible GPU, in turn."""
    from jaxframes_b200.batch import batch_partition_groupby
    rng = np.random.default_rng(77)
    k = rng.integers(0, 2**63, 1 << 20, dtype=np.uint64)
    ep = np.argsort(k, kind="stable")
    rows, off, keys, vals = _batch_inputs(12, 78)
    for d in range(torch.cuda.device_count()):
        with torch.cuda.device(d):
            sk, perm, used = P.learned_sort(k, mode="auto")
            assert used == 1, f"device {d}: learned path not taken (code {used})"
            np.testing.assert_array_equal(_np(perm), ep, err_msg=f"device {d}")
            kt = torch.from_numpy(keys).to(f"cuda:{d}")
            vt = torch.from_numpy(vals).to(f"cuda:{d}")
            ot = torch.from_numpy(off).to(f"cuda:{d}")
            b = batch_partition_groupby(kt, vt, ot, num_partitions=64)
            _check_batch(b, off, keys, vals, 64)


@pytest.mark.parametrize("dist", ["c4", "uniform", "sorted", "reversed", "equal", "few", "narrow"])
def test_learned_sort_matches_plain_and_oracle(P, dist):
    """The learned-CDF sort's output is the plain radix sort's, bit for bit."""
    rng = np.random.default_rng(len(dist))
    n = 1 << 21
    if dist == "c4":
        k = _c4_like(n)
    elif dist == "uniform":
        k = rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    elif dist == "sorted":
        k = np.sort(rng.integers(0, 2**63, n, dtype=np.uint64))
    elif dist == "reversed":
        k = np.sort(rng.integers(0, 2**63, n, dtype=np.uint64))[::-1].copy()
    elif dist == "equal":
        k = np.full(n, 77, dtype=np.uint64)
    elif dist == "few":
        k = rng.integers(0, 50, n).astype(np.uint64) * np.uint64(1 << 40)
    else:
        k = rng.integers(1 << 50, (1 << 50) + 100_000, n).astype(np.uint64)
    ep = np.argsort(k, kind="stable")
    sk, perm, used = P.learned_sort(k, mode="auto")
    np.testing.assert_array_equal(_np(perm), ep)
    np.testing.assert_array_equal(_np(sk), k[ep])
    sk2, perm2, used2 = P.learned_sort(k, mode="plain")
    assert used2 == 0
    np.testing.assert_array_equal(_np(perm2), ep)
    np.testing.assert_array_equal(_np(sk2), k[ep])
    if dist in ("c4", "uniform", "sorted"):
        assert used == 1, f"expected the learned path to be taken (code {used})"


def test_learned_sort_small_inputs_use_plain(P):
    for n in (0, 1, 5, 1000):
        k = np.random.default_rng(n).integers(0, 2**63, n, dtype=np.uint64)
        sk, perm, used = P.learned_sort(k)
        assert used == 0
        np.testing.assert_array_equal(_np(perm), np.argsort(k, kind="stable"))


# ------------------------------------------------------------------ batch ---
def _batch_inputs(nq, seed, max_rows=20000):
    rng = np.random.default_rng(seed)
    rows = np.floor(np.exp(rng.uniform(np.log(1), np.log(max_rows), nq))).astype(np.int64)
    rows[::7] = 0  # empty queries too
    off = np.zeros(nq + 1, dtype=np.int64)
    off[1:] = np.cumsum(rows)
    keys = np.concatenate([rng.integers(0, max(1, min(r // 4, 1 << 20)), r) for r in rows]).astype(np.int32)
    vals = rng.standard_normal(int(off[-1])).astype(np.float32)
    return rows, off, keys, vals


def _check_batch(b, off, keys, vals, P):
    for q in range(len(off) - 1):
        a, e = off[q], off[q + 1]
        k, v = keys[a:e], vals[a:e]
        po, pk, pv, gk, gs, gc = b.query(q)
        tgt, perm, eoffs = O.hash_partition([k], P)
        np.testing.assert_array_equal(_np(po), eoffs, err_msg=f"q{q} offsets")
        np.testing.assert_array_equal(_np(pk), k[perm], err_msg=f"q{q} part keys")
        np.testing.assert_array_equal(_np(pv), v[perm], err_msg=f"q{q} part values")
        ek, eo = O.groupby_aggregate(k, {"s": v, "c": v}, {"s": "sum", "c": "count"})
        np.testing.assert_array_equal(_np(gk), ek, err_msg=f"q{q} keys")
        np.testing.assert_array_equal(_np(gc), eo["c"], err_msg=f"q{q} counts")
        if len(ek):
            asum = O.groupby_aggregate(k, {"a": np.abs(v).astype(np.float64)}, {"a": "sum"})[1]["a"]
            assert (np.abs(_np(gs).astype(np.float64) - eo["s"]) <= asum * 2.0 ** -16 + 1e-30).all(), q


@pytest.mark.parametrize("P_", [256, 7, 1])
def test_batch_partition_groupby(P, P_):
    from jaxframes_b200.batch import batch_partition_groupby
    rows, off, keys, vals = _batch_inputs(40, 5 + P_)
    b = batch_partition_groupby(keys, vals, off, num_partitions=P_)
    _check_batch(b, off, keys, vals, P_)


@pytest.mark.parametrize("key_bits", [20, 28, 30])
def test_batch_key_spreads(P, key_bits):
    """Queries whose keys take each path of the per-query pipeline: one
    bucket of 4096 keys (no bucket pass), 12/13-bit boundaries, one and two
    bucket passes (keys over 20 bits), skewed buckets (many small buckets in
    a chunk after a few large ones), and keys too sparse for buckets (sorted
    by the whole key)."""
    from jaxframes_b200.batch import batch_partition_groupby
    rng = np.random.default_rng(key_bits)
    top = 1 << key_bits
    parts = [
        rng.integers(0, 4096, 9000),                         # kbits 12: one bucket
        np.full(5000, 4096),                                  # kbits 13, one key
        rng.integers(0, 1 << 13, 30000),                      # one bucket pass, two buckets
        rng.integers(0, min(top, 1 << 21), 600000),           # dense, 2 bucket passes when key_bits > 20
        np.concatenate([rng.integers(0, 8192, 300000),        # skewed: two heavy buckets, then
                        rng.integers(8192, 1 << 20, 3000)]),  # many light ones in the last chunks
        rng.integers(0, top, 5000),                           # sparse: whole-key passes
        np.array([top - 1, 0, top - 1, 5]),                  # extremes
        np.array([], dtype=np.int64),                         # empty
    ]
    rows = np.array([len(x) for x in parts], dtype=np.int64)
    off = np.zeros(len(parts) + 1, dtype=np.int64)
    off[1:] = np.cumsum(rows)
    keys = np.concatenate(parts).astype(np.int32)
    vals = rng.standard_normal(int(off[-1])).astype(np.float32)
    b = batch_partition_groupby(keys, vals, off, num_partitions=256, key_bits=key_bits)
    _check_batch(b, off, keys, vals, 256)


def test_batch_more_queries_than_the_device_orders(P):
    """Over 4096 queries the work queue takes them in index order instead of
    largest first; results are the same."""
    from jaxframes_b200.batch import batch_partition_groupby
    rng = np.random.default_rng(93)
    rows = rng.integers(0, 60, 5000)
    rows[::11] = 0
    off = np.zeros(len(rows) + 1, dtype=np.int64)
    off[1:] = np.cumsum(rows)
    keys = rng.integers(0, 40, int(off[-1])).astype(np.int32)
    vals = rng.standard_normal(int(off[-1])).astype(np.float32)
    b = batch_partition_groupby(keys, vals, off, num_partitions=16)
    _check_batch(b, off, keys, vals, 16)


def test_batch_graph_replay(P):
    """One CUDA-graph capture, replayed on new data in the same buffers."""
    import torch
    from jaxframes_b200.batch import BatchedGroupBy
    rows, off, keys, vals = _batch_inputs(30, 21)
    n = int(off[-1])
    b = BatchedGroupBy(n, len(rows), 256, 20)
    b.keys.copy_(torch.from_numpy(keys))
    b.values.copy_(torch.from_numpy(vals))
    b.query_offsets.copy_(torch.from_numpy(off))
    b.capture()
    rng = np.random.default_rng(99)
    keys2 = rng.integers(0, 1000, n).astype(np.int32)
    vals2 = rng.standard_normal(n).astype(np.float32)
    b.keys.copy_(torch.from_numpy(keys2))
    b.values.copy_(torch.from_numpy(vals2))
    b.replay()
    torch.cuda.synchronize()
    b.status()
    _check_batch(b, off, keys2, vals2, 256)


def test_batch_rejects_out_of_range_keys(P):
    from jaxframes_b200.batch import BatchedGroupBy
    from jaxframes_b200 import JfxError
    import torch
    b = BatchedGroupBy(100, 2, 256, 4)
    b.keys.copy_(torch.arange(100, dtype=torch.int32))  # keys up to 99 > 2^4
    b.values.zero_()
    b.query_offsets.copy_(torch.tensor([0, 50, 100]))
    b.run()
    with pytest.raises(JfxError):
        b.status()
