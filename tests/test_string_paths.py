"""String-key paths: dictionary codes (int32, null = -1) through the integer
kernels, against the oracle's restatement of core/string_fastpaths.py.

The known answers are the reference's own string tests
(tests/test_string_operations.py:31-110) with each string replaced by its
code in the sorted vocabulary, as core/string_encoding.py:37-51 encodes it."""

import numpy as np
import pytest
import torch

from oracle import jfx_oracle as O


def _codes(strings, vocab):
    return np.array([vocab.index(s) if s is not None else -1 for s in strings], dtype=np.int32)


# ---------------------------------------------------------- oracle KATs ---
def test_oracle_groupby_kats():
    # test_string_operations.py:31-53: categories b, a, b, c, a
    vocab = ["a", "b", "c"]
    k = _codes(["b", "a", "b", "c", "a"], vocab)
    v = np.array([10.0, 20.0, 5.0, 1.0, 7.0], dtype=np.float32)
    codes, out = O.groupby_encoded_strings(k, {"value": v}, {"value": "sum"}, 3)
    assert [vocab[c] for c in codes] == ["a", "b", "c"]
    assert out["value"].tolist() == [27.0, 15.0, 1.0]
    codes, out = O.groupby_encoded_strings(k, {"value": v}, {"value": "count"}, 3)
    assert out["value"].tolist() == [2, 2, 1] and out["value"].dtype == np.int32


def test_oracle_join_kats():
    # :55-74 many-to-one left join; the vocabularies align to (a, b, c, x)
    vocab = ["a", "b", "c", "x"]
    lk = _codes(["b", "a", "x", "b"], vocab)
    rk = _codes(["a", "b", "c"], vocab)
    codes, li, ri = O.join_encoded_strings(lk, rk, len(vocab), "left")
    assert [vocab[c] for c in codes] == ["b", "a", "x", "b"]
    assert li.tolist() == [0, 1, 2, 3] and ri.tolist() == [1, 0, -1, 1]
    # :76-93 inner join over different local vocabularies, aligned to (a, b, c)
    vocab = ["a", "b", "c"]
    codes, li, ri = O.join_encoded_strings(_codes(["b", "a", "b"], vocab), _codes(["c", "b", "a"], vocab), 3,
                                           "inner")
    lv, rv = np.array([1, 2, 3]), np.array([30, 20, 10])
    rows = sorted(zip([vocab[c] for c in codes], lv[li].tolist(), rv[ri].tolist()))
    assert rows == [("a", 2, 10), ("b", 1, 20), ("b", 3, 20)]
    # :95-110 outer join
    codes, li, ri = O.join_encoded_strings(_codes(["a", "b"], vocab), _codes(["b", "c"], vocab), 3, "outer")
    assert [vocab[c] for c in codes] == ["a", "b", "c"]
    assert li.tolist() == [0, 1, -1] and ri.tolist() == [-1, 0, 1]


def test_oracle_null_codes_match_each_other_and_many_to_many_order():
    # nulls take the code num_codes, so a null key joins null keys
    lk = np.array([1, -1, 0, 1], dtype=np.int32)
    rk = np.array([1, 1, -1, 2], dtype=np.int32)
    codes, li, ri = O.join_encoded_strings(lk, rk, 3, "outer")
    # code 0: left row 2 unmatched; code 1: rows (0, 3) x (0, 1); code 2:
    # right row 3 unmatched; null: (1, 2)
    assert codes.tolist() == [0, 1, 1, 1, 1, 2, -1]
    assert li.tolist() == [2, 0, 0, 3, 3, -1, 1]
    assert ri.tolist() == [-1, 0, 1, 0, 1, 3, 2]


def test_oracle_groupby_drops_nulls_and_out_of_vocabulary_codes():
    k = np.array([-1, 2, 5, 2, 0, -3], dtype=np.int32)
    v = np.arange(6, dtype=np.int32)
    codes, out = O.groupby_encoded_strings(k, {"s": v, "m": v}, {"s": "sum", "m": "mean"}, 4)
    assert codes.tolist() == [0, 2]
    assert out["s"].tolist() == [4, 4] and out["m"].dtype == np.float32
    assert out["m"].tolist() == [4.0, 2.0]


# -------------------------------------------------------------- product ---
@pytest.fixture(scope="module")
def S():
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jaxframes_b200 import build
    build.build()
    from jaxframes_b200 import string_fastpaths as S
    return S


def _np(t):
    return t.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n,vocab", [(0, 5), (1, 1), (1000, 17), (300_000, 5000), (100_000, 3)])
@pytest.mark.parametrize("vdt", [np.float32, np.int32, np.float64, np.int64])
def test_groupby_encoded_strings(S, n, vocab, vdt):
    rng = np.random.default_rng(n + vocab)
    k = rng.integers(-2, vocab + 2, n).astype(np.int32)  # nulls and out-of-vocabulary codes too
    v = (rng.standard_normal(n) * 100).astype(vdt) if np.issubdtype(vdt, np.floating) else \
        rng.integers(-1000, 1000, n).astype(vdt)
    aggs = {"s": "sum", "m": "mean", "lo": "min", "hi": "max", "c": "count"}
    vals = {c: v for c in aggs}
    codes, out = S.groupby_encoded_strings(k, vals, aggs, vocab)
    ecodes, eout = O.groupby_encoded_strings(k, vals, aggs, vocab)
    np.testing.assert_array_equal(_np(codes), ecodes)
    _, asum = O.groupby_encoded_strings(k, {"a": np.abs(v).astype(np.float64)}, {"a": "sum"}, vocab)
    asum, cnt = asum["a"], eout["c"]
    for c in aggs:
        g, e = _np(out[c]), eout[c]
        assert g.dtype == e.dtype, (c, g.dtype, e.dtype)
        if np.issubdtype(vdt, np.floating) and c == "s":
            assert (np.abs(g.astype(np.float64) - e) <= asum * 2.0 ** -16 + 1e-30).all()
        elif np.issubdtype(vdt, np.floating) and c == "m":
            assert (np.abs(g.astype(np.float64) - e) <= asum / cnt * 2.0 ** -16 + 1e-30).all()
        else:
            np.testing.assert_array_equal(g, e, err_msg=c)


@pytest.mark.gpu
@pytest.mark.parametrize("how", ["inner", "left", "right", "outer"])
@pytest.mark.parametrize("case", ["unique_right", "many", "nulls", "empty_left", "empty_right", "kats"])
def test_join_encoded_strings(S, how, case):
    rng = np.random.default_rng(["unique_right", "many", "nulls", "empty_left", "empty_right", "kats"].index(case))
    nc = 50
    if case == "unique_right":
        lk = rng.integers(-1, nc, 20_000).astype(np.int32)
        rk = rng.permutation(nc)[: nc - 7].astype(np.int32)
    elif case == "many":
        lk = rng.integers(0, nc, 3000).astype(np.int32)
        rk = rng.integers(0, nc, 500).astype(np.int32)
    elif case == "nulls":
        lk = rng.integers(-1, 8, 2000).astype(np.int32)
        rk = rng.integers(-1, 12, 300).astype(np.int32)
    elif case == "empty_left":
        lk = np.zeros(0, np.int32)
        rk = rng.integers(0, nc, 100).astype(np.int32)
    elif case == "empty_right":
        lk = rng.integers(0, nc, 100).astype(np.int32)
        rk = np.zeros(0, np.int32)
    else:
        lk = np.array([1, 0, 3, 1], np.int32)
        rk = np.array([0, 1, 2], np.int32)
        nc = 4
    plan = S.join_encoded_strings(lk, rk, nc, how)
    ec, el, er = O.join_encoded_strings(lk, rk, nc, how)
    np.testing.assert_array_equal(_np(plan.joined_codes), ec)
    np.testing.assert_array_equal(_np(plan.left_indices), el)
    np.testing.assert_array_equal(_np(plan.right_indices), er)


@pytest.mark.gpu
def test_string_join_payloads(S):
    vocab = ["a", "b", "c", "x"]
    lk = _codes(["b", "a", "x", "b"], vocab)
    rk = _codes(["a", "b", "c"], vocab)
    plan = S.join_encoded_strings(lk, rk, 4, "left")
    data, dtypes, _ = S.assemble_string_join_payloads(plan, {"left_value": np.array([1, 2, 3, 4], np.int32)},
                                                      {"right_value": np.array([10, 20, 30], np.int32)},
                                                      {"left_value": "int32"}, {"right_value": "int32"})
    assert _np(data["left_left_value"]).tolist() == [1, 2, 3, 4]
    r = _np(data["right_right_value"])
    assert r.dtype == np.float32 and r[[0, 1, 3]].tolist() == [20.0, 10.0, 20.0] and np.isnan(r[2])


@pytest.mark.gpu
def test_sortable_string_codes_sort_nulls_last(S):
    import jaxframes_b200.parallel_algorithms as P
    c = np.array([2, -1, 0, 1, -1, 2], np.int32)
    for desc in (False, True):
        k = S.sortable_string_codes(c, 3, desc)
        np.testing.assert_array_equal(_np(k), O.sortable_string_codes(c, 3, desc))
        perm = _np(P.ParallelRadixSort().argsort(k))
        np.testing.assert_array_equal(perm, np.argsort(O.sortable_string_codes(c, 3, desc), kind="stable"))
