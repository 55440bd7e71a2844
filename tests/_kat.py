"""Known-answer checks shared by the oracle tests and the GPU parity tests.

``check_kat(kat, impl)`` runs one vector of ``tests/golden/kat.json`` through an
implementation adaptor exposing

* ``parallel_sort(keys, values, ascending) -> (sorted_keys, sorted_values)``
* ``lexsort(keys, ascending) -> perm``
* ``groupby(keys, values, aggs) -> (unique_keys, {col: agg})``
* ``groupby_multi(keys, names, values, aggs) -> ({name: unique}, {col: agg})``
* ``join(lk, lv, rk, rv, how) -> (merged_keys, {name: payload})``
* ``join_multi(lk, rk, how) -> (left_idx, right_idx)``
* ``hash(keys) -> uint32 hashes``
* ``partition(keys, P) -> (targets, perm, offsets)``

with NumPy arrays in and out.
"""

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kat.json")


def load_kats():
    with open(GOLDEN) as f:
        return json.load(f)


def _arr(x, dt):
    return np.asarray(x, dtype=dt)


def _eq(got, exp, rtol=None):
    got = np.asarray(got)
    exp = np.asarray(exp)
    assert got.shape == exp.shape, (got.shape, exp.shape)
    if rtol is not None:
        np.testing.assert_allclose(got.astype(np.float64), exp.astype(np.float64), rtol=rtol)
    else:
        np.testing.assert_array_equal(got, exp)


def check_kat(k, impl):
    op = k["op"]
    dt = k.get("dtype", "int32")
    rtol = k.get("rtol")
    if op == "parallel_sort":
        keys = _arr(k["keys"], dt)
        vals = _arr(k["values"], np.int32) if "values" in k else None
        sk, sv = impl.parallel_sort(keys, vals, k.get("ascending", True))
        _eq(sk, _arr(k["expect_keys"], dt), rtol)
        if "expect_values" in k:
            _eq(sv, k["expect_values"])
    elif op == "lexsort":
        keys = [_arr(c, dt) for c in k["keys"]]
        perm = np.asarray(impl.lexsort(keys, k.get("ascending", True)))
        for col, exp in zip(keys, k.get("expect_cols", [])):
            if exp is not None:
                _eq(col[perm], _arr(exp, dt), 1e-6 if dt.startswith("float") else None)
        if "expect_payload" in k:
            if "payload" in k:
                _eq(np.asarray(k["payload"])[perm], k["expect_payload"])
            else:
                _eq(perm, k["expect_payload"])
    elif op == "groupby":
        keys = _arr(k["keys"], dt)
        vals = {c: _arr(v, k["vdtypes"][c]) for c, v in k["values"].items()}
        uk, out = impl.groupby(keys, vals, k["aggs"])
        _eq(uk, _arr(k["expect_keys"], dt))
        for c, e in k["expect"].items():
            _eq(out[c], e, rtol)
        for c, d in k.get("expect_dtype", {}).items():
            assert np.asarray(out[c]).dtype == np.dtype(d), (c, np.asarray(out[c]).dtype, d)
    elif op == "groupby_multi":
        keys = [_arr(c, dt) for c in k["keys"]]
        names = [f"k{i}" for i in range(len(keys))]
        vals = {c: _arr(v, k["vdtypes"][c]) for c, v in k["values"].items()}
        uk, out = impl.groupby_multi(keys, names, vals, k["aggs"])
        if "expect_num_groups" in k:
            assert len(uk[names[0]]) == k["expect_num_groups"]
        for n, e in zip(names, k.get("expect_cols", [])):
            _eq(uk[n], _arr(e, dt))
        for c, e in k.get("expect", {}).items():
            _eq(out[c], e, rtol)
        for c, tot in k.get("expect_total", {}).items():
            assert abs(float(np.sum(np.asarray(out[c], np.float64))) - tot) < 1e-6
        for c, d in k.get("expect_dtype", {}).items():
            assert np.asarray(out[c]).dtype == np.dtype(d), (c, np.asarray(out[c]).dtype, d)
    elif op == "join":
        lk, rk = _arr(k["lk"], dt), _arr(k["rk"], dt)
        lv = {c: _arr(v, np.int32) for c, v in k["lv"].items()}
        rv = {c: _arr(v, np.int32) for c, v in k["rv"].items()}
        mk, out = impl.join(lk, lv, rk, rv, k["how"])
        _eq(mk, _arr(k["expect_keys"], dt))
        for c, e in k["expect"].items():
            _eq(out[c], e)
        for c, d in k.get("expect_dtype", {}).items():
            assert np.asarray(out[c]).dtype == np.dtype(d), (c, np.asarray(out[c]).dtype, d)
    elif op == "join_multi":
        lk = [_arr(c, np.int32) for c in k["lk"]]
        rk = [_arr(c, np.int32) for c in k["rk"]]
        li, ri = impl.join_multi(lk, rk, k["how"])
        li, ri = np.asarray(li), np.asarray(ri)
        if "expect_pairs_sorted" in k:
            got = sorted(zip(li.tolist(), ri.tolist()))
            assert got == [tuple(p) for p in k["expect_pairs_sorted"]], got
        if "expect_num_pairs" in k:
            assert len(li) == k["expect_num_pairs"]
        if "expect_right_valid" in k:
            assert (ri >= 0).tolist() == k["expect_right_valid"]
    elif op == "hash":
        keys = [_arr(c, np.int32) for c in k["keys"]]
        h = np.asarray(impl.hash(keys))
        assert h.dtype == np.uint32
        if "expect_num_unique" in k:
            assert len(np.unique(h)) == k["expect_num_unique"]
        for a, b in k.get("expect_equal", []):
            assert h[a] == h[b]
        for a, b in k.get("expect_differ", []):
            assert h[a] != h[b]
        if "buckets" in k:
            cnt = np.bincount(h % k["buckets"], minlength=k["buckets"])
            avg = len(h) / k["buckets"]
            lo, hi = k["expect_balance"]
            assert (cnt > avg * lo).all() and (cnt < avg * hi).all(), cnt
    elif op == "hash_values":
        keys = [_arr(c, np.int32) for c in k["keys"]]
        _eq(np.asarray(impl.hash(keys)).astype(np.int64), np.asarray(k["expect"], np.int64))
    elif op == "partition":
        keys = [_arr(c, np.int32) for c in k["keys"]]
        tgt, perm, offs = impl.partition(keys, k["num_partitions"])
        _eq(np.asarray(tgt).astype(np.int64), k["expect_targets"])
        _eq(np.asarray(perm).astype(np.int64), k["expect_perm"])
        cnt = np.bincount(np.asarray(k["expect_targets"]), minlength=k["num_partitions"])
        _eq(np.diff(np.asarray(offs).astype(np.int64)), cnt)
    else:
        raise AssertionError(f"unknown op {op}")
