"""Writes ``tests/golden/kat.json``: the known-answer vectors the oracle is pinned on.

Part 1 copies the literal inputs and expected outputs that the reference's own
tests hard-code (each entry cites its test file and line).  The reference is
Python on JAX, which is not installed where these fixtures are made, so these
literals are the only outputs of the reference itself available; they pin the
oracle's sort order, group order, aggregate values and join pair order.

Part 2 adds vectors for behaviour the reference tests do not pin but its code
fixes (descending ties, count dtypes, the join's int->float payload
promotion, hash values).  Their expected values come from an independent
pure-Python evaluation written here (integer arithmetic with explicit masks,
list sorts), not from the NumPy oracle, so the oracle is checked against them.

Run:  python tests/golden/make_golden.py
"""

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
M32 = 0xFFFFFFFF


def _fmix32(h):
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M32
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M32
    h ^= h >> 16
    return h


def _py_hash(cols):
    """parallel_algorithms.py:69-136 evaluated with Python ints."""
    n = len(cols[0])
    out = []
    for r in range(n):
        if len(cols) == 1:
            out.append(_fmix32(cols[0][r] & M32))
            continue
        h = 0x1337
        for i, c in enumerate(cols):
            k = c[r] & M32
            h ^= (k * ((0x9E3779B1 + i) & M32)) & M32
            h = ((h << 13) | (h >> 19)) & M32
            h = (h * 0x85EBCA6B) & M32
        out.append(_fmix32(h))
    return out


def _py_stable_argsort(vals):
    return sorted(range(len(vals)), key=lambda i: (vals[i], i))


def reference_literals():
    np.random.seed(42)
    kat = []
    data = np.random.randint(0, 100, size=1000)
    kat.append(dict(name="sort_single_device", src="tests/test_parallel_algorithms.py:29-41",
                    op="parallel_sort", keys=data.tolist(), dtype="int32",
                    expect_keys=sorted(data.tolist())))
    kat.append(dict(name="sort_with_values", src="tests/test_parallel_algorithms.py:43-57",
                    op="parallel_sort", keys=[5, 2, 8, 1, 9, 3], dtype="int32",
                    values=[50, 20, 80, 10, 90, 30],
                    expect_keys=[1, 2, 3, 5, 8, 9], expect_values=[10, 20, 30, 50, 80, 90]))
    kat.append(dict(name="sort_descending", src="tests/test_parallel_algorithms.py:59-66",
                    op="parallel_sort", keys=[3, 1, 4, 1, 5, 9, 2, 6], dtype="int32", ascending=False,
                    expect_keys=[9, 6, 5, 4, 3, 2, 1, 1]))
    kat.append(dict(name="sort_float", src="tests/test_parallel_algorithms.py:68-75",
                    op="parallel_sort", keys=[3.14, 2.71, 1.41, 0.577, 2.71, 3.14], dtype="float32",
                    expect_keys=[0.577, 1.41, 2.71, 2.71, 3.14, 3.14], rtol=1e-6))
    kat.append(dict(name="sort_negative", src="tests/test_parallel_algorithms.py:77-84",
                    op="parallel_sort", keys=[3, -1, 4, -5, 0, 2, -3], dtype="int32",
                    expect_keys=[-5, -3, -1, 0, 2, 3, 4]))
    kat.append(dict(name="groupby_sum", src="tests/test_parallel_algorithms.py:90-105",
                    op="groupby", keys=[1, 2, 1, 3, 2, 1, 3], dtype="int32",
                    values={"col1": [10, 20, 30, 40, 50, 60, 70]}, vdtypes={"col1": "int32"},
                    aggs={"col1": "sum"}, expect_keys=[1, 2, 3], expect={"col1": [100, 70, 110]}))
    kat.append(dict(name="groupby_mean", src="tests/test_parallel_algorithms.py:107-119",
                    op="groupby", keys=[1, 2, 1, 2, 1], dtype="int32",
                    values={"col1": [10.0, 20.0, 30.0, 40.0, 50.0]}, vdtypes={"col1": "float32"},
                    aggs={"col1": "mean"}, expect_keys=[1, 2], expect={"col1": [30.0, 30.0]}, rtol=1e-6))
    kat.append(dict(name="groupby_max_min", src="tests/test_parallel_algorithms.py:121-138",
                    op="groupby", keys=[1, 2, 1, 2, 1], dtype="int32",
                    values={"col1": [10, 25, 30, 15, 20], "col2": [5, 8, 2, 9, 7]},
                    vdtypes={"col1": "int32", "col2": "int32"},
                    aggs={"col1": "max", "col2": "min"}, expect_keys=[1, 2],
                    expect={"col1": [30, 25], "col2": [2, 8]}))
    kat.append(dict(name="groupby_count", src="tests/test_parallel_algorithms.py:140-152",
                    op="groupby", keys=[1, 2, 1, 3, 2, 1], dtype="int32",
                    values={"col1": [10, 20, 30, 40, 50, 60]}, vdtypes={"col1": "int32"},
                    aggs={"col1": "count"}, expect_keys=[1, 2, 3], expect={"col1": [3, 2, 1]}))
    kat.append(dict(name="join_inner", src="tests/test_parallel_algorithms.py:158-182",
                    op="join", how="inner", lk=[1, 2, 3, 4], lv={"left_col": [10, 20, 30, 40]},
                    rk=[2, 3, 4, 5], rv={"right_col": [200, 300, 400, 500]}, dtype="int32",
                    expect_keys=[2, 3, 4],
                    expect={"left_left_col": [20, 30, 40], "right_right_col": [200, 300, 400]}))
    kat.append(dict(name="join_duplicates", src="tests/test_parallel_algorithms.py:184-208",
                    op="join", how="inner", lk=[1, 2, 2, 3], lv={"left_col": [10, 20, 25, 30]},
                    rk=[2, 2, 3, 4], rv={"right_col": [200, 250, 300, 400]}, dtype="int32",
                    expect_keys=[2, 2, 2, 2, 3],
                    expect={"left_left_col": [20, 20, 25, 25, 30],
                            "right_right_col": [200, 250, 200, 250, 300]}))
    kat.append(dict(name="join_left", src="tests/test_parallel_algorithms.py:210-230",
                    op="join", how="left", lk=[1, 2, 3], lv={"left_col": [10, 20, 30]},
                    rk=[2, 3, 4], rv={"right_col": [200, 300, 400]}, dtype="int32",
                    expect_keys=[1, 2, 3], expect={"left_left_col": [10, 20, 30]}))
    kat.append(dict(name="frame_sort_values", src="tests/test_parallel_algorithms.py:241-258",
                    op="parallel_sort", keys=[3, 1, 4, 1, 5, 9, 2, 6], dtype="int32",
                    values=[30, 10, 40, 15, 50, 90, 20, 60],
                    expect_keys=[1, 1, 2, 3, 4, 5, 6, 9], expect_values=[10, 15, 20, 30, 40, 50, 60, 90]))
    kat.append(dict(name="frame_groupby_sum", src="tests/test_parallel_algorithms.py:260-280",
                    op="groupby", keys=[1, 2, 1, 3, 2, 1], dtype="int32",
                    values={"value1": [10, 20, 30, 40, 50, 60], "value2": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]},
                    vdtypes={"value1": "int32", "value2": "float32"},
                    aggs={"value1": "sum", "value2": "sum"}, expect_keys=[1, 2, 3],
                    expect={"value1": [100, 70, 40], "value2": [10.0, 7.0, 4.0]}, rtol=1e-6))
    kat.append(dict(name="frame_merge", src="tests/test_parallel_algorithms.py:298-324",
                    op="join", how="inner", lk=[1, 2, 3], lv={"left_value": [10, 20, 30]},
                    rk=[2, 3, 4], rv={"right_value": [200, 300, 400]}, dtype="int32",
                    expect_keys=[2, 3],
                    expect={"left_left_value": [20, 30], "right_right_value": [200, 300]}))
    kat.append(dict(name="lexsort_two", src="tests/test_multi_column_operations.py:20-41",
                    op="lexsort", keys=[[3, 1, 2, 1, 3, 2], [5, 2, 1, 6, 3, 4]], dtype="int32",
                    payload=[10, 20, 30, 40, 50, 60],
                    expect_cols=[[1, 1, 2, 2, 3, 3], [2, 6, 1, 4, 3, 5]],
                    expect_payload=[20, 40, 30, 60, 50, 10]))
    kat.append(dict(name="lexsort_mixed", src="tests/test_multi_column_operations.py:43-60",
                    op="lexsort", keys=[[3, 1, 2, 1, 3, 2], [5, 2, 1, 6, 3, 4]], dtype="int32",
                    ascending=[True, False],
                    expect_cols=[[1, 1, 2, 2, 3, 3], [6, 2, 4, 1, 5, 3]]))
    kat.append(dict(name="lexsort_three", src="tests/test_multi_column_operations.py:62-81",
                    op="lexsort", keys=[[1, 1, 1, 2, 2, 2], [1, 1, 2, 1, 2, 2], [3, 1, 2, 5, 4, 6]],
                    dtype="int32", payload=[10, 20, 30, 40, 50, 60],
                    expect_cols=[None, None, [1, 3, 2, 5, 4, 6]],
                    expect_payload=[20, 10, 30, 40, 50, 60]))
    kat.append(dict(name="lexsort_float", src="tests/test_multi_column_operations.py:83-101",
                    op="lexsort", keys=[[1.5, 1.5, 2.3, 2.3, 0.5], [3.2, 1.1, 4.5, 2.2, 5.5]],
                    dtype="float32", payload=[1, 2, 3, 4, 5],
                    expect_cols=[[0.5, 1.5, 1.5, 2.3, 2.3], [5.5, 1.1, 3.2, 2.2, 4.5]],
                    expect_payload=[5, 2, 1, 4, 3]))
    kat.append(dict(name="groupby_two_sum", src="tests/test_multi_column_operations.py:107-126",
                    op="groupby_multi", keys=[[1, 1, 2, 2, 1, 2], [10, 10, 20, 20, 10, 20]], dtype="int32",
                    values={"value": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]}, vdtypes={"value": "float32"},
                    aggs={"value": "sum"}, expect_cols=[[1, 2], [10, 20]], expect={"value": [8.0, 13.0]},
                    rtol=1e-6))
    kat.append(dict(name="groupby_two_mean", src="tests/test_multi_column_operations.py:128-164",
                    op="groupby_multi", keys=[[1, 2, 1, 2, 1, 2], [1, 1, 1, 2, 2, 2]], dtype="int32",
                    values={"value": [10.0, 20.0, 30.0, 40.0, 50.0, 60.0]}, vdtypes={"value": "float32"},
                    aggs={"value": "mean"}, expect_cols=[[1, 1, 2, 2], [1, 2, 1, 2]],
                    expect={"value": [20.0, 50.0, 20.0, 50.0]}, rtol=1e-6))
    kat.append(dict(name="groupby_three", src="tests/test_multi_column_operations.py:166-180",
                    op="groupby_multi", keys=[[1, 1, 1, 2, 2, 2], [1, 1, 2, 1, 2, 2], [1, 2, 1, 1, 1, 2]],
                    dtype="int32", values={"value": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]},
                    vdtypes={"value": "float32"}, aggs={"value": "sum"}, expect_num_groups=6,
                    expect_total={"value": 21.0}))
    kat.append(dict(name="groupby_multi_aggs", src="tests/test_multi_column_operations.py:182-200",
                    op="groupby_multi", keys=[[1, 1, 2, 2, 1, 2], [10, 10, 20, 20, 10, 20]], dtype="int32",
                    values={"value1": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0],
                            "value2": [10.0, 20.0, 30.0, 40.0, 50.0, 60.0]},
                    vdtypes={"value1": "float32", "value2": "float32"},
                    aggs={"value1": "sum", "value2": "mean"}, expect_num_groups=2,
                    expect_cols=[[1, 2], [10, 20]],
                    expect={"value1": [8.0, 13.0], "value2": [80.0 / 3, 130.0 / 3]}, rtol=1e-5))
    kat.append(dict(name="join_multi_two_inner", src="tests/test_multi_column_operations.py:206-251",
                    op="join_multi", how="inner",
                    lk=[[1, 1, 2, 2], [10, 20, 10, 20]], rk=[[1, 2, 1, 2], [10, 10, 20, 30]],
                    expect_pairs_sorted=[[0, 0], [1, 2], [2, 1]]))
    kat.append(dict(name="join_multi_three", src="tests/test_multi_column_operations.py:253-275",
                    op="join_multi", how="inner",
                    lk=[[1, 1, 2], [2, 2, 3], [3, 4, 5]], rk=[[1, 1, 2], [2, 2, 3], [3, 4, 6]],
                    expect_num_pairs=2))
    kat.append(dict(name="join_multi_left", src="tests/test_multi_column_operations.py:277-303",
                    op="join_multi", how="left",
                    lk=[[1, 1, 2], [10, 20, 30]], rk=[[1, 2], [10, 40]],
                    expect_right_valid=[True, False, False]))
    kat.append(dict(name="hash_uniqueness", src="tests/test_distributed_multi_column.py:118-132",
                    op="hash", keys=[[1, 1, 2, 2], [10, 20, 10, 20]], expect_num_unique=4))
    kat.append(dict(name="hash_consistency", src="tests/test_distributed_multi_column.py:134-152",
                    op="hash", keys=[[1, 2, 1, 2], [10, 20, 10, 20]], expect_equal=[[0, 2], [1, 3]],
                    expect_differ=[[0, 1]]))
    kat.append(dict(name="hash_distribution", src="tests/test_distributed_multi_column.py:154-179",
                    op="hash", keys=[[i % 100 for i in range(1000)], [i % 50 for i in range(1000)]],
                    buckets=8, expect_balance=[0.5, 2.0]))
    return kat


def derived():
    """Vectors for behaviour fixed by the reference's code but untested there."""
    kat = []
    # descending single-key radix sort reverses the whole ascending result, so
    # ties come out in reverse original order (parallel_algorithms.py:552-555)
    keys = [2, 1, 2, 1, 2]
    asc = _py_stable_argsort(keys)
    kat.append(dict(name="desc_ties_reverse", src="parallel_algorithms.py:552-555", op="parallel_sort",
                    keys=keys, dtype="int32", values=list(range(5)), ascending=False,
                    expect_keys=[keys[i] for i in asc[::-1]], expect_values=asc[::-1]))
    # multi_column_lexsort ignores `ascending` for a single key (line 44-45)
    kat.append(dict(name="lexsort_single_ignores_desc", src="parallel_algorithms.py:44-45", op="lexsort",
                    keys=[[2, 1, 2, 1, 2]], dtype="int32", ascending=False, payload=[0, 1, 2, 3, 4],
                    expect_payload=_py_stable_argsort([2, 1, 2, 1, 2])))
    # descending integer key in a lexsort: max(arr) - arr wraps in int32 (line 61)
    big = [2147483647, -2147483648, 0, 5]
    wrapped = [((max(big) - v + 2**31) % 2**32) - 2**31 for v in big]
    kat.append(dict(name="lexsort_desc_wraps", src="parallel_algorithms.py:56-61", op="lexsort",
                    keys=[[0, 0, 0, 0], big], dtype="int32", ascending=[True, False], payload=[0, 1, 2, 3],
                    expect_payload=_py_stable_argsort(wrapped)))
    # count dtype: value dtype for one key (line 654-658), int32 for several (1220-1221)
    kat.append(dict(name="count_dtype_single", src="parallel_algorithms.py:654-658", op="groupby",
                    keys=[1, 2, 1], dtype="int32", values={"v": [1.5, 2.5, 3.5]}, vdtypes={"v": "float32"},
                    aggs={"v": "count"}, expect_keys=[1, 2], expect={"v": [2.0, 1.0]}, expect_dtype={"v": "float32"}))
    kat.append(dict(name="count_dtype_multi", src="parallel_algorithms.py:1220-1221", op="groupby_multi",
                    keys=[[1, 2, 1], [0, 0, 0]], dtype="int32", values={"v": [1.5, 2.5, 3.5]},
                    vdtypes={"v": "float32"}, aggs={"v": "count"}, expect_cols=[[1, 2], [0, 0]],
                    expect={"v": [2, 1]}, expect_dtype={"v": "int32"}))
    # inner join promotes integer payloads to float32 (line 1056-1073)
    kat.append(dict(name="join_int_payload_promoted", src="parallel_algorithms.py:1056-1073", op="join",
                    how="inner", lk=[7, 8], lv={"a": [16777217, 3]}, rk=[8, 7], rv={"b": [1, 2]}, dtype="int32",
                    expect_keys=[7, 8], expect={"left_a": [16777216.0, 3.0], "right_b": [2.0, 1.0]},
                    expect_dtype={"left_a": "float32", "right_b": "float32"}))
    # hash values on fixed inputs, computed with Python ints
    rng = np.random.default_rng(7)
    one = rng.integers(-2**31, 2**31, 64).tolist()
    two = [rng.integers(-2**31, 2**31, 64).tolist(), rng.integers(0, 1000, 64).tolist()]
    three = [rng.integers(0, 50, 64).tolist() for _ in range(3)]
    kat.append(dict(name="hash_values_one", src="parallel_algorithms.py:86-101", op="hash_values",
                    keys=[one], expect=_py_hash([one])))
    kat.append(dict(name="hash_values_two", src="parallel_algorithms.py:103-136", op="hash_values",
                    keys=two, expect=_py_hash(two)))
    kat.append(dict(name="hash_values_three", src="parallel_algorithms.py:103-136", op="hash_values",
                    keys=three, expect=_py_hash(three)))
    parts = [h % 256 for h in _py_hash([one])]
    kat.append(dict(name="partition_256", src="parallel_algorithms.py:163-182,214", op="partition",
                    keys=[one], num_partitions=256, expect_targets=parts,
                    expect_perm=_py_stable_argsort(parts)))
    return kat


def main():
    kat = reference_literals() + derived()
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=0)
    print(f"wrote {len(kat)} vectors")


if __name__ == "__main__":
    main()
