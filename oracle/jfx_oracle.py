"""CPU oracle for the jaxframes distributed-algorithms path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: the parity tests, the
``smoke()`` self-check and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it; the product (``jaxframes_b200``) never does.

It is a NumPy restatement of the semantics of
``src/jaxframes/distributed/parallel_algorithms.py`` in solenyaPickleman/jaxframes,
which is pure Python on JAX/XLA.  JAX is not importable where this runs, so the
restatement is pinned against the hard-coded known-answer vectors of the
reference's own tests (``tests/test_parallel_algorithms.py``,
``tests/test_multi_column_operations.py``,
``tests/test_distributed_multi_column.py``); see ``tests/golden/``.

JAX behaviours that the reference relies on and that are restated here:

* ``jnp.argsort`` is stable by default; floats are compared after -0.0 is
  folded onto +0.0 and every NaN onto one canonical NaN, which sorts last.
  ``np.argsort(kind="stable")`` has exactly that order.
* Type promotion follows JAX's lattice (int32 with a weak Python float gives
  the default float; int64 with float32 gives float32), with the default float
  being float32 unless ``x64`` is requested (``jax_enable_x64``).
* ``lax.max`` / ``lax.min`` propagate NaN.
"""

from __future__ import annotations

import numpy as np

__all__ = [
    "stable_argsort",
    "multi_column_lexsort",
    "radix_sort",
    "groupby_aggregate",
    "groupby_aggregate_multi_column",
    "sort_merge_join",
    "join_multi_column",
    "hash_multi_columns",
    "hash_partition",
    "compact_repartitioned_rows",
    "default_float",
    "groupby_encoded_strings",
    "join_encoded_strings",
    "sortable_string_codes",
]

_FLOATS = (np.float32, np.float64)


def default_float(x64: bool = False):
    """JAX's default float dtype: float64 under ``jax_enable_x64``, else float32."""
    return np.float64 if x64 else np.float32


def _is_float(a: np.ndarray) -> bool:
    return a.dtype.type in _FLOATS


def stable_argsort(a: np.ndarray) -> np.ndarray:
    """``jnp.argsort(a, stable=True)``: stable ascending, NaN last, -0.0 == +0.0."""
    a = np.asarray(a)
    if a.dtype == np.bool_:
        a = a.astype(np.uint8)
    return np.argsort(a, kind="stable").astype(np.int64)


def multi_column_lexsort(keys, ascending=True) -> np.ndarray:
    """parallel_algorithms.py:25-66.

    One key: plain stable argsort; ``ascending`` is ignored (line 44-45).
    Several keys: stable sorts from the last key to the first (line 55-64);
    a descending float key is negated, a descending integer key is rewritten as
    ``max(arr) - arr`` in the key's own dtype, which wraps on overflow
    (line 56-61).
    """
    keys = [np.asarray(k) for k in keys]
    if len(keys) == 1:
        return stable_argsort(keys[0])
    if isinstance(ascending, (bool, np.bool_)):
        ascending = [bool(ascending)] * len(keys)
    n = len(keys[0])
    indices = np.arange(n, dtype=np.int64)
    for arr, asc in zip(reversed(keys), reversed(list(ascending))):
        if not asc:
            if _is_float(arr):
                arr = -arr
            else:
                with np.errstate(over="ignore"):
                    arr = (arr.max() - arr).astype(arr.dtype) if n else arr
        sort_idx = stable_argsort(arr[indices])
        indices = indices[sort_idx]
    return indices


def _radix_order_key(keys: np.ndarray) -> np.ndarray:
    """The unsigned order the reference's LSD passes sort by (line 491-505).

    int32/int64 flip the sign bit, unsigned types are used as-is, and the
    narrow signed types (int8/int16) are NOT sign-flipped: ``keys >> shift``
    sign-extends them, so they order as their 32-bit two's-complement pattern
    read unsigned (non-negatives first, then negatives).
    """
    dt = keys.dtype
    if dt == np.int32:
        return keys.view(np.uint32) ^ np.uint32(0x80000000)
    if dt == np.int64:
        return keys.view(np.uint64) ^ np.uint64(1 << 63)
    if dt in (np.uint8, np.uint16, np.uint32, np.uint64):
        return keys
    if dt in (np.int8, np.int16):
        return keys.astype(np.int32).view(np.uint32)
    raise TypeError(f"radix sort does not support key dtype {dt}")


def radix_sort(keys, values=None, ascending=True):
    """``ParallelRadixSort.sort`` (parallel_algorithms.py:463-581).

    The LSD passes (one stable sort per 8-bit digit, line 508-549) amount to a
    stable ascending argsort on the transformed key.  Float keys are re-sorted
    with ``jnp.argsort(keys)`` (line 561).  ``ascending=False`` reverses the
    whole ascending result (line 552-555, 562-563), so equal keys come out in
    reverse original order.  Returns ``(sorted_keys, sorted_values)``.
    """
    keys = np.asarray(keys)
    if _is_float(keys):
        perm = stable_argsort(keys)
    else:
        perm = np.argsort(_radix_order_key(keys), kind="stable").astype(np.int64)
    if not ascending:
        perm = perm[::-1]
    sorted_keys = keys[perm]
    sorted_values = None if values is None else np.asarray(values)[perm]
    return sorted_keys, sorted_values


def _boundaries(sorted_cols) -> np.ndarray:
    """Group starts: row 0, then every row where any key differs (``!=``).

    parallel_algorithms.py:767-770 (one key) and :702-710 (several keys).  A NaN
    key differs from everything, itself included, so every NaN row starts a group.
    """
    n = len(sorted_cols[0])
    flags = np.zeros(n, dtype=bool)
    if n:
        flags[0] = True
    for c in sorted_cols:
        if n > 1:
            flags[1:] |= c[1:] != c[:-1]
    return flags


def _segment_max(vals, seg, g, is_min):
    """``jax.ops.segment_max/min`` / ``.at[].max/min`` with NaN propagation."""
    out = np.empty(g, dtype=vals.dtype)
    if _is_float(vals):
        fill = np.inf if is_min else -np.inf
    else:
        info = np.iinfo(vals.dtype)
        fill = info.max if is_min else info.min
    out[:] = fill
    if is_min:
        np.minimum.at(out, seg, vals)  # np.minimum propagates NaN like lax.min
    else:
        np.maximum.at(out, seg, vals)
    return out


def _segment_sum(vals, seg, g, dtype):
    """Sum per segment in ``dtype``.  Floats are summed in float64 and rounded
    once: the reference's float32 summation order is XLA's and is not pinned,
    so tests compare float sums within 2^-16 * sum(|x|) per group."""
    if np.issubdtype(dtype, np.floating):
        acc = np.zeros(g, dtype=np.float64)
        np.add.at(acc, seg, vals.astype(np.float64))
        return acc.astype(dtype)
    acc = np.zeros(g, dtype=dtype)
    with np.errstate(over="ignore"):
        np.add.at(acc, seg, vals.astype(dtype))
    return acc


def _mean_dtype_single(vdt, x64):
    # sums(v dtype) / maximum(counts(v dtype), 1): true division (line 634-643)
    if np.issubdtype(vdt, np.floating):
        return vdt
    return default_float(x64)


def _mean_dtype_multi(vdt):
    # sums(v dtype) / maximum(float32 counts, 1.0) (line 1216-1219): JAX promotes
    # any integer with float32 to float32; float64 stays float64.
    if vdt == np.float64:
        return np.float64
    return np.float32


def _aggregate(vals, seg, g, agg, multi, x64, sum64=None):
    vdt = vals.dtype.type
    if agg == "sum":
        return _segment_sum(vals, seg, g, vdt)
    if agg == "count":
        cnt = np.bincount(seg, minlength=g)
        return cnt.astype(np.int32 if multi else vdt)
    if agg == "mean":
        cnt = np.bincount(seg, minlength=g)
        if np.issubdtype(vdt, np.floating):
            s64 = np.zeros(g, dtype=np.float64)
            np.add.at(s64, seg, vals.astype(np.float64))
            out_dt = _mean_dtype_multi(vdt) if multi else vdt
            # the reference divides the value-dtype sum by the clamped count
            return (s64.astype(vdt) / np.maximum(cnt, 1).astype(vdt if not multi else np.float32)).astype(out_dt)
        s = _segment_sum(vals, seg, g, vdt)
        out_dt = _mean_dtype_multi(vdt) if multi else _mean_dtype_single(vdt, x64)
        return (s.astype(out_dt) / np.maximum(cnt, 1).astype(out_dt)).astype(out_dt)
    if agg == "max":
        return _segment_max(vals, seg, g, False)
    if agg == "min":
        return _segment_max(vals, seg, g, True)
    raise ValueError(f"Unsupported aggregation function: {agg}")


def groupby_aggregate(keys, values: dict, agg_funcs: dict, x64: bool = False):
    """``SortBasedGroupBy.groupby_aggregate`` (parallel_algorithms.py:733-803).

    Radix sort ascending (line 763), boundaries (767-770), unique keys in
    ascending order (773-774), then one aggregation per column with the value
    dtype for sum and for count (626-660).
    """
    keys = np.asarray(keys)
    if len(keys) == 0:
        return keys[:0], {c: np.asarray(a)[:0] for c, a in values.items()}
    sorted_keys, perm = radix_sort(keys, np.arange(len(keys)), True)
    flags = _boundaries([sorted_keys])
    g = int(flags.sum())
    seg = np.cumsum(flags) - 1
    uniq = sorted_keys[flags]
    out = {}
    for col, agg in agg_funcs.items():
        v = np.asarray(values[col])[perm]
        out[col] = _aggregate(v, seg, g, agg, multi=False, x64=x64)
    return uniq, out


def groupby_aggregate_multi_column(keys, key_names, values: dict, agg_funcs: dict, x64: bool = False):
    """``SortBasedGroupBy.groupby_aggregate_multi_column`` (:662-731) with
    ``_scatter_group_aggregate`` (:1212-1228): count is int32, mean divides by a
    float32 count."""
    keys = [np.asarray(k) for k in keys]
    if not keys or len(keys[0]) == 0:
        return ({n: k[:0] for n, k in zip(key_names, keys)},
                {c: np.asarray(a)[:0] for c, a in values.items()})
    idx = multi_column_lexsort(keys)
    sk = [k[idx] for k in keys]
    flags = _boundaries(sk)
    g = int(flags.sum())
    seg = np.cumsum(flags) - 1
    uniq = {n: k[flags] for n, k in zip(key_names, sk)}
    out = {}
    for col, agg in agg_funcs.items():
        v = np.asarray(values[col])[idx]
        out[col] = _aggregate(v, seg, g, agg, multi=True, x64=x64)
    return uniq, out


def _payload_nan_fill(col, idx, x64):
    """``jnp.where(idx >= 0, col[idx], nan)`` (parallel_algorithms.py:1056-1073):
    integers and bools become the default float even when every index is valid."""
    col = np.asarray(col)
    out_dt = col.dtype if _is_float(col) else default_float(x64)
    res = col[np.maximum(idx, 0)].astype(out_dt) if len(col) else np.zeros(len(idx), out_dt)
    res[idx < 0] = np.nan
    return res


def _equal_runs(sorted_keys):
    """Start index and length of each run of ``==`` keys (NaN never equal)."""
    flags = _boundaries([sorted_keys])
    starts = np.flatnonzero(flags)
    lens = np.diff(np.append(starts, len(sorted_keys)))
    return starts, lens


def inner_join_pairs(lk, rk):
    """Inner-join pairs in the reference's order (parallel_algorithms.py:987-994).

    ``jnp.where(sorted_left[:, None] == sorted_right[None, :])`` enumerates the
    match matrix row-major over the two SORTED sequences, i.e. pairs ordered by
    (key, left original index, right original index).  Restated with equal-run
    expansion instead of the nL x nR matrix; equal to the matrix version (a test
    checks both on small inputs).  Returns positions into the sorted orders and
    the two sort permutations.
    """
    lk = np.asarray(lk)
    rk = np.asarray(rk)
    sl, pl = radix_sort(lk, np.arange(len(lk)), True)
    sr, pr = radix_sort(rk, np.arange(len(rk)), True)
    lo = np.searchsorted(sr, sl, side="left")
    hi = np.searchsorted(sr, sl, side="right")
    cnt = hi - lo
    if _is_float(sl):
        cnt[np.isnan(sl)] = 0
    m = int(cnt.sum())
    li = np.repeat(np.arange(len(sl)), cnt)
    off = np.cumsum(cnt) - cnt
    ri = lo[li] + (np.arange(m) - off[li])
    return li, ri, sl, pl, sr, pr


def sort_merge_join(left_keys, left_values: dict, right_keys, right_values: dict,
                    how: str = "inner", x64: bool = False):
    """``ParallelSortMergeJoin.join`` (parallel_algorithms.py:938-1075).

    inner: every matching pair ordered by (key, left idx, right idx).
    left/right: each row of that side in sorted order with the FIRST match of
    the other side (``searchsorted``, line 1013-1034), -1 when none.
    outer: one row per distinct key (``jnp.unique``, line 999-1000, 1035-1046).
    Payloads are gathered with NaN fill and int->default-float promotion.
    Returns ``(merged_keys, {left_<col>, right_<col>})``.
    """
    lk = np.asarray(left_keys)
    rk = np.asarray(right_keys)
    if how == "inner":
        li, ri, sl, pl, sr, pr = inner_join_pairs(lk, rk)
        mk = sl[li]
        lidx = pl[li]
        ridx = pr[ri]
    else:
        sl, pl = radix_sort(lk, np.arange(len(lk)), True)
        sr, pr = radix_sort(rk, np.arange(len(rk)), True)
        if how == "left":
            mk = sl
            lidx = pl
            pos = np.searchsorted(sr, sl)
            ok = (pos < len(sr)) & (sr[np.minimum(pos, len(sr) - 1)] == sl) if len(sr) else np.zeros(len(sl), bool)
            ridx = np.where(ok, pr[np.minimum(pos, max(len(pr) - 1, 0))] if len(pr) else -1, -1)
        elif how == "right":
            mk = sr
            ridx = pr
            pos = np.searchsorted(sl, sr)
            ok = (pos < len(sl)) & (sl[np.minimum(pos, len(sl) - 1)] == sr) if len(sl) else np.zeros(len(sr), bool)
            lidx = np.where(ok, pl[np.minimum(pos, max(len(pl) - 1, 0))] if len(pl) else -1, -1)
        else:
            mk = np.unique(np.concatenate([sl, sr]))
            lp = np.searchsorted(sl, mk)
            rp = np.searchsorted(sr, mk)
            lok = (lp < len(sl)) & (sl[np.minimum(lp, len(sl) - 1)] == mk)
            rok = (rp < len(sr)) & (sr[np.minimum(rp, len(sr) - 1)] == mk)
            lidx = np.where(lok, pl[np.minimum(lp, len(pl) - 1)], -1)
            ridx = np.where(rok, pr[np.minimum(rp, len(pr) - 1)], -1)
    out = {}
    for c, a in left_values.items():
        out[f"left_{c}"] = _payload_nan_fill(a, lidx, x64)
    for c, a in right_values.items():
        out[f"right_{c}"] = _payload_nan_fill(a, ridx, x64)
    return mk, out, lidx, ridx


def join_multi_column(left_keys, right_keys, how="inner"):
    """Index pairs of ``join_multi_column`` (parallel_algorithms.py:868-917):
    matches in ORIGINAL row-major order, then unmatched left rows (left/outer)
    and unmatched right rows (right/outer), the missing side being -1."""
    lk = [np.asarray(k) for k in left_keys]
    rk = [np.asarray(k) for k in right_keys]
    nl, nr = len(lk[0]), len(rk[0])
    m = np.ones((nl, nr), dtype=bool)
    for a, b in zip(lk, rk):
        m &= a[:, None] == b[None, :]
    li, ri = np.nonzero(m)
    lun = np.flatnonzero(~m.any(axis=1))
    run = np.flatnonzero(~m.any(axis=0))
    if how == "inner":
        return li, ri
    if how == "left":
        return np.concatenate([li, lun]), np.concatenate([ri, -np.ones(len(lun), np.int64)])
    if how == "right":
        return np.concatenate([li, -np.ones(len(run), np.int64)]), np.concatenate([ri, run])
    return (np.concatenate([li, lun, -np.ones(len(run), np.int64)]),
            np.concatenate([ri, -np.ones(len(lun), np.int64), run]))


_M1 = np.uint32(0x85EBCA6B)
_M2 = np.uint32(0xC2B2AE35)
_P1 = np.uint32(0x9E3779B1)


def _key_as_u32(key: np.ndarray, multi: bool) -> np.ndarray:
    """Key to uint32 as the hash reads it (parallel_algorithms.py:89-93, 113-121)."""
    if key.dtype == np.float32:
        return key.view(np.uint32)
    if key.dtype == np.float64:
        if multi:
            return key.astype(np.float32).view(np.uint32)
        return key.view(np.uint32)  # the reference's single-key quirk: 2 words per row
    return key.astype(np.uint32)


def _fmix32(h: np.ndarray) -> np.ndarray:
    h = h ^ (h >> np.uint32(16))
    h = h * _M1
    h = h ^ (h >> np.uint32(13))
    h = h * _M2
    h = h ^ (h >> np.uint32(16))
    return h


def hash_multi_columns(keys) -> np.ndarray:
    """``hash_multi_columns`` (parallel_algorithms.py:69-136), uint32 wraparound.

    One key: the fmix32 finalizer.  Several keys: seed 0x1337, then per key i
    ``h ^= k_i * (0x9e3779b1 + i); h = rotl(h, 13); h *= 0x85ebca6b``, then fmix32.
    """
    keys = [np.asarray(k) for k in keys]
    with np.errstate(over="ignore"):
        if len(keys) == 1:
            return _fmix32(_key_as_u32(keys[0], False).astype(np.uint32))
        h = np.full(len(keys[0]), 0x1337, dtype=np.uint32)
        for i, k in enumerate(keys):
            ki = _key_as_u32(k, True).astype(np.uint32)
            h = h ^ (ki * (_P1 + np.uint32(i)))
            h = (h << np.uint32(13)) | (h >> np.uint32(19))
            h = h * _M1
        return _fmix32(h)


def hash_partition(keys, num_partitions: int):
    """One device's body of ``collective_hash_repartition`` with ndev := P
    (parallel_algorithms.py:163-182, 213-214): target = hash % P, then a stable
    counting sort by target.  Returns (targets int32, perm, offsets[P+1])."""
    h = hash_multi_columns(keys)
    tgt = (h % np.uint32(num_partitions)).astype(np.int32)
    perm = np.argsort(tgt, kind="stable").astype(np.int64)
    counts = np.bincount(tgt, minlength=num_partitions)
    offsets = np.zeros(num_partitions + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(counts)
    return tgt, perm, offsets


def compact_repartitioned_rows(keys, values, valid_mask):
    """``compact_repartitioned_rows`` (parallel_algorithms.py:277-293)."""
    valid_mask = np.asarray(valid_mask)
    if valid_mask.size == 0 or valid_mask.all():
        return keys, values
    pos = np.flatnonzero(valid_mask)
    return [np.asarray(k)[pos] for k in keys], {n: np.asarray(a)[pos] for n, a in values.items()}


# ------------------------------------------------ dictionary-encoded strings ---
# core/string_fastpaths.py: string columns are int32 dictionary codes into a
# lexicographically sorted vocabulary, null = -1 (core/string_encoding.py:37-51).

def string_agg_dtype(vals: np.ndarray, agg: str):
    """``_aggregation_output_dtype`` (string_fastpaths.py:151-157): mean is
    ``result_type(dtype, float32)``, count int32, the rest the value dtype."""
    if agg == "mean":
        return np.float64 if vals.dtype == np.float64 else np.float32
    if agg == "count":
        return np.int32
    return vals.dtype.type


def groupby_encoded_strings(keys, values: dict, agg_funcs: dict, vocab_size: int):
    """``groupby_encoded_strings`` (string_fastpaths.py:41-74) with
    ``_aggregate_by_code`` (:160-184).  Null codes (< 0) are dropped; codes of
    ``vocab_size`` or more are dropped too (``bincount(length=vocab_size)`` and
    the scatters drop out-of-range indices).  Groups are the observed codes in
    ascending order.  Sums accumulate in the value dtype (float sums here in
    float64, rounded once; the reference's scatter-add order is unpinned);
    mean = sum / count in the sum's dtype (integers: true division in the
    default float); min/max propagate NaN."""
    keys = np.asarray(keys)
    valid = (keys >= 0) & (keys < vocab_size)
    if not valid.any():
        return (keys[:0].copy(),
                {c: np.zeros(0, string_agg_dtype(np.asarray(values[c]), a)) for c, a in agg_funcs.items()})
    vk = keys[valid].astype(np.int64)
    counts = np.bincount(vk, minlength=vocab_size)[:vocab_size]
    observed = counts > 0
    codes = np.arange(vocab_size, dtype=keys.dtype)[observed]
    seg_of_code = np.cumsum(observed) - 1
    seg = seg_of_code[vk]
    g = int(observed.sum())
    cnt = counts[observed]
    out = {}
    for col, agg in agg_funcs.items():
        v = np.asarray(values[col])[valid]
        if agg == "count":
            out[col] = cnt.astype(np.int32)
        elif agg == "sum":
            out[col] = _segment_sum(v, seg, g, v.dtype.type)
        elif agg == "mean":
            s = _segment_sum(v, seg, g, v.dtype.type)
            od = string_agg_dtype(v, "mean")
            out[col] = (s.astype(od) / cnt.astype(od)).astype(od)
        elif agg in ("min", "max"):
            out[col] = _segment_max(v, seg, g, agg == "min")
        else:
            raise ValueError(f"Unsupported aggregation function: {agg}")
    return codes, out


def _string_domain(codes, null_code):
    c = np.asarray(codes)
    return np.where(c < 0, null_code, c).astype(np.int32)


def _restore_nulls(codes, null_code):
    return np.where(codes == null_code, -1, codes).astype(np.int32)


def join_encoded_strings(left_keys, right_keys, num_codes: int, how: str):
    """``join_encoded_strings`` (string_fastpaths.py:95-119): null codes become
    the extra code ``num_codes``, so nulls match nulls.  Returns
    ``(joined_codes, left_indices, right_indices)`` (-1: no row).

    Right side unique (every code at most once, :217-262): inner = matched left
    rows in left row order; left = every left row in order; right = matched
    left rows in order, then unmatched right rows ascending; outer = every left
    row in order, then unmatched right rows ascending.

    Otherwise (:265-309) codes ascending; per code the left-major cartesian
    product of its left rows and right rows (each in row order), or for left /
    right / outer joins the code's unmatched rows of one side."""
    if how not in ("inner", "left", "right", "outer"):
        raise ValueError(f"Unsupported join type: {how}")
    null = int(num_codes)
    ld = _string_domain(left_keys, null)
    rd = _string_domain(right_keys, null)
    size = null + 1
    rc = np.bincount(rd, minlength=size)
    nl, nr = len(ld), len(rd)
    if (rc <= 1).all():
        lookup = np.full(size, -1, dtype=np.int32)
        lookup[rd] = np.arange(nr, dtype=np.int32)
        lpos = np.arange(nl, dtype=np.int32)
        mr = lookup[ld] if nl else np.zeros(0, np.int32)
        ok = mr >= 0
        if how == "inner":
            return _restore_nulls(ld[ok], null), lpos[ok], mr[ok]
        if how == "left":
            return _restore_nulls(ld, null), lpos, mr
        hit = np.zeros(nr, dtype=bool)
        hit[mr[ok]] = True
        un = np.flatnonzero(~hit).astype(np.int32)
        neg = np.full(len(un), -1, dtype=np.int32)
        if how == "right":
            return (_restore_nulls(np.concatenate([ld[ok], rd[un]]), null), np.concatenate([lpos[ok], neg]),
                    np.concatenate([mr[ok], un]))
        return (_restore_nulls(np.concatenate([ld, rd[un]]), null), np.concatenate([lpos, neg]),
                np.concatenate([mr, un]))
    # several rows per code on the right: per code, in code order
    lo = np.argsort(ld, kind="stable").astype(np.int32)
    ro = np.argsort(rd, kind="stable").astype(np.int32)
    lcnt = np.bincount(ld, minlength=size)
    rcnt = np.bincount(rd, minlength=size)
    lst = np.concatenate([[0], np.cumsum(lcnt)])
    rst = np.concatenate([[0], np.cumsum(rcnt)])
    codes, li, ri = [], [], []
    for code in np.flatnonzero((lcnt > 0) | (rcnt > 0)):
        L = lo[lst[code]:lst[code + 1]]
        R = ro[rst[code]:rst[code + 1]]
        if len(L) and len(R):
            codes.append(np.full(len(L) * len(R), code, np.int32))
            li.append(np.repeat(L, len(R)))
            ri.append(np.tile(R, len(L)))
        elif len(L) and how in ("left", "outer"):
            codes.append(np.full(len(L), code, np.int32))
            li.append(L)
            ri.append(np.full(len(L), -1, np.int32))
        elif len(R) and how in ("right", "outer"):
            codes.append(np.full(len(R), code, np.int32))
            li.append(np.full(len(R), -1, np.int32))
            ri.append(R)
    if not codes:
        e = np.zeros(0, np.int32)
        return e, e.copy(), e.copy()
    return (_restore_nulls(np.concatenate(codes), null), np.concatenate(li).astype(np.int32),
            np.concatenate(ri).astype(np.int32))


def sortable_string_codes(codes, vocab_size: int, descending: bool = False):
    """``sortable_string_codes`` (string_encoding.py:115-124): lexical order,
    nulls last either way."""
    c = np.asarray(codes)
    if not descending:
        return np.where(c < 0, vocab_size, c)
    return np.where(c < 0, vocab_size, (vocab_size - 1) - c)
