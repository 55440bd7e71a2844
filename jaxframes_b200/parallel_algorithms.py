"""Drop-in for ``jaxframes.distributed.parallel_algorithms`` on one B200.

Same names, signatures, argument meaning, return structure and error
behaviour as ``src/jaxframes/distributed/parallel_algorithms.py``; every
computation runs in ``libjfx.so`` (hand-written sm_100a kernels, C ABI in
``include/jfx.h``).  Inputs may be torch tensors, NumPy arrays or any
``__dlpack__`` producer (jax arrays, CuPy); device arrays are imported
zero-copy.  Results are torch CUDA tensors (``jaxframes_b200.interop``
converts them back to jax arrays through DLPack when jax is present).

Dtype rules follow JAX with its default config: integer payloads of a join
are promoted to the default float, integer means are in the default float;
``config.x64 = True`` mirrors ``jax_enable_x64`` (default float = float64).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

from . import _lib
from ._lib import AGG_BITS, check

__all__ = [
    "config", "ShardingSpec", "multi_column_lexsort", "hash_multi_columns", "combine_keys_for_sorting",
    "collective_hash_repartition", "compact_repartitioned_rows", "ParallelRadixSort", "SortBasedGroupBy",
    "ParallelSortMergeJoin", "parallel_sort", "groupby_aggregate", "groupby_aggregate_multi_column",
    "sort_merge_join", "hash_partition", "learned_sort",
]


@dataclass
class _Config:
    x64: bool = False  # mirrors jax_enable_x64: default float is float64 when set

    def default_float(self):
        return torch.float64 if self.x64 else torch.float32


config = _Config()


@dataclass
class ShardingSpec:
    """Stand-in for ``jaxframes.distributed.sharding.ShardingSpec``
    (sharding.py:14-20).  ``mesh`` may be a jax Mesh, an int device count or
    None; only its size matters here.  ``row_sharding`` names the row axis."""

    mesh: Any = None
    row_sharding: str | None = "data"
    col_sharding: str | None = None

    @property
    def size(self) -> int:
        m = self.mesh
        if m is None:
            return 1
        if isinstance(m, int):
            return m
        return int(getattr(m, "size", 1))


# ------------------------------------------------------------------ tensors ---
_NP_OK = {np.dtype(d) for d in ("int8", "int16", "int32", "int64", "uint8", "uint16", "uint32",
                                "uint64", "float32", "float64", "bool")}


def as_device(x, device=None) -> torch.Tensor:
    """1-D contiguous CUDA tensor viewing ``x`` (zero-copy for device arrays)."""
    if not torch.cuda.is_available():
        raise _lib.JfxUnavailable("no CUDA device: the jfx kernels need a B200 (sm_100a); there is no CPU fallback")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if isinstance(x, torch.Tensor):
        t = x
    elif isinstance(x, np.ndarray):
        if x.dtype not in _NP_OK:
            raise TypeError(f"unsupported dtype {x.dtype}")
        t = torch.from_numpy(np.ascontiguousarray(x))
    elif hasattr(x, "__dlpack__"):
        t = torch.from_dlpack(x)
    else:
        t = torch.as_tensor(np.asarray(x))
    if t.dim() != 1:
        t = t.reshape(-1)
    if t.device != dev:
        t = t.to(dev, non_blocking=True)
    return t.contiguous()


def _stream():
    return _lib.stream_handle()


def _empty(n, dtype, like: torch.Tensor | None = None):
    dev = like.device if like is not None else torch.device("cuda", torch.cuda.current_device())
    return torch.empty(int(n), dtype=dtype, device=dev)


def _gather(src: torch.Tensor, idx: torch.Tensor, out_dtype=None) -> torch.Tensor:
    """``src[idx]`` with -1 -> NaN fill and dtype conversion (jfx_gather)."""
    L = _lib.lib()
    out_dtype = out_dtype or src.dtype
    out = _empty(idx.numel(), out_dtype, idx)
    check(L.jfx_gather(src.data_ptr() if src.numel() else None, _lib.jfx_dtype(src), src.numel(), idx.data_ptr(),
                       idx.numel(), out.data_ptr(), _lib.TORCH_TO_JFX[out_dtype], _stream()))
    return out


def _is_float(t: torch.Tensor) -> bool:
    return t.dtype in (torch.float32, torch.float64)


# ---------------------------------------------------------------- sorting ---
def _radix_sort_perm(keys: torch.Tensor, ascending: bool, want_keys: bool):
    L = _lib.lib()
    n = keys.numel()
    perm = _empty(n, torch.int32, keys)
    sk = _empty(n, keys.dtype, keys) if want_keys else None
    if n:
        from .autotune import applied
        ws = _lib.workspace(_lib.WS_SORT, n, device=keys.device)
        col = _lib.column(keys)
        with applied("sort", keys):
            check(L.jfx_sort(ctypes.byref(col), n, 1 if ascending else 0, perm.data_ptr(),
                             sk.data_ptr() if sk is not None else None, ws.data_ptr(), ws.numel(), _stream()))
    return perm, sk


def multi_column_lexsort(keys, ascending=True) -> torch.Tensor:
    """parallel_algorithms.py:25-66.  Stable lexicographic argsort (int32);
    a single key ignores ``ascending`` exactly as the reference does."""
    cols = [as_device(k) for k in keys]
    if not cols:
        raise ValueError("multi_column_lexsort needs at least one key")
    n = cols[0].numel()
    if isinstance(ascending, (bool, np.bool_)):
        ascending = [bool(ascending)] * len(cols)
    ascending = list(ascending)
    if len(ascending) != len(cols):
        raise ValueError("ascending must have one flag per key")
    perm = _empty(n, torch.int32, cols[0])
    if n == 0:
        return perm
    L = _lib.lib()
    arr = (_lib.Column * len(cols))(*[_lib.column(c, 0 if a else _lib.COL_DESC) for c, a in zip(cols, ascending)])
    ws = _lib.workspace(_lib.WS_SORT, n, device=cols[0].device)
    check(L.jfx_lexsort(arr, len(cols), n, perm.data_ptr(), ws.data_ptr(), ws.numel(), _stream()))
    return perm


def hash_multi_columns(keys) -> torch.Tensor:
    """parallel_algorithms.py:69-136 (uint32 per row).  A single float64 key is
    hashed word by word, two words per row, as the reference's ``view`` does."""
    cols = [as_device(k) for k in keys]
    if len(cols) == 1 and cols[0].dtype == torch.float64:
        cols = [cols[0].view(torch.uint32)]
    n = cols[0].numel()
    out = _empty(n, torch.uint32, cols[0])
    if n:
        L = _lib.lib()
        arr = (_lib.Column * len(cols))(*[_lib.column(c) for c in cols])
        check(L.jfx_hash_columns(arr, len(cols), n, out.data_ptr(), _stream()))
    return out


def combine_keys_for_sorting(keys) -> torch.Tensor:
    """parallel_algorithms.py:139-147: rank of each row in the lexicographic order."""
    idx = multi_column_lexsort(keys)
    n = idx.numel()
    ranks = torch.zeros(n, dtype=torch.int32, device=idx.device)
    ranks[idx.long()] = torch.arange(n, dtype=torch.int32, device=idx.device)
    return ranks


def hash_partition(keys, num_partitions: int):
    """One device's body of ``collective_hash_repartition`` with the device count
    set to ``num_partitions`` (parallel_algorithms.py:163-182, :213-214):
    ``target = hash % P`` and a stable counting sort by target.

    Returns ``(targets int32, perm int32, offsets int64[P+1])``: rows of
    partition p are ``perm[offsets[p]:offsets[p+1]]`` in original order."""
    cols = [as_device(k) for k in keys]
    n = cols[0].numel()
    tgt = _empty(n, torch.int32, cols[0])
    perm = _empty(n, torch.int32, cols[0])
    offs = _empty(num_partitions + 1, torch.int64, cols[0])
    L = _lib.lib()
    arr = (_lib.Column * len(cols))(*[_lib.column(c) for c in cols])
    ws = _lib.workspace(_lib.WS_PARTITION, max(n, 1), num_partitions, device=cols[0].device)
    check(L.jfx_hash_partition(arr, len(cols), n, int(num_partitions), tgt.data_ptr(), perm.data_ptr(),
                               offs.data_ptr(), ws.data_ptr(), ws.numel(), _stream()))
    return tgt, perm, offs


def collective_hash_repartition(keys, values, key_dtypes=None, value_dtypes=None, sharding_spec=None):
    """parallel_algorithms.py:185-274.  On one device (or without row sharding)
    the reference returns its inputs unchanged with an all-true mask
    (line 202-203); so does this.  Across ranks the exchange lives in
    ``jaxframes_b200.repartition.exchange_partitions``."""
    if not keys:
        return keys, values, torch.zeros(0, dtype=torch.bool, device="cuda")
    if sharding_spec is None or sharding_spec.size == 1 or not sharding_spec.row_sharding:
        k0 = as_device(keys[0])
        return keys, values, torch.ones(k0.numel(), dtype=torch.bool, device=k0.device)
    from .repartition import collective_repartition
    return collective_repartition(keys, values, sharding_spec)


def compact_repartitioned_rows(keys, values, valid_mask):
    """parallel_algorithms.py:277-293: keep the valid rows, in order."""
    m = as_device(valid_mask)
    if m.numel() == 0:
        return keys, values
    if bool(m.all()):
        return keys, values
    pos = torch.nonzero(m, as_tuple=False).reshape(-1).to(torch.int32)
    ks = [_gather(as_device(k), pos) for k in keys]
    vs = {n: _gather(as_device(a), pos) for n, a in values.items()}
    return ks, vs


class ParallelRadixSort:
    """parallel_algorithms.py:296-603 on the onesweep radix sort."""

    def __init__(self, sharding_spec=None, bits_per_pass: int = 8):
        self.sharding_spec = sharding_spec
        self.bits_per_pass = bits_per_pass  # digit width is chosen per key range; kept for API parity
        self.num_buckets = 2 ** bits_per_pass

    def sort(self, keys, values=None, ascending: bool = True):
        """Line 463-581: ``(sorted_keys, sorted_values)``; the order is a stable
        ascending argsort of the key (JAX float order for floats) and
        ``ascending=False`` reverses the whole result (ties reversed)."""
        k = as_device(keys)
        if k.dtype == torch.bool or k.dtype not in _lib.TORCH_TO_JFX:
            raise TypeError(f"radix sort does not support key dtype {k.dtype}")
        perm, sk = _radix_sort_perm(k, ascending, True)
        sv = None
        if values is not None:
            v = as_device(values)
            sv = _gather(v, perm)
        return sk, sv

    def sort_multi_column(self, keys, values=None, ascending=True):
        """Line 426-461: lexsort, then gather every key and value column."""
        idx = multi_column_lexsort(keys, ascending)
        sorted_keys = [_gather(as_device(k), idx) for k in keys]
        sorted_values = None
        if values is not None:
            sorted_values = {c: _gather(as_device(a), idx) for c, a in values.items()}
        return sorted_keys, sorted_values

    def argsort(self, keys, ascending: bool = True) -> torch.Tensor:
        """The permutation ``sort(keys, arange(n), ascending)[1]`` without the gather."""
        perm, _ = _radix_sort_perm(as_device(keys), ascending, False)
        return perm


def _value_dtype_rules(v: torch.Tensor, agg: str, multi: bool):
    """Output dtypes of one aggregation (parallel_algorithms.py:626-660, :1212-1228)."""
    fl = _is_float(v)
    if agg in ("sum", "min", "max"):
        return v.dtype
    if agg == "count":
        return torch.int32 if multi else v.dtype
    if agg == "mean":
        if multi:
            return torch.float64 if v.dtype == torch.float64 else torch.float32
        return v.dtype if fl else config.default_float()
    raise ValueError(f"Unsupported aggregation function: {agg}")


def _run_groupby(keys, values: dict, agg_funcs: dict, multi: bool, rules=None):
    """One jfx_groupby call.  ``rules(value, agg, multi)`` gives each output's
    dtype (default: the reference module's rules)."""
    rules = rules or _value_dtype_rules
    cols = [as_device(k) for k in keys]
    n = cols[0].numel()
    for c in cols:
        if c.numel() != n:
            raise ValueError("key columns differ in length")
    for col, agg in agg_funcs.items():
        if agg not in AGG_BITS:
            raise ValueError(f"Unsupported aggregation function: {agg}")
    # group the requested aggregations by source column: each source is read once
    srcs: dict[int, dict] = {}
    outputs = {}
    vals = {}
    for col, agg in agg_funcs.items():
        v = as_device(values[col])
        vals[col] = v
    uniq = [_empty(n, c.dtype, c) for c in cols]
    agg_cols = []
    for col, agg in agg_funcs.items():
        v = vals[col]
        odt = rules(v, agg, multi)
        out = _empty(n, odt, v)
        outputs[col] = out
        key = v.data_ptr()
        ent = srcs.get(key)
        if ent is None:
            ent = dict(tensor=v, aggs=0, outs={}, mean_dtype=_lib.F32, count_dtype=_lib.I32)
            srcs[key] = ent
        ent["aggs"] |= AGG_BITS[agg]
        ent["outs"][agg] = out
        if agg == "mean":
            ent["mean_dtype"] = _lib.TORCH_TO_JFX[odt]
        if agg == "count":
            ent["count_dtype"] = _lib.TORCH_TO_JFX[odt]
    # two requests of the same aggregation on one source (aliased columns)
    # need separate entries
    entries = []
    for ent in srcs.values():
        entries.append(ent)
    for col, agg in agg_funcs.items():
        v = vals[col]
        ent = srcs[v.data_ptr()]
        if ent["outs"][agg] is not outputs[col]:
            e2 = dict(tensor=v, aggs=AGG_BITS[agg], outs={agg: outputs[col]}, mean_dtype=_lib.F32,
                      count_dtype=_lib.I32)
            if agg == "mean":
                e2["mean_dtype"] = _lib.TORCH_TO_JFX[outputs[col].dtype]
            if agg == "count":
                e2["count_dtype"] = _lib.TORCH_TO_JFX[outputs[col].dtype]
            entries.append(e2)
    for ent in entries:
        t = ent["tensor"]
        if t.numel() != n:
            raise ValueError("value column length differs from the keys")
        o = ent["outs"]
        agg_cols.append(_lib.AggColumn(
            t.data_ptr(), _lib.jfx_dtype(t), ent["aggs"],
            o["sum"].data_ptr() if "sum" in o else None, o["mean"].data_ptr() if "mean" in o else None,
            o["count"].data_ptr() if "count" in o else None, o["min"].data_ptr() if "min" in o else None,
            o["max"].data_ptr() if "max" in o else None, ent["mean_dtype"], ent["count_dtype"]))
    G = ctypes.c_int64(0)
    if n:
        L = _lib.lib()
        karr = (_lib.Column * len(cols))(*[_lib.column(c) for c in cols])
        varr = (_lib.AggColumn * max(len(agg_cols), 1))(*agg_cols)
        uptrs = (ctypes.c_void_p * len(cols))(*[u.data_ptr() for u in uniq])
        ws = _lib.workspace(_lib.WS_GROUPBY, n, device=cols[0].device)
        check(L.jfx_groupby(karr, len(cols), n, 1 if multi else 0, varr, len(agg_cols), uptrs, ctypes.byref(G),
                            ws.data_ptr(), ws.numel(), _stream()))
    g = G.value
    # the kernels write into n-row buffers (G is known only after they ran);
    # when the groups are much fewer than the rows, copy the G rows out so the
    # caller does not keep the n-row storage alive
    fit = (lambda t: t[:g].clone()) if 2 * g < n else (lambda t: t[:g])
    return [fit(u) for u in uniq], {c: fit(outputs[c]) for c in agg_funcs}


class SortBasedGroupBy:
    """parallel_algorithms.py:606-803."""

    def __init__(self, sharding_spec=None):
        self.sharding_spec = sharding_spec
        self.sorter = ParallelRadixSort(sharding_spec)

    def groupby_aggregate(self, keys, values: dict, agg_funcs: dict):
        """Line 733-803: unique keys ascending and one aggregation per column;
        sum and count in the value dtype."""
        k = as_device(keys)
        if k.numel() == 0:
            return k[:0], {c: as_device(a)[:0] for c, a in values.items()}
        uniq, out = _run_groupby([k], values, agg_funcs, multi=False)
        return uniq[0], out

    def groupby_aggregate_multi_column(self, keys, key_names, values: dict, agg_funcs: dict):
        """Line 662-731: lexicographic group order; count is int32 and mean
        divides by a float32 count."""
        if not keys or as_device(keys[0]).numel() == 0:
            return ({n: as_device(k)[:0] for n, k in zip(key_names, keys)},
                    {c: as_device(a)[:0] for c, a in values.items()})
        uniq, out = _run_groupby(keys, values, agg_funcs, multi=True)
        return dict(zip(key_names, uniq)), out


def _payload_array(payloads, outs=None):
    arr = (_lib.JoinPayload * max(len(payloads), 1))()
    for k, (name, t, side, odt) in enumerate(payloads):
        arr[k] = _lib.JoinPayload(t.data_ptr() if t.numel() else None, t.numel(), _lib.jfx_dtype(t), side,
                                  outs[name].data_ptr() if outs is not None else None, _lib.TORCH_TO_JFX[odt], 0)
    return arr


def _join_prepare(lcols, rcols, how: str, payloads=None):
    """jfx_join_prepare (or jfx_join_prepare_payloads when the payload columns
    [(name, tensor, side, out dtype)] are given, at most 8): returns (plan,
    num_out, workspace); the workspace must outlive every later call that
    uses the plan."""
    L = _lib.lib()
    nl, nr = lcols[0].numel(), rcols[0].numel()
    ws = _lib.workspace(_lib.WS_JOIN, nl, nr, device=lcols[0].device)
    plan = _lib.JoinPlan()
    m = ctypes.c_int64(0)
    la = (_lib.Column * len(lcols))(*[_lib.column(c) for c in lcols])
    ra = (_lib.Column * len(rcols))(*[_lib.column(c) for c in rcols])
    if payloads:
        check(L.jfx_join_prepare_payloads(la, nl, ra, nr, len(lcols), _lib.JOIN_KINDS[how], _payload_array(payloads),
                                          len(payloads), ctypes.byref(plan), ctypes.byref(m), ws.data_ptr(),
                                          ws.numel(), _stream()))
    else:
        check(L.jfx_join_prepare(la, nl, ra, nr, len(lcols), _lib.JOIN_KINDS[how], ctypes.byref(plan),
                                 ctypes.byref(m), ws.data_ptr(), ws.numel(), _stream()))
    return plan, m.value, ws


def _join_expand(plan, m, like, key_cols=None):
    L = _lib.lib()
    li = _empty(m, torch.int32, like)
    ri = _empty(m, torch.int32, like)
    outs = [_empty(m, c.dtype, like) for c in key_cols] if key_cols else []
    if m:
        ptrs = (ctypes.c_void_p * max(len(outs), 1))(*[o.data_ptr() for o in outs]) if outs else None
        check(L.jfx_join_expand(ctypes.byref(plan), li.data_ptr(), ri.data_ptr(), ptrs, _stream()))
    return li, ri, outs


def _join_expand_gather(plan, m, like, key_col, payloads):
    """Merged keys plus the payload columns of ``join`` in one expand kernel
    per 8 payloads.  payloads: [(name, tensor, side 0/1, out dtype)]."""
    L = _lib.lib()
    mk = _empty(m, key_col.dtype, like)
    outs = {name: _empty(m, odt, like) for name, _, _, odt in payloads}
    if m:
        chunks = [payloads[i:i + 8] for i in range(0, len(payloads), 8)] or [[]]
        for ci, chunk in enumerate(chunks):
            keys = (ctypes.c_void_p * 1)(mk.data_ptr()) if ci == 0 else None
            check(L.jfx_join_expand_gather(ctypes.byref(plan), None, None, keys, _payload_array(chunk, outs),
                                           len(chunk), _stream()))
    return mk, outs


def _join_unmatched(plan, side: int, n: int, like):
    L = _lib.lib()
    out = _empty(max(n, 1), torch.int32, like)
    cnt = ctypes.c_int64(0)
    check(L.jfx_join_unmatched(ctypes.byref(plan), side, out.data_ptr(), n, ctypes.byref(cnt), _stream()))
    return out[:cnt.value]


def _same_dtypes(lcols, rcols):
    out_l, out_r = [], []
    for a, b in zip(lcols, rcols):
        if a.dtype != b.dtype:
            t = torch.promote_types(a.dtype, b.dtype)
            a, b = a.to(t), b.to(t)
        out_l.append(a)
        out_r.append(b)
    return out_l, out_r


def _coalesce(left: torch.Tensor, li: torch.Tensor, right: torch.Tensor, ri: torch.Tensor) -> torch.Tensor:
    """_coalesce_join_key (parallel_algorithms.py:1245-1251)."""
    if li.numel() == 0:
        return left[:0]
    L = _lib.lib()
    out = _empty(li.numel(), left.dtype, li)
    check(L.jfx_coalesce(left.data_ptr(), li.data_ptr(), left.numel(), right.data_ptr(), ri.data_ptr(), right.numel(),
                         li.numel(), _lib.jfx_dtype(left), out.data_ptr(), _stream()))
    return out


def _gather_join_column(arr: torch.Tensor, idx: torch.Tensor, dtype_name: str, all_valid: bool) -> torch.Tensor:
    """_gather_join_column (parallel_algorithms.py:1254-1278): string codes are
    filled with -1; with every index valid the column keeps its dtype;
    otherwise integers and bools become float32 with NaN where missing."""
    if idx.numel() == 0:
        return arr[:0]
    if dtype_name == "string" or all_valid:
        return _gather(arr, idx)
    return _gather(arr, idx, arr.dtype if _is_float(arr) else torch.float32)


class ParallelSortMergeJoin:
    """parallel_algorithms.py:806-1075."""

    def __init__(self, sharding_spec=None):
        self.sharding_spec = sharding_spec
        self.sorter = ParallelRadixSort(sharding_spec)

    def join_indices(self, left_keys, right_keys, how: str = "inner"):
        """(merged_keys, left_idx, right_idx) of ``join`` in the reference's row order."""
        if how not in _lib.JOIN_KINDS:
            raise ValueError(f"Unsupported join type: {how}")
        (lk,), (rk,) = _same_dtypes([as_device(left_keys)], [as_device(right_keys)])
        if how == "outer":
            return self._outer_indices(lk, rk)
        plan, m, ws = _join_prepare([lk], [rk], how)
        li, ri, (mk,) = _join_expand(plan, m, lk, [rk if how == "right" else lk])
        del ws
        return mk, li, ri

    def _outer_indices(self, lk, rk):
        # jnp.unique over both sides (line 999-1000), then the first match of
        # each side (searchsorted, line 1003-1046)
        L = _lib.lib()
        both = _empty(lk.numel() + rk.numel(), lk.dtype, lk)
        both[: lk.numel()].copy_(lk)
        both[lk.numel():].copy_(rk)
        uniq, _ = _run_groupby([both], {}, {}, multi=False)
        u = uniq[0]
        _, _, li = self.join_indices(u, lk, "left")
        _, _, ri = self.join_indices(u, rk, "left")
        return u, li, ri

    def join(self, left_keys, left_values: dict, right_keys, right_values: dict, how: str = "inner"):
        """Line 938-1075: ``(merged_keys, {left_<col>, right_<col>})``; payloads
        go through ``where(idx >= 0, col[idx], nan)``, so integer payloads
        become the default float even for an inner join."""
        if how not in _lib.JOIN_KINDS:
            raise ValueError(f"Unsupported join type: {how}")
        if how == "outer":
            mk, li, ri = self.join_indices(left_keys, right_keys, how)
            out = {}
            for c, a in left_values.items():
                t = as_device(a)
                out[f"left_{c}"] = _gather(t, li, t.dtype if _is_float(t) else config.default_float())
            for c, a in right_values.items():
                t = as_device(a)
                out[f"right_{c}"] = _gather(t, ri, t.dtype if _is_float(t) else config.default_float())
            return mk, out
        # the payload columns are handed to the prepare step, which carries
        # them through the sorts when they fit (8 at most per call), and are
        # written by the expand kernel
        lk, rk = as_device(left_keys), as_device(right_keys)
        payloads = []
        for c, a in left_values.items():
            t = as_device(a, lk.device)
            payloads.append((f"left_{c}", t, 0, t.dtype if _is_float(t) else config.default_float()))
        for c, a in right_values.items():
            t = as_device(a, lk.device)
            payloads.append((f"right_{c}", t, 1, t.dtype if _is_float(t) else config.default_float()))
        (lk,), (rk,) = _same_dtypes([lk], [rk])
        plan, m, ws = _join_prepare([lk], [rk], how, payloads if 0 < len(payloads) <= 8 else None)
        mk, out = _join_expand_gather(plan, m, lk, rk if how == "right" else lk, payloads)
        del ws
        return mk, out

    def join_multi_indices(self, left_keys, right_keys, how: str = "inner"):
        """Index pairs of ``join_multi_column`` (parallel_algorithms.py:868-917):
        matches in ORIGINAL row-major order (left row, then right row), then the
        unmatched left rows (left/outer) and unmatched right rows (right/outer),
        the missing side being -1."""
        if how not in _lib.JOIN_KINDS:
            raise ValueError(f"Unsupported join type: {how}")
        lcols, rcols = _same_dtypes([as_device(k) for k in left_keys], [as_device(k) for k in right_keys])
        plan, m, ws = _join_prepare(lcols, rcols, "outer" if how in ("right", "outer") else "inner")
        li, ri, _ = _join_expand(plan, m, lcols[0])
        if m:
            order = multi_column_lexsort([li, ri])
            li, ri = _gather(li, order), _gather(ri, order)
        nl, nr = lcols[0].numel(), rcols[0].numel()
        lun = _join_unmatched(plan, 0, nl, li) if how in ("left", "outer") else li[:0]
        run = _join_unmatched(plan, 1, nr, li) if how in ("right", "outer") else li[:0]
        del ws
        neg = lambda k: torch.full((k,), -1, dtype=torch.int32, device=li.device)
        if how == "inner":
            return li, ri
        if how == "left":
            return torch.cat([li, lun]), torch.cat([ri, neg(lun.numel())])
        if how == "right":
            return torch.cat([li, neg(run.numel())]), torch.cat([ri, run])
        return (torch.cat([li, lun, neg(run.numel())]), torch.cat([ri, neg(lun.numel()), run]))

    def join_multi_column(self, left_keys, left_key_names, left_values, right_keys, right_key_names, right_values,
                          how: str = "inner", left_key_dtypes=None, right_key_dtypes=None, left_value_dtypes=None,
                          right_value_dtypes=None):
        """Line 826-936: keys coalesced left-first, payloads gathered with -1
        (string codes) or NaN fill."""
        li, ri = self.join_multi_indices(left_keys, right_keys, how)
        lcols, rcols = _same_dtypes([as_device(k) for k in left_keys], [as_device(k) for k in right_keys])
        l_ok = how in ("inner", "left") or bool((li >= 0).all())
        r_ok = how in ("inner", "right") or bool((ri >= 0).all())
        keys = {name: _coalesce(lc, li, rc, ri) for name, lc, rc in zip(left_key_names, lcols, rcols)}
        vals = {}
        for name, arr in left_values.items():
            t = as_device(arr)
            dn = (left_value_dtypes or {}).get(name, str(t.dtype))
            vals[f"left_{name}"] = _gather_join_column(t, li, dn, l_ok)
        for name, arr in right_values.items():
            t = as_device(arr)
            dn = (right_value_dtypes or {}).get(name, str(t.dtype))
            vals[f"right_{name}"] = _gather_join_column(t, ri, dn, r_ok)
        return keys, vals


def learned_sort(keys, mode: str = "auto"):
    """Learned-CDF partitioned sort of uint64 keys (no reference counterpart):
    ``(sorted_keys, perm int32, learned_used)``, identical to the plain radix
    sort.  ``mode``: "auto" (learned with plain fallback) or "plain".
    ``learned_used`` is 1 for the learned path, 0 for plain, negative for a
    fallback (-1 model check failed, -3 large-bucket list full)."""
    k = as_device(keys)
    if k.dtype != torch.uint64:
        raise TypeError(f"learned_sort takes uint64 keys, got {k.dtype}")
    n = k.numel()
    out = _empty(n, torch.uint64, k)
    perm = _empty(n, torch.int32, k)
    used = ctypes.c_int32(0)
    if n:
        L = _lib.lib()
        ws = _lib.workspace(_lib.WS_LEARNED, n, device=k.device)
        check(L.jfx_learned_sort(k.data_ptr(), n, out.data_ptr(), perm.data_ptr(), 0 if mode == "auto" else 1,
                                 ctypes.byref(used), ws.data_ptr(), ws.numel(), _stream()))
    return out, perm, int(used.value)


def _default_spec(sharding_spec):
    return sharding_spec if sharding_spec is not None else ShardingSpec(mesh=None, row_sharding=None)


def parallel_sort(arr, sharding_spec=None, values=None, ascending: bool = True):
    """parallel_algorithms.py:1079-1114."""
    sorter = ParallelRadixSort(_default_spec(sharding_spec))
    sk, sv = sorter.sort(arr, values, ascending)
    if values is None:
        return sk
    return sk, sv


def groupby_aggregate(keys, values, agg_funcs, sharding_spec=None):
    """parallel_algorithms.py:1117-1148."""
    return SortBasedGroupBy(_default_spec(sharding_spec)).groupby_aggregate(keys, values, agg_funcs)


def groupby_aggregate_multi_column(keys, key_names, values, agg_funcs, sharding_spec=None):
    """parallel_algorithms.py:1151-1169."""
    return SortBasedGroupBy(_default_spec(sharding_spec)).groupby_aggregate_multi_column(
        keys, key_names, values, agg_funcs)


def sort_merge_join(left_keys, left_values, right_keys, right_values, how: str = "inner", sharding_spec=None):
    """parallel_algorithms.py:1172-1209."""
    return ParallelSortMergeJoin(_default_spec(sharding_spec)).join(left_keys, left_values, right_keys,
                                                                    right_values, how)
