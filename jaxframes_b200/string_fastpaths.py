"""Dictionary-encoded string keys on the B200 kernels.

jaxframes keeps a string column as int32 codes into a lexicographically
sorted vocabulary with null = -1 (core/string_encoding.py:37-51), and its
eager string groupby and join (core/string_fastpaths.py) work on those codes
with ``bincount`` scatters and a per-code Python loop.  Here the same
functions run on the integer kernels: the groupby is ``jfx_groupby`` over the
codes, the join is the sort-merge join over the codes with null mapped to
the extra code ``num_codes`` (so nulls match nulls, as in the reference),
and the reference's row orders are rebuilt with stable radix sorts.

Results are torch CUDA tensors; ``StringJoinPlan`` holds the joined codes
(null back to -1) and the row indices of each side (-1: no row).
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import parallel_algorithms as P

SUPPORTED_STRING_GROUPBY_AGGS = {"sum", "mean", "min", "max", "count"}
SUPPORTED_STRING_JOIN_HOW = {"inner", "left", "right", "outer"}


@dataclass(frozen=True)
class StringJoinPlan:
    """string_fastpaths.py:17-23."""

    joined_codes: torch.Tensor
    left_indices: torch.Tensor
    right_indices: torch.Tensor


def _string_rules(v: torch.Tensor, agg: str, multi: bool):
    """``_aggregation_output_dtype`` (string_fastpaths.py:151-157)."""
    if agg not in SUPPORTED_STRING_GROUPBY_AGGS:
        raise ValueError(f"Unsupported aggregation function: {agg}")
    if agg == "mean":
        return torch.float64 if v.dtype == torch.float64 else torch.float32
    if agg == "count":
        return torch.int32
    return v.dtype


def groupby_encoded_strings(keys, values: dict, agg_funcs: dict, vocab_size: int):
    """``groupby_encoded_strings`` (string_fastpaths.py:41-74): observed codes
    ascending, null codes (< 0) and codes outside the vocabulary dropped;
    count int32, mean in ``result_type(value, float32)``."""
    k = P.as_device(keys)
    vals = {c: P.as_device(values[c], k.device) for c in agg_funcs}
    if k.numel() == 0:
        return k[:0], {c: P._empty(0, _string_rules(vals[c], a, False), k) for c, a in agg_funcs.items()}
    uniq, out = P._run_groupby([k], vals, agg_funcs, multi=False, rules=_string_rules)
    codes = uniq[0]
    # groups ascend, so the in-vocabulary codes are one slice [lo, hi)
    bounds = torch.searchsorted(codes, torch.tensor([0, int(vocab_size)], dtype=codes.dtype, device=codes.device))
    lo, hi = (int(x) for x in bounds.tolist())
    return codes[lo:hi], {c: t[lo:hi] for c, t in out.items()}


def _domain(codes: torch.Tensor, null_code: int) -> torch.Tensor:
    return torch.where(codes < 0, torch.full_like(codes, null_code), codes).to(torch.int32)


def _restore(codes: torch.Tensor, null_code: int) -> torch.Tensor:
    return torch.where(codes == null_code, torch.full_like(codes, -1), codes).to(torch.int32)


def _take(t: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
    return P._gather(t, idx)


def _stable_order(key: torch.Tensor) -> torch.Tensor:
    return P.ParallelRadixSort().argsort(key)


def _right_is_unique(rd: torch.Tensor) -> bool:
    if rd.numel() < 2:
        return True
    sk, _ = P.ParallelRadixSort().sort(rd)
    return not bool((sk[1:] == sk[:-1]).any())


def join_encoded_strings(left_keys, right_keys, num_codes: int, how: str) -> StringJoinPlan:
    """``join_encoded_strings`` (string_fastpaths.py:95-119) on the join kernels.

    Right side unique (:217-262): inner = matched left rows in left row order;
    left = every left row in order; right / outer = those, then the unmatched
    right rows ascending.  Otherwise (:265-309): codes ascending, per code the
    left-major product of its rows (the sort-merge join's pair order), or the
    code's unmatched rows of one side for left / right / outer joins."""
    if how not in SUPPORTED_STRING_JOIN_HOW:
        raise ValueError(f"Unsupported join type: {how}")
    null = int(num_codes)
    lk = P.as_device(left_keys)
    rk = P.as_device(right_keys, lk.device)
    ld, rd = _domain(lk, null), _domain(rk, null)
    j = P.ParallelSortMergeJoin()
    neg = lambda k: torch.full((k,), -1, dtype=torch.int32, device=lk.device)
    rows = lambda k: torch.arange(k, dtype=torch.int32, device=lk.device)
    unique = _right_is_unique(rd)
    if ld.numel() == 0 or rd.numel() == 0:
        # one side empty: nothing matches; the other side's rows are kept by
        # left / right / outer joins, in row order when the right side is
        # unique and by code (row order inside a code) otherwise
        if how == "inner" or (how == "left" and ld.numel() == 0) or (how == "right" and rd.numel() == 0) or \
                ld.numel() + rd.numel() == 0:
            e = ld[:0]
            return StringJoinPlan(e, e.clone(), e.clone())
        if ld.numel():
            li, ri, codes = rows(ld.numel()), neg(ld.numel()), ld
        else:
            li, ri, codes = neg(rd.numel()), rows(rd.numel()), rd
        if not unique and ld.numel() == 0:
            order = _stable_order(codes)
            codes, ri = _take(codes, order), _take(ri, order)
        return StringJoinPlan(_restore(codes, null), li, ri)
    if unique:
        # join_multi_indices emits matches in left row order (one right row
        # each), then the unmatched left rows, then the unmatched right rows
        li, ri = j.join_multi_indices([ld], [rd], how)
        m = li.numel()
        if how in ("left", "outer"):
            nun_r = int((li < 0).sum()) if how == "outer" else 0
            head = m - nun_r  # matched + unmatched left rows: every left row once
            order = _stable_order(li[:head])
            li = torch.cat([_take(li[:head], order), li[head:]])
            ri = torch.cat([_take(ri[:head], order), ri[head:]])
        codes = P._coalesce(ld, li, rd, ri) if m else ld[:0]
        return StringJoinPlan(_restore(codes, null), li, ri)
    # several right rows per code: pairs in (code, left row, right row) order
    plan, m, ws = P._join_prepare([ld], [rd], "outer")
    li, ri, (codes,) = P._join_expand(plan, m, ld, [ld])
    parts_c, parts_l, parts_r = [codes], [li], [ri]
    if how in ("left", "outer"):
        ul = P._join_unmatched(plan, 0, ld.numel(), ld)
        parts_c.append(_take(ld, ul))
        parts_l.append(ul)
        parts_r.append(neg(ul.numel()))
    if how in ("right", "outer"):
        ur = P._join_unmatched(plan, 1, rd.numel(), ld)
        parts_c.append(_take(rd, ur))
        parts_l.append(neg(ur.numel()))
        parts_r.append(ur)
    del ws
    codes, li, ri = torch.cat(parts_c), torch.cat(parts_l), torch.cat(parts_r)
    if len(parts_c) > 1 and codes.numel():
        # a code's rows are all pairs or all unmatched rows of one side, so a
        # stable sort by code puts each list's rows at their code
        order = _stable_order(codes)
        codes, li, ri = _take(codes, order), _take(li, order), _take(ri, order)
    return StringJoinPlan(_restore(codes, null), li, ri)


def assemble_string_join_payloads(plan: StringJoinPlan, left_values: dict, right_values: dict,
                                  left_dtypes: dict, right_dtypes: dict):
    """``assemble_string_join_payloads`` (string_fastpaths.py:122-148) with
    ``_gather_join_payload`` (:357-378): string payloads filled with -1, other
    columns kept when every row matched, else integers and bools promoted to
    float32 with NaN where a row is missing."""
    data = {"key_codes": plan.joined_codes}
    dtypes = {"key_codes": "string"}
    l_ok = bool((plan.left_indices >= 0).all()) if plan.left_indices.numel() else True
    r_ok = bool((plan.right_indices >= 0).all()) if plan.right_indices.numel() else True
    for name, arr in left_values.items():
        t = P.as_device(arr)
        data[f"left_{name}"] = P._gather_join_column(t, plan.left_indices, left_dtypes[name], l_ok)
        dtypes[f"left_{name}"] = left_dtypes[name]
    for name, arr in right_values.items():
        t = P.as_device(arr)
        data[f"right_{name}"] = P._gather_join_column(t, plan.right_indices, right_dtypes[name], r_ok)
        dtypes[f"right_{name}"] = right_dtypes[name]
    return data, dtypes, {}


def sortable_string_codes(codes, vocab_size: int, descending: bool = False) -> torch.Tensor:
    """``sortable_string_codes`` (string_encoding.py:115-124): lexical order,
    nulls last either way; the result sorts with ``ParallelRadixSort``."""
    c = P.as_device(codes)
    null = torch.full_like(c, int(vocab_size))
    if not descending:
        return torch.where(c < 0, null, c)
    return torch.where(c < 0, null, (int(vocab_size) - 1) - c)
