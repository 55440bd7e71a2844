"""The hot path across ranks: one process per GPU, ``torch.distributed``
(NCCL for CUDA tensors) for the exchange, the single-GPU kernels for the
local work.

* ``distributed_join``: both sides are repartitioned by
  ``hash_multi_columns(keys) % world`` and joined locally -- the order of
  ``DistributedJaxFrame.merge`` (distributed/frame.py:814-855:
  ``collective_hash_repartition`` + ``compact_repartitioned_rows`` on each
  side, then ``sort_merge_join`` / ``join_multi_column``).  Rows of one key
  meet on one rank, so the union of the ranks' outputs is the global join.
* ``distributed_groupby``: the group keys are repartitioned the same way and
  grouped locally (distributed/frame.py:971-999); each group lives on one
  rank.
* ``distributed_sort``: a sample sort, which the reference leaves as a TODO
  that falls back to a local lexsort (multi_column_distributed.py:36-58):
  every rank contributes a strided sample of its keys, the gathered sample
  gives ``world - 1`` splitters, each row goes to the rank of its key range
  (equal keys to one rank), and the received rows -- ordered by source rank,
  then by source row -- are sorted stably.  Rank r then holds the r-th block
  of the global stable order (``ascending=False``: of its reverse).

The partition, gather and local operators are injectable so that the
exchange logic runs with CPU ``gloo`` ranks in tests; by default they are the
CUDA path (``hash_partition``, ``jfx_gather``, ``sort_merge_join``,
``groupby_aggregate*``, ``ParallelRadixSort``).
"""

from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist

from .repartition import exchange_partitions


def _world(group):
    return dist.get_world_size(group)


def distributed_join(left_keys, left_values: dict, right_keys, right_values: dict, how: str = "inner",
                     group=None, local_join: Callable | None = None, partition: Callable | None = None,
                     take: Callable | None = None):
    """Hash-repartitioned join.  ``left_keys`` / ``right_keys``: one key
    column (tensor) or a list of them.  Returns this rank's part of the join:
    ``(merged_keys, values)`` for one key column, as ``sort_merge_join``
    (parallel_algorithms.py:1172-1209); ``(keys dict, values)`` for several,
    as ``join_multi_column`` (:826-936)."""
    single = isinstance(left_keys, torch.Tensor)
    lk = [left_keys] if single else list(left_keys)
    rk = [right_keys] if single else list(right_keys)
    lk, lv, _ = exchange_partitions(lk, dict(left_values), group=group, local_partition=partition, take=take)
    rk, rv, _ = exchange_partitions(rk, dict(right_values), group=group, local_partition=partition, take=take)
    if local_join is None:
        from . import parallel_algorithms as P
        if single:
            return P.sort_merge_join(lk[0], lv, rk[0], rv, how)
        names = [f"key{i}" for i in range(len(lk))]
        return P.ParallelSortMergeJoin().join_multi_column(lk, names, lv, rk, names, rv, how)
    return local_join(lk[0] if single else lk, lv, rk[0] if single else rk, rv, how)


def distributed_groupby(keys, values: dict, agg_funcs: dict, key_names=None, group=None,
                        local_groupby: Callable | None = None, partition: Callable | None = None,
                        take: Callable | None = None):
    """Hash-repartitioned groupby; this rank's groups, keys ascending.  One
    key column (tensor): ``groupby_aggregate``'s result (:1117-1148); a list:
    ``groupby_aggregate_multi_column``'s (:1151-1169)."""
    single = isinstance(keys, torch.Tensor)
    ks = [keys] if single else list(keys)
    vals = {c: values[c] for c in agg_funcs}
    ks, vals, _ = exchange_partitions(ks, vals, group=group, local_partition=partition, take=take)
    if local_groupby is None:
        from . import parallel_algorithms as P
        if single:
            return P.groupby_aggregate(ks[0], vals, agg_funcs)
        names = key_names or [f"key{i}" for i in range(len(ks))]
        return P.groupby_aggregate_multi_column(ks, names, vals, agg_funcs)
    return local_groupby(ks[0] if single else ks, vals, agg_funcs)


# ----------------------------------------------------------------- sort ---
def order_key(t: torch.Tensor) -> torch.Tensor:
    """int64 whose signed order is ParallelRadixSort's order of ``t``
    (parallel_algorithms.py:495-501, :583-603): integers by value, floats in
    the float total order with -0.0 == +0.0 and every NaN last."""
    if t.dtype in (torch.float32, torch.float64):
        x = t.to(torch.float64)
        x = torch.where(x == 0, torch.zeros_like(x), x)
        b = x.view(torch.int64)
        b = torch.where(torch.isnan(x), torch.full_like(b, 0x7FF8000000000000), b)
        # sign-magnitude bits -> two's-complement order: a negative float's
        # magnitude bits are flipped, so a larger magnitude sorts lower
        return torch.where(b < 0, b ^ 0x7FFFFFFFFFFFFFFF, b)
    if t.dtype == torch.uint64:
        return t.view(torch.int64) ^ torch.iinfo(torch.int64).min
    if t.dtype == torch.uint32:
        return t.to(torch.int64) & 0xFFFFFFFF
    return t.to(torch.int64)


def splitters_from_sample(sample: torch.Tensor, world: int) -> torch.Tensor:
    """``world - 1`` splitters (order keys) at the sample's quantiles."""
    s, _ = torch.sort(sample)
    if s.numel() == 0 or world == 1:
        return s[:0]
    idx = (torch.arange(1, world, device=s.device) * s.numel()) // world
    return s[idx.clamp(max=s.numel() - 1)]


def _gpu_stable_argsort(ok: torch.Tensor) -> torch.Tensor:
    from .parallel_algorithms import ParallelRadixSort
    return ParallelRadixSort().argsort(ok)


def distributed_sort(keys: torch.Tensor, values: dict | None = None, ascending: bool = True, group=None,
                     samples_per_rank: int = 1024, argsort: Callable | None = None, take: Callable | None = None,
                     local_sort: Callable | None = None):
    """Sample sort across ranks.  Returns this rank's block of the global
    stable order: ``(sorted_keys, sorted_values)`` as ``ParallelRadixSort.sort``
    (parallel_algorithms.py:463-581) would return for the concatenation of all
    ranks' rows, split at the splitters."""
    world = _world(group)
    argsort = argsort or _gpu_stable_argsort
    ok = order_key(keys)
    n = ok.numel()
    dev = ok.device
    S = int(samples_per_rank)
    # a strided sample of this rank's keys (S order keys and how many are real)
    if n:
        pos = (torch.arange(S, device=dev, dtype=torch.int64) * n) // S
        smp = ok[pos]
    else:
        smp = torch.zeros(S, dtype=torch.int64, device=dev)
    cnt = torch.tensor([min(n, S) if n else 0], dtype=torch.int64, device=dev)
    all_smp = [torch.empty_like(smp) for _ in range(world)]
    all_cnt = [torch.empty_like(cnt) for _ in range(world)]
    dist.all_gather(all_smp, smp, group=group)
    dist.all_gather(all_cnt, cnt, group=group)
    pool = torch.cat([s[: (S if int(c) else 0)] for s, c in zip(all_smp, all_cnt)])
    spl = splitters_from_sample(pool, world)
    # destination: the number of splitters below the key (equal keys share a rank)
    dest = torch.searchsorted(spl, ok, right=False).to(torch.int32) if world > 1 else torch.zeros(
        n, dtype=torch.int32, device=dev)
    if not ascending:
        dest = (world - 1) - dest
    # rows grouped by destination, original order inside each group
    perm = argsort(dest)
    counts = torch.bincount(dest.to(torch.int64), minlength=world)
    offsets = torch.zeros(world + 1, dtype=torch.int64, device=dev)
    offsets[1:] = torch.cumsum(counts, 0)

    def fixed(_keys, _world):
        return dest, perm, offsets

    vals = dict(values or {})
    (rkeys,), rvals, _ = exchange_partitions([keys], vals, group=group, local_partition=fixed, take=take)
    if local_sort is not None:
        return local_sort(rkeys, rvals, ascending)
    from .parallel_algorithms import ParallelRadixSort, _gather
    p = ParallelRadixSort().argsort(rkeys, ascending)
    return _gather(rkeys, p), {c: _gather(v, p) for c, v in rvals.items()} if values is not None else None
