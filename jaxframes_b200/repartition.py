"""Hash repartition across ranks: the multi-device body of
``collective_hash_repartition`` (parallel_algorithms.py:185-274).

Per rank: ``target = hash_multi_columns(keys) % world`` and a stable counting
sort by target (the same kernel as ``hash_partition``), then one exchange of
the per-destination counts and one variable-count ``all_to_all_single`` per
column.  The reference pads every destination bucket to the local row count
(``_bucketize_local_column``, :163-182) and returns a validity mask; here the
exchange moves only real rows, so the mask is all true and
``compact_repartitioned_rows`` is a no-op.  Row order on the receiving rank is
the reference's compacted order: by source rank, then by the source's
original row order.

One process per GPU; ``torch.distributed`` must be initialised (NCCL for CUDA
tensors).  ``local_partition`` can be replaced (tests pass a CPU restatement
to exercise the exchange with ``gloo`` ranks).
"""

from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist


def _gpu_partition(keys, world):
    from .parallel_algorithms import hash_partition
    return hash_partition(keys, world)


def _gpu_take(col: torch.Tensor, perm: torch.Tensor) -> torch.Tensor:
    from .parallel_algorithms import _gather
    return _gather(col, perm)


def exchange_partitions(keys: list, values: dict, group=None,
                        local_partition: Callable | None = None,
                        take: Callable | None = None):
    """Sends every row to rank ``hash(keys) % world``.

    Returns ``(keys, values, valid_mask)`` with the received rows.
    """
    world = dist.get_world_size(group)
    part = local_partition or _gpu_partition
    take = take or _gpu_take
    tgt, perm, offsets = part(keys, world)
    offsets = torch.as_tensor(offsets)
    send_counts = (offsets[1:] - offsets[:-1]).to(torch.int64)
    dev = keys[0].device
    send_counts = send_counts.to(dev)
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts, group=group)
    send_splits = send_counts.tolist()
    recv_splits = recv_counts.tolist()
    total = int(sum(recv_splits))

    def move(col: torch.Tensor) -> torch.Tensor:
        send = take(col, perm)
        recv = torch.empty(total, dtype=col.dtype, device=col.device)
        dist.all_to_all_single(recv, send, recv_splits, send_splits, group=group)
        return recv

    out_keys = [move(k) for k in keys]
    out_vals = {name: move(v) for name, v in values.items()}
    mask = torch.ones(total, dtype=torch.bool, device=dev)
    return out_keys, out_vals, mask


def collective_repartition(keys, values, sharding_spec, group=None):
    """``collective_hash_repartition`` for a row-sharded spec across ranks."""
    from .parallel_algorithms import as_device
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("collective_hash_repartition across devices needs torch.distributed initialised "
                           "(one process per GPU)")
    ks = [as_device(k) for k in keys]
    vs = {n: as_device(v) for n, v in values.items()}
    return exchange_partitions(ks, vs, group=group)
