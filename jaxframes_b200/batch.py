"""Batched hash partition + groupby over many independent queries.

One call (``jfx_batch_partition_groupby``) runs, for every query, the
one-device body of ``collective_hash_repartition`` with P partitions
(parallel_algorithms.py:163-182, :213-214) and
``SortBasedGroupBy.groupby_aggregate`` sum and count (:733-803), on all
queries' rows at once, in one persistent kernel launch (a device work queue
of the queries, one CTA per query).  The launch never synchronises with the
host, so ``BatchedGroupBy.capture()`` records it as one CUDA graph and
``replay()`` re-runs it on new data placed in the same input buffers.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import check
from .parallel_algorithms import as_device


class BatchedGroupBy:
    """Fixed-shape batch: ``n`` rows in ``nq`` queries, ``P`` partitions,
    keys in [0, 2^key_bits).  Input buffers ``keys`` (int32), ``values``
    (float32) and ``query_offsets`` (int64, nq+1) live on the device; fill
    them and call ``run()`` (or ``replay()`` after ``capture()``)."""

    def __init__(self, n: int, nq: int, num_partitions: int = 256, key_bits: int = 20, device=None):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.n, self.nq, self.P, self.key_bits = int(n), int(nq), int(num_partitions), int(key_bits)
        e = lambda k, dt: torch.empty(max(int(k), 1), dtype=dt, device=dev)
        self.keys = e(n, torch.int32)
        self.values = e(n, torch.float32)
        self.query_offsets = e(nq + 1, torch.int64)
        self.part_keys = e(n, torch.int32)
        self.part_values = e(n, torch.float32)
        self.part_offsets = e(nq * (num_partitions + 1), torch.int64)
        self.group_keys = e(n, torch.int32)
        self.group_sums = e(n, torch.float32)
        self.group_counts = e(n, torch.float32)
        self.group_offsets = e(nq + 1, torch.int64)
        self.ws = _lib.workspace(_lib.WS_BATCH, n, nq, device=dev)
        self.graph = None

    def run(self, stream=None):
        L = _lib.lib()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(L.jfx_batch_partition_groupby(
            self.keys.data_ptr(), self.values.data_ptr(), self.query_offsets.data_ptr(), self.nq, self.n, self.P,
            self.key_bits, self.part_keys.data_ptr(), self.part_values.data_ptr(), self.part_offsets.data_ptr(),
            self.group_keys.data_ptr(), self.group_sums.data_ptr(), self.group_counts.data_ptr(),
            self.group_offsets.data_ptr(), self.ws.data_ptr(), self.ws.numel(), s))

    def status(self):
        """Raises if the last run saw a key outside [0, 2^key_bits)."""
        L = _lib.lib()
        check(L.jfx_batch_status(self.ws.data_ptr(), self.ws.numel(), torch.cuda.current_stream().cuda_stream))

    def capture(self):
        """Records one run as a CUDA graph (after one eager run)."""
        self.run()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                self.run(stream=side.cuda_stream)
        torch.cuda.current_stream().wait_stream(side)
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    def query(self, q: int):
        """Per-query views: (partition offsets relative to the query start,
        partitioned keys, values, group keys, sums, counts)."""
        qo = self.query_offsets[q:q + 2].tolist()
        go = self.group_offsets[q:q + 2].tolist()
        po = self.part_offsets[q * (self.P + 1):(q + 1) * (self.P + 1)] - qo[0]
        return (po, self.part_keys[qo[0]:qo[1]], self.part_values[qo[0]:qo[1]], self.group_keys[go[0]:go[1]],
                self.group_sums[go[0]:go[1]], self.group_counts[go[0]:go[1]])


def batch_partition_groupby(keys, values, query_offsets, num_partitions: int = 256, key_bits: int | None = None):
    """Eager helper: copies the inputs into a ``BatchedGroupBy`` and runs it."""
    k = as_device(keys).to(torch.int32)
    v = as_device(values).to(torch.float32)
    qo = as_device(query_offsets).to(torch.int64)
    n = int(qo[-1].item())
    if key_bits is None:
        mx = int(k.max().item()) if n else 0
        key_bits = max(1, mx.bit_length())
    b = BatchedGroupBy(n, qo.numel() - 1, num_partitions, key_bits, device=k.device)
    b.keys[:n].copy_(k[:n])
    b.values[:n].copy_(v[:n])
    b.query_offsets.copy_(qo)
    b.run()
    b.status()
    return b
