"""The cross-rank exchange of the hash repartition with world_size-2 ``gloo``
ranks on CPU.  The per-rank partition is the oracle (CPU), injected; the
exchange (count all_to_all, variable all_to_all per column, order) is the
product code under test."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import jfx_oracle as O


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_partition(keys, world):
    tgt, perm, offs = O.hash_partition([k.numpy() for k in keys], world)
    return torch.from_numpy(tgt), torch.from_numpy(perm), torch.from_numpy(offs)


def _take(col, perm):
    return col[perm.long()]


def _rank_data(rank, n=1000):
    rng = np.random.default_rng(100 + rank)
    k1 = rng.integers(-50, 50, n).astype(np.int32)
    k2 = rng.integers(0, 7, n).astype(np.int64)
    v = rng.standard_normal(n).astype(np.float32)
    return k1, k2, v


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from jaxframes_b200.repartition import exchange_partitions
        k1, k2, v = _rank_data(rank)
        keys, vals, mask = exchange_partitions([torch.from_numpy(k1), torch.from_numpy(k2)],
                                               {"v": torch.from_numpy(v)},
                                               local_partition=_oracle_partition, take=_take)
        q.put((rank, keys[0].numpy(), keys[1].numpy(), vals["v"].numpy(), mask.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_exchange_matches_reference_order(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        r, a, b, c, m = q.get(timeout=120)
        got[r] = (a, b, c, m)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # expected: rank d receives, from each source s in order, the rows of s
    # whose hash % world == d, in s's original order
    data = [_rank_data(r) for r in range(world)]
    for d in range(world):
        ek1, ek2, ev = [], [], []
        for s in range(world):
            k1, k2, v = data[s]
            t = O.hash_multi_columns([k1, k2]) % world
            sel = np.flatnonzero(t == d)
            ek1.append(k1[sel])
            ek2.append(k2[sel])
            ev.append(v[sel])
        a, b, c, m = got[d]
        np.testing.assert_array_equal(a, np.concatenate(ek1))
        np.testing.assert_array_equal(b, np.concatenate(ek2))
        np.testing.assert_array_equal(c, np.concatenate(ev))
        assert m.all()
    assert sum(len(got[d][0]) for d in range(world)) == 1000 * world
