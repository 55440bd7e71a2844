"""The multi-rank drivers (jaxframes_b200.distributed) with CPU ``gloo``
ranks.  The per-rank kernels are replaced by the oracle (CPU); what is under
test is the product's composition: hash repartition of both join sides, then
the local join (distributed/frame.py:814-855); repartition of the group keys,
then the local groupby (:971-999); and the sample sort (splitters from a
gathered sample, exchange by key range, local stable sort), which the
reference leaves as a TODO (multi_column_distributed.py:36-58).  Each rank's
output is compared with the single-process oracle on all ranks' rows."""

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


def _partition(keys, world):
    tgt, perm, offs = O.hash_partition([k.numpy() for k in keys], world)
    return torch.from_numpy(tgt), torch.from_numpy(perm), torch.from_numpy(offs)


def _take(col, perm):
    return col[perm.long()]


def _local_join(lk, lv, rk, rv, how):
    mk, out, _, _ = O.sort_merge_join(lk.numpy(), {c: v.numpy() for c, v in lv.items()}, rk.numpy(),
                                      {c: v.numpy() for c, v in rv.items()}, how)
    return mk, out


def _local_groupby(keys, vals, aggs):
    if isinstance(keys, torch.Tensor):
        return O.groupby_aggregate(keys.numpy(), {c: v.numpy() for c, v in vals.items()}, aggs)
    names = [f"k{i}" for i in range(len(keys))]
    return O.groupby_aggregate_multi_column([k.numpy() for k in keys], names,
                                            {c: v.numpy() for c, v in vals.items()}, aggs)


def _argsort(dest):
    return torch.from_numpy(np.argsort(dest.numpy(), kind="stable"))


def _local_sort(keys, vals, ascending):
    k = keys.numpy()
    sk, perm = O.radix_sort(k, np.arange(len(k)), ascending)
    return sk, {c: v.numpy()[perm] for c, v in vals.items()}


def _rank_data(rank, world):
    rng = np.random.default_rng(200 + rank)
    nl, nr = 3000 + 17 * rank, 1000 + 5 * rank
    lk = rng.integers(0, 1500, nl).astype(np.int64)
    lv = rng.standard_normal(nl).astype(np.float32)
    rk = rng.integers(0, 1500, nr).astype(np.int64)
    rv = rng.integers(-1000, 1000, nr).astype(np.int32)
    gk1 = rng.integers(-40, 40, nl).astype(np.int32)
    gk2 = rng.integers(0, 5, nl).astype(np.int64)
    sk = rng.standard_normal(nl).astype(np.float32)
    sk[::13] = sk[5]  # ties across ranks
    sk[::101] = np.nan
    return dict(lk=lk, lv=lv, rk=rk, rv=rv, gk1=gk1, gk2=gk2, sk=sk)


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from jaxframes_b200.distributed import distributed_groupby, distributed_join, distributed_sort
        d = {k: torch.from_numpy(v) for k, v in _rank_data(rank, world).items()}
        res = {}
        for how in ("inner", "left"):
            res["join_" + how] = distributed_join(d["lk"], {"lv": d["lv"]}, d["rk"], {"rv": d["rv"]}, how,
                                                  local_join=_local_join, partition=_partition, take=_take)
        res["gb1"] = distributed_groupby(d["gk1"], {"v": d["lv"], "c": d["lv"]}, {"v": "sum", "c": "count"},
                                         local_groupby=_local_groupby, partition=_partition, take=_take)
        res["gb2"] = distributed_groupby([d["gk1"], d["gk2"]], {"v": d["lv"], "m": d["lv"]},
                                         {"v": "sum", "m": "max"}, local_groupby=_local_groupby,
                                         partition=_partition, take=_take)
        for asc in (True, False):
            res[f"sort_{asc}"] = distributed_sort(d["sk"], {"row": torch.arange(len(d["sk"])) + rank * 10**6},
                                                  ascending=asc, samples_per_rank=64, argsort=_argsort,
                                                  take=_take, local_sort=_local_sort)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module", params=[2, 3])
def ranks(request):
    world = request.param
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        r, res = q.get(timeout=180)
        got[r] = res
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    data = [_rank_data(r, world) for r in range(world)]
    allv = {k: np.concatenate([d[k] for d in data]) for k in data[0]}
    return world, got, allv


def _owner(keys, world):
    return O.hash_multi_columns(keys) % world


@pytest.mark.parametrize("how", ["inner", "left"])
def test_join_union_of_ranks_is_the_global_join(ranks, how):
    world, got, a = ranks
    emk, eout, _, _ = O.sort_merge_join(a["lk"], {"lv": a["lv"]}, a["rk"], {"rv": a["rv"]}, how)
    own = _owner([emk], world)
    total = 0
    for d in range(world):
        mk, out = got[d]["join_" + how]
        sel = own == d
        np.testing.assert_array_equal(mk, emk[sel])
        for c in eout:
            np.testing.assert_array_equal(out[c], eout[c][sel], err_msg=c)
        total += len(mk)
    assert total == len(emk)


def test_groupby_groups_split_across_ranks(ranks):
    world, got, a = ranks
    ek, eout = O.groupby_aggregate(a["gk1"], {"v": a["lv"], "c": a["lv"]}, {"v": "sum", "c": "count"})
    own = _owner([ek], world)
    for d in range(world):
        uk, out = got[d]["gb1"]
        np.testing.assert_array_equal(uk, ek[own == d])
        for c in eout:
            np.testing.assert_array_equal(out[c], eout[c][own == d], err_msg=c)
    ek, eout = O.groupby_aggregate_multi_column([a["gk1"], a["gk2"]], ["k0", "k1"], {"v": a["lv"], "m": a["lv"]},
                                                {"v": "sum", "m": "max"})
    own = _owner([ek["k0"], ek["k1"]], world)
    for d in range(world):
        uk, out = got[d]["gb2"]
        np.testing.assert_array_equal(uk["k0"], ek["k0"][own == d])
        np.testing.assert_array_equal(uk["k1"], ek["k1"][own == d])
        for c in eout:
            np.testing.assert_array_equal(out[c], eout[c][own == d], err_msg=c)


@pytest.mark.parametrize("asc", [True, False])
def test_sample_sort_concatenation_is_the_global_stable_sort(ranks, asc):
    world, got, a = ranks
    # global rows in (rank, local row) order, tagged with rank * 10^6 + row
    rows = np.concatenate([np.arange(len(_rank_data(r, world)["sk"])) + r * 10**6 for r in range(world)])
    ek, erow = O.radix_sort(a["sk"], rows, asc)
    gk = np.concatenate([got[d][f"sort_{asc}"][0] for d in range(world)])
    grow = np.concatenate([got[d][f"sort_{asc}"][1]["row"] for d in range(world)])
    np.testing.assert_array_equal(gk.view(np.uint32), ek.view(np.uint32))
    np.testing.assert_array_equal(grow, erow)
    sizes = [len(got[d][f"sort_{asc}"][0]) for d in range(world)]
    assert min(sizes) > 0  # the splitters spread the rows


def test_order_key_matches_the_radix_order():
    from jaxframes_b200.distributed import order_key
    x = np.array([3.0, -0.0, 0.0, -1.5, np.nan, np.inf, -np.inf, 1e-30, -1e-30, 2.0], dtype=np.float32)
    ok = order_key(torch.from_numpy(x)).numpy()
    _, perm = O.radix_sort(x, np.arange(len(x)))
    np.testing.assert_array_equal(np.argsort(ok, kind="stable"), perm)
    u = np.array([0, 2**63, 2**64 - 1, 5, 2**63 - 1], dtype=np.uint64)
    np.testing.assert_array_equal(np.argsort(order_key(torch.from_numpy(u)).numpy(), kind="stable"),
                                  np.argsort(u, kind="stable"))
