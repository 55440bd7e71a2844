#!/usr/bin/env python
"""Benchmark of the jaxframes distributed-algorithms hot path on B200.

Headline workload: sort-merge inner join, left 10M rows (int64 key uniform in
[0, 5M), float32 payload), right 5M rows (key = a permutation of 0..5M-1,
int32 payload over the full int32 range), output (left_idx, right_idx) pairs
plus the gathered payloads -- one step is one ``ParallelSortMergeJoin.join``
through the public API.  Inputs are synthetic (``np.random.default_rng(43)``)
and larger than L2 (180 MB resident), so no L2 flush is needed between steps.

``value`` = input rows (left + right) per second over the whole job with
inputs resident in HBM; ``e2e`` = the same through the API from pinned host
buffers, host<->device copies included.  ``--impl reference`` times the
reference's algorithm on the host CPU (the NumPy restatement; jaxframes itself
needs jax, which is not installed) on a bounded sample.

Prints one JSON line (rank 0).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NL, NR = 10_000_000, 5_000_000
METRIC = "sort-merge inner join throughput (input rows/s)"
WORKLOAD = "sort-merge inner join 10M x 5M int64 keys, f32 + i32 payloads"


def make_join_inputs(nl=NL, nr=NR, seed=43):
    rng = np.random.default_rng(seed)
    lk = rng.integers(0, nr, nl, dtype=np.int64)
    lv = rng.standard_normal(nl, dtype=np.float32)
    rk = rng.permutation(nr).astype(np.int64)
    rv = rng.integers(-2**31, 2**31, nr, dtype=np.int64).astype(np.int32)
    return lk, lv, rk, rv


def make_join_shard(rank, world, nl=NL, nr=NR):
    """Rank ``rank``'s shard of the join scaled to ``world`` ranks (weak
    scaling): ``nl`` left rows with keys uniform in [0, world * nr) and ``nr``
    right rows holding the keys [rank * nr, (rank + 1) * nr) in random order,
    so that the right keys of all ranks are one permutation of
    0..world * nr - 1 and every left row matches exactly one right row.  With
    world == 1 this is ``make_join_inputs``."""
    if world == 1:
        return make_join_inputs(nl, nr)
    rng = np.random.default_rng(43 + 1000 * rank)
    lk = rng.integers(0, world * nr, nl, dtype=np.int64)
    lv = rng.standard_normal(nl, dtype=np.float32)
    rk = (rng.permutation(nr) + rank * nr).astype(np.int64)
    rv = rng.integers(-2**31, 2**31, nr, dtype=np.int64).astype(np.int32)
    return lk, lv, rk, rv


def c3_inputs(n=100_000_000, seed=44):
    """Multi-key groupby input: k1 truncated Zipf(s=1.1) over 1M ranks mapped
    through a permutation, k2 uniform in [0, 64), v1 N(0,1) float32, v2 uniform
    int64 in [-1e6, 1e6]."""
    rng = np.random.default_rng(seed)
    ranks = np.arange(1, 1_000_001, dtype=np.float64)
    cdf = np.cumsum(ranks ** -1.1)
    cdf /= cdf[-1]
    perm = rng.permutation(1_000_000).astype(np.int32)
    k1 = perm[np.searchsorted(cdf, rng.random(n))]
    k2 = rng.integers(0, 64, n, dtype=np.int64).astype(np.int32)
    v1 = rng.standard_normal(n, dtype=np.float32)
    v2 = rng.integers(-1_000_000, 1_000_001, n, dtype=np.int64)
    return k1, k2, v1, v2


def c4_keys(nblocks=65_536, block=4096, seed=45):
    """Skewed uint64 keys: blocks of 4096 assigned by a permutation to 40%
    floor(lognormal(20, 2)), 40% floored continuous power law (s = 1.2) on
    [1, 2^40], 20% ascending runs from a uniform start in [0, 2^63) with 5% of
    positions swapped inside the run."""
    rng = np.random.default_rng(seed)
    n_ln = int(nblocks * 0.4)
    n_zf = int(nblocks * 0.4)
    n_run = nblocks - n_ln - n_zf
    kinds = rng.permutation(nblocks)
    out = np.empty((nblocks, block), dtype=np.uint64)
    ln = np.floor(rng.lognormal(20.0, 2.0, size=(n_ln, block)))
    out[kinds[:n_ln]] = np.clip(ln, 0, 2.0 ** 63).astype(np.uint64)
    s_, m_ = 1.2, 2.0 ** 40
    u = rng.random((n_zf, block))
    zf = np.floor((1.0 - u * (1.0 - m_ ** (1.0 - s_))) ** (1.0 / (1.0 - s_)))
    out[kinds[n_ln:n_ln + n_zf]] = zf.astype(np.uint64)
    start = rng.integers(0, 2 ** 63, n_run, dtype=np.uint64)
    runs = start[:, None] + np.arange(block, dtype=np.uint64)[None, :]
    rows = np.arange(n_run)
    for _ in range(int(round(0.05 * block))):
        i = rng.integers(0, block, n_run)
        j = rng.integers(0, block, n_run)
        a, b = runs[rows, i].copy(), runs[rows, j].copy()
        runs[rows, i], runs[rows, j] = b, a
    out[kinds[n_ln + n_zf:]] = runs
    return out.reshape(-1)


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one
# k_onesweep launch of this workload, averaged over the six radix passes of
# one join call: 544.7 MB over 6 launches in an ncu capture of those launches
# (`--metrics dram__bytes_read.sum,dram__bytes_write.sum -k regex:k_onesweep
# -s 30 -c 6` around `bench.py --profile --steps 1 --warmup 5`); the writes
# that are still in L2 when a launch ends are not counted.
ONESWEEP_DRAM_BYTES_PER_LAUNCH = 90.8e6


def join_model_bytes(nl, nr, m):
    """Algorithmic bytes of the join: SORT(L) + SORT(R) + merge read + output,
    with K = 8 (int64 key), I = 4, P = ceil(23 / 11) = 3 passes."""
    K, I, P = 8, 4, 3
    sort = lambda n: n * (8 + (K + I) + (P - 1) * 2 * (K + I))
    return sort(nl) + sort(nr) + (nl + nr) * (K + I) + m * (2 * I + K + 4 + 4 + 4 + 4)


# ------------------------------------------------------------------ clocks ---
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- CPU legs ---
def cpu_join_sample(nl, nr, seconds=10.0):
    """Single-threaded oracle join on a sample; rows/s."""
    from oracle import jfx_oracle as O
    lk, lv, rk, rv = make_join_inputs(nl, nr, seed=44)
    reps, t0 = 0, time.perf_counter()
    while True:
        O.sort_merge_join(lk, {"lv": lv}, rk, {"rv": rv}, "inner")
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds or reps >= 50:
            break
    return (nl + nr) * reps / el, reps


_REF = {}


def _ref_worker(p):
    from oracle import jfx_oracle as O
    lk, lv, rk, rv, lp, rp = (_REF[k] for k in ("lk", "lv", "rk", "rv", "lp", "rp"))
    li = np.flatnonzero(lp == p)
    ri = np.flatnonzero(rp == p)
    mk, out, _, _ = O.sort_merge_join(lk[li], {"lv": lv[li]}, rk[ri], {"rv": rv[ri]}, "inner")
    return len(mk)


def run_reference(args):
    """The reference's algorithm on the host CPU: the oracle restatement of
    ParallelSortMergeJoin.join on a sample of the workload, hash-partitioned
    across all available cores (one process per core)."""
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0))
    nl, nr = NL // 5, NR // 5
    lk, lv, rk, rv = make_join_inputs(nl, nr, seed=44)
    _REF.update(lk=lk, lv=lv, rk=rk, rv=rv, lp=(lk % cores).astype(np.int32), rp=(rk % cores).astype(np.int32))
    ctx = mp.get_context("fork")  # this arm never initialises CUDA
    times = []
    with ctx.Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            m = sum(pool.map(_ref_worker, range(cores)))
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
    ms = 1000 * statistics.mean(times)
    value = (nl + nr) / (ms / 1000)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{nl} x {nr} rows per step", "parallelism": f"{cores} processes"},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": cores, "kind": "port",
                         "sample": f"inner join {nl} x {nr} rows, hash-partitioned over {cores} processes; "
                                   "NumPy restatement of parallel_algorithms.py:938-1075 (jax not installed)"},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "matched_rows": m,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- parity ---
def check_join_parity(mk, out, lk, lv, rk, rv):
    """The join's merged keys and payloads against the oracle's
    ParallelSortMergeJoin.join (parallel_algorithms.py:938-1075), bit-exact."""
    from oracle import jfx_oracle as O
    t0 = time.perf_counter()
    emk, eout, _, _ = O.sort_merge_join(lk, {"lv": lv}, rk, {"rv": rv}, "inner")
    ok = mk.numel() == len(emk) and np.array_equal(mk.cpu().numpy(), emk)
    for c, e in eout.items():
        g = out[c].cpu().numpy()
        ok = ok and g.dtype == e.dtype and np.array_equal(g.view(np.uint8), e.view(np.uint8))
    return {"ok": bool(ok), "against": "oracle, bit-exact", "rows": int(len(emk)),
            "check_s": round(time.perf_counter() - t0, 1)}


def stable_argsort_ok(keys, perm):
    """On the device: ``perm`` is the stable ascending argsort of uint64
    ``keys`` -- a permutation, keys non-decreasing along it, and equal keys in
    ascending row order.  These three properties determine the stable argsort
    uniquely, so this is the same check as comparing with
    ``np.argsort(kind="stable")``."""
    import torch
    n = keys.numel()
    p = perm.long()
    if n == 0:
        return True
    if int(p.min()) < 0 or int(p.max()) >= n:
        return False
    seen = torch.zeros(n, dtype=torch.bool, device=keys.device)
    seen[p] = True
    if not bool(seen.all()):
        return False
    del seen
    s = keys.view(torch.int64)[p] ^ torch.iinfo(torch.int64).min  # unsigned order as signed
    ok = bool((s[1:] >= s[:-1]).all())
    ties = s[1:] == s[:-1]
    ok = ok and bool((p[1:] > p[:-1])[ties].all())
    return ok


def check_groupby_parity(k1, k2, v1, v2, got_keys, got):
    """groupby_aggregate_multi_column (:662-731, :1212-1242) against the
    oracle: keys, counts, min/max and integer sums bit-exact, float32 sums
    within 2^-16 * sum(|x|) per group, means within that over the count."""
    from oracle import jfx_oracle as O
    t0 = time.perf_counter()
    hv = {f"v1_{a}": v1 for a in ("sum", "mean", "min", "max", "count")}
    hv.update({f"v2_{a}": v2 for a in ("sum", "mean", "min", "max", "count")})
    aggs = {c: c.split("_")[1] for c in hv}
    hv["abs_v1"] = np.abs(v1).astype(np.float64)
    ek, eout = O.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], hv, dict(aggs, abs_v1="sum"))
    ok = all(np.array_equal(got_keys[k], ek[k]) for k in ("k1", "k2"))
    asum, cnt = eout["abs_v1"], eout["v1_count"]
    for c in aggs:
        g, e = got[c], eout[c]
        if not ok or g.dtype != e.dtype or len(g) != len(e):
            ok = False
            break
        if c == "v1_sum":
            ok = bool((np.abs(g.astype(np.float64) - e) <= asum * 2.0 ** -16 + 1e-30).all())
        elif c == "v1_mean":
            ok = bool((np.abs(g.astype(np.float64) - e) <= asum / cnt * 2.0 ** -16 + 1e-30).all())
        else:
            ok = bool(np.array_equal(g, e))
    return {"ok": bool(ok), "against": "oracle (float32 sums within 2^-16 sum|x|)", "groups": int(len(ek["k1"])),
            "check_s": round(time.perf_counter() - t0, 1)}


# ------------------------------------------------------------------- GPU ---
def run_gpu(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from jaxframes_b200 import build as b
    if rank == 0 or world == 1:
        b.build()
    if world > 1:
        dist.barrier()
    from jaxframes_b200 import _lib
    import jaxframes_b200.parallel_algorithms as P
    L = _lib.load_library()

    lk, lv, rk, rv = make_join_shard(rank, world)
    dev = torch.device("cuda", local)
    d_lk, d_lv = torch.from_numpy(lk).to(dev), torch.from_numpy(lv).to(dev)
    d_rk, d_rv = torch.from_numpy(rk).to(dev), torch.from_numpy(rv).to(dev)
    joiner = P.ParallelSortMergeJoin()

    def join(a, av, b, bv):
        # one GPU: the join itself; several: both sides repartitioned by
        # hash(key) % world over NCCL, then the local join on every rank
        if world == 1:
            return joiner.join(a, av, b, bv, "inner")
        from jaxframes_b200.distributed import distributed_join
        return distributed_join(a, av, b, bv, "inner")

    def step():
        return join(d_lk, {"lv": d_lv}, d_rk, {"rv": d_rv})

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        mk, out = step()
    torch.cuda.synchronize()
    m_rows = int(mk.numel())

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    launches0 = L.jfx_launch_count()
    L.jfx_timing_enable(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        mk, out = step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    launches = int(L.jfx_launch_count() - launches0)
    import ctypes
    pms, pl, pb = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
    L.jfx_timing_read(ctypes.byref(pms), ctypes.byref(pl), ctypes.byref(pb))
    L.jfx_timing_enable(0)
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    if args.profile:
        if rank == 0:
            print(json.dumps({"workload": "join", "ms_per_step": ms, "value": (NL + NR) / (ms / 1e3)}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    # end to end: pinned host buffers in, results back to the host
    h = [torch.from_numpy(x).pin_memory() for x in (lk, lv, rk, rv)]
    h2d = sum(x.numel() * x.element_size() for x in h)

    # results land in pinned host buffers (allocated once, like a caller
    # streaming results would); the copies are inside the timed region
    outs_h = {}

    def e2e_step():
        if world == 1:
            mk, out = joiner.join(h[0], {"lv": h[1]}, h[2], {"rv": h[3]}, "inner")
        else:
            a, av, b, bv = (x.to(dev, non_blocking=True) for x in h)
            mk, out = join(a, {"lv": av}, b, {"rv": bv})
        res = [mk, out["left_lv"], out["right_rv"]]
        nbytes = 0
        for i, t in enumerate(res):
            buf = outs_h.get(i)
            if buf is None or buf.numel() < t.numel() or buf.dtype != t.dtype:
                buf = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
                outs_h[i] = buf
            buf[: t.numel()].copy_(t, non_blocking=True)
            nbytes += t.numel() * t.element_size()
        torch.cuda.current_stream().synchronize()
        return nbytes

    for _ in range(max(1, args.warmup // 2)):
        d2h = e2e_step()
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 5))
    f0.record()
    for _ in range(e2e_steps):
        d2h = e2e_step()
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    pass_ms = pms.value / max(pl.value, 1)
    pass_bytes = pb.value / max(pl.value, 1)
    achieved = pass_bytes / (pass_ms / 1000) / 1e9 if pass_ms > 0 else None
    rows = (NL + NR) * world
    value = rows / (ms / 1000)
    model = join_model_bytes(NL, NR, m_rows)

    # parity of the timed call's output against the oracle at full size
    # (outside the timed region).  Several ranks: each rank checks its local
    # join on the rows the exchange brought it (the exchange itself is
    # checked with gloo ranks in the tests); the flags are AND-ed over ranks.
    parity = None
    if not args.no_check:
        if world == 1:
            parity = check_join_parity(mk, out, lk, lv, rk, rv)
        else:
            from jaxframes_b200.repartition import exchange_partitions
            (xl,), xlv, _ = exchange_partitions([d_lk], {"lv": d_lv})
            (xr,), xrv, _ = exchange_partitions([d_rk], {"rv": d_rv})
            parity = check_join_parity(mk, out, xl.cpu().numpy(), xlv["lv"].cpu().numpy(), xr.cpu().numpy(),
                                       xrv["rv"].cpu().numpy())
            ok = torch.tensor([1 if parity["ok"] else 0], device=dev)
            rows_all = torch.tensor([int(mk.numel())], device=dev)
            dist.all_reduce(ok, op=dist.ReduceOp.MIN)
            dist.all_reduce(rows_all, op=dist.ReduceOp.SUM)
            parity.update(ok=bool(ok.item()), against="oracle, bit-exact, per rank on its exchanged rows",
                          rows=int(rows_all.item()), expected_rows=NL * world)
            parity["ok"] = parity["ok"] and parity["rows"] == NL * world

    extra = {}
    if args.extra and rank == 0 and world == 1:
        extra = run_extra(args, P, dev, hbm, check=not args.no_check)

    if rank == 0:
        cpu_v, reps = cpu_join_sample(NL // 10, NR // 10, seconds=args.cpu_seconds)
        line = {
            "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "left_rows": NL * world, "right_rows": NR * world,
                       "rows_per_rank": [NL, NR], "output_rows_rank0": m_rows,
                       "parallelism": (f"hash-repartitioned over {world} ranks (NCCL all_to_all, then local join)"
                                       if world > 1 else "single"),
                       "l2": "inputs 180 MB per rank > 126 MB L2, no flush"},
            "model_gbs": model / (ms / 1000) / 1e9,
            "model_frac": model / (ms / 1000) / 1e9 / hbm,
            "roofline": {"bound": "hbm", "kernel": "k_onesweep (radix pass)", "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": ONESWEEP_DRAM_BYTES_PER_LAUNCH, "traffic_unit": "bytes per launch (ncu)",
                         "algorithmic_bytes_per_launch": pass_bytes, "peak_source": peak_src,
                         "launches": int(pl.value), "avg_launch_ms": pass_ms},
            "e2e": {"value": (NL + NR) * world / (e2e_ms / 1000), "unit": "rows/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
            "gpu_launches": launches,
            "parity_checked": bool(parity and parity["ok"]),
            "parity": parity,
            "clocks": clocks,
            "cpu_baseline": {"value": cpu_v, "unit": "rows/s", "cores": 1, "kind": "port",
                             "sample": f"inner join {NL // 10} x {NR // 10} rows x {reps} reps, single-threaded "
                                       "NumPy restatement (jax not installed)"},
        }
        if extra:
            line["extra"] = extra
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_secondary(args):
    """One secondary config timed alone (used for profiling and tuning)."""
    import torch
    torch.cuda.set_device(0)
    from jaxframes_b200 import build as b
    b.build()
    import jaxframes_b200.parallel_algorithms as P
    dev = torch.device("cuda", 0)
    if args.workload == "batch":
        run_batch(args, dev)
        return
    if args.workload == "groupby":
        n = args.n or 100_000_000
        k1, k2, v1, v2 = [torch.from_numpy(x).to(dev) for x in c3_inputs(n)]
        vals = {f"v1_{a}": v1 for a in ("sum", "mean", "min", "max", "count")}
        vals.update({f"v2_{a}": v2 for a in ("sum", "mean", "min", "max", "count")})
        aggs = {c: c.split("_")[1] for c in vals}
        fn = lambda: P.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], vals, aggs)
        unit_rows = n
    elif args.workload == "groupby1m":
        n = args.n or 1_000_000
        rng = np.random.default_rng(42)
        k = torch.from_numpy(rng.integers(0, 1000, n).astype(np.int32)).to(dev)
        v = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(dev)
        fn = lambda: P.groupby_aggregate(k, {"v": v, "c": v}, {"v": "sum", "c": "count"})
        unit_rows = n
    elif args.workload == "learned":
        n = args.n or (1 << 28)
        keys = torch.from_numpy(c4_keys(nblocks=max(1, n // 4096))).to(dev)
        n = keys.numel()
        res = {}
        for mode in ("plain", "auto"):
            fn = lambda: P.learned_sort(keys, mode=mode)
            for _ in range(args.warmup):
                out = fn()
            torch.cuda.synchronize()
            a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(args.steps):
                out = fn()
            b2.record()
            torch.cuda.synchronize()
            res[mode] = {"ms": a.elapsed_time(b2) / args.steps, "learned_used": int(out[2])}
        same = bool(torch.equal(P.learned_sort(keys, mode="plain")[1], P.learned_sort(keys, mode="auto")[1]))
        print(json.dumps({"workload": "learned", "rows": n, "plain": res["plain"], "learned": res["auto"],
                          "identical_perm": same, "speedup": res["plain"]["ms"] / res["auto"]["ms"]}), flush=True)
        return
    else:
        n = args.n or (1 << 28)
        rng = np.random.default_rng(45)
        keys = torch.from_numpy(rng.integers(0, 2**63, n, dtype=np.uint64)).to(dev)
        s = P.ParallelRadixSort()
        fn = lambda: s.argsort(keys)
        unit_rows = n
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        fn()
    b2.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b2) / args.steps
    print(json.dumps({"workload": args.workload, "rows": n, "ms_per_step": ms, "rows_per_s": unit_rows / (ms / 1e3)}),
          flush=True)


def c5_batch(dev, total_rows=0, nq=2048):
    """The batched workload: 2048 queries with row counts
    floor(exp(uniform(ln 1e3, ln 4e6))) (about 1e9 rows; scaled to about
    ``total_rows`` when given), int32 keys uniform in [0, min(rows // 4, 1e6)),
    float32 N(0, 1) values, hash partition to 256 partitions then groupby-sum.
    Inputs are generated on the device from a seeded generator straight into a
    ``BatchedGroupBy``'s buffers; returns it and the host row offsets."""
    import torch
    from jaxframes_b200.batch import BatchedGroupBy
    rng = np.random.default_rng(46)
    rows = np.floor(np.exp(rng.uniform(np.log(1e3), np.log(4e6), nq))).astype(np.int64)
    if total_rows:  # scaled-down batch with the same shape of row counts
        rows = np.maximum(1, np.floor(rows * (total_rows / rows.sum()))).astype(np.int64)
    off = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
    n = int(off[-1])
    b = BatchedGroupBy(n, nq, 256, 20, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(46)
    for q in range(nq):
        span = int(max(1, min(rows[q] // 4, 1_000_000)))
        b.keys[off[q]:off[q + 1]] = torch.randint(0, span, (int(rows[q]),), generator=g, device=dev,
                                                  dtype=torch.int32)
    torch.randn(n, generator=g, device=dev, out=b.values[:n])
    b.query_offsets.copy_(torch.from_numpy(off))
    return b, off


def check_batch_queries(b, off, queries, num_partitions=256):
    """Per-query parity of a batched run against the oracle: partition
    offsets, partitioned keys and values and group keys and counts bit-exact,
    sums within 2^-16 * sum(|x|) per group.  Returns the number of rows
    checked; raises AssertionError on a mismatch."""
    from oracle import jfx_oracle as O
    rows = 0
    for q in queries:
        a, e = int(off[q]), int(off[q + 1])
        k = b.keys[a:e].cpu().numpy()
        v = b.values[a:e].cpu().numpy()
        po, pk, pv, gk, gs, gc = (t.cpu().numpy() for t in b.query(q))
        _, perm, eoffs = O.hash_partition([k], num_partitions)
        assert np.array_equal(po, eoffs), f"query {q}: partition offsets"
        assert np.array_equal(pk, k[perm]) and np.array_equal(pv, v[perm]), f"query {q}: partitioned rows"
        ek, eo = O.groupby_aggregate(k, {"s": v, "c": v, "a": np.abs(v).astype(np.float64)},
                                     {"s": "sum", "c": "count", "a": "sum"})
        assert np.array_equal(gk, ek) and np.array_equal(gc, eo["c"]), f"query {q}: groups"
        assert (np.abs(gs.astype(np.float64) - eo["s"]) <= eo["a"] * 2.0 ** -16 + 1e-30).all(), f"query {q}: sums"
        rows += e - a
    return rows


def batch_check_queries(off, count=64, seed=47):
    """A seeded subset of the queries that includes the largest one."""
    nq = len(off) - 1
    largest = int(np.argmax(np.diff(off)))
    others = np.delete(np.arange(nq), largest)
    pick = np.random.default_rng(seed).choice(others, size=min(count, nq) - 1, replace=False).tolist()
    return sorted(pick + [largest])


def run_batch(args, dev):
    """Batched hash partition (256 partitions) + groupby-sum over 2048 queries
    (``c5_batch``); one CUDA-graph replay per step."""
    import torch
    b, off = c5_batch(dev, args.n)
    nq = len(off) - 1
    n = int(off[-1])
    b.capture()
    for _ in range(args.warmup):
        b.replay()
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        b.replay()
    e.record()
    torch.cuda.synchronize()
    b.status()
    ms = a.elapsed_time(e) / args.steps
    groups = int(b.group_offsets[nq].item())
    model = 56 * n + 8 * groups  # partition 16 + sort 28 + groupby 12 bytes per row, 8 per group
    print(json.dumps({"workload": "batch", "queries": nq, "rows": n, "groups": groups, "ms_per_step": ms,
                      "rows_per_s": n / (ms / 1e3), "model_gbs": model / (ms / 1e3) / 1e9,
                      "graph": "one CUDA graph replay per step"}), flush=True)


def run_extra(args, P, dev, hbm=6650.0, check=True):
    """The other configurations, each timed on the device (CUDA events, inputs
    resident, larger than L2 except the 1M-row groupby) and checked against
    the oracle outside the timed region.  Model bytes follow the fixed
    per-row byte model of each operator (sort, groupby, batch); ``frac`` is
    model GB/s over the measured HBM copy bandwidth."""
    import torch
    out = {}

    def timeit(fn, steps, warm=1):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b2.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b2) / steps

    def roof(model, ms):
        gbs = model / (ms / 1e3) / 1e9
        return {"bound": "hbm", "model_bytes": model, "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm}

    from oracle import jfx_oracle as O
    try:
        rng = np.random.default_rng(42)
        n = 1_000_000
        kh = rng.integers(0, 1000, n).astype(np.int32)
        vh = rng.standard_normal(n).astype(np.float32)
        k, v = torch.from_numpy(kh).to(dev), torch.from_numpy(vh).to(dev)
        ms = timeit(lambda: P.groupby_aggregate(k, {"v": v, "c": v}, {"v": "sum", "c": "count"}), 5)
        res = {"ms": ms, "rows_per_s": n / (ms / 1e3), "roofline": roof(n * 24 + 1000 * 12, ms)}
        if check:
            uk, o = P.groupby_aggregate(k, {"v": v, "c": v}, {"v": "sum", "c": "count"})
            ek, eo = O.groupby_aggregate(kh, {"v": vh, "c": vh, "a": np.abs(vh).astype(np.float64)},
                                         {"v": "sum", "c": "count", "a": "sum"})
            ok = (np.array_equal(uk.cpu().numpy(), ek) and np.array_equal(o["c"].cpu().numpy(), eo["c"])
                  and bool((np.abs(o["v"].cpu().numpy().astype(np.float64) - eo["v"]) <= eo["a"] * 2.0 ** -16).all()))
            res["parity_checked"] = bool(ok)
        out["groupby_sum_1M"] = res
    except Exception as e:  # report, do not hide
        out["groupby_sum_1M"] = {"error": repr(e)}
    try:
        hk1, hk2, hv1, hv2 = c3_inputs()
        k1, k2, v1, v2 = [torch.from_numpy(x).to(dev) for x in (hk1, hk2, hv1, hv2)]
        vals = {f"v1_{a}": v1 for a in ("sum", "mean", "min", "max", "count")}
        vals.update({f"v2_{a}": v2 for a in ("sum", "mean", "min", "max", "count")})
        aggs = {c: c.split("_")[1] for c in vals}
        ms = timeit(lambda: P.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], vals, aggs), 3)
        uk, o = P.groupby_aggregate_multi_column([k1, k2], ["k1", "k2"], vals, aggs)
        g = int(uk["k1"].numel())
        n = k1.numel()
        # SORT(N, K=4, Kraw=8) with P = ceil(26 / 11) = 3 passes, the value
        # reads, and 60 bytes of key and aggregate outputs per group
        model = n * (8 + 8 + 2 * 2 * 8) + n * (4 + 4 + 4 + 8) + g * 60
        res = {"ms": ms, "rows_per_s": n / (ms / 1e3), "groups": g, "model_gbs": model / (ms / 1e3) / 1e9,
               "roofline": roof(model, ms)}
        got_keys = {kk: t.cpu().numpy() for kk, t in uk.items()}
        got = {c: t.cpu().numpy() for c, t in o.items()}
        del k1, k2, v1, v2, vals, uk, o
        torch.cuda.empty_cache()
        if check:
            res["parity"] = check_groupby_parity(hk1, hk2, hv1, hv2, got_keys, got)
            res["parity_checked"] = res["parity"]["ok"]
        out["groupby_multikey_100M"] = res
        del hk1, hk2, hv1, hv2, got, got_keys
    except Exception as e:
        out["groupby_multikey_100M"] = {"error": repr(e)}
    try:
        rng = np.random.default_rng(45)
        n = 1 << 28
        keys = torch.from_numpy(rng.integers(0, 2**63, n, dtype=np.uint64)).to(dev)
        s = P.ParallelRadixSort()
        ms = timeit(lambda: s.argsort(keys), 2)
        model = n * (8 + 12 + 5 * 24)
        res = {"ms": ms, "keys_per_s": n / (ms / 1e3), "model_gbs": model / (ms / 1e3) / 1e9,
               "roofline": roof(model, ms)}
        if check:
            res["parity_checked"] = stable_argsort_ok(keys, s.argsort(keys))
        out["sort_u64_256M_uniform"] = res
        del keys
        torch.cuda.empty_cache()
    except Exception as e:
        out["sort_u64_256M_uniform"] = {"error": repr(e)}
    try:
        keys = torch.from_numpy(c4_keys()).to(dev)
        n = keys.numel()
        model = n * (8 + 12 + 5 * 24)  # the plain sort's model bytes, the denominator of both forms
        res = {"rows": n}
        for mode in ("plain", "auto"):
            ms = timeit(lambda: P.learned_sort(keys, mode=mode), 3)
            res["learned" if mode == "auto" else "plain"] = {"ms": ms, "model_gbs": model / (ms / 1e3) / 1e9}
        sk_p, perm_p, _ = P.learned_sort(keys, mode="plain")
        del sk_p
        sk_l, perm_l, used = P.learned_sort(keys, mode="auto")
        res["learned_used"] = used
        res["identical_perm"] = bool(torch.equal(perm_p, perm_l))
        del sk_l, perm_l
        res["speedup"] = res["plain"]["ms"] / res["learned"]["ms"]
        res["roofline"] = roof(model, res["learned"]["ms"])
        if check:
            res["parity_checked"] = res["identical_perm"] and stable_argsort_ok(keys, perm_p)
        out["learned_c4_256M"] = res
        del keys, perm_p
        torch.cuda.empty_cache()
    except Exception as e:
        out["learned_c4_256M"] = {"error": repr(e)}
    try:
        b, off = c5_batch(dev)
        nq, n = len(off) - 1, int(off[-1])
        b.capture()
        ms = timeit(b.replay, 3, warm=2)
        b.status()
        groups = int(b.group_offsets[nq].item())
        model = 56 * n + 8 * groups  # partition 16 + sort 28 + groupby 12 bytes per row, 8 per group
        res = {"ms": ms, "queries": nq, "rows": n, "groups": groups, "rows_per_s": n / (ms / 1e3),
               "model_gbs": model / (ms / 1e3) / 1e9, "roofline": roof(model, ms),
               "graph": "one CUDA graph replay per step"}
        if check:
            qs = batch_check_queries(off)
            try:
                rows = check_batch_queries(b, off, qs)
                res["parity_checked"] = True
                res["parity"] = {"ok": True, "queries": len(qs), "rows": rows, "includes_largest": True}
            except AssertionError as e:
                res["parity_checked"] = False
                res["parity"] = {"ok": False, "error": str(e)}
        out["batch_c5_2048q"] = res
        del b
        torch.cuda.empty_cache()
    except Exception as e:
        out["batch_c5_2048q"] = {"error": repr(e)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="jfx", choices=["jfx", "reference"])
    ap.add_argument("--extra", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--workload", default="join", choices=["join", "groupby", "sort", "groupby1m", "learned", "batch"],
                    help="join = the headline; the others time one secondary config alone")
    ap.add_argument("--n", type=int, default=0, help="rows for --workload groupby/sort (0 = config size)")
    ap.add_argument("--profile", action="store_true", help="timed steps only (no e2e, CPU leg or extras)")
    ap.add_argument("--no-check", action="store_true", help="skip the parity checks against the oracle")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference(args)
    elif args.workload != "join":
        run_secondary(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
