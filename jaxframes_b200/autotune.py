"""Autotuner for the radix kernels (no counterpart in the reference).

Chooses, per (operation, key dtype, size bucket, skew bucket, GPU name):

* the widest radix digit per pass (8, 9, 10 or 11 bits): wider digits mean
  fewer passes over HBM but larger per-tile histograms and look-back;
* learned-CDF versus plain radix sort for uint64 keys.

Candidates are timed on the device with CUDA events; winners are cached in a
JSON file (``$JFX_TUNE_CACHE`` or ``~/.cache/jaxframes_b200/tune.json``).
With ``enable()``, the sort / groupby / join entry points of
``parallel_algorithms`` apply the cached choice for their inputs; without a
cached entry they keep the library defaults.
"""

from __future__ import annotations

import contextlib
import ctypes
import json
import math
import os
import threading

import numpy as np

from . import _lib

DIGIT_CANDIDATES = (8, 9, 10, 11)
_state = threading.local()
_enabled = False


def cache_path() -> str:
    return os.environ.get("JFX_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "jaxframes_b200",
                                                          "tune.json"))


def size_bucket(n: int) -> int:
    """log2 bucket of the row count."""
    return int(math.log2(max(int(n), 1)))


def skew_bucket(distinct_fraction: float) -> int:
    """0: mostly distinct keys, 1: moderate duplication, 2: heavy duplication."""
    if distinct_fraction >= 0.9:
        return 0
    if distinct_fraction >= 0.5:
        return 1
    return 2


def estimate_skew(keys, sample: int = 65536) -> int:
    """Skew bucket from the distinct fraction of a strided sample."""
    import torch
    k = keys if isinstance(keys, torch.Tensor) else torch.as_tensor(np.asarray(keys))
    n = k.numel()
    if n == 0:
        return 0
    step = max(1, n // sample)
    s = k[::step][:sample]
    if s.dtype in (torch.uint32, torch.uint64, torch.uint16):
        s = s.view(torch.int32 if s.dtype == torch.uint32 else torch.int64 if s.dtype == torch.uint64 else torch.int16)
    d = torch.unique(s).numel()
    return skew_bucket(d / s.numel())


class Autotuner:
    def __init__(self, path: str | None = None, gpu_name: str | None = None, timer=None):
        self.path = path or cache_path()
        self.gpu = gpu_name
        self.timer = timer  # callable(fn) -> ms; default: CUDA events
        self.table: dict[str, dict] = {}
        if os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    self.table = json.load(f)
            except (OSError, ValueError):
                self.table = {}

    def _gpu(self) -> str:
        if self.gpu is None:
            import torch
            self.gpu = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
        return self.gpu

    def key(self, op: str, dtype: str, n: int, skew: int) -> str:
        return f"{self._gpu()}|{op}|{dtype}|{size_bucket(n)}|{skew}"

    def lookup(self, op: str, dtype: str, n: int, skew: int) -> dict | None:
        return self.table.get(self.key(op, dtype, n, skew))

    def record(self, op: str, dtype: str, n: int, skew: int, choice: dict) -> None:
        self.table[self.key(op, dtype, n, skew)] = choice
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.table, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def _time(self, fn, trials: int) -> float:
        if self.timer is not None:
            return self.timer(fn)
        import torch
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(trials):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / trials

    def tune_sort(self, keys, trials: int = 3, candidates=DIGIT_CANDIDATES) -> dict:
        """Times the radix argsort of ``keys`` with each digit width."""
        from .parallel_algorithms import ParallelRadixSort, as_device
        k = as_device(keys)
        skew = estimate_skew(k)
        sorter = ParallelRadixSort()
        times = {}
        for bits in candidates:
            with tuning(max_digit_bits=bits):
                times[bits] = self._time(lambda: sorter.argsort(k), trials)
        best = min(times, key=times.get)
        choice = {"max_digit_bits": int(best), "ms": {str(b): t for b, t in times.items()}}
        self.record("sort", str(k.dtype), k.numel(), skew, choice)
        return choice

    def tune_learned(self, keys, trials: int = 3) -> dict:
        """Times learned-CDF versus plain radix sort of uint64 ``keys``."""
        from .parallel_algorithms import as_device, learned_sort
        k = as_device(keys)
        skew = estimate_skew(k)
        t_plain = self._time(lambda: learned_sort(k, mode="plain"), trials)
        t_learn = self._time(lambda: learned_sort(k, mode="auto"), trials)
        choice = {"learned": bool(t_learn < t_plain), "ms_plain": t_plain, "ms_learned": t_learn}
        self.record("learned", str(k.dtype), k.numel(), skew, choice)
        return choice


@contextlib.contextmanager
def tuning(max_digit_bits: int | None = None, two_phase: bool | None = None, spin_limit_us: int | None = None):
    """Applies a tuning to this thread's libjfx calls for the block."""
    L = _lib.load_library()
    old = _lib.Tuning()
    _lib.check(L.jfx_get_tuning(ctypes.byref(old)))
    new = _lib.Tuning(old.max_digit_bits if max_digit_bits is None else int(max_digit_bits),
                      old.two_phase if two_phase is None else int(bool(two_phase)),
                      old.spin_limit_us if spin_limit_us is None else int(spin_limit_us), 0)
    _lib.check(L.jfx_set_tuning(ctypes.byref(new)))
    try:
        yield
    finally:
        _lib.check(L.jfx_set_tuning(ctypes.byref(old)))


_tuner: Autotuner | None = None


def enable(path: str | None = None) -> Autotuner:
    """Makes the entry points apply cached choices."""
    global _enabled, _tuner
    _tuner = Autotuner(path)
    _enabled = True
    return _tuner


def disable() -> None:
    global _enabled
    _enabled = False


@contextlib.contextmanager
def applied(op: str, keys):
    """Context used by the entry points: the cached digit width, if any."""
    if not _enabled or _tuner is None:
        yield
        return
    choice = _tuner.lookup(op, str(keys.dtype), keys.numel(), estimate_skew(keys))
    if not choice or "max_digit_bits" not in choice:
        yield
        return
    with tuning(max_digit_bits=choice["max_digit_bits"]):
        yield
