"""Autotuner bookkeeping on CPU (timings injected), and one GPU tuning run."""

import json

import numpy as np
import pytest
import torch

from jaxframes_b200 import autotune


def test_buckets():
    assert autotune.size_bucket(1) == 0 and autotune.size_bucket(1 << 20) == 20
    assert autotune.size_bucket((1 << 20) + 5) == 20
    assert autotune.skew_bucket(1.0) == 0 and autotune.skew_bucket(0.6) == 1 and autotune.skew_bucket(0.01) == 2


def test_estimate_skew_cpu_tensor():
    assert autotune.estimate_skew(np.arange(100000, dtype=np.int64)) == 0
    assert autotune.estimate_skew(np.zeros(100000, dtype=np.int32)) == 2


def test_cache_roundtrip(tmp_path):
    p = str(tmp_path / "t.json")
    t = autotune.Autotuner(p, gpu_name="B200-test")
    assert t.lookup("sort", "torch.int32", 1000, 0) is None
    t.record("sort", "torch.int32", 1000, 0, {"max_digit_bits": 9})
    t2 = autotune.Autotuner(p, gpu_name="B200-test")
    assert t2.lookup("sort", "torch.int32", 1000, 0) == {"max_digit_bits": 9}
    assert t2.lookup("sort", "torch.int32", 600, 0) == {"max_digit_bits": 9}  # same size bucket (2^9)
    assert t2.lookup("sort", "torch.int32", 1000, 0) is not None
    other = autotune.Autotuner(p, gpu_name="other-gpu")
    assert other.lookup("sort", "torch.int32", 1000, 0) is None
    assert "B200-test|sort|torch.int32|9|0" in json.load(open(p))


@pytest.mark.gpu
def test_tune_sort_on_gpu(tmp_path):
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from jaxframes_b200 import build
    build.build()
    import jaxframes_b200.parallel_algorithms as P
    t = autotune.Autotuner(str(tmp_path / "t.json"))
    k = np.random.default_rng(0).integers(0, 2**40, 1 << 20, dtype=np.int64)
    choice = t.tune_sort(k, trials=1)
    assert choice["max_digit_bits"] in autotune.DIGIT_CANDIDATES
    ref = np.argsort(k, kind="stable")
    for bits in autotune.DIGIT_CANDIDATES:
        with autotune.tuning(max_digit_bits=bits):
            perm = P.ParallelRadixSort().argsort(k)
        np.testing.assert_array_equal(perm.cpu().numpy(), ref)
    autotune._tuner = t
    autotune._enabled = True
    try:
        np.testing.assert_array_equal(P.ParallelRadixSort().argsort(k).cpu().numpy(), ref)
    finally:
        autotune.disable()
