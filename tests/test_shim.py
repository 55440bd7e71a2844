"""The jaxframes rebinding shim against stand-in modules (jax is absent).

The stand-ins mirror how the reference binds the replaced names: a module
that imports inside its functions (core/frame.py, lazy/codegen.py) reads the
patched attribute at call time, while distributed/frame.py:20-24 and
multi_column_distributed.py:13-19 bind names once with ``from ... import``."""

import sys
import types

import pytest
import torch

from jaxframes_b200 import _lib
from jaxframes_b200 import parallel_algorithms as P
from jaxframes_b200 import shim


def _fake_module(name="fake_parallel_algorithms"):
    m = types.ModuleType(name)
    for n in shim.REPLACED:
        if n[0].isupper():
            setattr(m, n, type(n, (), {}))
        else:
            def f(*a, **k):
                return "jax path"
            f.__name__ = n
            setattr(m, n, f)
    m.collective_hash_repartition = object()
    m.untouched = object()
    return m


@pytest.fixture
def fake_pkg():
    pa = _fake_module("fake_jf.distributed.parallel_algorithms")
    # distributed/frame.py:20-24 and multi_column_distributed.py:13-19 bind at import
    frame = types.ModuleType("fake_jf.distributed.frame")
    for n in ("groupby_aggregate", "parallel_sort", "sort_merge_join", "compact_repartitioned_rows"):
        setattr(frame, n, getattr(pa, n))
    frame.collective_hash_repartition = pa.collective_hash_repartition
    mcd = types.ModuleType("fake_jf.distributed.multi_column_distributed")
    for n in ("ParallelSortMergeJoin", "SortBasedGroupBy", "multi_column_lexsort", "compact_repartitioned_rows"):
        setattr(mcd, n, getattr(pa, n))
    mods = {pa.__name__: pa, frame.__name__: frame, mcd.__name__: mcd}
    sys.modules.update(mods)
    yield pa, frame, mcd
    for k in mods:
        sys.modules.pop(k, None)


def test_install_replaces_the_hot_path_symbols_and_uninstall_restores(fake_pkg):
    m, _, _ = fake_pkg
    before = {n: getattr(m, n) for n in shim.REPLACED}
    originals = shim.install(m, from_torch=lambda t: t)
    assert set(originals) == set(shim.REPLACED)
    for n in shim.REPLACED:
        assert getattr(m, n) is not before[n]
        assert getattr(m, n).__name__ == getattr(P, n).__name__
    assert isinstance(m.ParallelRadixSort(None), P.ParallelRadixSort)
    shim.uninstall(m, originals)
    for n in shim.REPLACED:
        assert getattr(m, n) is before[n]


def test_modules_that_bound_names_at_import_are_rebound(fake_pkg):
    pa, frame, mcd = fake_pkg
    orig_frame = dict(vars(frame))
    orig_mcd = dict(vars(mcd))
    inst = shim.install(pa, from_torch=lambda t: t)
    try:
        # distributed/frame.py's bindings now reach the B200 path
        for n in ("groupby_aggregate", "parallel_sort", "sort_merge_join", "compact_repartitioned_rows"):
            assert getattr(frame, n) is getattr(pa, n)
            assert getattr(frame, n).__wrapped__ is getattr(P, n)
        # DistributedMultiColumnOps' classes and lexsort too
        assert issubclass(mcd.ParallelSortMergeJoin, P.ParallelSortMergeJoin)
        assert issubclass(mcd.SortBasedGroupBy, P.SortBasedGroupBy)
        assert mcd.multi_column_lexsort.__wrapped__ is P.multi_column_lexsort
        # names outside the replaced set are left alone
        assert frame.collective_hash_repartition is orig_frame["collective_hash_repartition"]
        # a call through the rebound name runs the product path, which has no
        # CPU fallback: without a GPU it raises instead of returning "jax path"
        if not torch.cuda.is_available():
            with pytest.raises(_lib.JfxUnavailable):
                frame.parallel_sort([3, 1, 2])
    finally:
        shim.uninstall(pa, inst)
    assert dict(vars(frame)) == orig_frame
    assert dict(vars(mcd)) == orig_mcd


def test_a_module_imported_after_install_sees_the_replacement(fake_pkg):
    pa, _, _ = fake_pkg
    inst = shim.install(pa, from_torch=lambda t: t)
    try:
        late = types.ModuleType("fake_jf.lazy.codegen")
        late.multi_column_lexsort = pa.multi_column_lexsort  # "from ... import" after install
        assert late.multi_column_lexsort.__wrapped__ is P.multi_column_lexsort
    finally:
        shim.uninstall(pa, inst)


def test_results_are_converted_back():
    seen = []
    conv = lambda t: seen.append(t) or ("converted", t)
    out = shim._convert({"a": [1, 2], "b": (3,)}, conv)
    assert out == {"a": [1, 2], "b": (3,)} and not seen
