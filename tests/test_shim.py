"""The jaxframes rebinding shim against a stand-in module (jax is absent)."""

import types

from jaxframes_b200 import parallel_algorithms as P
from jaxframes_b200 import shim


def _fake_module():
    m = types.ModuleType("fake_parallel_algorithms")
    for name in shim.REPLACED:
        setattr(m, name, object())
    m.untouched = object()
    return m


def test_install_replaces_the_hot_path_symbols_and_uninstall_restores():
    m = _fake_module()
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


def test_results_are_converted_back():
    seen = []
    conv = lambda t: seen.append(t) or ("converted", t)
    out = shim._convert({"a": [1, 2], "b": (3,)}, conv)
    assert out == {"a": [1, 2], "b": (3,)} and not seen
