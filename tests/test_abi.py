"""C ABI checks that need no GPU: the library loads, exports every function
``include/jfx.h`` declares, and rejects bad arguments on the host side."""

import ctypes
import os
import re

import pytest

from jaxframes_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(jfx_[a-z0-9_]+)\s*\(", src))
    return names


@pytest.fixture(scope="module")
def lib():
    from jaxframes_b200 import build
    build.build()
    return _lib.load_library()


def test_every_declared_symbol_is_exported(lib):
    declared = _declared()
    assert declared, "no declarations found"
    for name in sorted(declared):
        assert hasattr(lib, name), name


def test_binding_covers_header(lib):
    assert _declared() == set(_lib.SIGNATURES)


def test_version_and_limits(lib):
    assert lib.jfx_version() >= 1
    assert lib.jfx_max_rows() == (1 << 30) - 1


def test_workspace_sizes_grow_with_rows(lib):
    for kind in (_lib.WS_SORT, _lib.WS_GROUPBY, _lib.WS_PARTITION):
        a = lib.jfx_workspace_size(kind, 1000, 256)
        b = lib.jfx_workspace_size(kind, 1_000_000, 256)
        assert 0 < a < b
    assert lib.jfx_workspace_size(_lib.WS_JOIN, 10, 5) > 0
    assert lib.jfx_workspace_size(99, 10, 5) == 0


def test_host_side_argument_errors(lib):
    col = _lib.Column(None, _lib.I32, 0)
    st = lib.jfx_sort(ctypes.byref(col), -1, 1, None, None, None, 0, None)
    assert st == -1 and b"negative" in lib.jfx_last_error()
    st = lib.jfx_sort(ctypes.byref(col), 1 << 31, 1, None, None, None, 0, None)
    assert st == -5
    st = lib.jfx_sort(None, 10, 1, None, None, None, 0, None)
    assert st == -1
    # zero rows is a no-op on the host
    assert lib.jfx_sort(ctypes.byref(col), 0, 1, ctypes.c_void_p(8), None, None, 0, None) == 0
    st = lib.jfx_hash_partition(ctypes.byref(col), 1, 10, 0, None, None, None, None, 0, None)
    assert st == -1
    g = ctypes.c_int64(7)
    st = lib.jfx_groupby(ctypes.byref(col), 2, 10, 0, None, 0, None, ctypes.byref(g), None, 0, None)
    assert st == -1 and b"single-key" in lib.jfx_last_error()
    plan = _lib.JoinPlan()
    assert lib.jfx_join_expand(ctypes.byref(plan), None, None, None, None) == -1


def test_compute_without_gpu_raises():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from jaxframes_b200 import parallel_sort, JfxUnavailable
    import numpy as np
    with pytest.raises(JfxUnavailable):
        parallel_sort(np.arange(5, dtype=np.int32))
