"""Rebinds jaxframes' distributed-algorithms functions to the B200 kernels.

``install()`` replaces, inside ``jaxframes.distributed.parallel_algorithms``,
the symbols its callers use (core/frame.py:1171-1201, :1300-1319, :1416-1525,
:748-893; distributed/frame.py:709, :814-855, :971-999; lazy/codegen.py:488,
:558, :616) with wrappers that take jax arrays, import them zero-copy into
torch through DLPack, run the CUDA path and hand the results back as jax
arrays through DLPack.  The callers stay unchanged.

jax is not a dependency of this package; ``install`` takes the module and the
two DLPack converters as arguments so it can be exercised without jax.
"""

from __future__ import annotations

import types

from . import parallel_algorithms as P

REPLACED = [
    "multi_column_lexsort", "hash_multi_columns", "combine_keys_for_sorting", "compact_repartitioned_rows",
    "ParallelRadixSort", "SortBasedGroupBy", "ParallelSortMergeJoin", "parallel_sort", "groupby_aggregate",
    "groupby_aggregate_multi_column", "sort_merge_join",
]


def _convert(obj, to_host):
    if isinstance(obj, dict):
        return {k: _convert(v, to_host) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        out = [_convert(v, to_host) for v in obj]
        return type(obj)(out) if isinstance(obj, tuple) else out
    if hasattr(obj, "__dlpack__") and hasattr(obj, "dtype"):
        return to_host(obj)
    return obj


def _wrap_fn(fn, from_torch):
    def wrapped(*args, **kwargs):
        return _convert(fn(*args, **kwargs), from_torch)
    wrapped.__name__ = fn.__name__
    wrapped.__doc__ = fn.__doc__
    return wrapped


def _wrap_class(cls, from_torch):
    class Wrapped(cls):
        pass
    for name in dir(cls):
        if name.startswith("_"):
            continue
        attr = getattr(cls, name)
        if callable(attr):
            def make(meth):
                def m(self, *a, **k):
                    return _convert(meth(self, *a, **k), from_torch)
                m.__name__ = meth.__name__
                m.__doc__ = meth.__doc__
                return m
            setattr(Wrapped, name, make(attr))
    Wrapped.__name__ = cls.__name__
    return Wrapped


def install(module: types.ModuleType | None = None, from_torch=None):
    """Patches ``module`` (default: ``jaxframes.distributed.parallel_algorithms``).

    ``from_torch`` converts a torch CUDA tensor to the caller's array type
    (default: ``jax.dlpack.from_dlpack``).  Inputs need no converter: the
    CUDA path imports any ``__dlpack__`` producer zero-copy.
    Returns the dict of replaced originals (for ``uninstall``)."""
    if module is None:
        import importlib
        module = importlib.import_module("jaxframes.distributed.parallel_algorithms")
    if from_torch is None:
        import jax.dlpack
        from_torch = jax.dlpack.from_dlpack
    originals = {}
    for name in REPLACED:
        if not hasattr(module, name):
            continue
        originals[name] = getattr(module, name)
        impl = getattr(P, name)
        if isinstance(impl, type):
            setattr(module, name, _wrap_class(impl, from_torch))
        else:
            setattr(module, name, _wrap_fn(impl, from_torch))
    return originals


def uninstall(module, originals: dict):
    for name, obj in originals.items():
        setattr(module, name, obj)
