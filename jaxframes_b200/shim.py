"""Rebinds jaxframes' distributed-algorithms functions to the B200 kernels.

``install()`` replaces, inside ``jaxframes.distributed.parallel_algorithms``,
the symbols its callers use (core/frame.py:1171-1201, :1300-1319, :1416-1525,
:748-893; distributed/frame.py:709, :814-855, :971-999; lazy/codegen.py:488,
:558, :616) with wrappers that take jax arrays, import them zero-copy into
torch through DLPack, run the CUDA path and hand the results back as jax
arrays through DLPack.  The callers stay unchanged.

Callers that import inside a function (core/frame.py, lazy/codegen.py,
distributed/frame.py:793 and :991) read the module attribute at call time and
so see the replacement.  Two modules bind names once, at their own import:
``distributed/frame.py:20-24`` (``groupby_aggregate``, ``parallel_sort``,
``sort_merge_join``, ``compact_repartitioned_rows``) and
``distributed/multi_column_distributed.py:13-19`` (``ParallelSortMergeJoin``,
``SortBasedGroupBy``, ``multi_column_lexsort``, ``compact_repartitioned_rows``).
``install()`` therefore also walks ``sys.modules`` and rebinds every module
attribute that still refers to one of the replaced originals (an identity
check, so nothing else is touched); ``uninstall()`` puts those back too.
Modules imported after ``install()`` pick up the replacements themselves.

``collective_hash_repartition`` is not replaced: on one device the reference
returns its inputs unchanged (parallel_algorithms.py:202-203), and across
devices the reference exchanges inside one JAX process while this package
runs one process per GPU (``jaxframes_b200.repartition``).

jax is not a dependency of this package; ``install`` takes the module and the
DLPack converter as arguments so it can be exercised without jax.
"""

from __future__ import annotations

import sys
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
    wrapped.__wrapped__ = fn
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
    Wrapped.__qualname__ = cls.__qualname__
    return Wrapped


class Installed(dict):
    """Replaced originals by name, plus ``rebound``: the (module, name,
    original) triples of other modules' bindings that ``install`` rebound."""

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.rebound: list[tuple[types.ModuleType, str, object]] = []


def _rebind_importers(module, originals: dict, replacements: dict, installed: Installed):
    by_id = {id(obj): name for name, obj in originals.items()}
    for mod in list(sys.modules.values()):
        if mod is None or mod is module or not isinstance(mod, types.ModuleType):
            continue
        try:
            items = list(vars(mod).items())
        except TypeError:
            continue
        for attr, val in items:
            name = by_id.get(id(val))
            if name is None or val is not originals[name]:
                continue
            setattr(mod, attr, replacements[name])
            installed.rebound.append((mod, attr, val))


def install(module: types.ModuleType | None = None, from_torch=None, rebind_importers: bool = True):
    """Patches ``module`` (default: ``jaxframes.distributed.parallel_algorithms``)
    and, with ``rebind_importers``, every loaded module that bound one of the
    replaced names with ``from ... import``.

    ``from_torch`` converts a torch CUDA tensor to the caller's array type
    (default: ``jax.dlpack.from_dlpack``).  Inputs need no converter: the
    CUDA path imports any ``__dlpack__`` producer zero-copy.
    Returns the replaced originals (an ``Installed`` dict, for ``uninstall``)."""
    if module is None:
        import importlib
        module = importlib.import_module("jaxframes.distributed.parallel_algorithms")
    if from_torch is None:
        import jax.dlpack
        from_torch = jax.dlpack.from_dlpack
    installed = Installed()
    replacements = {}
    for name in REPLACED:
        if not hasattr(module, name):
            continue
        installed[name] = getattr(module, name)
        impl = getattr(P, name)
        rep = _wrap_class(impl, from_torch) if isinstance(impl, type) else _wrap_fn(impl, from_torch)
        replacements[name] = rep
        setattr(module, name, rep)
    if rebind_importers:
        _rebind_importers(module, dict(installed), replacements, installed)
    return installed


def uninstall(module, originals: dict):
    """Undoes ``install``: the module's names and every rebound binding."""
    for name, obj in originals.items():
        setattr(module, name, obj)
    for mod, attr, obj in getattr(originals, "rebound", []):
        setattr(mod, attr, obj)
