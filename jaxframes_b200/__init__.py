"""jaxframes_b200 -- B200-native (sm_100a) kernels for jaxframes' distributed
algorithms layer: stable LSD radix sort, sort-based groupby, sort-merge join
and hash partitioning, behind the API of
``jaxframes.distributed.parallel_algorithms``.
"""

from . import parallel_algorithms
from ._lib import JfxError, JfxUnavailable, load_library
from .parallel_algorithms import (
    ParallelRadixSort,
    ParallelSortMergeJoin,
    ShardingSpec,
    SortBasedGroupBy,
    collective_hash_repartition,
    combine_keys_for_sorting,
    compact_repartitioned_rows,
    config,
    groupby_aggregate,
    groupby_aggregate_multi_column,
    hash_multi_columns,
    hash_partition,
    multi_column_lexsort,
    parallel_sort,
    sort_merge_join,
)

__all__ = [
    "parallel_algorithms", "JfxError", "JfxUnavailable", "load_library", "ParallelRadixSort",
    "ParallelSortMergeJoin", "ShardingSpec", "SortBasedGroupBy", "collective_hash_repartition",
    "combine_keys_for_sorting", "compact_repartitioned_rows", "config", "groupby_aggregate",
    "groupby_aggregate_multi_column", "hash_multi_columns", "hash_partition", "multi_column_lexsort",
    "parallel_sort", "sort_merge_join",
]
