// batch.cuh -- many independent queries in one stream of kernels: per query,
// the one-device body of collective_hash_repartition with P partitions
// (parallel_algorithms.py:163-182, :213-214) followed by
// SortBasedGroupBy.groupby_aggregate sum and count (:733-803).
//
// All queries' rows are concatenated.  Segmented onesweep passes (radix.cuh,
// PassArgs.segmented) never let a tile straddle a query: the look-back chains
// within a query and every digit offset is per query.  Pass 0 partitions by
// fmix32(key) % P and moves (key, value); the key passes sort each query by
// key; the last pass tags each key with its query id so one run of the
// groupby kernels covers the whole batch (groups never cross queries) with
// the values already in sorted order.  Nothing synchronises with the host, so
// the whole sequence can be captured in one CUDA graph.
#pragma once

#include "groupby.cuh"

namespace jfx {

constexpr int kBatchRB = 10;  // digit width of the batched passes (RADIX 1024)
constexpr int kBatchTile = PassLayout<u32, kBatchRB>::TILE;  // rows per tile of every batched pass

__global__ void k_seg_setup(const int64_t* qoff, u32 nq, u64* row_base, u32* tile_cnt, u32* err) {
  for (u32 q = blockIdx.x * blockDim.x + threadIdx.x; q <= nq; q += gridDim.x * blockDim.x) {
    row_base[q] = (u64)qoff[q];
    if (q < nq) {
      const int64_t rows = qoff[q + 1] - qoff[q];
      if (rows < 0) {
        atomicOr(err, DERR_BOUNDS);
        tile_cnt[q] = 0;
      } else {
        tile_cnt[q] = (u32)((rows + kBatchTile - 1) / kBatchTile);
      }
    }
  }
}

__global__ void k_seg_tile_map(const u32* tile_base, const u32* tile_cnt, u32 nq, u32* tile_seg) {
  for (u32 q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
    for (u32 t = 0; t < tile_cnt[q]; ++t) tile_seg[tile_base[q] + t] = q;
}

struct SegHistArgs {
  const int32_t* keys;
  const u64* row_base;
  const u32* tile_base;
  const u32* tile_seg;
  const u32* total_tiles;
  u32* hist;        // [nseg][npass][RADIX]
  u32* err;
  int npass;        // pass 0: partition digit; passes 1..: key digits
  u32 modulus;
  int key_bits;
  int shift[8];
  int width[8];
};

template <int RB>
__global__ void __launch_bounds__(256) k_hist_seg(SegHistArgs a) {
  constexpr int RADIX = 1 << RB;
  extern __shared__ u32 sh[];
  const int total = a.npass * RADIX;
  const u32 tiles = *a.total_tiles;
  for (u32 t = blockIdx.x; t < tiles; t += gridDim.x) {
    for (int i = threadIdx.x; i < total; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    const u32 q = a.tile_seg[t];
    const u64 r0 = a.row_base[q] + (u64)(t - a.tile_base[q]) * kBatchTile;
    const u64 r1 = min(a.row_base[q + 1], r0 + kBatchTile);
    for (u64 r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const u32 raw = (u32)a.keys[r];
      if (raw >= (1u << a.key_bits)) atomicOr(a.err, DERR_BOUNDS);  // key outside [0, 2^key_bits)
      atomicAdd(&sh[fmix32_d(raw) % a.modulus], 1u);
      for (int p = 1; p < a.npass; ++p) atomicAdd(&sh[p * RADIX + ((raw >> a.shift[p]) & ((1u << a.width[p]) - 1u))], 1u);
    }
    __syncthreads();
    u32* h = a.hist + (u64)q * total;
    for (int i = threadIdx.x; i < total; i += blockDim.x)
      if (sh[i]) atomicAdd(&h[i], sh[i]);
    __syncthreads();
  }
}

// Partition offsets of every query: row_base[q] + digit offsets of pass 0.
__global__ void k_part_offsets(const u64* row_base, const u32* bin_base, u32 nq, int npass, int radix, u32 P,
                               int64_t* out) {
  const u64 total = (u64)nq * (P + 1);
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (u64)gridDim.x * blockDim.x) {
    const u32 q = (u32)(i / (P + 1)), p = (u32)(i % (P + 1));
    out[i] = p < P ? (int64_t)(row_base[q] + bin_base[(u64)q * npass * radix + p]) : (int64_t)row_base[q + 1];
  }
}

// Group offsets of every query: groups are ordered by (query, key), so the
// first group of query q is the lower bound of q in the groups' query ids.
__global__ void k_group_offsets(const u32* group_q, const u32* ngroups, u32 nq, int64_t* out) {
  const u32 G = *ngroups;
  for (u32 q = blockIdx.x * blockDim.x + threadIdx.x; q <= nq; q += gridDim.x * blockDim.x) {
    u32 lo = 0, hi = G;
    while (lo < hi) {
      const u32 mid = (lo + hi) >> 1;
      if (group_q[mid] < q) lo = mid + 1;
      else hi = mid;
    }
    out[q] = lo;
  }
}

}  // namespace jfx
