// groupby.cuh -- sort-based groupby: segment-boundary flags over the sorted
// packed keys, then a segmented reduction of each value column gathered
// through the sort permutation (or carried through the sort).
//
// Replaces SortBasedGroupBy.groupby_aggregate (parallel_algorithms.py:733-803,
// boundary flags :767-770, host group count :772, nonzero/cumsum :773-777,
// jax.ops.segment_* :626-660) and groupby_aggregate_multi_column (:662-731,
// _scatter_group_aggregate :1212-1228).
//
// k_group_count counts group starts per warp of 32 * kGroupIPT sorted rows; an
// exclusive scan of the counts numbers the groups; k_group_starts writes each
// group's first row and key columns; k_group_agg reduces each group's rows
// with one thread per group (a warp or a CTA for larger groups), so outputs
// are written by consecutive threads for consecutive groups.  Float sums are accumulated in float64 in row order and rounded
// once, so results are deterministic.
#pragma once

#include "radix.cuh"

namespace jfx {

constexpr int kMaxVals = 16;
constexpr int kGroupIPT = 8;

enum : int { VK_F = 0, VK_I = 1, VK_U = 2 };

struct ValDesc {
  const void* ptr;
  const void* ptr_hi;  // carried 8-byte values: high words (ptr: low words)
  int carried;         // values were carried through the sort as u32 words
  int dtype;
  int kind;
  u32 aggs;
  int mean_dtype;
  int count_dtype;
  int count_via_f32;  // multi-key mean divides by a float32 count
  void* out_sum;
  void* out_mean;
  void* out_count;
  void* out_min;
  void* out_max;
};

struct GroupArgs {
  const void* skeys;  // sorted packed keys (K)
  const u32* perm;    // sorted row ids
  u64 n;
  u32* warp_count;    // per-warp number of group starts (k_group_count)
  const u32* warp_base;  // exclusive scan of warp_count
  PackDesc pack;
  void* uniq_out[kMaxCols];
  int nvals;
  ValDesc v[kMaxVals];
  int values_sorted;  // value columns are already in sorted order (perm unused)
};

// NaN test on the packed key: a float key column holding the canonical NaN.
template <typename K>
__device__ __forceinline__ bool packed_has_nan(const PackDesc& pd, K k) {
  if (!pd.nan_cols) return false;
  for (int j = 0; j < pd.ncols; ++j) {
    if (!((pd.nan_cols >> j) & 1)) continue;
    const ColDesc& c = pd.c[j];
    const u64 nant = c.dtype == JFX_F32 ? (u64)kF32NanT : kF64NanT;
    if (c.bits == 0) {
      if (c.tmin == nant) return true;
      continue;
    }
    const u64 field = ((u64)k >> c.shift) & (c.bits >= 64 ? ~0ull : ((1ull << c.bits) - 1ull));
    if (field + c.tmin == nant) return true;
  }
  return false;
}

template <typename K>
__device__ __forceinline__ bool row_flag(const GroupArgs& a, const K* sk, u64 row) {
  const K k = sk[row];
  if (row == 0) return true;
  return k != sk[row - 1] || packed_has_nan<K>(a.pack, k);
}

template <typename K>
__global__ void __launch_bounds__(256) k_group_count(GroupArgs a, u64 nwarps) {
  const u64 w = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nwarps) return;
  const K* sk = (const K*)a.skeys;
  const u64 wbeg = w * 32 * kGroupIPT, wend = min(a.n, wbeg + 32 * kGroupIPT);
  u32 cnt = 0;
  K kv[kGroupIPT], kl[kGroupIPT];
#pragma unroll
  for (int s = 0; s < kGroupIPT; ++s) {
    const u64 row = wbeg + (u64)s * 32 + lane;
    kv[s] = row < wend ? sk[row] : (K)0;
    kl[s] = (lane == 0 && row < wend && row > 0) ? sk[row - 1] : (K)0;
  }
#pragma unroll
  for (int s = 0; s < kGroupIPT; ++s) {
    const u64 row = wbeg + (u64)s * 32 + lane;
    K kp = __shfl_up_sync(0xffffffffu, kv[s], 1);
    if (lane == 0) kp = kl[s];
    const bool f = row < wend && (row == 0 || kv[s] != kp || packed_has_nan<K>(a.pack, kv[s]));
    cnt += __popc(__ballot_sync(0xffffffffu, f));
  }
  if (lane == 0) a.warp_count[w] = cnt;
}

// ---- per-kind partial state: sum, min, max (64-bit words) and row count ----
template <int KIND>
struct Agg {
  u64 sum, mn, mx;
  u32 cnt;
};

template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_identity() {
  Agg<KIND> s;
  s.cnt = 0;
  if (KIND == VK_F) {
    s.sum = __double_as_longlong(0.0);
    s.mn = __double_as_longlong(__longlong_as_double(0x7ff0000000000000ll));   // +inf
    s.mx = __double_as_longlong(__longlong_as_double((long long)0xfff0000000000000ull));  // -inf
  } else if (KIND == VK_I) {
    s.sum = 0;
    s.mn = 0x7fffffffffffffffull;
    s.mx = 0x8000000000000000ull;
  } else {
    s.sum = 0;
    s.mn = ~0ull;
    s.mx = 0ull;
  }
  return s;
}

// a precedes b in row order; ties keep a.
template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_combine(const Agg<KIND>& a, const Agg<KIND>& b) {
  Agg<KIND> r;
  r.cnt = a.cnt + b.cnt;
  if (KIND == VK_F) {
    const double as = __longlong_as_double(a.sum), bs = __longlong_as_double(b.sum);
    r.sum = __double_as_longlong(as + bs);
    const double an = __longlong_as_double(a.mn), bn = __longlong_as_double(b.mn);
    const double ax = __longlong_as_double(a.mx), bx = __longlong_as_double(b.mx);
    // lax.min / lax.max propagate NaN
    r.mn = (an != an) ? a.mn : (bn != bn) ? b.mn : (bn < an ? b.mn : a.mn);
    r.mx = (ax != ax) ? a.mx : (bx != bx) ? b.mx : (bx > ax ? b.mx : a.mx);
  } else if (KIND == VK_I) {
    r.sum = a.sum + b.sum;
    r.mn = ((long long)b.mn < (long long)a.mn) ? b.mn : a.mn;
    r.mx = ((long long)b.mx > (long long)a.mx) ? b.mx : a.mx;
  } else {
    r.sum = a.sum + b.sum;
    r.mn = b.mn < a.mn ? b.mn : a.mn;
    r.mx = b.mx > a.mx ? b.mx : a.mx;
  }
  return r;
}

// The row's value as the 64-bit word the partial state holds.
template <int KIND>
__device__ __forceinline__ u64 value_word(const ValDesc& v, u64 row) {
  if (v.carried) {
    const u32 lo = __ldg((const u32*)v.ptr + row);
    if (dtype_size(v.dtype) == 8) {
      const u64 w = (u64)lo | ((u64)__ldg((const u32*)v.ptr_hi + row) << 32);
      return KIND == VK_F ? w : w;  // f64 bits / i64 / u64 as stored
    }
    if (KIND == VK_F) return __double_as_longlong((double)__uint_as_float(lo));
    if (KIND == VK_I) return (u64)(long long)(int)lo;
    return (u64)lo;
  }
  if (KIND == VK_F) {
    const double x = v.dtype == JFX_F32 ? (double)__ldg((const float*)v.ptr + row) : __ldg((const double*)v.ptr + row);
    return __double_as_longlong(x);
  }
  if (KIND == VK_I) {
    switch (v.dtype) {
      case JFX_I8: return (u64)(long long)((const signed char*)v.ptr)[row];
      case JFX_I16: return (u64)(long long)((const short*)v.ptr)[row];
      case JFX_I32: return (u64)(long long)__ldg((const int*)v.ptr + row);
      default: return (u64)__ldg((const long long*)v.ptr + row);
    }
  }
  switch (v.dtype) {
    case JFX_U8: case JFX_BOOL: return ((const unsigned char*)v.ptr)[row];
    case JFX_U16: return ((const unsigned short*)v.ptr)[row];
    case JFX_U32: return __ldg((const unsigned*)v.ptr + row);
    default: return __ldg((const u64*)v.ptr + row);
  }
}

template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_of(const ValDesc& v, u64 row) {
  Agg<KIND> s;
  s.cnt = 1;
  u64 w;
  if (KIND == VK_F) {
    double x = v.dtype == JFX_F32 ? (double)__ldg((const float*)v.ptr + row) : __ldg((const double*)v.ptr + row);
    w = __double_as_longlong(x);
  } else if (KIND == VK_I) {
    long long x;
    switch (v.dtype) {
      case JFX_I8: x = ((const signed char*)v.ptr)[row]; break;
      case JFX_I16: x = ((const short*)v.ptr)[row]; break;
      case JFX_I32: x = __ldg((const int*)v.ptr + row); break;
      default: x = __ldg((const long long*)v.ptr + row); break;
    }
    w = (u64)x;
  } else {
    switch (v.dtype) {
      case JFX_U8: case JFX_BOOL: w = ((const unsigned char*)v.ptr)[row]; break;
      case JFX_U16: w = ((const unsigned short*)v.ptr)[row]; break;
      case JFX_U32: w = __ldg((const unsigned*)v.ptr + row); break;
      default: w = __ldg((const u64*)v.ptr + row); break;
    }
  }
  s.sum = s.mn = s.mx = w;
  return s;
}

__device__ __forceinline__ void store_float(void* base, int dtype, u64 i, double x) {
  if (dtype == JFX_F32) ((float*)base)[i] = (float)x;
  else ((double*)base)[i] = x;
}

// Value of the group's sum in the value dtype, as a double (for the mean).
template <int KIND>
__device__ __forceinline__ double sum_in_value_dtype(const ValDesc& v, u64 sum) {
  if (KIND == VK_F) {
    double s = __longlong_as_double(sum);
    return v.dtype == JFX_F32 ? (double)(float)s : s;
  }
  // integer sums wrap in the value dtype
  const int bits = dtype_bits(v.dtype);
  if (KIND == VK_I) {
    long long x = bits >= 64 ? (long long)sum : ((long long)(sum << (64 - bits)) >> (64 - bits));
    return (double)x;
  }
  u64 x = bits >= 64 ? sum : (sum & ((1ull << bits) - 1ull));
  return (double)x;
}

template <int KIND>
__device__ __forceinline__ void agg_finalize(const ValDesc& v, u64 g, const Agg<KIND>& s) {
  if (v.aggs & JFX_AGG_SUM) {
    if (KIND == VK_F) store_float(v.out_sum, v.dtype, g, __longlong_as_double(s.sum));
    else store_raw(v.out_sum, v.dtype, g, s.sum);
  }
  if (v.aggs & JFX_AGG_MEAN) {
    double c = v.count_via_f32 ? (double)(float)s.cnt : (double)s.cnt;
    if (v.mean_dtype == JFX_F32) {
      // float32 arithmetic: float(sum in value dtype) / float(count)
      float num;
      if (KIND == VK_F) num = (float)sum_in_value_dtype<KIND>(v, s.sum);
      else if (KIND == VK_I) {
        const int bits = dtype_bits(v.dtype);
        long long x = bits >= 64 ? (long long)s.sum : ((long long)(s.sum << (64 - bits)) >> (64 - bits));
        num = (float)x;
      } else {
        const int bits = dtype_bits(v.dtype);
        u64 x = bits >= 64 ? s.sum : (s.sum & ((1ull << bits) - 1ull));
        num = (float)x;
      }
      ((float*)v.out_mean)[g] = num / (float)c;
    } else {
      double num;
      if (KIND == VK_F) num = sum_in_value_dtype<KIND>(v, s.sum);
      else if (KIND == VK_I) {
        const int bits = dtype_bits(v.dtype);
        long long x = bits >= 64 ? (long long)s.sum : ((long long)(s.sum << (64 - bits)) >> (64 - bits));
        num = (double)x;
      } else {
        const int bits = dtype_bits(v.dtype);
        u64 x = bits >= 64 ? s.sum : (s.sum & ((1ull << bits) - 1ull));
        num = (double)x;
      }
      ((double*)v.out_mean)[g] = num / c;
    }
  }
  if (v.aggs & JFX_AGG_COUNT) {
    switch (v.count_dtype) {
      case JFX_F32: ((float*)v.out_count)[g] = (float)s.cnt; break;
      case JFX_F64: ((double*)v.out_count)[g] = (double)s.cnt; break;
      default: store_raw(v.out_count, v.count_dtype, g, (u64)s.cnt); break;
    }
  }
  if (v.aggs & JFX_AGG_MIN) {
    if (KIND == VK_F) store_float(v.out_min, v.dtype, g, __longlong_as_double(s.mn));
    else store_raw(v.out_min, v.dtype, g, s.mn);
  }
  if (v.aggs & JFX_AGG_MAX) {
    if (KIND == VK_F) store_float(v.out_max, v.dtype, g, __longlong_as_double(s.mx));
    else store_raw(v.out_max, v.dtype, g, s.mx);
  }
}

// ------------------------------------------------- group-parallel reduce ---
// After k_group_count and the scan of its per-warp counts, k_group_starts
// writes every group's first row (and the group's key columns), and
// k_group_agg reduces each group's rows: thread g of the grid owns group g,
// so every output column is written with consecutive threads on consecutive
// groups.  A group of more than kSmallGroup rows is reduced by the whole warp
// instead, and one of more than kWarpGroup rows (the heavy keys of a skewed
// column) by a whole CTA in k_group_big, many at once; both read coalesced and combine the
// rows in row order.

constexpr u32 kSmallGroup = 32;

template <typename K>
__global__ void __launch_bounds__(256) k_group_starts(GroupArgs a, u64 nwarps, u32* starts) {
  const u64 w = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nwarps) return;
  const K* sk = (const K*)a.skeys;
  const u64 wbeg = w * 32 * kGroupIPT, wend = min(a.n, wbeg + 32 * kGroupIPT);
  const u32 lt = lanemask_lt();
  u32 gbase = a.warp_base[w];
  K kv[kGroupIPT];
#pragma unroll
  for (int q = 0; q < kGroupIPT; ++q) {
    const u64 row = wbeg + (u64)q * 32 + lane;
    kv[q] = row < wend ? sk[row] : (K)0;
  }
  K carry = wbeg > 0 ? sk[wbeg - 1] : (K)0;  // the row before this step's first row
#pragma unroll
  for (int q = 0; q < kGroupIPT; ++q) {
    const u64 row = wbeg + (u64)q * 32 + lane;
    K kp = __shfl_up_sync(0xffffffffu, kv[q], 1);
    if (lane == 0) kp = carry;
    carry = __shfl_sync(0xffffffffu, kv[q], 31);
    const bool f = row < wend && (row == 0 || kv[q] != kp || packed_has_nan<K>(a.pack, kv[q]));
    const u32 bal = __ballot_sync(0xffffffffu, f);
    if (f) {
      const u32 gid = gbase + __popc(bal & lt);
      starts[gid] = (u32)row;
      for (int jc = 0; jc < a.pack.ncols; ++jc) {
        const ColDesc& cd = a.pack.c[jc];
        if (!a.uniq_out[jc]) continue;
        if (dtype_is_float(cd.dtype)) {
          // original bits of the group's first row (-0.0 vs +0.0, NaN payloads)
          const u32 krow = a.perm ? a.perm[row] : (u32)row;
          store_raw(a.uniq_out[jc], cd.dtype, gid, load_raw(cd.ptr, cd.dtype, krow));
        } else {
          const u64 field =
              cd.bits ? (((u64)kv[q] >> cd.shift) & (cd.bits >= 64 ? ~0ull : ((1ull << cd.bits) - 1ull))) : 0ull;
          store_raw(a.uniq_out[jc], cd.dtype, gid, untransform_int(cd.dtype, cd.flags, field + cd.tmin));
        }
      }
    }
    gbase += __popc(bal);
  }
}

// starts[G] = n: the end of the last group (G read on the device).
__global__ void k_group_end(u32* starts, const u32* total, u64 n) { starts[*total] = (u32)n; }

template <int KIND>
__device__ __forceinline__ u64 row_value(const GroupArgs& a, const ValDesc& v, u64 row) {
  return value_word<KIND>(v, a.values_sorted ? row : (u64)a.perm[row]);
}

// Rows [s, e) folded in row order by one thread.
template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_rows(const GroupArgs& a, const ValDesc& v, bool need_vals, u32 s, u32 e) {
  Agg<KIND> acc = agg_identity<KIND>();
  constexpr int U = 4;  // loads issued together
  for (u32 r0 = s; r0 < e; r0 += U) {
    u64 w[U];
#pragma unroll
    for (int u = 0; u < U; ++u) w[u] = (need_vals && r0 + u < e) ? row_value<KIND>(a, v, r0 + u) : 0ull;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (r0 + u >= e) break;
      Agg<KIND> r;
      r.cnt = 1;
      r.sum = r.mn = r.mx = w[u];
      acc = agg_combine<KIND>(acc, r);
    }
  }
  return acc;
}

// Ordered combine of the warp's per-lane states: lane order, result in lane 0.
template <int KIND>
__device__ __forceinline__ Agg<KIND> warp_combine_ordered(Agg<KIND> acc, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    Agg<KIND> up;
    up.sum = __shfl_down_sync(0xffffffffu, acc.sum, o);
    up.mn = __shfl_down_sync(0xffffffffu, acc.mn, o);
    up.mx = __shfl_down_sync(0xffffffffu, acc.mx, o);
    up.cnt = __shfl_down_sync(0xffffffffu, acc.cnt, o);
    if ((lane & (2 * o - 1)) == 0 && lane + o < 32) acc = agg_combine<KIND>(acc, up);
  }
  return acc;
}

// Rows [s, e) folded by the whole warp in row order, reading coalesced: each
// round covers 32 * kWarpRun consecutive rows, lane l folding the kWarpRun
// rows from s + round + l * kWarpRun; the 32 lane states combine in lane
// order and the round's state joins the running one.  Valid in lane 0.
// Rows [j0, min(j0 + R, e)) folded in row order, every load issued first.
template <int KIND, int R>
__device__ __forceinline__ Agg<KIND> fold_run(const GroupArgs& a, const ValDesc& v, bool need_vals, u32 j0, u32 e) {
  u64 w[R];
#pragma unroll
  for (int u = 0; u < R; ++u) w[u] = (need_vals && j0 + u < e) ? row_value<KIND>(a, v, j0 + u) : 0ull;
  Agg<KIND> part = agg_identity<KIND>();
#pragma unroll
  for (int u = 0; u < R; ++u) {
    if (j0 + u < e) {
      Agg<KIND> r;
      r.cnt = 1;
      r.sum = r.mn = r.mx = w[u];
      part = agg_combine<KIND>(part, r);
    }
  }
  return part;
}

constexpr int kWarpRun = 8;
template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_rows_warp(const GroupArgs& a, const ValDesc& v, bool need_vals, u32 s,
                                                   u32 e, int lane) {
  Agg<KIND> acc = agg_identity<KIND>();
  for (u32 r0 = s; r0 < e; r0 += 32 * kWarpRun) {
    const u32 j0 = min(e, r0 + (u32)lane * kWarpRun);
    Agg<KIND> part = warp_combine_ordered<KIND>(fold_run<KIND, kWarpRun>(a, v, need_vals, j0, e), lane);
    if (lane == 0) acc = agg_combine<KIND>(acc, part);
  }
  return acc;
}

// Groups of more than kWarpGroup rows are listed by k_group_agg and reduced by
// k_group_big, one CTA each.
constexpr u32 kWarpGroup = 512;

template <int KIND>
__device__ __forceinline__ void agg_column(const GroupArgs& a, int c, bool valid, u32 g, u32 s, u32 e, bool mid,
                                           int lane) {
  const ValDesc& v = a.v[c];
  const bool need_vals = (v.aggs & ~JFX_AGG_COUNT) != 0;
  if (valid && e - s <= kSmallGroup) agg_finalize<KIND>(v, g, agg_rows<KIND>(a, v, need_vals, s, e));
  for (u32 m = __ballot_sync(0xffffffffu, mid); m; m &= m - 1) {
    const int L = __ffs(m) - 1;
    const u32 gs = __shfl_sync(0xffffffffu, s, L), ge = __shfl_sync(0xffffffffu, e, L);
    const u32 gg = __shfl_sync(0xffffffffu, g, L);
    const Agg<KIND> r = agg_rows_warp<KIND>(a, v, need_vals, gs, ge, lane);
    if (lane == 0) agg_finalize<KIND>(v, gg, r);
  }
}

// big: [0] count, then group ids (capacity n / kWarpGroup + 1).
__global__ void __launch_bounds__(256) k_group_agg(GroupArgs a, const u32* starts, const u32* total, u32* big) {
  const u32 G = *total;
  const int lane = threadIdx.x & 31;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 g0 = (u64)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); g0 < G; g0 += stride) {
    const u64 g = g0 + lane;
    const bool valid = g < G;
    const u32 s = valid ? starts[g] : 0u, e = valid ? starts[g + 1] : 0u;
    const bool large = valid && e - s > kWarpGroup;
    const bool mid = valid && !large && e - s > kSmallGroup;
    if (large) big[1 + atomicAdd(&big[0], 1u)] = (u32)g;
    for (int c = 0; c < a.nvals; ++c) {
      switch (a.v[c].kind) {
        case VK_F: agg_column<VK_F>(a, c, valid && !large, (u32)g, s, e, mid, lane); break;
        case VK_I: agg_column<VK_I>(a, c, valid && !large, (u32)g, s, e, mid, lane); break;
        default: agg_column<VK_U>(a, c, valid && !large, (u32)g, s, e, mid, lane); break;
      }
    }
  }
}

// One listed group per CTA, in rounds of kBigRun * blockDim.x consecutive
// rows: thread t loads rows round + t * kBigRun .. + kBigRun (all loads issued
// before the first is used) and folds them; the threads' states combine in
// thread order (warps in lane order, then the warps in order through shared
// memory) and join the running state in thread 0.
constexpr int kBigRun = 8;
template <int KIND>
__device__ __forceinline__ void big_column(const GroupArgs& a, int c, u32 g, u32 s, u32 e, u64* sh) {
  const ValDesc& v = a.v[c];
  const bool need_vals = (v.aggs & ~JFX_AGG_COUNT) != 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  Agg<KIND> acc = agg_identity<KIND>();
  for (u32 r0 = s; r0 < e; r0 += kBigRun * blockDim.x) {
    const u32 j0 = min(e, r0 + threadIdx.x * kBigRun);
    Agg<KIND> part = warp_combine_ordered<KIND>(fold_run<KIND, kBigRun>(a, v, need_vals, j0, e), lane);
    if (lane == 0) {
      sh[4 * warp] = part.sum;
      sh[4 * warp + 1] = part.mn;
      sh[4 * warp + 2] = part.mx;
      sh[4 * warp + 3] = part.cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int q = 0; q < warps; ++q) {
        Agg<KIND> x;
        x.sum = sh[4 * q];
        x.mn = sh[4 * q + 1];
        x.mx = sh[4 * q + 2];
        x.cnt = (u32)sh[4 * q + 3];
        acc = agg_combine<KIND>(acc, x);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) agg_finalize<KIND>(v, g, acc);
}

__global__ void __launch_bounds__(256) k_group_big(GroupArgs a, const u32* starts, const u32* big) {
  __shared__ u64 sh[4 * 32];
  const u32 count = big[0];
  for (u32 i = blockIdx.x; i < count; i += gridDim.x) {
    const u32 g = big[1 + i];
    const u32 s = starts[g], e = starts[g + 1];
    for (int c = 0; c < a.nvals; ++c) {
      switch (a.v[c].kind) {
        case VK_F: big_column<VK_F>(a, c, g, s, e, sh); break;
        case VK_I: big_column<VK_I>(a, c, g, s, e, sh); break;
        default: big_column<VK_U>(a, c, g, s, e, sh); break;
      }
    }
  }
}

// ---------------------------------------------------- device-wide scan ---
// Exclusive scan of m u32 values into T (u32 or u64); *total = sum.
template <typename T>
__global__ void __launch_bounds__(1024) k_scan_reduce(const u32* in, u64 m, T* partial) {
  __shared__ T sh[32];
  const u64 base = (u64)blockIdx.x * 4096;
  T s = 0;
  for (int k = 0; k < 4; ++k) {
    u64 i = base + (u64)k * 1024 + threadIdx.x;
    if (i < m) s += (T)in[i];
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    T x = sh[threadIdx.x];
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = x;
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_scan_partials(T* partial, u64 nb, T* total) {
  __shared__ T sh[32];
  T carry = 0;
  for (u64 b0 = 0; b0 < nb; b0 += 1024) {
    u64 i = b0 + threadIdx.x;
    T x = i < nb ? partial[i] : 0;
    T inc = x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      T wv = sh[lane];
      T wi = wv;
      for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += y;
      }
      sh[lane] = wi - wv;
    }
    __syncthreads();
    T ex = inc - x + sh[warp] + carry;
    if (i < nb) partial[i] = ex;
    __syncthreads();
    if (threadIdx.x == 1023) sh[0] = ex + x;
    __syncthreads();
    carry = sh[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_scan_apply(const u32* in, u64 m, const T* partial, T* out) {
  __shared__ T sh[32];
  const u64 base = (u64)blockIdx.x * 4096;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // each thread: 4 consecutive items
  T v[4], s = 0;
  for (int k = 0; k < 4; ++k) {
    u64 i = base + (u64)threadIdx.x * 4 + k;
    v[k] = i < m ? (T)in[i] : 0;
    s += v[k];
  }
  T inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T wv = sh[lane];
    T wi = wv;
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    sh[lane] = wi - wv;
  }
  __syncthreads();
  T ex = inc - s + sh[warp] + partial[blockIdx.x];
  for (int k = 0; k < 4; ++k) {
    u64 i = base + (u64)threadIdx.x * 4 + k;
    if (i < m) out[i] = ex;
    ex += v[k];
  }
}

template <typename T>
inline int device_exclusive_scan(const u32* in, u64 m, T* out, T* total, T* partial, cudaStream_t s) {
  u64 nb = (m + 4095) / 4096;
  if (nb == 0) {
    JFX_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
    return JFX_OK;
  }
  k_scan_reduce<T><<<(unsigned)nb, 1024, 0, s>>>(in, m, partial), note_launch();
  k_scan_partials<T><<<1, 1024, 0, s>>>(partial, nb, total), note_launch();
  k_scan_apply<T><<<(unsigned)nb, 1024, 0, s>>>(in, m, partial, out), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}
inline u64 scan_partials_count(u64 m) { return (m + 4095) / 4096 + 1; }

}  // namespace jfx
