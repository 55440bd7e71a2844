// groupby.cuh -- sort-based groupby: segment-boundary flags over the sorted
// packed keys, then a warp-level segmented reduction of each value column
// gathered through the sort permutation.
//
// Replaces SortBasedGroupBy.groupby_aggregate (parallel_algorithms.py:733-803,
// boundary flags :767-770, host group count :772, nonzero/cumsum :773-777,
// jax.ops.segment_* :626-660) and groupby_aggregate_multi_column (:662-731,
// _scatter_group_aggregate :1212-1228).
//
// Every warp owns 32*IPT consecutive sorted rows.  A group that starts and
// ends inside one warp is written by that warp.  A group that crosses a warp
// boundary leaves one partial record per warp it touches (at most two per
// warp); k_group_fixup combines those records in row order.  Float sums are
// accumulated in float64 and rounded once, so results are deterministic.
#pragma once

#include "radix.cuh"

namespace jfx {

constexpr int kMaxVals = 16;
constexpr int kGroupIPT = 8;
constexpr u32 kEmptySlot = 0xffffffffu;

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
  u32* slot_gid;      // [2 * warps]
  u32* slot_started;  // [2 * warps]
  u64* slot_state;    // [nvals][4][2 * warps]: sum, min, max, count
  u64 nslots;
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

template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_shfl_up(const Agg<KIND>& s, int o) {
  Agg<KIND> r;
  r.sum = __shfl_up_sync(0xffffffffu, s.sum, o);
  r.mn = __shfl_up_sync(0xffffffffu, s.mn, o);
  r.mx = __shfl_up_sync(0xffffffffu, s.mx, o);
  r.cnt = __shfl_up_sync(0xffffffffu, s.cnt, o);
  return r;
}
template <int KIND>
__device__ __forceinline__ Agg<KIND> agg_shfl(const Agg<KIND>& s, int src) {
  Agg<KIND> r;
  r.sum = __shfl_sync(0xffffffffu, s.sum, src);
  r.mn = __shfl_sync(0xffffffffu, s.mn, src);
  r.mx = __shfl_sync(0xffffffffu, s.mx, src);
  r.cnt = __shfl_sync(0xffffffffu, s.cnt, src);
  return r;
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

template <int KIND>
__device__ __forceinline__ void slot_store(const GroupArgs& a, int c, u64 slot, u32 gid, u32 started,
                                           const Agg<KIND>& s) {
  u64* st = a.slot_state + (u64)c * 4 * a.nslots;
  st[slot] = s.sum;
  st[a.nslots + slot] = s.mn;
  st[2 * a.nslots + slot] = s.mx;
  st[3 * a.nslots + slot] = s.cnt;
  if (c == 0) {
    a.slot_gid[slot] = gid;
    a.slot_started[slot] = started;
  }
}

// The value of sorted row `pos` (carried columns: lo/hi words already read).
template <int KIND>
__device__ __forceinline__ u64 carried_word(const ValDesc& v, u32 lo, u32 hi) {
  if (dtype_size(v.dtype) == 8) return (u64)lo | ((u64)hi << 32);
  if (KIND == VK_F) return __double_as_longlong((double)__uint_as_float(lo));
  if (KIND == VK_I) return (u64)(long long)(int)lo;
  return (u64)lo;
}

// One value column over the warp's rows, lane-sequential: lane l owns the
// kGroupIPT consecutive rows r0.. (bit j of fl: row r0+j starts a group).
// Pass 1 folds each lane's rows after its last group start; a segmented
// scan across the 32 lanes gives every lane the part of its first group that
// lies in earlier lanes; pass 2 walks the lane's rows again and writes each
// group where it ends.  Groups that begin in an earlier warp or run past the
// warp end leave slot records for k_group_fixup, as before.
template <int KIND>
__device__ __forceinline__ void reduce_lane_column(const GroupArgs& a, int c, u64 w, u64 r0, int nv, u32 fl,
                                                   u32 gfirst, bool last_lane, bool end_closes, bool next_flag,
                                                   const u32 (&pr)[kGroupIPT]) {
  const ValDesc& v = a.v[c];
  const int lane = threadIdx.x & 31;
  const bool need_vals = (v.aggs & ~JFX_AGG_COUNT) != 0;
  u64 word[kGroupIPT];
  if (need_vals) {
    if (v.carried) {
      u32 lo[kGroupIPT], hi[kGroupIPT];
      const bool wide = dtype_size(v.dtype) == 8;
      if (nv == kGroupIPT) {
#pragma unroll
        for (int q = 0; q < kGroupIPT / 4; ++q) {
          reinterpret_cast<uint4*>(lo)[q] = __ldg(reinterpret_cast<const uint4*>((const u32*)v.ptr + r0) + q);
          if (wide) reinterpret_cast<uint4*>(hi)[q] = __ldg(reinterpret_cast<const uint4*>((const u32*)v.ptr_hi + r0) + q);
        }
      } else {
#pragma unroll
        for (int j = 0; j < kGroupIPT; ++j) {
          lo[j] = j < nv ? __ldg((const u32*)v.ptr + r0 + j) : 0u;
          hi[j] = (wide && j < nv) ? __ldg((const u32*)v.ptr_hi + r0 + j) : 0u;
        }
      }
#pragma unroll
      for (int j = 0; j < kGroupIPT; ++j) word[j] = carried_word<KIND>(v, lo[j], wide ? hi[j] : 0u);
    } else {
#pragma unroll
      for (int j = 0; j < kGroupIPT; ++j) word[j] = j < nv ? value_word<KIND>(v, pr[j]) : 0ull;
    }
  }
  // pass 1: the lane's rows after its last group start (all rows without one)
  Agg<KIND> tail = agg_identity<KIND>();
#pragma unroll
  for (int j = 0; j < kGroupIPT; ++j) {
    if (j >= nv) break;
    if ((fl >> j) & 1u) tail = agg_identity<KIND>();
    Agg<KIND> r;
    r.cnt = 1;
    r.sum = r.mn = r.mx = need_vals ? word[j] : 0ull;
    tail = agg_combine<KIND>(tail, r);
  }
  // segmented inclusive scan over lanes: a lane with a group start restarts
  Agg<KIND> run = tail;
  bool seg = fl != 0u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const Agg<KIND> up = agg_shfl_up<KIND>(run, o);
    const bool useg = __shfl_up_sync(0xffffffffu, seg, o);
    if (lane >= o && !seg) {
      run = agg_combine<KIND>(up, run);
      seg = useg;
    }
  }
  // the part of the lane's first group in earlier lanes, and whether that
  // group began inside this warp
  Agg<KIND> cur = agg_shfl_up<KIND>(run, 1);
  bool cur_started = __shfl_up_sync(0xffffffffu, seg, 1);
  bool cur_rows = lane > 0;
  if (lane == 0) {
    cur = agg_identity<KIND>();
    cur_started = false;
  }
  u32 cur_gid = gfirst - 1u;
  // pass 2: write every group that ends inside the lane
#pragma unroll 1
  for (int j = 0; j < nv; ++j) {
    if ((fl >> j) & 1u) {
      if (cur_rows) {
        if (cur_started) agg_finalize<KIND>(v, cur_gid, cur);
        else slot_store<KIND>(a, c, 2 * w, cur_gid, 0u, cur);  // the warp's first group, begun earlier
      }
      cur = agg_identity<KIND>();
      cur_started = true;
      cur_gid = gfirst + __popc(fl & ((1u << j) - 1u));
    }
    Agg<KIND> r;
    r.cnt = 1;
    r.sum = r.mn = r.mx = need_vals ? word[j] : 0ull;
    cur = agg_combine<KIND>(cur, r);
    cur_rows = true;
  }
  if (nv == 0) return;
  // the group open at the lane end ends here if the next lane starts a group,
  // or at the warp end when the row after the warp starts one
  if (last_lane ? end_closes : next_flag) {
    if (cur_started) agg_finalize<KIND>(v, cur_gid, cur);
    else slot_store<KIND>(a, c, 2 * w, cur_gid, 0u, cur);
  } else if (last_lane) {
    slot_store<KIND>(a, c, 2 * w + 1, cur_gid, cur_started ? 1u : 0u, cur);  // open past the warp end
  }
}

template <typename K>
__global__ void __launch_bounds__(256, 4) k_group_reduce(GroupArgs a, u64 nwarps) {  // 4 CTAs per SM
  const u64 w = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nwarps) return;  // whole warps exit together
  const K* sk = (const K*)a.skeys;
  const u64 wbeg = w * 32 * kGroupIPT, wend = min(a.n, wbeg + 32 * kGroupIPT);
  const u64 r0 = wbeg + (u64)lane * kGroupIPT;
  const int nv = r0 >= wend ? 0 : (int)min((u64)kGroupIPT, wend - r0);
  K kv[kGroupIPT];
  if (nv == kGroupIPT && (kGroupIPT * sizeof(K)) % 16 == 0) {
#pragma unroll
    for (int q = 0; q < kGroupIPT * (int)sizeof(K) / 16; ++q)
      reinterpret_cast<uint4*>(kv)[q] = __ldg(reinterpret_cast<const uint4*>(sk + r0) + q);
  } else {
#pragma unroll
    for (int j = 0; j < kGroupIPT; ++j) kv[j] = j < nv ? sk[r0 + j] : (K)0;
  }
  u32 pr[kGroupIPT];
  if (!a.values_sorted) {
#pragma unroll
    for (int j = 0; j < kGroupIPT; ++j) pr[j] = j < nv ? a.perm[r0 + j] : 0u;
  } else {
#pragma unroll
    for (int j = 0; j < kGroupIPT; ++j) pr[j] = (u32)(r0 + j);
  }
  // group starts: the key differs from the previous row's (a NaN key is a group of its own)
  K prev = __shfl_up_sync(0xffffffffu, kv[kGroupIPT - 1], 1);
  if (lane == 0) prev = wbeg > 0 ? sk[wbeg - 1] : (K)0;
  u32 fl = 0;
#pragma unroll
  for (int j = 0; j < kGroupIPT; ++j) {
    const K kp = j ? kv[j - 1] : prev;
    const bool f = j < nv && (r0 + j == 0 || kv[j] != kp || packed_has_nan<K>(a.pack, kv[j]));
    fl |= (u32)f << j;
  }
  // group id of the lane's first start: warp base + starts in earlier lanes
  const u32 cnt = __popc(fl);
  u32 inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  const u32 gfirst = a.warp_base[w] + inc - cnt;
  // unique key columns of every group starting in the lane
  for (u32 m = fl; m; m &= m - 1) {
    const int j = __ffs(m) - 1;
    const u32 gid = gfirst + __popc(fl & ((1u << j) - 1u));
    const u64 row = r0 + j;
    for (int jc = 0; jc < a.pack.ncols; ++jc) {
      const ColDesc& cd = a.pack.c[jc];
      if (!a.uniq_out[jc]) continue;
      if (dtype_is_float(cd.dtype)) {
        // original bits of the group's first row (-0.0 vs +0.0, NaN payloads)
        const u32 krow = a.perm ? a.perm[row] : (u32)row;
        store_raw(a.uniq_out[jc], cd.dtype, gid, load_raw(cd.ptr, cd.dtype, krow));
      } else {
        const u64 field = cd.bits ? (((u64)kv[j] >> cd.shift) & (cd.bits >= 64 ? ~0ull : ((1ull << cd.bits) - 1ull))) : 0ull;
        store_raw(a.uniq_out[jc], cd.dtype, gid, untransform_int(cd.dtype, cd.flags, field + cd.tmin));
      }
    }
  }
  const int last = (int)((wend - 1 - wbeg) / kGroupIPT);  // lane holding the warp's last row
  const bool end_closes = wend < a.n ? row_flag<K>(a, sk, wend) : true;
  const bool next_flag = __shfl_down_sync(0xffffffffu, fl & 1u, 1) != 0u;
  for (int c = 0; c < a.nvals; ++c) {
    switch (a.v[c].kind) {
      case VK_F: reduce_lane_column<VK_F>(a, c, w, r0, nv, fl, gfirst, lane == last, end_closes, next_flag, pr); break;
      case VK_I: reduce_lane_column<VK_I>(a, c, w, r0, nv, fl, gfirst, lane == last, end_closes, next_flag, pr); break;
      default: reduce_lane_column<VK_U>(a, c, w, r0, nv, fl, gfirst, lane == last, end_closes, next_flag, pr); break;
    }
  }
}

template <int KIND>
__device__ __forceinline__ Agg<KIND> slot_load(const GroupArgs& a, int c, u64 i) {
  const u64* st = a.slot_state + (u64)c * 4 * a.nslots;
  Agg<KIND> s;
  s.sum = st[i];
  s.mn = st[a.nslots + i];
  s.mx = st[2 * a.nslots + i];
  s.cnt = (u32)st[3 * a.nslots + i];
  return s;
}

// The records [i, end) of group g (empty records skipped), combined in row
// order by one warp: lane l folds a contiguous share of the records, then a
// tree in lane order joins the shares, so a group spanning many warps costs
// its record count / 32 steps, not one step per record.
template <int KIND>
__device__ void fixup_column(const GroupArgs& a, int c, u64 i, u64 end, u32 g, int lane) {
  const u64 cnt = end - i, share = (cnt + 31) / 32;
  const u64 j0 = i + (u64)lane * share, j1 = min(end, j0 + share);
  Agg<KIND> s = agg_identity<KIND>();
  for (u64 j = j0; j < j1; ++j)
    if (a.slot_gid[j] == g) s = agg_combine<KIND>(s, slot_load<KIND>(a, c, j));
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    Agg<KIND> up;
    up.sum = __shfl_down_sync(0xffffffffu, s.sum, o);
    up.mn = __shfl_down_sync(0xffffffffu, s.mn, o);
    up.mx = __shfl_down_sync(0xffffffffu, s.mx, o);
    up.cnt = __shfl_down_sync(0xffffffffu, s.cnt, o);
    if ((lane & (2 * o - 1)) == 0 && lane + o < 32) s = agg_combine<KIND>(s, up);
  }
  if (lane == 0) agg_finalize<KIND>(a.v[c], g, s);
}

// For every partial record that holds a group's first row, a warp finds the
// group's following records (same group id, not a group start; empty
// records in between) 32 at a time and combines them.  Warps take the
// records 32 at a time over a grid sized to the GPU, so the mostly empty or
// continuing records cost a ballot, not a warp launch each.
__global__ void __launch_bounds__(256) k_group_fixup(GroupArgs a) {
  // a warp takes 32 records at a time (grid-stride) and handles the ones
  // that hold a group's first row, one after the other
  const int lane = threadIdx.x & 31;
  const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 base = (((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < a.nslots; base += nw * 32) {
    const u64 jl = base + lane;
    const u32 gl = jl < a.nslots ? a.slot_gid[jl] : kEmptySlot;
    u32 todo = __ballot_sync(0xffffffffu, gl != kEmptySlot && a.slot_started[jl]);
    while (todo) {
      const int l = __ffs(todo) - 1;
      todo &= todo - 1;
      const u64 i = base + l;
      const u32 g = __shfl_sync(0xffffffffu, gl, l);
      u64 end = a.nslots;
      for (u64 b = i + 1; b < a.nslots; b += 32) {
        const u64 j = b + lane;
        bool stop = j >= a.nslots;
        if (!stop) {
          const u32 gj = a.slot_gid[j];
          stop = gj != kEmptySlot && (gj != g || a.slot_started[j]);
        }
        const u32 sm = __ballot_sync(0xffffffffu, stop);
        if (sm) {
          end = b + __ffs(sm) - 1;
          break;
        }
      }
      for (int c = 0; c < a.nvals; ++c) {
        switch (a.v[c].kind) {
          case VK_F: fixup_column<VK_F>(a, c, i, end, g, lane); break;
          case VK_I: fixup_column<VK_I>(a, c, i, end, g, lane); break;
          default: fixup_column<VK_U>(a, c, i, end, g, lane); break;
        }
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
