// join.cuh -- sort-merge join over the two sorted packed key runs.
//
// Replaces ParallelSortMergeJoin.join (parallel_algorithms.py:938-1075).  The
// reference finds inner matches with an nL x nR broadcast matrix
// (:989-994); here both sides are radix sorted with one shared key packing,
// a count pass finds, for every sorted left row, its equal-key run in the
// sorted right side (binary search inside a shared-memory window of the right
// run that the CTA's left tile can reach), an exclusive scan turns counts into
// output offsets, and an expand pass writes the pairs with a load-balanced
// search of the offsets.  Pair order is the matrix's row-major order:
// (key, left row, right row).  left/right joins keep the first match
// (searchsorted, :1013-1034).
#pragma once

#include "groupby.cuh"

namespace jfx {

constexpr int kJoinThreads = 256, kJoinIPT = 8, kJoinTile = kJoinThreads * kJoinIPT;

template <typename K>
__device__ __forceinline__ u64 lower_bound_g(const K* a, u64 lo, u64 hi, K x) {
  while (lo < hi) {
    u64 mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
template <typename K>
__device__ __forceinline__ u64 upper_bound_g(const K* a, u64 lo, u64 hi, K x) {
  while (lo < hi) {
    u64 mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// For each sorted A row: lo = first B position with key >= A[i], cnt = number
// of B keys equal to A[i] (0 for a NaN key, which equals nothing).
// Warp-cooperative search: the first i in [lo, hi) with !(a[i] < x) (UPPER:
// !(a[i] <= x)), or hi.  Each round the 32 lanes probe 32 evenly spaced
// positions and the ballot narrows the range 32-fold, so a search over n
// keys costs about log32(n) dependent loads instead of log2(n).
template <typename K, bool UPPER>
__device__ __forceinline__ u64 warp_bound(const K* a, u64 lo, u64 hi, K x, int lane) {
  while (hi - lo > 32) {
    const u64 step = (hi - lo + 31) / 32;
    const u64 idx = lo + (u64)(lane + 1) * step - 1;
    bool p = false;
    if (idx < hi) {
      const K v = a[idx];
      p = UPPER ? !(x < v) : (v < x);
    }
    const u32 c = __popc(__ballot_sync(0xffffffffu, p));  // probes 0..c-1 hold
    const u64 nlo = lo + (u64)c * step;
    hi = min(hi, nlo + step - 1);  // probe c (if any) fails
    if (c == 32) hi = min(hi, lo + 32 * step);
    lo = nlo;
    if (lo > hi) lo = hi;
  }
  bool p = false;
  if (lo + lane < hi) {
    const K v = a[lo + lane];
    p = UPPER ? !(x < v) : (v < x);
  }
  return lo + __popc(__ballot_sync(0xffffffffu, p));
}

// Window of B that the A tile of each count CTA can reach: [lower_bound of
// its first key, upper_bound of its last key).  One warp per tile.
template <typename K>
__global__ void k_join_windows(const K* A, u64 na, const K* B, u64 nb, u64 tiles, u64* win) {
  const int lane = threadIdx.x & 31;
  const u64 warps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 t = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tiles; t += warps) {
    const u64 a0 = t * kJoinTile, a1 = min(na, a0 + kJoinTile);
    const u64 lo = warp_bound<K, false>(B, 0, nb, A[a0], lane);
    const u64 hi = warp_bound<K, true>(B, lo, nb, A[a1 - 1], lane);
    if (lane == 0) {
      win[2 * t] = lo;
      win[2 * t + 1] = hi;
    }
  }
}

// First i in [lo, n) with a[i] >= x (n if none), for x >= every a[< lo]:
// exponential steps from lo, then a binary search inside the last step.
template <typename K>
__device__ __forceinline__ u64 gallop_lower(const K* a, u64 lo, u64 n, K x) {
  if (lo >= n || !(a[lo] < x)) return lo;
  u64 prev = lo, step = 1;  // a[prev] < x
  while (prev + step < n && a[prev + step] < x) {
    prev += step;
    step <<= 1;
  }
  return lower_bound_g<K>(a, prev + 1, min(n, prev + step), x);
}
// First i in [lo, n) with a[i] > x (n if none), given a[lo] <= x.
template <typename K>
__device__ __forceinline__ u64 gallop_upper(const K* a, u64 lo, u64 n, K x) {
  u64 prev = lo, step = 1;  // a[prev] <= x
  while (prev + step < n && a[prev + step] <= x) {
    prev += step;
    step <<= 1;
  }
  return upper_bound_g<K>(a, prev + 1, min(n, prev + step), x);
}

// Sum and maximum of the per-row match counts: warp and block reductions,
// then one atomic pair per CTA into one of kJoinStatSlots slot pairs
// (stats[2 s] += sum, stats[2 s + 1] = max), so no single word takes every
// CTA's atomics; the host combines the slots.  Every thread of the CTA calls
// it (the reduction uses full warps and a barrier).
constexpr int kJoinStatSlots = 64;
__device__ __forceinline__ void join_count_stats(unsigned long long sum, u32 mx, unsigned long long* stats) {
  __shared__ unsigned long long ssum[kJoinThreads / 32];
  __shared__ u32 smx[kJoinThreads / 32];
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    ssum[threadIdx.x >> 5] = sum;
    smx[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kJoinThreads / 32; ++w) {
      sum += ssum[w];
      mx = max(mx, smx[w]);
    }
    unsigned long long* slot = stats + 2 * (blockIdx.x % kJoinStatSlots);
    if (sum) atomicAdd(&slot[0], sum);
    if (mx) atomicMax(&slot[1], (unsigned long long)mx);
  }
}

// Count pass.  Each thread takes kJoinIPT consecutive sorted A rows (their
// keys ascend), finds the first one's position in the CTA's B window by a
// binary search and every later one by galloping forward from the previous
// position, so a row costs O(1) probes when keys are dense and O(log gap)
// otherwise.  Loads and stores are 16-byte vectors.
template <typename K>
__global__ void __launch_bounds__(kJoinThreads) k_join_count(const K* A, u64 na, const K* B, u64 nb,
                                                            const u64* windows, u32* lo_out, u32* cnt_out,
                                                            PackDesc pd, unsigned long long* stats) {
  constexpr int CAP = (32 * 1024) / sizeof(K);
  __shared__ K win[CAP];
  const u64 a0 = (u64)blockIdx.x * kJoinTile;
  const u64 a1 = min(na, a0 + kJoinTile);
  const u64 wlo = windows[2 * blockIdx.x], whi = windows[2 * blockIdx.x + 1], wn = whi - wlo;
  const bool in_smem = wn <= (u64)CAP;
  if (in_smem)
    for (u64 i = threadIdx.x; i < wn; i += kJoinThreads) win[i] = B[wlo + i];
  const u64 r0 = a0 + (u64)threadIdx.x * kJoinIPT;
  const bool full = r0 + kJoinIPT <= a1;
  K xs[kJoinIPT];
  if (full) {
    static_assert(kJoinIPT * sizeof(K) % 16 == 0, "vector loads");
#pragma unroll
    for (int v = 0; v < kJoinIPT * (int)sizeof(K) / 16; ++v)
      reinterpret_cast<uint4*>(xs)[v] = __ldg(reinterpret_cast<const uint4*>(A + r0) + v);
  } else {
#pragma unroll
    for (int k = 0; k < kJoinIPT; ++k) xs[k] = r0 + k < a1 ? A[r0 + k] : (K)0;
  }
  __syncthreads();
  const K* W = in_smem ? win : B + wlo;
  unsigned long long sum = 0;
  u32 mx = 0;
  if (r0 < a1) {
    u32 los[kJoinIPT], cnts[kJoinIPT];
    u64 j = lower_bound_g<K>(W, 0, wn, xs[0]);
    u32 c = (j < wn && W[j] == xs[0]) ? (u32)(gallop_upper<K>(W, j, wn, xs[0]) - j) : 0u;
#pragma unroll
    for (int k = 0; k < kJoinIPT; ++k) {
      if (k > 0 && xs[k] != xs[k - 1]) {
        j = gallop_lower<K>(W, j, wn, xs[k]);
        c = (j < wn && W[j] == xs[k]) ? (u32)(gallop_upper<K>(W, j, wn, xs[k]) - j) : 0u;
      }
      los[k] = (u32)(wlo + j);
      cnts[k] = (pd.nan_cols && packed_has_nan<K>(pd, xs[k])) ? 0u : c;
    }
    if (full) {
#pragma unroll
      for (int v = 0; v < kJoinIPT / 4; ++v) {
        reinterpret_cast<uint4*>(lo_out + r0)[v] = reinterpret_cast<const uint4*>(los)[v];
        reinterpret_cast<uint4*>(cnt_out + r0)[v] = reinterpret_cast<const uint4*>(cnts)[v];
      }
    } else {
#pragma unroll
      for (int k = 0; k < kJoinIPT; ++k)
        if (r0 + k < a1) {
          lo_out[r0 + k] = los[k];
          cnt_out[r0 + k] = cnts[k];
        }
    }
#pragma unroll
    for (int k = 0; k < kJoinIPT; ++k)
      if (r0 + k < a1) {
        sum += cnts[k];
        mx = max(mx, cnts[k]);
      }
  }
  if (stats) join_count_stats(sum, mx, stats);  // every thread of the CTA
}

// out[i] = src[r] converted to odt, or the join's fill when r is out of range
// (r < 0: no match): NaN for a float output, -1 (all bits set) otherwise.
// Integer payloads promoted to float32 are rounded once, straight from the
// integer.  The per-element rule of jfx_gather.
// Split in two so that a thread can issue the loads of several rows before
// any store: gather_load reads the raw bits (0 for a missing row),
// gather_store converts and writes them.
__device__ __forceinline__ u64 gather_load(const void* src, int sdt, u64 n_src, long long r) {
  return (r >= 0 && (u64)r < n_src) ? load_raw(src, sdt, (u64)r) : 0ull;
}
__device__ __forceinline__ void gather_store(u64 raw, bool valid, int sdt, void* out, int odt, u64 i) {
  if (!valid) {
    if (odt == JFX_F32) ((float*)out)[i] = __int_as_float(0x7fc00000);
    else if (odt == JFX_F64) ((double*)out)[i] = __longlong_as_double(0x7ff8000000000000ll);
    else store_raw(out, odt, i, ~0ull);
    return;
  }
  if (odt == sdt) {
    store_raw(out, odt, i, raw);
    return;
  }
  double x;
  switch (sdt) {
    case JFX_F32: x = __uint_as_float((u32)raw); break;
    case JFX_F64: x = __longlong_as_double((long long)raw); break;
    case JFX_I8: x = (signed char)raw; break;
    case JFX_I16: x = (short)raw; break;
    case JFX_I32: x = (int)raw; break;
    case JFX_I64: x = (double)(long long)raw; break;
    case JFX_U8: case JFX_BOOL: x = (unsigned char)raw; break;
    case JFX_U16: x = (unsigned short)raw; break;
    case JFX_U32: x = (unsigned)raw; break;
    default: x = (double)raw; break;
  }
  if (odt == JFX_F32) {
    float f;
    switch (sdt) {  // integers round straight to float32 (double rounding can differ)
      case JFX_I64: f = (float)(long long)raw; break;
      case JFX_U64: f = (float)raw; break;
      case JFX_I32: f = (float)(int)raw; break;
      case JFX_U32: f = (float)(unsigned)raw; break;
      default: f = (float)x; break;
    }
    ((float*)out)[i] = f;
  } else if (odt == JFX_F64) {
    ((double*)out)[i] = x;
  } else {
    store_raw(out, odt, i, (u64)(long long)x);
  }
}
__device__ __forceinline__ void gather_elem(const void* src, int sdt, u64 n_src, long long r, void* out, int odt,
                                            u64 i) {
  gather_store(gather_load(src, sdt, n_src, r), r >= 0 && (u64)r < n_src, sdt, out, odt, i);
}

// Payload columns gathered by the expand kernels as they write each output
// row (the separate gathers of ParallelSortMergeJoin.join, :1056-1073).
// A payload is either gathered by row id from its column (src), or was
// carried through its side's sort as 32-bit words (cw0, and cw1 for an
// 8-byte dtype) and is read at the row's sorted position, which the expand
// kernels reach in nearly sequential order.
constexpr int kMaxJoinPayloads = 8;
struct JoinPayloads {
  int n;
  int swap;      // the A side of the expand is the right table
  int gathered;  // some payload is gathered by row id (the kernels need the row ids)
  const void* src[kMaxJoinPayloads];
  const u32* cw0[kMaxJoinPayloads];  // carried words in sorted order, or null
  const u32* cw1[kMaxJoinPayloads];
  void* out[kMaxJoinPayloads];
  u64 n_src[kMaxJoinPayloads];
  int sdt[kMaxJoinPayloads], odt[kMaxJoinPayloads];
  int side[kMaxJoinPayloads];  // 0: the left table's column, 1: the right table's
  int kind[kMaxJoinPayloads];  // PayloadKind: the conversion, fixed per column
};

// Conversions of a payload column, chosen on the host so that the kernels'
// inner loops carry no per-element dtype dispatch.
enum PayloadKind : int {
  PK_GENERIC = 0,  // gather_store
  PK_SAME4 = 1,    // 4-byte copy (fill: -1 bits, or NaN for float32)
  PK_SAME8 = 2,    // 8-byte copy (fill: -1 bits, or NaN for float64)
  PK_I32_F32 = 3,
  PK_U32_F32 = 4,
  PK_I64_F32 = 5,
  PK_U64_F32 = 6,
};
inline int payload_kind(int sdt, int odt) {
  if (sdt == odt) return dtype_size(sdt) == 4 ? PK_SAME4 : dtype_size(sdt) == 8 ? PK_SAME8 : PK_GENERIC;
  if (odt == JFX_F32) {
    switch (sdt) {
      case JFX_I32: return PK_I32_F32;
      case JFX_U32: return PK_U32_F32;
      case JFX_I64: return PK_I64_F32;
      case JFX_U64: return PK_U64_F32;
    }
  }
  return PK_GENERIC;
}

// Writes every payload of U outputs o[u] (valid when ok[u]); ra / rb are the
// A / B row ids and pa / pb their sorted positions (-1: no row).  Per payload
// the U loads go out before the stores (the compiler cannot move loads across
// stores that may alias).
template <int U>
__device__ __forceinline__ void write_payloads(const JoinPayloads& p, const u64* o, const bool* ok,
                                               const long long* ra, const long long* rb, const long long* pa,
                                               const long long* pb) {
  for (int k = 0; k < p.n; ++k) {
    const bool right = p.side[k] != p.swap;  // the row comes from the B side
    const u32* w0 = p.cw0[k];
    const u32* w1 = p.cw1[k];
    u64 raw[U];
    bool valid[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long r = w0 ? (right ? pb[u] : pa[u]) : (right ? rb[u] : ra[u]);
      valid[u] = ok[u] && r >= 0 && (w0 || (u64)r < p.n_src[k]);
      raw[u] = 0ull;
      if (valid[u]) {
        if (w0) raw[u] = (u64)w0[r] | (w1 ? (u64)w1[r] << 32 : 0ull);
        else raw[u] = load_raw(p.src[k], p.sdt[k], (u64)r);
      }
    }
    const float fnan = __int_as_float(0x7fc00000);
    switch (p.kind[k]) {
      case PK_SAME4: {
        const u32 fill = p.odt[k] == JFX_F32 ? 0x7fc00000u : 0xffffffffu;
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) ((u32*)p.out[k])[o[u]] = valid[u] ? (u32)raw[u] : fill;
        break;
      }
      case PK_SAME8: {
        const u64 fill = p.odt[k] == JFX_F64 ? 0x7ff8000000000000ull : ~0ull;
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) ((u64*)p.out[k])[o[u]] = valid[u] ? raw[u] : fill;
        break;
      }
      case PK_I32_F32:
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) ((float*)p.out[k])[o[u]] = valid[u] ? (float)(int)raw[u] : fnan;
        break;
      case PK_U32_F32:
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) ((float*)p.out[k])[o[u]] = valid[u] ? (float)(u32)raw[u] : fnan;
        break;
      case PK_I64_F32:
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) ((float*)p.out[k])[o[u]] = valid[u] ? (float)(long long)raw[u] : fnan;
        break;
      case PK_U64_F32:
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) ((float*)p.out[k])[o[u]] = valid[u] ? (float)raw[u] : fnan;
        break;
      default:
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) gather_store(raw[u], valid[u], p.sdt[k], p.out[k], p.odt[k], o[u]);
    }
  }
}

// Merged key columns written by the expand kernels (A side's key values).
struct JoinKeyOut {
  int ncols;
  int float_key;        // some requested key column is float: written from its original row
  // one requested 4- or 8-byte integer key column: out = ((packed >> shift) &
  // mask) + tmin, sign bit flipped back (untransform_int), stored as fast_size bytes
  int fast_size;
  u64 fast_flip;
  void* out[kMaxCols];  // per column output, or null
  ColDesc c[kMaxCols];  // A side's columns with the shared packing
};

template <typename K>
__device__ __forceinline__ void write_join_key(const JoinKeyOut& ko, u64 o, K packed, u32 row) {
  if (ko.fast_size) {
    const ColDesc& c = ko.c[0];
    const u64 field = (((u64)packed >> c.shift) & (c.bits >= 64 ? ~0ull : ((1ull << c.bits) - 1ull))) + c.tmin;
    if (ko.fast_size == 8) ((u64*)ko.out[0])[o] = field ^ ko.fast_flip;
    else ((u32*)ko.out[0])[o] = (u32)field ^ (u32)ko.fast_flip;
    return;
  }
  for (int j = 0; j < ko.ncols; ++j) {
    if (!ko.out[j]) continue;
    const ColDesc& c = ko.c[j];
    if (dtype_is_float(c.dtype)) {
      store_raw(ko.out[j], c.dtype, o, load_raw(c.ptr, c.dtype, row));
    } else {
      const u64 field = c.bits ? (((u64)packed >> c.shift) & (c.bits >= 64 ? ~0ull : ((1ull << c.bits) - 1ull))) : 0ull;
      store_raw(ko.out[j], c.dtype, o, untransform_int(c.dtype, c.flags, field + c.tmin));
    }
  }
}

// Inner join: output o belongs to the sorted A row i with off[i] <= o < off[i+1].
// Rows of A used by each expand CTA's output tile: [row of its first output,
// one past the row of its last output).  One warp per tile.
__global__ void k_expand_windows(const u64* off, u64 na, u64 m, u64 tile0, u64 tiles, u64* win) {
  const int lane = threadIdx.x & 31;
  const u64 warps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 t = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tiles; t += warps) {
    const u64 o0 = (tile0 + t) * kJoinTile, o1 = min(m, o0 + kJoinTile);
    const u64 i0 = warp_bound<u64, true>(off, 0, na, o0, lane) - 1;
    const u64 i1 = warp_bound<u64, true>(off, i0, na, o1 - 1, lane);
    if (lane == 0) {
      win[2 * t] = i0;
      win[2 * t + 1] = i1;
    }
  }
}

// Each thread writes kJoinIPT consecutive outputs: one binary search finds
// the A row of the first, later ones gallop forward from it.
template <typename K>
__global__ void __launch_bounds__(kJoinThreads) k_join_expand_inner(const u64* off, u64 na, u64 m,
                                                                   const u64* windows, const u32* lo,
                                                                   const u32* pA, const u32* pB, const K* skA,
                                                                   int32_t* a_out, int32_t* b_out,
                                                                   JoinKeyOut ko, JoinPayloads pay, u64 tile0) {
  constexpr int CAP = 4096;
  __shared__ u64 win[CAP];
  const u64 o0 = (tile0 + blockIdx.x) * kJoinTile;
  const u64 o1 = min(m, o0 + kJoinTile);
  const u64 i0 = windows[2 * blockIdx.x], i1 = windows[2 * blockIdx.x + 1], wn = i1 - i0;
  const bool in_smem = wn <= (u64)CAP;
  if (in_smem)
    for (u64 i = threadIdx.x; i < wn; i += kJoinThreads) win[i] = off[i0 + i];
  __syncthreads();
  const u64 ob = o0 + (u64)threadIdx.x * kJoinIPT;
  if (ob >= o1) return;
  const u64* OW = in_smem ? win : off + i0;
  // rows: the owner of output o is the last r with OW[r] <= o (empty rows
  // share their successor's offset and are skipped by that rule)
  u64 ii[kJoinIPT], jj[kJoinIPT];
  u64 r = upper_bound_g<u64>(OW, 0, wn, ob) - 1;
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 o = ob + k;
    if (k > 0 && r + 1 < wn && OW[r + 1] <= o) r = gallop_upper<u64>(OW, r + 1, wn, o) - 1;
    ii[k] = i0 + r;
    jj[k] = o - OW[r];
  }
  const bool idx_out = a_out && b_out;
  const bool rows = idx_out || pay.gathered || ko.float_key;  // row ids needed
  u32 ra[kJoinIPT], lo_k[kJoinIPT];
  K kk[kJoinIPT];
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    ra[k] = 0xffffffffu;
    if (ob + k >= o1) continue;
    if (rows) ra[k] = pA[ii[k]];
    lo_k[k] = lo[ii[k]];
    kk[k] = skA[ii[k]];
  }
  int32_t rb[kJoinIPT];
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    rb[k] = -1;
    if (ob + k >= o1) continue;
    if (rows) rb[k] = (int32_t)pB[(u64)lo_k[k] + jj[k]];
  }
  const bool vec = idx_out && ob + kJoinIPT <= o1 &&
                   ((((uintptr_t)(a_out + ob)) | ((uintptr_t)(b_out + ob))) & 15) == 0;
  if (vec) {
#pragma unroll
    for (int v = 0; v < kJoinIPT / 4; ++v) {
      reinterpret_cast<uint4*>(a_out + ob)[v] = reinterpret_cast<const uint4*>(ra)[v];
      reinterpret_cast<uint4*>(b_out + ob)[v] = reinterpret_cast<const uint4*>(rb)[v];
    }
  }
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 o = ob + k;
    if (o >= o1) continue;
    if (idx_out && !vec) {
      a_out[o] = (int32_t)ra[k];
      b_out[o] = rb[k];
    }
    write_join_key<K>(ko, o, kk[k], ra[k]);
  }
  if (pay.n) {
    u64 oo[kJoinIPT];
    bool ok[kJoinIPT];
    long long la[kJoinIPT], lb[kJoinIPT], qa[kJoinIPT], qb[kJoinIPT];
#pragma unroll
    for (int k = 0; k < kJoinIPT; ++k) {
      oo[k] = ob + k;
      ok[k] = ob + k < o1;
      la[k] = ok[k] && rows ? (long long)ra[k] : -1;
      lb[k] = ok[k] && rows ? (long long)rb[k] : -1;
      qa[k] = ok[k] ? (long long)ii[k] : -1;
      qb[k] = ok[k] ? (long long)lo_k[k] + (long long)jj[k] : -1;
    }
    write_payloads<kJoinIPT>(pay, oo, ok, la, lb, qa, qb);
  }
}

// Inner join where every A row has exactly one match (m == na and no count
// above 1, as in a many-to-one join against unique keys): output i is sorted
// A row i, so no offsets or searches are needed.  U rows per thread, each
// round's loads issued together.
template <typename K>
__global__ void __launch_bounds__(256) k_join_expand_unique(u64 na, const u32* lo, const u32* pA, const u32* pB,
                                                           const K* skA, int32_t* a_out, int32_t* b_out,
                                                           JoinKeyOut ko, JoinPayloads pay) {
  constexpr int U = 4;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  const bool rows = a_out || b_out || pay.gathered || ko.float_key;  // row ids needed
  for (u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; i0 < na; i0 += stride * U) {
    u32 ra[U], l[U];
    K kk[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 i = i0 + (u64)u * stride;
      ra[u] = 0xffffffffu;
      if (i < na) {
        if (rows) ra[u] = pA[i];
        l[u] = lo[i];
        kk[u] = skA[i];
      }
    }
    u32 rb[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      rb[u] = 0xffffffffu;
      if (rows && i0 + (u64)u * stride < na) rb[u] = pB[l[u]];
    }
    u64 oo[U];
    bool ok[U];
    long long la[U], lb[U], qa[U], qb[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      oo[u] = i0 + (u64)u * stride;
      ok[u] = oo[u] < na;
      la[u] = ok[u] && rows ? (long long)ra[u] : -1;
      lb[u] = ok[u] && rows ? (long long)rb[u] : -1;
      qa[u] = ok[u] ? (long long)oo[u] : -1;
      qb[u] = ok[u] ? (long long)l[u] : -1;
    }
    if (pay.n) write_payloads<U>(pay, oo, ok, la, lb, qa, qb);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!ok[u]) break;
      const u64 i = oo[u];
      if (a_out) a_out[i] = (int32_t)ra[u];
      if (b_out) b_out[i] = (int32_t)rb[u];
      write_join_key<K>(ko, i, kk[u], ra[u]);
    }
  }
}

// k_join_expand_unique for its common form: every payload carried through
// the sorts (no row ids needed), one 4/8-byte integer key column, and a
// conversion without per-element dtype dispatch.  Loads and stores only what
// that form needs, in few registers, so more warps hide the load latency.
template <typename K>
__global__ void __launch_bounds__(256) k_join_expand_unique_carried(u64 na, const u32* lo, const K* skA,
                                                                    JoinKeyOut ko, JoinPayloads pay) {
  constexpr int U = 4;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  const ColDesc& kc = ko.c[0];
  const u64 kmask = kc.bits >= 64 ? ~0ull : ((1ull << kc.bits) - 1ull);
  for (u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; i0 < na; i0 += stride * U) {
    u32 l[U];
    K kk[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 i = i0 + (u64)u * stride;
      if (i < na) {
        l[u] = __ldg(lo + i);
        kk[u] = __ldg(skA + i);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 i = i0 + (u64)u * stride;
      if (i >= na) break;
      const u64 field = (((u64)kk[u] >> kc.shift) & kmask) + kc.tmin;
      if (ko.fast_size == 8) ((u64*)ko.out[0])[i] = field ^ ko.fast_flip;
      else ((u32*)ko.out[0])[i] = (u32)field ^ (u32)ko.fast_flip;
    }
    for (int k = 0; k < pay.n; ++k) {
      const bool right = pay.side[k] != pay.swap;
      const u32* w0 = pay.cw0[k];
      const u32* w1 = pay.cw1[k];
      u64 raw[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 i = i0 + (u64)u * stride;
        raw[u] = 0ull;
        if (i < na) {
          const u64 r = right ? (u64)l[u] : i;
          raw[u] = (u64)__ldg(w0 + r) | (w1 ? (u64)__ldg(w1 + r) << 32 : 0ull);
        }
      }
      void* out = pay.out[k];
      const int kind = pay.kind[k];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 i = i0 + (u64)u * stride;
        if (i >= na) break;
        switch (kind) {
          case PK_SAME4: ((u32*)out)[i] = (u32)raw[u]; break;
          case PK_SAME8: ((u64*)out)[i] = raw[u]; break;
          case PK_I32_F32: ((float*)out)[i] = (float)(int)raw[u]; break;
          case PK_U32_F32: ((float*)out)[i] = (float)(u32)raw[u]; break;
          case PK_I64_F32: ((float*)out)[i] = (float)(long long)raw[u]; break;
          default: ((float*)out)[i] = (float)raw[u]; break;  // PK_U64_F32
        }
      }
    }
  }
}

// left / right join: one output per sorted A row, first match in B or -1.
template <typename K>
__global__ void __launch_bounds__(256) k_join_expand_first(u64 na, const u32* lo, const u32* cnt,
                                                          const u32* pA, const u32* pB, const K* skA,
                                                          int32_t* a_out, int32_t* b_out, JoinKeyOut ko,
                                                          JoinPayloads pay) {
  const bool rows = a_out || b_out || pay.gathered || ko.float_key;  // row ids needed
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (u64)gridDim.x * blockDim.x) {
    const u32 c = cnt[i], l = lo[i];
    const u32 ra = rows ? pA[i] : 0xffffffffu;
    const int32_t rb = c ? (rows ? (int32_t)pB[l] : 0) : -1;
    if (a_out) a_out[i] = (int32_t)ra;
    if (b_out) b_out[i] = rb;
    write_join_key<K>(ko, i, skA[i], ra);
    if (pay.n) {
      const u64 oo[1] = {i};
      const bool ok[1] = {true};
      const long long la[1] = {rows ? (long long)ra : -1}, lb[1] = {rows ? (long long)rb : -1};
      const long long qa[1] = {(long long)i}, qb[1] = {c ? (long long)l : -1};
      write_payloads<1>(pay, oo, ok, la, lb, qa, qb);
    }
  }
}

// ------------------------------------------------------------------ gather ---
// out[i] = src[idx[i]] converted to out_dtype; idx < 0 -> NaN (float out) or -1.
__global__ void __launch_bounds__(256) k_gather(const void* src, int sdt, u64 n_src, const int32_t* idx, u64 n,
                                               void* out, int odt) {
  // same-dtype fast path: indices of U items, then their values, then stores
  constexpr int U = 8;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  if (odt == sdt) {
    for (u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * U) {
      int32_t r[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 i = i0 + (u64)u * stride;
        r[u] = i < n ? idx[i] : -1;
      }
      u64 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) v[u] = (r[u] >= 0 && (u64)r[u] < n_src) ? load_raw(src, sdt, (u64)r[u]) : 0ull;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 i = i0 + (u64)u * stride;
        if (i >= n) break;
        if (r[u] >= 0 && (u64)r[u] < n_src) store_raw(out, odt, i, v[u]);
        else if (odt == JFX_F32) ((float*)out)[i] = __int_as_float(0x7fc00000);
        else if (odt == JFX_F64) ((double*)out)[i] = __longlong_as_double(0x7ff8000000000000ll);
        else store_raw(out, odt, i, ~0ull);
      }
    }
    return;
  }
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    gather_elem(src, sdt, n_src, (long long)idx[i], out, odt, i);
}

// flag[pA[i]] = 1 for sorted A rows without a match (original row order).
__global__ void __launch_bounds__(256) k_mark_unmatched(const u32* cnt, const u32* pA, u64 na, u32* flag) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (u64)gridDim.x * blockDim.x)
    flag[pA[i]] = cnt[i] == 0 ? 1u : 0u;
}

// out[off[r]] = r for every flagged row r (stable compaction).
__global__ void __launch_bounds__(256) k_compact_rows(const u32* flag, const u32* off, u64 n, int32_t* out) {
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (u64)gridDim.x * blockDim.x)
    if (flag[r]) out[off[r]] = (int32_t)r;
}

// _coalesce_join_key (parallel_algorithms.py:1245-1251): left key when the
// left index is valid, else the right key.
__global__ void __launch_bounds__(256) k_coalesce(const void* a, const int32_t* ia, u64 na, const void* b,
                                                 const int32_t* ib, u64 nb, u64 n, int dt, void* out) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const int32_t x = ia[i];
    u64 v = 0;
    if (x >= 0 && (u64)x < na) v = load_raw(a, dt, x);
    else {
      const int32_t y = ib[i] < 0 ? 0 : ib[i];
      if ((u64)y < nb) v = load_raw(b, dt, y);
    }
    store_raw(out, dt, i, v);
  }
}

__global__ void __launch_bounds__(256) k_hash(PackDesc pd, u64 n, u32* out) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    out[i] = hash_row(pd, i);
}

__global__ void k_offsets_from_base(const u32* base, int p, u64 n, int64_t* out) {
  for (int i = threadIdx.x; i <= p; i += blockDim.x) out[i] = i < p ? (int64_t)base[i] : (int64_t)n;
}

}  // namespace jfx
