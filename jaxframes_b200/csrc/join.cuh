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
// Window of B that the A tile of each count CTA can reach: [lower_bound of
// its first key, upper_bound of its last key).  One thread per tile, all
// searches in parallel (a CTA would otherwise start with a serial search).
template <typename K>
__global__ void k_join_windows(const K* A, u64 na, const K* B, u64 nb, u64 tiles, u64* win) {
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += (u64)gridDim.x * blockDim.x) {
    const u64 a0 = t * kJoinTile, a1 = min(na, a0 + kJoinTile);
    const u64 lo = lower_bound_g<K>(B, 0, nb, A[a0]);
    win[2 * t] = lo;
    win[2 * t + 1] = upper_bound_g<K>(B, lo, nb, A[a1 - 1]);
  }
}

template <typename K>
__global__ void __launch_bounds__(kJoinThreads) k_join_count(const K* A, u64 na, const K* B, u64 nb,
                                                            const u64* windows, u32* lo_out, u32* cnt_out,
                                                            PackDesc pd) {
  constexpr int CAP = (32 * 1024) / sizeof(K);
  __shared__ K win[CAP];
  const u64 a0 = (u64)blockIdx.x * kJoinTile;
  const u64 a1 = min(na, a0 + kJoinTile);
  const u64 wlo = windows[2 * blockIdx.x], whi = windows[2 * blockIdx.x + 1], wn = whi - wlo;
  const bool in_smem = wn <= (u64)CAP;
  if (in_smem)
    for (u64 i = threadIdx.x; i < wn; i += kJoinThreads) win[i] = B[wlo + i];
  __syncthreads();
  K xs[kJoinIPT];
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 i = a0 + (u64)k * kJoinThreads + threadIdx.x;
    xs[k] = i < a1 ? A[i] : (K)0;
  }
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 i = a0 + (u64)k * kJoinThreads + threadIdx.x;
    if (i >= a1) break;
    const K x = xs[k];
    u64 l, h;
    if (in_smem) {
      l = lower_bound_g<K>(win, 0, wn, x);
      h = upper_bound_g<K>(win, l, wn, x);
    } else {
      l = lower_bound_g<K>(B + wlo, 0, wn, x);
      h = upper_bound_g<K>(B + wlo, l, wn, x);
    }
    u32 c = (u32)(h - l);
    if (pd.nan_cols && packed_has_nan<K>(pd, x)) c = 0;
    lo_out[i] = (u32)(wlo + l);
    cnt_out[i] = c;
  }
}

// Merged key columns written by the expand kernels (A side's key values).
struct JoinKeyOut {
  int ncols;
  void* out[kMaxCols];  // per column output, or null
  ColDesc c[kMaxCols];  // A side's columns with the shared packing
};

template <typename K>
__device__ __forceinline__ void write_join_key(const JoinKeyOut& ko, u64 o, K packed, u32 row) {
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
// one past the row of its last output).
__global__ void k_expand_windows(const u64* off, u64 na, u64 m, u64 tile0, u64 tiles, u64* win) {
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += (u64)gridDim.x * blockDim.x) {
    const u64 o0 = (tile0 + t) * kJoinTile, o1 = min(m, o0 + kJoinTile);
    const u64 i0 = upper_bound_g<u64>(off, 0, na, o0) - 1;
    win[2 * t] = i0;
    win[2 * t + 1] = upper_bound_g<u64>(off, i0, na, o1 - 1);
  }
}

template <typename K>
__global__ void __launch_bounds__(kJoinThreads) k_join_expand_inner(const u64* off, u64 na, u64 m,
                                                                   const u64* windows, const u32* lo,
                                                                   const u32* pA, const u32* pB, const K* skA,
                                                                   int32_t* a_out, int32_t* b_out,
                                                                   JoinKeyOut ko, u64 tile0) {
  constexpr int CAP = 4096;
  __shared__ u64 win[CAP];
  const u64 o0 = (tile0 + blockIdx.x) * kJoinTile;
  const u64 o1 = min(m, o0 + kJoinTile);
  const u64 i0 = windows[2 * blockIdx.x], i1 = windows[2 * blockIdx.x + 1], wn = i1 - i0;
  const bool in_smem = wn <= (u64)CAP;
  if (in_smem)
    for (u64 i = threadIdx.x; i < wn; i += kJoinThreads) win[i] = off[i0 + i];
  __syncthreads();
  // three rounds so each round's loads are all in flight together
  u64 ii[kJoinIPT], jj[kJoinIPT];
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 o = o0 + (u64)k * kJoinThreads + threadIdx.x;
    ii[k] = 0;
    jj[k] = 0;
    if (o >= o1) continue;
    u64 r;
    if (in_smem) r = upper_bound_g<u64>(win, 0, wn, o) - 1;
    else r = upper_bound_g<u64>(off + i0, 0, wn, o) - 1;
    ii[k] = i0 + r;
    jj[k] = o - (in_smem ? win[r] : off[i0 + r]);  // offset inside the row's run
  }
  u32 ra[kJoinIPT], lo_k[kJoinIPT];
  K kk[kJoinIPT];
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 o = o0 + (u64)k * kJoinThreads + threadIdx.x;
    if (o >= o1) continue;
    ra[k] = pA[ii[k]];
    lo_k[k] = lo[ii[k]];
    kk[k] = skA[ii[k]];
  }
  u32 rb[kJoinIPT];
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 o = o0 + (u64)k * kJoinThreads + threadIdx.x;
    if (o >= o1) continue;
    rb[k] = pB[(u64)lo_k[k] + jj[k]];
  }
#pragma unroll
  for (int k = 0; k < kJoinIPT; ++k) {
    const u64 o = o0 + (u64)k * kJoinThreads + threadIdx.x;
    if (o >= o1) continue;
    a_out[o] = (int32_t)ra[k];
    b_out[o] = (int32_t)rb[k];
    write_join_key<K>(ko, o, kk[k], ra[k]);
  }
}

// left / right join: one output per sorted A row, first match in B or -1.
template <typename K>
__global__ void __launch_bounds__(256) k_join_expand_first(u64 na, const u32* lo, const u32* cnt,
                                                          const u32* pA, const u32* pB, const K* skA,
                                                          int32_t* a_out, int32_t* b_out, JoinKeyOut ko) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (u64)gridDim.x * blockDim.x) {
    const u32 ra = pA[i];
    a_out[i] = (int32_t)ra;
    b_out[i] = cnt[i] ? (int32_t)pB[lo[i]] : -1;
    write_join_key<K>(ko, i, skA[i], ra);
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
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const int32_t r = idx[i];
    if (r < 0 || (u64)r >= n_src) {
      if (odt == JFX_F32) ((float*)out)[i] = __int_as_float(0x7fc00000);
      else if (odt == JFX_F64) ((double*)out)[i] = __longlong_as_double(0x7ff8000000000000ll);
      else store_raw(out, odt, i, ~0ull);
      continue;
    }
    if (odt == sdt) {
      store_raw(out, odt, i, load_raw(src, sdt, r));
      continue;
    }
    // conversion (integer/bool payload promoted to a float)
    double x;
    switch (sdt) {
      case JFX_F32: x = ((const float*)src)[r]; break;
      case JFX_F64: x = ((const double*)src)[r]; break;
      case JFX_I8: x = ((const signed char*)src)[r]; break;
      case JFX_I16: x = ((const short*)src)[r]; break;
      case JFX_I32: x = ((const int*)src)[r]; break;
      case JFX_I64: x = (double)((const long long*)src)[r]; break;
      case JFX_U8: case JFX_BOOL: x = ((const unsigned char*)src)[r]; break;
      case JFX_U16: x = ((const unsigned short*)src)[r]; break;
      case JFX_U32: x = ((const unsigned*)src)[r]; break;
      default: x = (double)((const unsigned long long*)src)[r]; break;
    }
    if (odt == JFX_F32) {
      // round the integer straight to float32 (double rounding can differ)
      float f;
      switch (sdt) {
        case JFX_I64: f = (float)((const long long*)src)[r]; break;
        case JFX_U64: f = (float)((const unsigned long long*)src)[r]; break;
        case JFX_I32: f = (float)((const int*)src)[r]; break;
        case JFX_U32: f = (float)((const unsigned*)src)[r]; break;
        default: f = (float)x; break;
      }
      ((float*)out)[i] = f;
    } else if (odt == JFX_F64) {
      ((double*)out)[i] = x;
    } else {
      store_raw(out, odt, i, (u64)(long long)x);
    }
  }
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
