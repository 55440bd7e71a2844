// learned.cuh -- learned-CDF partitioned sort of uint64 keys.  No counterpart
// in the reference; its output is defined as the plain radix sort's.
//
// 1. A strided sample (1 key in 100) is sorted by the plain radix sort; the
//    sample ranks are the labels.
// 2. A two-level piecewise-linear model is fitted by least squares: a root
//    linear model on model_feature(x) picks one of 4096 leaves; each leaf is a
//    line rank ~ base + slope * (x - x0) clamped to the leaf's rank range
//    (radix.cuh: model_pos).  Slopes are forced >= 0 and leaf ranges are
//    disjoint and increasing, so the predicted position is monotone in x;
//    k_leaf_finalize verifies it.
// 3. Stable radix passes over the bits of the predicted position (not of x)
//    move (key, row id) pairs: ceil(log2(n) / 11) passes instead of
//    ceil(63 / 11).
// 4. The position is monotone, so keys with different positions are already
//    in order and only runs of equal position can hold inversions.
//    k_fix_find lists the runs that hold one; k_fix_small (a warp per run)
//    and k_fix_medium (a block radix sort per run) sort them by key -- equal
//    keys keep row order because every pass is stable.  A run longer than
//    kFixMaxRun, a full run list or a failed check make the caller fall back
//    to the plain radix sort.  Either way the output equals the plain sort's.
#pragma once

#include "radix.cuh"

namespace jfx {

constexpr int kSampleStride = 100;

__global__ void k_sample(const u64* keys, u64 stride, u64 s, u64* out) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (u64)gridDim.x * blockDim.x)
    out[i] = keys[i * stride];
}

// Root fit, pass 1: acc[0] = sum of the feature over the sorted sample.
__global__ void __launch_bounds__(256) k_root_sum(const u64* sx, u64 s, double* acc) {
  double a = 0;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (u64)gridDim.x * blockDim.x)
    a += model_feature(sx[i]);
  for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&acc[0], a);
}

// Root fit, pass 2: centred covariance of (feature, rank) and feature variance.
__global__ void __launch_bounds__(256) k_root_cov(const u64* sx, u64 s, double* acc) {
  const double mf = acc[0] / (double)s, mr = 0.5 * (double)(s - 1);
  double c = 0, v = 0;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (u64)gridDim.x * blockDim.x) {
    const double df = model_feature(sx[i]) - mf;
    c += df * ((double)i - mr);
    v += df * df;
  }
  for (int o = 16; o; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc[1], c);
    atomicAdd(&acc[2], v);
  }
}

// Root line: leaf coordinate = L/s * (mr + slope * (f - mf)).
__global__ void k_root_solve(const double* acc, u64 s, ModelRef* m, Leaf* leaves) {
  const double mf = acc[0] / (double)s, mr = 0.5 * (double)(s - 1);
  double slope = acc[2] > 0 ? acc[1] / acc[2] : 0.0;
  if (!(slope >= 0)) slope = 0;
  const double k = (double)kLeaves / (double)s;
  m->ra = slope * k;
  m->rb = (mr - slope * mf) * k;
  m->leaves = leaves;
}

// First and one-past-last sample index of every leaf (the sample is sorted
// and the leaf index is monotone, so each leaf's points are contiguous).
__global__ void k_leaf_bounds(const u64* sx, u64 s, const ModelRef* mp, u32* first, u32* last) {
  const ModelRef m = *mp;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < s; i += (u64)gridDim.x * blockDim.x) {
    const int l = model_leaf(m, sx[i]);
    if (i == 0 || model_leaf(m, sx[i - 1]) != l) first[l] = (u32)i;
    if (i + 1 == s || model_leaf(m, sx[i + 1]) != l) last[l] = (u32)(i + 1);
  }
}

// Sum of v over the block (256 threads); every thread gets the total.
__device__ __forceinline__ double block_sum256(double v, double* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // red is free (an earlier call's readers are done)
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) t += red[w];
  return t;
}

// Least-squares line rank ~ base + slope * (x - x0) per leaf, one block per
// leaf: the leaves' sample counts are very uneven on skewed keys (a leaf can
// hold a tenth of the sample when many keys are equal).
__global__ void __launch_bounds__(256) k_leaf_fit(const u64* sx, const u32* first, const u32* last, double* fit) {
  __shared__ double red[8];
  const int l = blockIdx.x;
  const u32 s0 = first[l];
  if (s0 == 0xffffffffu) return;
  const u32 e0 = last[l];
  const u64 x0 = sx[s0];
  const double cnt = (double)(e0 - s0);
  double sd = 0;
  for (u32 i = s0 + threadIdx.x; i < e0; i += 256) sd += (double)(sx[i] - x0);
  sd = block_sum256(sd, red);
  const double md = sd / cnt, mr = 0.5 * ((double)s0 + (double)(e0 - 1));
  double c = 0, v = 0;
  for (u32 i = s0 + threadIdx.x; i < e0; i += 256) {
    const double dd = (double)(sx[i] - x0) - md;
    c += dd * ((double)i - mr);
    v += dd * dd;
  }
  c = block_sum256(c, red);
  v = block_sum256(v, red);
  if (threadIdx.x == 0) {
    double slope = v > 0 ? c / v : 0.0;
    if (!(slope >= 0)) slope = 0;
    fit[2 * l] = slope;
    fit[2 * l + 1] = mr - slope * md;  // rank predicted at x0
  }
}

// Leaf table in output positions.  An empty leaf collapses onto the start of
// the next non-empty one.  ok[0] is cleared if the model is not monotone.
__global__ void __launch_bounds__(1024) k_leaf_finalize(const u64* sx, u64 s, u64 n, const u32* first,
                                                        const u32* last, const double* fit, Leaf* leaves,
                                                        u32* ok) {
  // n here is the range of predicted positions (a multiple of the row count:
  // finer positions make distinct keys collide less often)
  __shared__ u32 nf[kLeaves];
  const double scale = (double)n / (double)s;
  for (int l = threadIdx.x; l < kLeaves; l += 1024) nf[l] = first[l] == 0xffffffffu ? (u32)s : first[l];
  __syncthreads();
  for (int off = 1; off < kLeaves; off <<= 1) {  // suffix minimum
    u32 tmp[kLeaves / 1024];
#pragma unroll
    for (int k = 0; k < kLeaves / 1024; ++k) {
      const int l = threadIdx.x + k * 1024;
      tmp[k] = l + off < kLeaves ? min(nf[l], nf[l + off]) : nf[l];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kLeaves / 1024; ++k) nf[threadIdx.x + k * 1024] = tmp[k];
    __syncthreads();
  }
  for (int l = threadIdx.x; l < kLeaves; l += 1024) {
    Leaf lf;
    const bool empty = first[l] == 0xffffffffu;
    const u32 s0 = empty ? nf[l] : first[l];
    const u32 e0 = empty ? nf[l] : last[l];
    lf.lo = (u32)fmin((double)n, floor((double)s0 * scale));
    lf.hi = (u32)fmin((double)n, floor((double)e0 * scale));
    if (lf.hi < lf.lo) lf.hi = lf.lo;
    if (empty) {
      lf.x0 = 0;
      lf.slope = 0;
      lf.base = (double)lf.lo;
    } else {
      lf.x0 = sx[s0];
      lf.slope = fit[2 * l] * scale;
      lf.base = fit[2 * l + 1] * scale;
    }
    if (!(lf.slope >= 0) || !(lf.base == lf.base)) atomicExch(ok, 0u);
    leaves[l] = lf;
  }
  __syncthreads();
  for (int l = threadIdx.x; l + 1 < kLeaves; l += 1024) {
    if (leaves[l].hi > leaves[l + 1].lo || leaves[l].lo > leaves[l + 1].lo) atomicExch(ok, 0u);
  }
}

// Predicted position of every key, in row order.
__global__ void __launch_bounds__(256) k_model_positions(const u64* keys, u64 n, const ModelRef* mp, u32* pos) {
  const ModelRef m = *mp;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  constexpr int U = 4;
  for (u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * U) {
    u64 k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) k[u] = i0 + u * stride < n ? __ldg(keys + i0 + u * stride) : 0ull;
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (i0 + u * stride < n) pos[i0 + u * stride] = model_pos(m, k[u]);
  }
}

// ------------------------------------------------------------------ fix-up ---
constexpr int kFindTile = 2048, kFindThreads = 256;
constexpr int kFixMaxRun = 6144;   // longest run the shared-memory block sort takes
constexpr u32 kFixLongMax = 1u << 20;  // longest run the global-memory sort takes
constexpr int kFixSmall = 32;      // runs up to this length: one warp

struct FixLists {
  u32* small;       // [cap_small][2] (start, end)
  u32* medium;      // [cap_medium][2]
  u32* lng;         // [cap_long][2]
  u32* counts;      // [0] small, [1] medium, [2] overflow flag, [3] long
  u32* last_start;  // [tiles] last run start in the tile, or ~0
  u32* carried_inv; // [tiles] first inversion of the run carried into the tile, or ~0
  u32* scanned_to;  // [tiles] position up to which the tile's last run was scanned
  u32 cap_small, cap_medium, cap_long;
};

// counts[2] bits: why the fix-up cannot finish (the caller falls back)
enum : u32 { FIX_LONG_RUN = 1u, FIX_SMALL_FULL = 2u, FIX_MEDIUM_FULL = 4u };

__device__ __forceinline__ void fix_record(const FixLists& L, u64 s, u64 e) {
  const u64 len = e - s;
  if (len > (u64)kFixLongMax) {
    atomicOr(&L.counts[2], FIX_LONG_RUN);
    return;
  }
  if (len > (u64)kFixMaxRun) {
    const u32 r = atomicAdd(&L.counts[3], 1u);
    if (r >= L.cap_long) { atomicOr(&L.counts[2], FIX_MEDIUM_FULL); return; }
    L.lng[2 * r] = (u32)s;
    L.lng[2 * r + 1] = (u32)e;
    return;
  }
  if (len <= (u64)kFixSmall) {
    const u32 r = atomicAdd(&L.counts[0], 1u);
    if (r >= L.cap_small) { atomicOr(&L.counts[2], FIX_SMALL_FULL); return; }
    L.small[2 * r] = (u32)s;
    L.small[2 * r + 1] = (u32)e;
  } else {
    const u32 r = atomicAdd(&L.counts[1], 1u);
    if (r >= L.cap_medium) { atomicOr(&L.counts[2], FIX_MEDIUM_FULL); return; }
    L.medium[2 * r] = (u32)s;
    L.medium[2 * r + 1] = (u32)e;
  }
}

// Lists the runs of equal predicted position that start in this CTA's tile
// and contain an inversion.
// First set bit of the bitmap w in [lo, hi), or hi: a word at a time.
__device__ __forceinline__ u32 first_bit_in(const u32* w, u32 lo, u32 hi) {
  for (u32 q = lo; q < hi;) {
    const u32 bits = w[q >> 5] >> (q & 31);
    if (bits) {
      const u32 r = q + __ffs(bits) - 1;
      return r < hi ? r : hi;
    }
    q = (q | 31) + 1;
  }
  return hi;
}

__global__ void __launch_bounds__(kFindThreads) k_fix_find(u64* keys, u32* vals, const u32* spos, u64 n,
                                                           FixLists L) {
  __shared__ u64 sk[kFindTile + 1];
  __shared__ u32 sp[kFindTile + 1];
  __shared__ u32 sv[kFindTile + 1];
  __shared__ u32 fb[kFindTile / 32 + 2], ib[kFindTile / 32 + 2];
  __shared__ int s_open;
  const u64 t0 = (u64)blockIdx.x * kFindTile;
  const u64 t1 = min(n, t0 + kFindTile);
  const u64 base = t0 ? t0 - 1 : 0;
  const u32 len = (u32)(t1 - base);  // window: [base, t1)
  for (u32 i = threadIdx.x; i < len; i += kFindThreads) {
    sk[i] = keys[base + i];
    sp[i] = spos[base + i];
  }
  if (threadIdx.x == 0) s_open = -1;
  __syncthreads();
  // bit i of fb: window position i starts a run; of ib: it is an inversion
  const int lane = threadIdx.x & 31;
  for (u32 w0 = (threadIdx.x >> 5) * 32; w0 < len; w0 += kFindThreads) {
    const u32 i = w0 + lane;
    bool f = false, v = false;
    if (i < len) {
      if (base + i == 0) f = true;
      else if (i > 0) {
        f = sp[i] != sp[i - 1];
        v = !f && sk[i - 1] > sk[i];
      }
    }
    const u32 bf = __ballot_sync(0xffffffffu, f), bi = __ballot_sync(0xffffffffu, v);
    if (lane == 0) {
      fb[w0 >> 5] = bf;
      ib[w0 >> 5] = bi;
    }
  }
  __syncthreads();
  const u32 off = t0 ? 1u : 0u;
  const u32 nwords = (len + 31) >> 5;
  if (threadIdx.x == 0) {
    // tile summary: last run start, and the first inversion of the run that
    // was carried in from earlier tiles (positions before the first start)
    u32 first = len, lastp = 0xffffffffu;
    for (u32 w = 0; w < nwords; ++w) {
      u32 b = fb[w];
      if (w == 0 && off) b &= ~1u;
      if (b) {
        if (first == len) first = (w << 5) + __ffs(b) - 1;
        lastp = (w << 5) + 31 - __clz(b);
      }
    }
    const u32 cq = first_bit_in(ib, off, first);
    const u32 cinv = cq < first ? cq : 0xffffffffu;
    L.last_start[blockIdx.x] = lastp == 0xffffffffu ? lastp : (u32)(base + lastp);
    L.carried_inv[blockIdx.x] = cinv == 0xffffffffu ? cinv : (u32)(base + cinv);
  }
  for (u32 i = off + threadIdx.x; i < len; i += kFindThreads) {
    if (!((fb[i >> 5] >> (i & 31)) & 1u)) continue;
    // next run start after i inside the window
    u32 e = len;
    u32 w = i >> 5;
    u32 bits = fb[w] & ~((2u << (i & 31)) - 1u);
    if ((i & 31) == 31) bits = 0;
    while (true) {
      if (bits) {
        e = (w << 5) + __ffs(bits) - 1;
        break;
      }
      if (++w >= nwords) break;
      bits = fb[w];
    }
    if (e > len) e = len;
    if (e == len && t1 < n) {  // continues past the tile: finished by warp 0
      s_open = (int)i;
      continue;
    }
    if (first_bit_in(ib, i + 1, e) >= e) continue;  // no inversion in the run
    if (e - i > (u32)kFixSmall) {
      fix_record(L, base + i, base + e);
      continue;
    }
    // a short run inside the window: stable insertion sort here, then write back
    for (u32 q = i; q < e; ++q) sv[q] = vals[base + q];
    for (u32 q = i + 1; q < e; ++q) {
      const u64 k = sk[q];
      const u32 v = sv[q];
      u32 r = q;
      while (r > i && sk[r - 1] > k) {
        sk[r] = sk[r - 1];
        sv[r] = sv[r - 1];
        --r;
      }
      sk[r] = k;
      sv[r] = v;
    }
    for (u32 q = i; q < e; ++q) {
      keys[base + q] = sk[q];
      vals[base + q] = sv[q];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) L.scanned_to[blockIdx.x] = (u32)t1;
  if (s_open < 0 || threadIdx.x >= 32) return;
  // the last run of the tile continues past it: scan on, 32 keys at a time.
  // A run whose keys are all equal so far holds no inversion; past
  // kFixMaxRun such a run is left to k_fix_check.  A run with distinct keys
  // is scanned to its end (at most kFixLongMax).
  const u32 i = (u32)s_open;
  const u32 p0 = sp[i];
  const u64 k0 = sk[i];
  bool inv = first_bit_in(ib, i + 1, len) < len, distinct = false;
  for (u32 q = i + 1 + lane; q < len; q += 32) distinct |= sk[q] != k0;
  distinct = __any_sync(0xffffffffu, distinct);
  u64 prev_key = sk[len - 1];
  u64 pos = t1;
  u64 e = n;
  bool ended = false;
  constexpr int CH = 8;  // 32-key chunks loaded per round trip
  bool done = false;
  while (pos < n && !done) {
    u64 kc[CH];
    bool sc[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const u64 q = pos + 32 * c + lane;
      kc[c] = q < n ? keys[q] : 0;
      sc[c] = q < n && spos[q] == p0;
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      if (done || pos >= n) break;
      const u64 k = kc[c];
      const u32 bs = __ballot_sync(0xffffffffu, sc[c]);
      const u64 kp = __shfl_up_sync(0xffffffffu, k, 1);
      const u64 km = lane == 0 ? prev_key : kp;
      const u32 run_lanes = ~bs ? (u32)(__ffs(~bs) - 1) : 32u;
      const bool mine = (u32)lane < run_lanes;
      inv |= __ballot_sync(0xffffffffu, mine && km > k) != 0;
      distinct |= __ballot_sync(0xffffffffu, mine && k != k0) != 0;
      if (run_lanes < 32) {
        e = pos + run_lanes;
        ended = true;
        done = true;
        break;
      }
      prev_key = __shfl_sync(0xffffffffu, k, 31);
      pos += 32;
      const u64 scanned = pos - (base + i);
      if ((!distinct && !inv && scanned > (u64)kFixMaxRun) || scanned > (u64)kFixLongMax) {
        e = pos;
        done = true;
        break;
      }
    }
  }
  if (pos >= n) ended = true;
  if (lane == 0) {
    L.scanned_to[blockIdx.x] = (u32)(ended ? n : e);
    if (inv) fix_record(L, base + i, ended ? e : (u64)n + kFixLongMax);  // unended + inversion: too long
  }
}

// A run carried into a tile with an inversion the run's owner did not scan
// (more than kFixMaxRun past the run start) means overflow.
__global__ void k_fix_check(u64 tiles, FixLists L) {
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += (u64)gridDim.x * blockDim.x) {
    const u32 inv = L.carried_inv[t];
    if (inv == 0xffffffffu) continue;
    u32 start = 0xffffffffu;
    for (u64 k = 1; k <= t && k <= (u64)(kFixLongMax / kFindTile + 2); ++k) {
      start = L.last_start[t - k];
      if (start != 0xffffffffu) break;
    }
    // the owner of the run is the nearest earlier tile with a run start; it
    // scanned the run up to scanned_to (its inversions there are handled)
    u32 owner_scan = 0;
    for (u64 k = 1; k <= t && k <= (u64)(kFixLongMax / kFindTile + 2); ++k)
      if (L.last_start[t - k] != 0xffffffffu) {
        owner_scan = L.scanned_to[t - k];
        break;
      }
    if (start == 0xffffffffu || inv >= owner_scan) atomicOr(&L.counts[2], FIX_LONG_RUN);
  }
}

// Sorts each short run by key with one warp (rank counting).
__global__ void __launch_bounds__(256) k_fix_small(u64* keys, u32* vals, FixLists L) {
  const u32 cnt = min(L.counts[0], L.cap_small);
  const int lane = threadIdx.x & 31;
  for (u64 r = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < cnt; r += ((u64)gridDim.x * blockDim.x) >> 5) {
    const u32 s = L.small[2 * r], e = L.small[2 * r + 1];
    const u32 m = e - s;
    u64 k = 0;
    u32 v = 0;
    if ((u32)lane < m) {
      k = keys[s + lane];
      v = vals[s + lane];
    }
    u32 rank = 0;
    for (u32 q = 0; q < m; ++q) {
      const u64 kq = __shfl_sync(0xffffffffu, k, q);
      rank += (kq < k) || (kq == k && q < (u32)lane);
    }
    __syncwarp();
    if ((u32)lane < m) {
      keys[s + rank] = k;
      vals[s + rank] = v;
    }
  }
}

// Sorts each medium run with a block-wide stable LSD radix sort in shared
// memory (8-bit digits of key - min over bit_length(max - min) bits).
constexpr int kFixMedThreads = 256;
__global__ void __launch_bounds__(kFixMedThreads) k_fix_medium(u64* keys, u32* vals, FixLists L) {
  extern __shared__ __align__(16) unsigned char smem[];
  u64* ka = (u64*)smem;                  // [kFixMaxRun]
  u64* kb = ka + kFixMaxRun;             // [kFixMaxRun]
  uint16_t* ia = (uint16_t*)(kb + kFixMaxRun);  // [kFixMaxRun] local indices
  uint16_t* ib2 = ia + kFixMaxRun;
  u32* sv = (u32*)(ib2 + kFixMaxRun);    // [kFixMaxRun] values
  u32* wh = sv + kFixMaxRun;             // [8][256]
  u32* tot = wh + 8 * 256;               // [256]
  __shared__ u64 s_min, s_max;
  __shared__ u32 scan_scratch[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 cnt = min(L.counts[1], L.cap_medium);
  for (u32 r = blockIdx.x; r < cnt; r += gridDim.x) {
    const u32 s = L.medium[2 * r], e = L.medium[2 * r + 1];
    const u32 m = e - s;
    if (tid == 0) {
      s_min = ~0ull;
      s_max = 0;
    }
    __syncthreads();
    u64 lmin = ~0ull, lmax = 0;
    for (u32 j = tid; j < m; j += kFixMedThreads) {
      const u64 k = keys[s + j];
      ka[j] = k;
      ia[j] = (uint16_t)j;
      sv[j] = vals[s + j];
      lmin = k < lmin ? k : lmin;
      lmax = k > lmax ? k : lmax;
    }
    atomicMin(&s_min, lmin);
    atomicMax(&s_max, lmax);
    __syncthreads();
    const u64 mn = s_min;
    const int bits = bit_length(s_max - mn);
    const u32 seg = (m + 7) / 8;  // warp w sorts positions [w*seg, (w+1)*seg) in order
    u64 *src = ka, *dst = kb;
    uint16_t *isrc = ia, *idst = ib2;
    for (int sh = 0; sh < bits; sh += 8) {
      for (int i = tid; i < 8 * 256; i += kFixMedThreads) wh[i] = 0;
      __syncthreads();
      const u32 w0 = warp * seg, w1 = min(m, w0 + seg);
      for (u32 j = w0 + lane; j < w1; j += 32) atomicAdd(&wh[warp * 256 + (u32)(((src[j] - mn) >> sh) & 255u)], 1u);
      __syncthreads();
      for (int d = tid; d < 256; d += kFixMedThreads) {
        u32 run = 0;
        for (int w = 0; w < 8; ++w) {
          const u32 c = wh[w * 256 + d];
          wh[w * 256 + d] = run;
          run += c;
        }
        tot[d] = run;
      }
      __syncthreads();
      block_exclusive_scan<kFixMedThreads, 256>(tot, scan_scratch);
      for (int d = tid; d < 256; d += kFixMedThreads)
        for (int w = 0; w < 8; ++w) wh[w * 256 + d] += tot[d];
      __syncthreads();
      const u32 lt = lanemask_lt(), gt = lanemask_gt();
      for (u32 j0 = w0; j0 < w1; j0 += 32) {
        const u32 j = j0 + lane;
        const bool in = j < w1;
        const u32 d = in ? (u32)(((src[j] - mn) >> sh) & 255u) : 256u;
        // lanes with the same digit: one ballot per digit bit (faster than
        // match.any here); lanes past the segment end form their own group
        u32 peers = __ballot_sync(0xffffffffu, in);
        if (!in) peers = ~peers;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const u32 bit = (d >> b) & 1u;
          const u32 bb = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? bb : ~bb;
        }
        const u32 prior = in ? wh[warp * 256 + d] : 0u;
        const u32 dst_i = prior + __popc(peers & lt);
        __syncwarp();
        if (in && !(peers & gt)) wh[warp * 256 + d] = prior + __popc(peers);
        __syncwarp();
        if (in) {
          dst[dst_i] = src[j];
          idst[dst_i] = isrc[j];
        }
      }
      __syncthreads();
      u64* t = src;
      src = dst;
      dst = t;
      uint16_t* ti = isrc;
      isrc = idst;
      idst = ti;
    }
    for (u32 j = tid; j < m; j += kFixMedThreads) {
      keys[s + j] = src[j];
      vals[s + j] = sv[isrc[j]];
    }
    __syncthreads();
  }
}

// Sorts each long run (kFixMaxRun < length <= kFixLongMax) with one CTA: a
// stable LSD radix sort of 8-bit digits of key - min, ping-ponging between
// the run's place in the output and the same positions of a scratch array.
__global__ void __launch_bounds__(kFixMedThreads) k_fix_long(u64* keys, u32* vals, u64* tkeys, u32* tvals,
                                                             FixLists L) {
  __shared__ u32 hist[256];
  __shared__ u32 wh[8][256];
  __shared__ u64 s_min, s_max;
  __shared__ u32 scan_scratch[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 cnt = min(L.counts[3], L.cap_long);
  for (u32 r = blockIdx.x; r < cnt; r += gridDim.x) {
    const u32 s = L.lng[2 * r], e = L.lng[2 * r + 1];
    if (tid == 0) {
      s_min = ~0ull;
      s_max = 0;
    }
    __syncthreads();
    u64 lmin = ~0ull, lmax = 0;
    for (u32 j = s + tid; j < e; j += kFixMedThreads) {
      const u64 k = keys[j];
      lmin = k < lmin ? k : lmin;
      lmax = k > lmax ? k : lmax;
    }
    atomicMin(&s_min, lmin);
    atomicMax(&s_max, lmax);
    __syncthreads();
    const u64 mn = s_min;
    const int bits = bit_length(s_max - mn);
    u64 *ks = keys, *kd = tkeys;
    u32 *vs = vals, *vd = tvals;
    for (int sh = 0; sh < bits; sh += 8) {
      for (int i = tid; i < 256; i += kFixMedThreads) hist[i] = 0;
      __syncthreads();
      for (u32 j = s + tid; j < e; j += kFixMedThreads) atomicAdd(&hist[(u32)(((ks[j] - mn) >> sh) & 255u)], 1u);
      __syncthreads();
      block_exclusive_scan<kFixMedThreads, 256>(hist, scan_scratch);  // hist: running base per digit
      // chunks of 256 rows in order; inside a chunk, warp w takes rows
      // [w*32, w*32+32) so warps are in row order too
      const u32 lt = lanemask_lt();
      for (u32 c0 = s; c0 < e; c0 += kFixMedThreads) {
        for (int i = tid; i < 8 * 256; i += kFixMedThreads) (&wh[0][0])[i] = 0;
        __syncthreads();
        const u32 j = c0 + tid;
        const bool in = j < e;
        const u64 k = in ? ks[j] : 0;
        const u32 v = in ? vs[j] : 0;
        const u32 d = in ? (u32)(((k - mn) >> sh) & 255u) : 256u;
        u32 peers = __ballot_sync(0xffffffffu, in);
        if (!in) peers = ~peers;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const u32 bit = (d >> b) & 1u;
          const u32 bb = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? bb : ~bb;
        }
        const u32 rank = __popc(peers & lt);
        if (in && !(peers & lanemask_gt())) wh[warp][d] = __popc(peers);
        __syncthreads();
        // offset of this warp's first row of digit d: earlier warps of the chunk
        u32 before = 0;
        if (in)
          for (int w = 0; w < warp; ++w) before += wh[w][d];
        if (in) {
          const u32 dst = s + hist[d] + before + rank;
          kd[dst] = k;
          vd[dst] = v;
        }
        __syncthreads();
        if (tid < 256) {
          u32 tot = 0;
          for (int w = 0; w < 8; ++w) tot += wh[w][tid];
          hist[tid] += tot;
        }
        __syncthreads();
      }
      u64* tk = ks;
      ks = kd;
      kd = tk;
      u32* tv = vs;
      vs = vd;
      vd = tv;
    }
    if (ks != keys) {  // odd number of passes: the run ended up in the scratch
      for (u32 j = s + tid; j < e; j += kFixMedThreads) {
        keys[j] = ks[j];
        vals[j] = vs[j];
      }
    }
    __syncthreads();
  }
}

constexpr size_t kFixMediumSmem = (size_t)kFixMaxRun * (8 + 8 + 2 + 2 + 4) + (8 * 256 + 256) * 4;

}  // namespace jfx
