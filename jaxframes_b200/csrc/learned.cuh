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
// 3. The predicted position's top bits name a bucket of about 2048 rows.
//    Two stable radix passes over the bucket id (not over the key's 64 bits)
//    move (key, row id) pairs into bucket order, row order inside a bucket.
// 4. The model is monotone, so every key of a bucket is <= every key of the
//    next bucket and only the order inside a bucket is left: k_bucket_sort
//    sorts each bucket of up to kBucketCap rows in shared memory by the key
//    bits that vary inside it (stable, so equal keys keep row order); a
//    bucket of more rows is listed, and the host sorts its rows with the
//    plain stable radix sort.  A failed model check makes the caller fall
//    back to the plain radix sort.  Either way the output equals the plain
//    sort's.
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

// Predicted position of every key >> shift (its bucket), in row order.
__global__ void __launch_bounds__(256) k_model_positions(const u64* keys, u64 n, const ModelRef* mp, int shift,
                                                         u32* pos) {
  const ModelRef m = *mp;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  constexpr int U = 8;  // keys in flight per thread (the leaf loads depend on them)
  for (u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * U) {
    u64 k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) k[u] = i0 + u * stride < n ? __ldg(keys + i0 + u * stride) : 0ull;
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (i0 + u * stride < n) pos[i0 + u * stride] = model_pos(m, k[u]) >> shift;
  }
}

// ------------------------------------------------------------- buckets ---
constexpr int kBucketShift = 13;  // positions in [0, 4n): 8192 positions, about 2048 rows, per bucket
constexpr int kBucketThreads = 256, kBucketIPT = 16;
constexpr u32 kBucketCap = kBucketThreads * kBucketIPT;  // rows one CTA sorts in shared memory
constexpr u32 kBucketSmallCap = kBucketThreads * 8;       // buckets the 8-item instantiation takes
constexpr u32 kBucketLargeMax = 4096;                     // large buckets listed per call
constexpr u32 kLargeCtaMax = 1u << 20;  // larger buckets: the multi-CTA radix sort, one call each
constexpr u32 kLargeChunk = 1u << 16;   // rows per CTA of the large buckets' min/max

// starts[c] = first row of bucket c in the bucket-sorted ids sb[0..n), for
// c in [0, nb]; an empty bucket starts where the next non-empty one does.
// Thread t takes rows 4t .. 4t + 3 with one 16-byte load (sb is 256-byte
// aligned), and the thread whose rows reach n also writes the buckets that
// start at n (the empty ones after the last row).
__global__ void k_bucket_starts(const u32* sb, u64 n, u32 nb, u32* starts) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; 4 * t <= n; t += stride) {
    const u64 i0 = 4 * t;
    u32 v[4];
    if (i0 + 4 <= n) {
      const uint4 q = __ldg(reinterpret_cast<const uint4*>(sb) + t);
      v[0] = q.x;
      v[1] = q.y;
      v[2] = q.z;
      v[3] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = i0 + k < n ? sb[i0 + k] : nb;
    }
    u32 prev = i0 == 0 ? 0xffffffffu : __ldg(sb + i0 - 1);  // lo = prev + 1 wraps to 0 for row 0
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const u64 i = i0 + k;
      if (i > n) break;
      const u32 lo = prev + 1u;  // buckets that start at row i
      const u32 hi = i == n ? nb : v[k];
      for (u32 c = lo; c <= hi && c <= nb; ++c) starts[c] = (u32)i;
      prev = v[k];
    }
  }
}

struct BucketArgs {
  u64* keys;           // in/out: rows in bucket order (row order inside a bucket)
  u32* ids;            // in/out: their row ids
  const u32* starts;   // [nb + 1]
  u32 nb;
  u32* large;          // [kBucketLargeMax][2] buckets of more than kBucketCap rows: (start, end),
                       // or null: such buckets are left to another launch
  u32* counts;         // [0] large buckets found
  u32 min_rows;        // buckets of at most this many rows are left to another launch
};

// Min and max key of rows [s, e), by the whole CTA (red: 2 * warps words).
__device__ __forceinline__ void block_minmax(const u64* keys, u32 s, u32 e, u64* red, u64& mn, u64& mx) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  mn = ~0ull;
  mx = 0ull;
  // eight independent loads in flight per thread, then the remainder
  constexpr int U = 8;
  u32 j = s + threadIdx.x;
  for (; j + (U - 1) * blockDim.x < e; j += U * blockDim.x) {
    u64 k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) k[u] = __ldg(keys + j + u * blockDim.x);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      mn = k[u] < mn ? k[u] : mn;
      mx = k[u] > mx ? k[u] : mx;
    }
  }
  for (; j < e; j += blockDim.x) {
    const u64 k = keys[j];
    mn = k < mn ? k : mn;
    mx = k > mx ? k : mx;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const u64 a2 = __shfl_xor_sync(0xffffffffu, mn, o), b2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mn = a2 < mn ? a2 : mn;
    mx = b2 > mx ? b2 : mx;
  }
  if (lane == 0) {
    red[warp] = mn;
    red[warps + warp] = mx;
  }
  __syncthreads();
  mn = red[0];
  mx = red[warps];
  for (int w = 1; w < warps; ++w) {
    mn = red[w] < mn ? red[w] : mn;
    mx = red[warps + w] > mx ? red[warps + w] : mx;
  }
  __syncthreads();
}

template <int IPT>
constexpr size_t bucket_smem() {
  return (size_t)kBucketThreads * IPT * (8 + 4) + (size_t)2 * 8 * 256 * 4 + 256 * 4 + 32 * 4 + 16 * 8;
}

// One bucket at a time per CTA: a stable LSD radix sort of key - min in
// shared memory over bit_length(max - min) bits, 8 bits per pass.  Warp w
// owns the bucket's rows [w * seg, (w + 1) * seg), seg = ceil(m / 8); item i
// of lane l is row w * seg + 32 i + l, so (warp, item, lane) order is row
// order and the warp ranking keeps equal digits in row order.
// IPT = 8 takes buckets of min_rows + 1 .. 2048 rows (most buckets, in fewer
// registers); IPT = 16 takes 2049 .. 4096 rows and lists the larger ones.
template <int IPT>
__global__ void __launch_bounds__(kBucketThreads, IPT <= 8 ? 3 : 2) k_bucket_sort(BucketArgs a) {
  constexpr int RADIX = 256, WARPS = kBucketThreads / 32;
  constexpr u32 CAP = (u32)kBucketThreads * IPT;
  extern __shared__ __align__(16) unsigned char smem[];
  u64* skeys = (u64*)smem;                       // [CAP]
  u32* sids = (u32*)(skeys + CAP);               // [CAP]
  u32* whist = sids + CAP;                       // [WARPS][RADIX] counters
  u32* wmask = whist + WARPS * RADIX;            // [WARPS][RADIX] peer masks
  u32* sexcl = wmask + WARPS * RADIX;            // [RADIX]
  u32* sscan = sexcl + RADIX;                    // [32]
  u64* sred = (u64*)(sscan + 32);                // [16] per-warp min / max
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < WARPS * RADIX; i += kBucketThreads) wmask[i] = 0u;
  for (u32 b = blockIdx.x; b < a.nb; b += gridDim.x) {
    const u32 s = a.starts[b], e = a.starts[b + 1], m = e - s;
    if (m <= 1 || m <= a.min_rows) continue;
    if (m > CAP) {  // listed for k_bucket_sort_large or the host
      if (a.large && tid == 0) {
        const u32 r = atomicAdd(&a.counts[0], 1u);
        if (r < kBucketLargeMax) {
          a.large[2 * r] = s;
          a.large[2 * r + 1] = e;
        }
      }
      continue;
    }
    const u32 seg = (m + WARPS - 1) / WARPS;
    const u32 w0 = min(m, warp * seg), wn = min(seg, m - w0);  // this warp's rows [w0, w0 + wn)
    u64 k[IPT];
    u32 id[IPT];
    u64 mn = ~0ull, mx = 0ull;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 r = i * 32 + lane;
      const bool in = r < wn;
      k[i] = in ? a.keys[s + w0 + r] : 0ull;
      id[i] = in ? a.ids[s + w0 + r] : 0u;
      if (in) {
        mn = k[i] < mn ? k[i] : mn;
        mx = k[i] > mx ? k[i] : mx;
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const u64 a2 = __shfl_xor_sync(0xffffffffu, mn, o), b2 = __shfl_xor_sync(0xffffffffu, mx, o);
      mn = a2 < mn ? a2 : mn;
      mx = b2 > mx ? b2 : mx;
    }
    if (lane == 0) {
      sred[warp] = mn;
      sred[WARPS + warp] = mx;
    }
    __syncthreads();
    mn = sred[0];
    mx = sred[WARPS];
#pragma unroll
    for (int w = 1; w < WARPS; ++w) {
      mn = sred[w] < mn ? sred[w] : mn;
      mx = sred[WARPS + w] > mx ? sred[WARPS + w] : mx;
    }
    const int bits = bit_length(mx - mn);
    __syncthreads();  // sred is read by all before the next bucket writes it
    if (bits == 0) continue;  // one key: the rows are in row order already
    u32* wh = whist + warp * RADIX;
    for (int sh = 0; sh < bits; sh += 8) {
      for (int i = lane; i < RADIX; i += 32) wh[i] = 0u;
      __syncwarp();
      u32 rd[IPT];
#pragma unroll
      for (int i = 0; i < IPT; ++i) rd[i] = (u32)(i * 32 + lane) < wn ? (u32)((k[i] - mn) >> sh) & 255u : (u32)RADIX;
      warp_rank_or<IPT, RADIX>(rd, wh, wmask + warp * RADIX, lane);
      __syncthreads();
      // per digit: exclusive prefix over warps, then over digits
      {
        const int d = tid;  // RADIX == threads
        u32 run = 0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
          const u32 c = whist[w * RADIX + d];
          whist[w * RADIX + d] = run;
          run += c;
        }
        sexcl[d] = run;
      }
      __syncthreads();
      block_exclusive_scan<kBucketThreads, RADIX>(sexcl, sscan);
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        if (rd[i] != kNoRank) {
          const u32 d = rd[i] >> 16;
          const u32 slot = sexcl[d] + wh[d] + (rd[i] & 0xffffu);
          skeys[slot] = k[i];
          sids[slot] = id[i];
        }
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const u32 r = i * 32 + lane;
        if (r < wn) {
          k[i] = skeys[w0 + r];
          id[i] = sids[w0 + r];
        }
      }
      __syncthreads();  // skeys / whist are rewritten by the next pass
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 r = i * 32 + lane;
      if (r < wn) {
        a.keys[s + w0 + r] = k[i];
        a.ids[s + w0 + r] = id[i];
      }
    }
  }
}

struct LargeArgs {
  u64* keys;           // in/out (the bucket's rows)
  u32* ids;
  u64* tkeys;          // scratch, same positions
  u32* tids;
  const u32* spans;    // [count][2] (start, end) of buckets holding more than one key
  const u64* mins;     // [count] their smallest key
  const u32* bits;     // [count] bit_length(max - min)
  u32 count;
};

// Min and max key of every listed large bucket: one CTA per chunk of
// kLargeChunk rows (chunks: [r, start, end] triples), atomics into mm[2r],
// mm[2r + 1] (set to ~0 / 0 beforehand).
__global__ void __launch_bounds__(256) k_large_minmax(const u64* keys, const u32* chunks, u32 nchunks, u64* mm) {
  __shared__ u64 red[16];
  for (u32 c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const u32 r = chunks[3 * c], s = chunks[3 * c + 1], e = chunks[3 * c + 2];
    u64 mn, mx;
    block_minmax(keys, s, e, red, mn, mx);
    if (threadIdx.x == 0) {
      atomicMin(&mm[2 * r], mn);
      atomicMax(&mm[2 * r + 1], mx);
    }
  }
}

__global__ void k_init_pairs(u64* mm, u32 count) {
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    mm[2 * i] = ~0ull;
    mm[2 * i + 1] = 0ull;
  }
}

// The large buckets of at most kLargeCtaMax rows that hold more than one key,
// one CTA each: a stable LSD radix sort of key - min, 8 bits per pass,
// through the scratch arrays.  Per pass a counting read gives each digit's
// first position; then chunks of kBucketCap rows in row order are ranked as
// in k_bucket_sort (warp w owns rows [512 w, 512 w + 512) of the chunk) and
// written to the digit's next positions, so equal digits keep row order
// across chunks.
__global__ void __launch_bounds__(kBucketThreads) k_bucket_sort_large(LargeArgs a) {
  constexpr int IPT = kBucketIPT, RADIX = 256, WARPS = kBucketThreads / 32, SEG = 32 * IPT;
  __shared__ u32 whist[WARPS * RADIX];
  __shared__ u32 wmask[WARPS * RADIX];
  __shared__ u32 sbase[RADIX], stot[RADIX], sscan[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < WARPS * RADIX; i += kBucketThreads) wmask[i] = 0u;
  for (u32 r = blockIdx.x; r < a.count; r += gridDim.x) {
    const u32 s = a.spans[2 * r], e = a.spans[2 * r + 1];
    const u64 mn = a.mins[r];
    const int bits = (int)a.bits[r];
    u64* ks = a.keys;
    u32* is = a.ids;
    u64* kd = a.tkeys;
    u32* id = a.tids;
    for (int sh = 0; sh < bits; sh += 8) {
      sbase[tid] = 0u;
      __syncthreads();
      for (u32 j = s + tid; j < e; j += kBucketThreads) atomicAdd(&sbase[(u32)((ks[j] - mn) >> sh) & 255u], 1u);
      __syncthreads();
      block_exclusive_scan<kBucketThreads, RADIX>(sbase, sscan);
      u32* wh = whist + warp * RADIX;
      for (u32 c0 = s; c0 < e; c0 += kBucketCap) {
        for (int i = lane; i < RADIX; i += 32) wh[i] = 0u;
        __syncwarp();
        const u32 w0 = c0 + warp * SEG;
        u64 k[IPT];
        u32 v[IPT], rd[IPT];
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
          const u32 j = w0 + i * 32 + lane;
          const bool in = j < e && j >= w0;  // j >= w0 guards the 32-bit wrap
          k[i] = in ? ks[j] : 0ull;
          v[i] = in ? is[j] : 0u;
          rd[i] = in ? (u32)((k[i] - mn) >> sh) & 255u : (u32)RADIX;
        }
        warp_rank_or<IPT, RADIX>(rd, wh, wmask + warp * RADIX, lane);
        __syncthreads();
        {
          u32 run = 0;
#pragma unroll
          for (int w = 0; w < WARPS; ++w) {
            const u32 c = whist[w * RADIX + tid];
            whist[w * RADIX + tid] = run;
            run += c;
          }
          stot[tid] = run;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
          if (rd[i] != kNoRank) {
            const u32 d = rd[i] >> 16;
            const u32 dst = s + sbase[d] + wh[d] + (rd[i] & 0xffffu);
            kd[dst] = k[i];
            id[dst] = v[i];
          }
        }
        __syncthreads();
        sbase[tid] += stot[tid];
        __syncthreads();
      }
      u64* tk = ks;
      ks = kd;
      kd = tk;
      u32* tv = is;
      is = id;
      id = tv;
    }
    if (ks != a.keys) {  // an odd number of passes left the rows in the scratch
      for (u32 j = s + tid; j < e; j += kBucketThreads) {
        a.keys[j] = ks[j];
        a.ids[j] = is[j];
      }
    }
    __syncthreads();
  }
}

}  // namespace jfx
