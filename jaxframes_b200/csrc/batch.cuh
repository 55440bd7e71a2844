// batch.cuh -- many independent queries in ONE persistent kernel: per query,
// the one-device body of collective_hash_repartition with P partitions
// (parallel_algorithms.py:163-182, :213-214) followed by
// SortBasedGroupBy.groupby_aggregate sum and count (:733-803).
//
// k_batch_queue is launched once with as many CTAs as the GPU holds at a
// time.  Its work queue is the list of queries, largest first (ordered on
// the device by CTA 0 before the others start); a CTA takes the next query
// with an atomic ticket and runs the query's whole pipeline itself:
//   0. one read of the query's keys: the partition histogram, the histograms
//      of the bucket digits (key >> 12, 8 bits at a time), the largest key
//      and the key range check (the histograms of a permutation are the
//      same, so no later pass counts again);
//   1. one read of (key, value) in chunks of kQueueChunk rows, each chunk
//      ranked per warp, staged in shared memory in digit order and written
//      out in coalesced digit runs, twice: the stable partition by
//      fmix32(key) % P into the caller's partitioned outputs, and the first
//      bucket pass into scratch (more bucket passes for keys over 20 bits);
//   2. groups: the rows are in bucket order (4096 keys per bucket), so a
//      shared-memory table of 4096 float64 sums and counts takes one bucket
//      at a time and writes its groups out in key order when the next
//      bucket starts.  A query whose buckets would hold fewer than 1024 rows
//      on average is sorted by its whole key instead (8-bit LSD passes) and
//      its groups found from the boundaries of the sorted keys.
// Group sums are accumulated in float64 and rounded once.  When every query
// is done (a counter the CTAs wait on, bounded by progress), CTA 0 scans the
// queries' group counts into the packed group offsets and all CTAs copy the
// staged groups into the packed outputs.  Nothing synchronises with the
// host, so the single launch can be captured in a CUDA graph.
#pragma once

#include "groupby.cuh"

namespace jfx {

constexpr int kQueueThreads = 256, kQueueIPT = 16;
constexpr u32 kQueueChunk = kQueueThreads * kQueueIPT;  // rows per chunk
constexpr u32 kQueueSortMax = kQueueChunk;             // queries ordered by size on the device (more: index order)
// Groups of bucketed rows: a shared-memory table of kWin keys (one bucket,
// key >> kWinBits); it shares the chunk staging space of the passes.
constexpr int kWinBits = 12;
constexpr u32 kWin = 1u << kWinBits;
static_assert(kWin == kQueueChunk, "the group table and the pass staging share space");
// Buckets are used when the query has at least this many rows per bucket on
// average (or a single bucket); sparser queries sort by the whole key.
constexpr u64 kDenseRowsPerBucket = 1024;

struct QueueArgs {
  const int32_t* keys;
  const float* values;
  const int64_t* qoff;   // [nq + 1]
  u64 n;                 // rows of the batch (qoff[nq])
  u32 nq;
  u32 P;                 // partitions, <= 256
  int key_bits;          // keys must lie in [0, 2^key_bits)
  int32_t* part_keys;    // [n]
  float* part_values;    // [n]
  int64_t* part_offsets; // [nq * (P + 1)]
  int32_t* group_keys;   // [n] packed: query q's groups at [group_offsets[q], group_offsets[q+1])
  float* group_sums;
  float* group_counts;
  int64_t* group_offsets;  // [nq + 1]
  u32* sk[2];            // [n] scratch keys (ping-pong)
  u32* sv[2];            // [n] scratch value bits
  u32* tkeys;            // [n] staging of each query's groups at its first row
  double* tsums;         // [n]
  u32* tcnts;            // [n]
  u32* qgroups;          // [nq] groups of each query
  u32* order;            // [nq] query processing order
  u32* ctl;              // [0] ticket, [1] queries done, [2] order ready, [3] offsets ready (zeroed)
  u32* err;
  u64 spin_ns;
  u32 withhold_order;    // failure injection: CTA 0 never publishes the query order
};

// Bounded wait (thread 0) until *p >= target; false after spin_ns without
// *p advancing or when another CTA already reported a timeout.  The bound is
// on progress, not on the whole wait: the queries done counter advances as
// long as some CTA still works.
__device__ __forceinline__ bool queue_wait(const u32* p, u32 target, u32* err, u64 spin_ns) {
  u32 seen = ld_relaxed(p);
  if (seen >= target) return true;
  u64 t0 = globaltimer_ns();
  for (u32 spins = 1;; ++spins) {
    const u32 now = ld_relaxed(p);
    if (now >= target) return true;
    if (now != seen) {
      seen = now;
      t0 = globaltimer_ns();
    }
    __nanosleep(256);
    if ((spins & 63u) == 0) {
      if (ld_relaxed(err) & DERR_TIMEOUT) return false;
      if (globaltimer_ns() - t0 > spin_ns) {
        atomicOr(err, DERR_TIMEOUT);
        return false;
      }
    }
  }
}

// Partition of a key: fmix32(key) % P, a mask when P is a power of two.
__device__ __forceinline__ u32 part_of(u32 key, u32 P) {
  const u32 h = fmix32_d(key);
  return (P & (P - 1u)) == 0u ? (h & (P - 1u)) : h % P;
}

struct QueueShared {
  u32 whist[8 * 256];
  u32 wmask[8 * 256];
  // row 0: partition counts; rows 1..3: counts of the bucket digits
  // (key >> (kWinBits + 8 p)) & 255; row 4: scratch of the full-key passes.
  // Scanned in place into the running bases of a pass.
  u32 hist[5 * 256];
  u32 tot[256];
  u32 cexcl[256];
  u32 scan[32];
  u32 red[16];
  u32 flag[2];
  u32 maxkey;
  u32 q;
  // groups: float64 sums and counts of a chunk (sorted rows) or of a window
  // of kWin keys (bucketed rows); passes: the chunk's keys and values staged
  // in digit order (lsum)
  double lsum[kQueueChunk + 1];
  u32 lcnt[kQueueChunk + 1];
};

// Row counts of the query's rows [q0, q1) per partition (S.hist row 0) and
// per bucket digit p < ndig (row p + 1), the largest key in S.maxkey; a key
// above lim raises DERR_BOUNDS.  Loads are coalesced (item i of thread t is
// row c0 + i * kQueueThreads + t); a warp whose valid items share one digit
// adds them with one atomic.
__device__ void queue_hist(QueueShared& S, const u32* ks, u64 q0, u64 q1, u32 P, int ndig, u32 lim, u32* err) {
  constexpr int IPT = kQueueIPT;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < 5 * 256; i += kQueueThreads) S.hist[i] = 0u;
  if (tid == 0) S.maxkey = 0u;
  __syncthreads();
  u32 mx = 0u;
  bool bad = false;
  for (u64 c0 = q0; c0 < q1; c0 += kQueueChunk) {
    u32 k[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u64 j = c0 + (u64)i * kQueueThreads + tid;
      k[i] = j < q1 ? ks[j] : 0u;
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const bool valid = c0 + (u64)i * kQueueThreads + tid < q1;
      const u32 vb = __ballot_sync(0xffffffffu, valid);
      if (vb == 0u) continue;  // warp-uniform: lane 0 is valid whenever any lane is
      bad |= valid && k[i] > lim;
      mx = valid && k[i] > mx ? k[i] : mx;
      for (int b = 0; b <= ndig; ++b) {
        const u32 d = b == 0 ? part_of(k[i], P) : (k[i] >> (kWinBits + 8 * (b - 1))) & 255u;
        const u32 d0 = __shfl_sync(0xffffffffu, d, 0);
        if (__all_sync(0xffffffffu, !valid || d == d0)) {
          if (lane == 0) atomicAdd(&S.hist[256 * b + d0], (u32)__popc(vb));
        } else if (valid) {
          atomicAdd(&S.hist[256 * b + d], 1u);
        }
      }
    }
  }
  if (bad) atomicOr(err, DERR_BOUNDS);
  atomicMax(&S.maxkey, mx);
  __syncthreads();
}

// Row counts of rows [q0, q1) of ks by dig(key) into row[0..255].
template <typename Dig>
__device__ void queue_count(QueueShared& S, u32* row, const u32* ks, u64 q0, u64 q1, Dig dig) {
  constexpr int IPT = kQueueIPT;
  const int tid = threadIdx.x;
  row[tid] = 0u;
  __syncthreads();
  for (u64 c0 = q0; c0 < q1; c0 += kQueueChunk) {
    u32 k[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u64 j = c0 + (u64)i * kQueueThreads + tid;
      k[i] = j < q1 ? ks[j] : 0u;
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i)
      if (c0 + (u64)i * kQueueThreads + tid < q1) atomicAdd(&row[dig(k[i])], 1u);
  }
  __syncthreads();
}

// One chunk of a stable pass: the chunk's items (item i of warp w, lane l:
// row c0 + w * 32 * kQueueIPT + 32 i + l) ranked per warp by dig(key), staged
// in shared memory in digit order (row order inside a digit), then written
// by consecutive threads to consecutive rows of each digit's run at
// q0 + base[d] + the digit's rows so far, so that the global writes are
// coalesced.  base[d] advances by the chunk's count of d.
template <typename Dig>
__device__ __forceinline__ void chunk_scatter(QueueShared& S, u32* base, const u32 (&k)[kQueueIPT],
                                              const u32 (&v)[kQueueIPT], u64 c0, u64 q0, u64 q1, u32* dk,
                                              u32* dv, u32* err, Dig dig) {
  constexpr int IPT = kQueueIPT, RADIX = 256, WARPS = kQueueThreads / 32, SEG = 32 * IPT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  u32* wh = S.whist + warp * RADIX;
  for (int i = lane; i < RADIX; i += 32) wh[i] = 0u;
  __syncwarp();
  const u64 w0 = c0 + (u64)warp * SEG;
  u32 rd[IPT];
#pragma unroll
  for (int i = 0; i < IPT; ++i) rd[i] = w0 + (u64)i * 32 + lane < q1 ? dig(k[i]) : (u32)RADIX;
  warp_rank_or<IPT, RADIX>(rd, wh, S.wmask + warp * RADIX, lane);
  __syncthreads();
  {
    // per digit (thread = digit): earlier warps' counts, and the chunk total
    u32 run = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
      const u32 c = S.whist[w * RADIX + tid];
      S.whist[w * RADIX + tid] = run;
      run += c;
    }
    S.tot[tid] = run;
    S.cexcl[tid] = run;
  }
  block_exclusive_scan<kQueueThreads, RADIX>(S.cexcl, S.scan);  // the chunk's digit starts
  u32* stk = reinterpret_cast<u32*>(S.lsum);
  u32* stv = stk + kQueueChunk;
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    if (rd[i] != kNoRank) {
      const u32 d = rd[i] >> 16;
      const u32 pos = S.cexcl[d] + wh[d] + (rd[i] & 0xffffu);
      stk[pos] = k[i];
      stv[pos] = v[i];
    }
  }
  __syncthreads();
  const u32 cn = (u32)min((u64)kQueueChunk, q1 - c0);
  for (u32 j = tid; j < cn; j += kQueueThreads) {
    const u32 kk = stk[j];
    const u32 d = dig(kk);  // recomputed from the staged key (cheaper than staging it)
    const u64 dst = q0 + base[d] + (j - S.cexcl[d]);
    if (dst >= q1) {  // only reachable if the counts and the pass disagree
      atomicOr(err, DERR_BOUNDS);
      continue;
    }
    dk[dst] = kk;
    dv[dst] = stv[j];
  }
  __syncthreads();
  // thread d advances digit d's base; the next chunk reads it only after its
  // ranking barrier, and a reader after the pass synchronises first
  base[tid] += S.tot[tid];
}

// A stable pass of rows [q0, q1) of (ks, vs) by dig1 into (dk1, dv1) whose
// digit counts are base1[0..255] (scanned in place; base1 ends as each
// digit's end), and, from the same read, by dig2 into (dk2, dv2) when base2
// is given.
template <typename D1, typename D2>
__device__ void queue_pass(QueueShared& S, const u32* ks, const u32* vs, u64 q0, u64 q1, u32* err, u32* base1,
                           u32* dk1, u32* dv1, D1 dig1, u32* base2, u32* dk2, u32* dv2, D2 dig2) {
  constexpr int IPT = kQueueIPT, SEG = 32 * IPT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  block_exclusive_scan<kQueueThreads, 256>(base1, S.scan);
  if (base2) block_exclusive_scan<kQueueThreads, 256>(base2, S.scan);
  for (u64 c0 = q0; c0 < q1; c0 += kQueueChunk) {
    const u64 w0 = c0 + (u64)warp * SEG;
    u32 k[IPT], v[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u64 j = w0 + (u64)i * 32 + lane;
      k[i] = j < q1 ? ks[j] : 0u;
      v[i] = j < q1 ? vs[j] : 0u;
    }
    chunk_scatter(S, base1, k, v, c0, q0, q1, dk1, dv1, err, dig1);
    if (base2) chunk_scatter(S, base2, k, v, c0, q0, q1, dk2, dv2, err, dig2);
  }
}

// Writes the groups of the window (keys win * kWin + e for every table entry
// e with a count) in key order at q0 + gbase + their rank, and clears the
// table.  Warp w owns entries [w * kWin / 8, (w + 1) * kWin / 8), lane l
// entry 32 r + l of them; ranks come from ballots and the warps' totals.
// Returns the window's number of groups.
__device__ u32 queue_flush(QueueShared& S, u32 win, u64 q0, u32 gbase, const QueueArgs& a) {
  constexpr int WARPS = kQueueThreads / 32, ROWS = kWin / kQueueThreads;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 e0 = (u32)warp * (kWin / WARPS);
  u32 wt = 0;
#pragma unroll
  for (int r = 0; r < ROWS; ++r) wt += __popc(__ballot_sync(0xffffffffu, S.lcnt[e0 + r * 32 + lane] != 0u));
  if (lane == 0) S.red[WARPS + warp] = wt;
  __syncthreads();
  u32 run = gbase, tot = 0;
#pragma unroll
  for (int w = 0; w < WARPS; ++w) {
    const u32 t = S.red[WARPS + w];
    run += w < warp ? t : 0u;
    tot += t;
  }
  const u32 lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    const u32 e = e0 + (u32)r * 32 + lane;
    const u32 c = S.lcnt[e];
    const u32 b = __ballot_sync(0xffffffffu, c != 0u);
    if (c) {
      const u64 g = q0 + run + (u32)__popc(b & lt);
      a.tkeys[g] = (win << kWinBits) | e;
      a.tsums[g] = S.lsum[e];
      a.tcnts[g] = c;
      S.lsum[e] = 0.0;
      S.lcnt[e] = 0u;
    }
    run += (u32)__popc(b);
  }
  __syncthreads();
  return tot;
}

// Groups of rows [q0, q1) of (ks, vs) sorted by key >> kWinBits (bucket
// order, any order inside a bucket): a table of kWin float64 sums and counts
// in shared memory takes one window (bucket) at a time; a chunk's items of
// the current window are added, then, while items of later buckets remain,
// the window is written out in key order and moves to the smallest bucket
// left.  Sums are accumulated in float64.  Returns the number of groups.
__device__ u32 queue_dense_groups(QueueShared& S, const u32* ks, const u32* vs, u64 q0, u64 q1,
                                  const QueueArgs& a) {
  constexpr int IPT = kQueueIPT, WARPS = kQueueThreads / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (u32 j = tid; j < kWin; j += kQueueThreads) {
    S.lsum[j] = 0.0;
    S.lcnt[j] = 0u;
  }
  u32 win = q1 > q0 ? ks[q0] >> kWinBits : 0u;
  u32 gbase = 0;
  __syncthreads();
  for (u64 c0 = q0; c0 < q1; c0 += kQueueChunk) {
    u32 k[IPT], v[IPT], left = 0u;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u64 j = c0 + (u64)i * kQueueThreads + tid;
      const bool in = j < q1;
      k[i] = in ? ks[j] : 0u;
      v[i] = in ? vs[j] : 0u;
      left |= (u32)in << i;
    }
    while (true) {
      u32 nxt = 0xffffffffu;
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        if ((left >> i) & 1u) {
          const u32 b = k[i] >> kWinBits;
          if (b == win) {
            const u32 e = k[i] & (kWin - 1u);
            atomicAdd(&S.lsum[e], (double)__uint_as_float(v[i]));
            atomicAdd(&S.lcnt[e], 1u);
            left &= ~(1u << i);
          } else {
            nxt = min(nxt, b);
          }
        }
      }
      nxt = __reduce_min_sync(0xffffffffu, nxt);
      if (lane == 0) S.red[warp] = nxt;
      __syncthreads();
      u32 m = S.red[0];
#pragma unroll
      for (int w = 1; w < WARPS; ++w) m = min(m, S.red[w]);
      __syncthreads();
      if (m == 0xffffffffu) break;  // the chunk is used up; the window stays open
      gbase += queue_flush(S, win, q0, gbase, a);
      win = m;
    }
  }
  gbase += queue_flush(S, win, q0, gbase, a);
  return gbase;
}

// Groups of the sorted rows [q0, q1) of (ks, vs): keys and float64 sums and
// counts staged at q0 + group id.  Returns the number of groups (thread 0).
__device__ u32 queue_groups(QueueShared& S, const u32* ks, const u32* vs, u64 q0, u64 q1, const QueueArgs& a) {
  constexpr int IPT = kQueueIPT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  u32 gbase = 0;  // groups started before the chunk
  for (u64 c0 = q0; c0 < q1; c0 += kQueueChunk) {
    const u64 c1 = min(q1, c0 + kQueueChunk);
    // thread t owns the chunk's rows c0 + t * IPT .. + IPT (consecutive)
    const u64 r0 = c0 + (u64)tid * IPT;
    // every key and value of the thread's rows is loaded before the first
    // shared-memory atomic below (a load after one would wait for it)
    u32 k[IPT], vb[IPT], fl = 0;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      k[i] = r0 + i < c1 ? ks[r0 + i] : 0u;
      vb[i] = r0 + i < c1 ? vs[r0 + i] : 0u;
    }
    const u32 kprev = (r0 < c1 && r0 > q0) ? ks[r0 - 1] : ~0u;
    const bool cont = !(c0 == q0) && ks[c0] == ks[c0 - 1];  // chunk opens inside a group
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 p = i ? k[i - 1] : kprev;
      if (r0 + i < c1 && (r0 + i == q0 || k[i] != p)) fl |= 1u << i;
    }
    // inclusive count of group starts before each thread: block scan
    const u32 cnt = __popc(fl);
    u32 x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) S.scan[warp] = x;
    for (u32 j = tid; j <= kQueueChunk; j += kQueueThreads) {
      S.lsum[j] = 0.0;
      S.lcnt[j] = 0u;
    }
    __syncthreads();
    if (warp == 0) {
      const u32 w = lane < kQueueThreads / 32 ? S.scan[lane] : 0u;
      u32 z = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= o) z += y;
      }
      if (lane < kQueueThreads / 32) S.scan[lane] = z - w;
      if (lane == kQueueThreads / 32 - 1) S.flag[0] = z;  // starts in the chunk
    }
    __syncthreads();
    // local group index of row r: starts up to r - 1 (0 when the chunk's
    // first row continues the previous chunk's last group)
    u32 local = S.scan[warp] + x - cnt;  // starts before this thread's first row
    // a run of the thread's rows in one group is summed in registers and
    // added to the group's shared-memory partial once
    double run = 0.0;
    u32 rc = 0u, li = 0u;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      if (r0 + i >= c1) break;
      const float v = __uint_as_float(vb[i]);
      if ((fl >> i) & 1u) {
        if (rc) {
          atomicAdd(&S.lsum[li], run);
          atomicAdd(&S.lcnt[li], rc);
        }
        ++local;
        run = 0.0;
        rc = 0u;
        a.tkeys[q0 + gbase + local - 1] = k[i];
      }
      li = cont ? local : local - 1;  // 0: the continued group
      run += (double)v;
      ++rc;
    }
    if (rc) {
      atomicAdd(&S.lsum[li], run);
      atomicAdd(&S.lcnt[li], rc);
    }
    __syncthreads();
    const u32 starts = S.flag[0];
    const u32 nloc = starts + (cont ? 1u : 0u);
    for (u32 j = tid; j < nloc; j += kQueueThreads) {
      if (cont && j == 0) {  // completes the previous chunk's last group
        a.tsums[q0 + gbase - 1] += S.lsum[0];
        a.tcnts[q0 + gbase - 1] += S.lcnt[0];
      } else {
        const u32 g = gbase + j - (cont ? 1u : 0u);
        a.tsums[q0 + g] = S.lsum[j];
        a.tcnts[q0 + g] = S.lcnt[j];
      }
    }
    gbase += starts;
    __syncthreads();
  }
  return gbase;
}

__global__ void __launch_bounds__(kQueueThreads, 2) k_batch_queue(QueueArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  QueueShared& S = *reinterpret_cast<QueueShared*>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < 8 * 256; i += kQueueThreads) S.wmask[i] = 0u;
  // 0. CTA 0 orders the queries by size, largest first (ties by index): a
  // query's place is the number of queries that go before it
  if (blockIdx.x == 0) {
    const bool sorted = a.nq <= kQueueSortMax;
    int64_t* sizes = reinterpret_cast<int64_t*>(S.lsum);  // free until the first query
    if (sorted)
      for (u32 q = tid; q < a.nq; q += kQueueThreads) sizes[q] = a.qoff[q + 1] - a.qoff[q];
    __syncthreads();
    for (u32 q = tid; q < a.nq; q += kQueueThreads) {
      if (!sorted) {
        a.order[q] = q;
        continue;
      }
      const int64_t m = sizes[q];
      u32 rank = 0;
      for (u32 p = 0; p < a.nq; ++p) rank += (sizes[p] > m || (sizes[p] == m && p < q)) ? 1u : 0u;
      a.order[rank] = q;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0 && !a.withhold_order) atomicExch(&a.ctl[2], 1u);
  }
  if (tid == 0) S.flag[1] = queue_wait(&a.ctl[2], 1u, a.err, a.spin_ns) ? 1u : 0u;
  __syncthreads();
  if (!S.flag[1]) return;
  __threadfence();  // the order CTA 0 published is read after its flag
  // 1. the queue
  while (true) {
    if (tid == 0) S.q = atomicAdd(&a.ctl[0], 1u);
    __syncthreads();
    const u32 t = S.q;
    __syncthreads();
    if (t >= a.nq) break;
    const u32 q = ld_relaxed(a.order + t);
    const int64_t s64 = a.qoff[q], e64 = a.qoff[q + 1];
    // a decreasing or out-of-range offset is an error; the query is clamped
    const u64 q0 = min((u64)max(s64, (int64_t)0), a.n);
    const u64 q1 = e64 > s64 ? min((u64)e64, a.n) : q0;
    if ((e64 < s64 || s64 < 0 || (u64)e64 > a.n) && tid == 0) atomicOr(a.err, DERR_BOUNDS);
    const u32* keys = (const u32*)a.keys;
    const u32* vals = (const u32*)a.values;
    // 0. histograms, largest key, range check
    const u32 P = a.P;
    const int kb = a.key_bits <= 0 ? 0 : min(a.key_bits, 32);
    const int ndig = kb > kWinBits ? min(3, (kb - kWinBits + 7) >> 3) : 0;
    const u32 lim = kb >= 32 ? 0xffffffffu : kb <= 0 ? 0u : (1u << kb) - 1u;
    queue_hist(S, keys, q0, q1, P, ndig, lim, a.err);
    // keys above the declared width are an error (already raised); the
    // passes cover the declared width only
    const int kbits = min(bit_length(S.maxkey), kb);
    const bool dense = kbits <= kWinBits || q1 - q0 >= (kDenseRowsPerBucket << (kbits - kWinBits));
    u32* part_k = (u32*)a.part_keys;
    u32* part_v = (u32*)a.part_values;
    const auto pdig = [P](u32 kk) { return part_of(kk, P); };
    const u32* ks = part_k;
    const u32* vs = part_v;
    int pp = 0;
    if (dense && kbits > kWinBits) {
      // 1a. stable partition by fmix32(key) % P and, from the same read,
      // the first bucket pass; then the bucket passes above it
      queue_pass(S, keys, vals, q0, q1, a.err, S.hist, part_k, part_v, pdig, S.hist + 256, a.sk[0], a.sv[0],
                 [](u32 kk) { return (kk >> kWinBits) & 255u; });
      ks = a.sk[0];
      vs = a.sv[0];
      pp = 1;
      for (int sh = kWinBits + 8; sh < kbits; sh += 8, pp ^= 1) {
        const auto dg = [sh](u32 kk) { return (kk >> sh) & 255u; };
        queue_pass(S, ks, vs, q0, q1, a.err, S.hist + 256 * (1 + (sh - kWinBits) / 8), a.sk[pp], a.sv[pp], dg,
                   (u32*)nullptr, (u32*)nullptr, (u32*)nullptr, dg);
        ks = a.sk[pp];
        vs = a.sv[pp];
      }
    } else {
      // 1a. stable partition; 1b. for sparse keys, stable LSD passes of 8
      // bits over the whole key, each counted first
      queue_pass(S, keys, vals, q0, q1, a.err, S.hist, part_k, part_v, pdig, (u32*)nullptr, (u32*)nullptr,
                 (u32*)nullptr, pdig);
      if (!dense) {
        for (int sh = 0; sh < kbits; sh += 8, pp ^= 1) {
          const auto dg = [sh](u32 kk) { return (kk >> sh) & 255u; };
          queue_count(S, S.hist + 4 * 256, ks, q0, q1, dg);
          queue_pass(S, ks, vs, q0, q1, a.err, S.hist + 4 * 256, a.sk[pp], a.sv[pp], dg, (u32*)nullptr,
                     (u32*)nullptr, (u32*)nullptr, dg);
          ks = a.sk[pp];
          vs = a.sv[pp];
        }
      }
    }
    // hist row 0 now holds each partition's end; a partition starts where
    // the previous one ends
    __syncthreads();
    if (tid < (int)P) a.part_offsets[(u64)q * (P + 1) + tid] = (int64_t)(q0 + (tid ? S.hist[tid - 1] : 0u));
    if (tid == 0) a.part_offsets[(u64)q * (P + 1) + P] = (int64_t)q1;
    // 1c. groups: a shared-memory table per bucket, or boundaries of the
    // sorted keys
    const u32 G = dense ? queue_dense_groups(S, ks, vs, q0, q1, a) : queue_groups(S, ks, vs, q0, q1, a);
    // every thread's staged groups reach the device before the query counts
    // as done
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      a.qgroups[q] = G;
      __threadfence();
      atomicAdd(&a.ctl[1], 1u);
    }
    __syncthreads();
  }
  // 2. every query done: CTA 0 writes the packed group offsets, then every
  // CTA copies a share of the queries' staged groups
  if (tid == 0) S.flag[1] = queue_wait(&a.ctl[1], a.nq, a.err, a.spin_ns) ? 1u : 0u;
  __syncthreads();
  if (!S.flag[1]) return;
  if (blockIdx.x == 0) {
    u64 run = 0;
    for (u32 q0 = 0; q0 < a.nq; q0 += kQueueThreads) {
      const u32 q = q0 + tid;
      const u32 g = q < a.nq ? __ldcg(a.qgroups + q) : 0u;
      u32 x = g;
      const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) S.scan[warp] = x;
      __syncthreads();
      if (warp == 0) {
        const u32 w = lane < kQueueThreads / 32 ? S.scan[lane] : 0u;
        u32 z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const u32 y = __shfl_up_sync(0xffffffffu, z, o);
          if (lane >= o) z += y;
        }
        if (lane < kQueueThreads / 32) S.scan[lane] = z - w;
        if (lane == kQueueThreads / 32 - 1) S.flag[0] = z;
      }
      __syncthreads();
      if (q < a.nq) a.group_offsets[q] = (int64_t)(run + S.scan[warp] + x - g);
      run += S.flag[0];
      __syncthreads();
    }
    if (tid == 0) a.group_offsets[a.nq] = (int64_t)run;
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(&a.ctl[3], 1u);
  }
  if (tid == 0) S.flag[1] = queue_wait(&a.ctl[3], 1u, a.err, a.spin_ns) ? 1u : 0u;
  __syncthreads();
  if (!S.flag[1]) return;
  __threadfence();
  for (u32 q = blockIdx.x; q < a.nq; q += gridDim.x) {
    const u64 q0 = min((u64)max(a.qoff[q], (int64_t)0), a.n);
    const u64 o = (u64)__ldcg(a.group_offsets + q);
    const u32 G = __ldcg(a.qgroups + q);
    for (u32 g = tid; g < G; g += kQueueThreads) {
      a.group_keys[o + g] = (int32_t)__ldcg(a.tkeys + q0 + g);
      a.group_sums[o + g] = (float)__ldcg(a.tsums + q0 + g);
      a.group_counts[o + g] = (float)__ldcg(a.tcnts + q0 + g);
    }
  }
}

}  // namespace jfx
