// batch.cuh -- many independent queries in ONE persistent kernel: per query,
// the one-device body of collective_hash_repartition with P partitions
// (parallel_algorithms.py:163-182, :213-214) followed by
// SortBasedGroupBy.groupby_aggregate sum and count (:733-803).
//
// k_batch_queue is launched once with as many CTAs as the GPU holds at a
// time.  Its work queue is the list of queries, largest first (ordered on
// the device by CTA 0 before the others start); a CTA takes the next query
// with an atomic ticket and runs the query's whole pipeline itself:
//   0. one read of the query's keys: the partition histogram, the histogram
//      of every key byte the passes will use, the largest key and the key
//      range check (the histograms of a permutation are the same, so no
//      later pass counts again);
//   1. partition: a stable scatter of (key, value) by fmix32(key) % P in
//      chunks of kQueueChunk rows (each chunk ranked per warp, chunks in row
//      order) into the caller's partitioned outputs;
//   2. sort by key: stable LSD passes of 8 bits over the query's key width
//      (the bit length of its largest key), chunked the same way, between two
//      scratch buffers;
//   3. groupby: boundary flags over the sorted keys, group ids by a block
//      scan, per-chunk float64 sums and counts in shared memory (a thread
//      sums its runs in registers first), flushed to a per-query staging
//      area (a group that crosses chunks is completed by the next chunk: one
//      CTA walks the query in order).
// When every query is done (a counter the CTAs wait on, bounded), CTA 0
// scans the queries' group counts into the packed group offsets and all CTAs
// copy the staged groups into the packed outputs.  Nothing synchronises with
// the host, so the single launch can be captured in a CUDA graph.
#pragma once

#include "groupby.cuh"

namespace jfx {

constexpr int kQueueThreads = 256, kQueueIPT = 16;
constexpr u32 kQueueChunk = kQueueThreads * kQueueIPT;  // rows per chunk
constexpr u32 kQueueSortMax = kQueueChunk;             // queries ordered by size on the device (more: index order)

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

struct QueueShared {
  u32 whist[8 * 256];
  u32 wmask[8 * 256];
  u32 hist[5 * 256];  // partition, then key bytes 0..3; scanned in place into running bases
  u32 tot[256];
  u32 scan[32];
  u32 flag[2];
  u32 maxkey;
  u32 q;
  double lsum[kQueueChunk + 1];  // per-chunk group partials
  u32 lcnt[kQueueChunk + 1];
};

// Row counts of the query's rows [q0, q1) per partition (S.hist row 0) and
// per key byte b < nbytes (row b + 1), the largest key in S.maxkey; a key
// above lim raises DERR_BOUNDS.  A warp whose valid items share one digit
// adds them with one atomic.
__device__ void queue_hist(QueueShared& S, const u32* ks, u64 q0, u64 q1, u32 P, int nbytes, u32 lim, u32* err) {
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
      for (int b = 0; b <= nbytes; ++b) {
        const u32 d = b == 0 ? fmix32_d(k[i]) % P : (k[i] >> (8 * (b - 1))) & 255u;
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

// One stable pass of rows [q0, q1) by an 8-bit digit (dig(key)) whose row
// counts are base[0..255]: an exclusive scan of them in place, then chunks
// in row order.  Writes (key, value) to (dk, dv) at q0 + the row's stable
// position; base ends as each digit's end.
template <typename Dig>
__device__ void queue_pass(QueueShared& S, u32* base, const u32* ks, const u32* vs, u32* dk, u32* dv, u64 q0, u64 q1,
                           Dig dig) {
  constexpr int IPT = kQueueIPT, RADIX = 256, WARPS = kQueueThreads / 32, SEG = 32 * IPT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  block_exclusive_scan<kQueueThreads, RADIX>(base, S.scan);
  u32* wh = S.whist + warp * RADIX;
  for (u64 c0 = q0; c0 < q1; c0 += kQueueChunk) {
    for (int i = lane; i < RADIX; i += 32) wh[i] = 0u;
    __syncwarp();
    const u64 w0 = c0 + (u64)warp * SEG;
    u32 k[IPT], v[IPT], rd[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u64 j = w0 + i * 32 + lane;
      const bool in = j < q1;
      k[i] = in ? ks[j] : 0u;
      v[i] = in ? vs[j] : 0u;
      rd[i] = in ? dig(k[i]) : (u32)RADIX;
    }
    warp_rank_or<IPT, RADIX>(rd, wh, S.wmask + warp * RADIX, lane);
    __syncthreads();
    {
      u32 run = 0;
#pragma unroll
      for (int w = 0; w < WARPS; ++w) {
        const u32 c = S.whist[w * RADIX + tid];
        S.whist[w * RADIX + tid] = run;
        run += c;
      }
      S.tot[tid] = run;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      if (rd[i] != kNoRank) {
        const u32 d = rd[i] >> 16;
        const u64 dst = q0 + base[d] + wh[d] + (rd[i] & 0xffffu);
        dk[dst] = k[i];
        dv[dst] = v[i];
      }
    }
    __syncthreads();
    base[tid] += S.tot[tid];
    __syncthreads();
  }
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
    if (tid == 0) atomicExch(&a.ctl[2], 1u);
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
    const int nbytes = a.key_bits <= 0 ? 0 : min(4, (a.key_bits + 7) >> 3);
    const u32 lim = a.key_bits >= 32 ? 0xffffffffu : a.key_bits <= 0 ? 0u : (1u << a.key_bits) - 1u;
    queue_hist(S, keys, q0, q1, P, nbytes, lim, a.err);
    // 1a. stable partition by fmix32(key) % P
    queue_pass(S, S.hist, keys, vals, (u32*)a.part_keys, (u32*)a.part_values, q0, q1,
               [P](u32 kk) { return fmix32_d(kk) % P; });
    // hist row 0 now holds each partition's end; a partition starts where
    // the previous one ends
    if (tid < (int)P) a.part_offsets[(u64)q * (P + 1) + tid] = (int64_t)(q0 + (tid ? S.hist[tid - 1] : 0u));
    if (tid == 0) a.part_offsets[(u64)q * (P + 1) + P] = (int64_t)q1;
    __syncthreads();
    // 1b. stable LSD passes over the query's key bits (bytes whose counts
    // were taken: keys above the declared width are an error, already raised)
    const int kbits = min(bit_length(S.maxkey), 8 * nbytes);
    const u32* ks = (const u32*)a.part_keys;
    const u32* vs = (const u32*)a.part_values;
    int pp = 0;
    for (int sh = 0; sh < kbits; sh += 8, pp ^= 1) {
      queue_pass(S, S.hist + 256 * (1 + sh / 8), ks, vs, a.sk[pp], a.sv[pp], q0, q1,
                 [sh](u32 kk) { return (kk >> sh) & 255u; });
      ks = a.sk[pp];
      vs = a.sv[pp];
    }
    // 1c. groups
    const u32 G = queue_groups(S, ks, vs, q0, q1, a);
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
