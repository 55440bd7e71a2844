// radix.cuh -- onesweep stable LSD radix sort for sm_100a.
//
// Replaces the reference's per-digit XLA comparison sorts
// (ParallelRadixSort._compute_local_histogram / _compute_global_offsets /
// _redistribute_data, parallel_algorithms.py:319-424, driven by lax.scan at
// :508-549) with:
//   1. one upsweep that reads the key columns once and builds the digit
//      histograms of every pass (k_hist),
//   2. an exclusive scan of each histogram (k_hist_scan),
//   3. one chained-scan kernel per pass (k_onesweep): a CTA takes the next
//      tile id from an atomic counter, ranks its keys with warp match-any
//      ballots (stable), publishes its per-digit counts, resolves its global
//      offsets by decoupled look-back over the preceding tiles (every wait is
//      bounded and reports DERR_TIMEOUT), sorts the tile by digit in shared
//      memory and writes each digit run contiguously.
// Keys are the columns packed into one unsigned word (bit-packing each
// column's (value - min) after an order-preserving transform), so a
// multi-column lexicographic sort is one radix sort over ceil(bits / 11)
// passes whenever the packed width fits 64 bits.
#pragma once

#include "common.cuh"

namespace jfx {

// No tile (tile ids stay below 2^30).
constexpr u32 kNoTile = 0xffffffffu;

// look-back status word: [31:30] flag, [29:0] count
constexpr u32 ST_AGG = 1u << 30, ST_INC = 2u << 30, ST_ERR = 3u << 30, ST_CNT = (1u << 30) - 1;

// 256 threads per tile.  Items per thread: 8 (2048-row tiles) for the
// common 8/9-bit digits with one payload word -- fewer registers, more CTAs
// per SM -- and 16 otherwise, where the digit histograms and staged words
// make a bigger tile pay.
template <int RB, int NW = 1>
struct RadixCfg {
  static constexpr int THREADS = 256;
  static constexpr int IPT = (NW == 1 && RB <= 9) ? 8 : 16;
};

constexpr int kMaxWords = 4;  // payload words a pass can carry per row

template <typename K, int RB, int NW = 1>
struct PassLayout {
  static constexpr int THREADS = RadixCfg<RB, NW>::THREADS, IPT = RadixCfg<RB, NW>::IPT;
  static constexpr int RADIX = 1 << RB, WARPS = THREADS / 32, TILE = THREADS * IPT;
  static constexpr size_t HIST_BYTES = (size_t)WARPS * RADIX * 4;
  static constexpr size_t KEY_BYTES = (size_t)TILE * sizeof(K);
  static constexpr size_t A_BYTES = HIST_BYTES > KEY_BYTES ? HIST_BYTES : KEY_BYTES;
  static constexpr size_t PAY_BYTES = (size_t)NW * TILE * 4;  // payload staged in row order
  static constexpr size_t IDX_BYTES = (size_t)TILE * 2;       // sorted slot -> staging slot
  static constexpr size_t DIG_BYTES = (size_t)TILE * 2;
  // Ranking by per-warp peer masks in shared memory (OR_RANK, digits of up to
  // 9 bits) or by one ballot per digit bit (wider digits, whose mask rows
  // would not fit).  The mask rows live only during the ranking and share
  // their bytes with the slot and digit arrays written after it.
  static constexpr bool OR_RANK = RB <= 9;
  static constexpr size_t MASK_BYTES = OR_RANK ? (size_t)WARPS * RADIX * 4 : 0;
  static constexpr size_t R_BYTES =
      MASK_BYTES > IDX_BYTES + DIG_BYTES ? MASK_BYTES : IDX_BYTES + DIG_BYTES;
  static constexpr size_t SMEM = A_BYTES + PAY_BYTES + R_BYTES + 2 * (size_t)RADIX * 4 + 64 * 4;
};

// Stable rank of each item among the warp's items of the same digit.  Item i
// of lane l is row 32 i + l of the warp's rows, so (item, lane) order is row
// order.  wh: this warp's counter row (wh[d] = the digit's items already
// counted; advanced here); wm: this warp's mask row, zero on entry and left
// zero.  Lanes of one digit set their bits in wm[d] with a shared-memory OR,
// read the peer mask back, and the highest peer advances wh[d] for the group
// and clears wm[d].  A warp whose valid items share one digit (sorted or
// constant keys, where the ORs would all hit one word) takes a shortcut.
// In place: rd[i] is the item's digit on entry (RADIX: no item) and on exit
// (digit << 16) | (counter value before the item + its rank among its
// peers), or kNoRank for no item.
constexpr u32 kNoRank = 0xffffffffu;
template <int IPT, int RADIX>
__device__ __forceinline__ void warp_rank_or(u32 (&rd)[IPT], u32* wh, u32* wm, int lane) {
  const u32 lt = lanemask_lt(), bit = 1u << lane;
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    const u32 d = rd[i];
    const bool valid = d < (u32)RADIX;
    const u32 d0 = __shfl_sync(0xffffffffu, d, 0);
    u32 rank;
    if (__all_sync(0xffffffffu, d == d0)) {
      // one digit for the whole warp (or no valid item at all)
      const u32 before = valid ? wh[d] : 0u;
      __syncwarp();
      if (valid && lane == 31) wh[d] = before + 32u;
      rank = before + (u32)lane;
    } else {
      if (valid) atomicOr(&wm[d], bit);
      __syncwarp();
      const u32 peers = valid ? wm[d] : 0u;
      const u32 before = valid ? wh[d] : 0u;
      __syncwarp();
      if (valid && (peers >> lane) == 1u) {
        wm[d] = 0u;
        wh[d] = before + (u32)__popc(peers);
      }
      rank = before + (u32)__popc(peers & lt);
    }
    __syncwarp();
    rd[i] = valid ? (d << 16) | rank : kNoRank;
  }
}

// The same ranking with every other item ranked by ballots instead of the
// shared-memory masks (one ballot per digit bit, the highest peer advances
// the counter with a shared-memory atomic): the mask ranking loads the
// shared-memory pipe and the ballot ranking the integer pipe, and in a radix
// pass whose shared-memory traffic is already high, splitting the items
// between the two keeps either from saturating.  Same counters, same output.
template <int IPT, int RADIX, int RB>
__device__ __forceinline__ void warp_rank_mixed(u32 (&rd)[IPT], u32* wh, u32* wm, int lane) {
  const u32 lt = lanemask_lt(), bit = 1u << lane;
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    const u32 d = rd[i];
    const bool valid = d < (u32)RADIX;
    u32 rank;
    if (i & 1) {
      u32 peers = __ballot_sync(0xffffffffu, valid);
      if (!valid) peers = ~peers;
#pragma unroll
      for (int b = 0; b < RB; ++b) {
        const u32 db = (d >> b) & 1u;
        const u32 bb = __ballot_sync(0xffffffffu, db);
        peers &= db ? bb : ~bb;
      }
      const int leader = 31 - __clz(peers);
      u32 prior = 0;
      if (valid && lane == leader) prior = atomicAdd(&wh[d], (u32)__popc(peers));
      prior = __shfl_sync(0xffffffffu, prior, leader);
      rank = prior + (u32)__popc(peers & lt);
      __syncwarp();
    } else {
      const u32 d0 = __shfl_sync(0xffffffffu, d, 0);
      if (__all_sync(0xffffffffu, d == d0)) {
        const u32 before = valid ? wh[d] : 0u;
        __syncwarp();
        if (valid && lane == 31) wh[d] = before + 32u;
        rank = before + (u32)lane;
      } else {
        if (valid) atomicOr(&wm[d], bit);
        __syncwarp();
        const u32 peers = valid ? wm[d] : 0u;
        const u32 before = valid ? wh[d] : 0u;
        __syncwarp();
        if (valid && (peers >> lane) == 1u) {
          wm[d] = 0u;
          wh[d] = before + (u32)__popc(peers);
        }
        rank = before + (u32)__popc(peers & lt);
      }
      __syncwarp();
    }
    rd[i] = valid ? (d << 16) | rank : kNoRank;
  }
}

// Where the first pass reads payload word w of row r: *(u32*)(ptr + r*stride + off);
// a null ptr means the row id itself.
struct PayloadSrc {
  const unsigned char* ptr;
  u32 stride;
  u32 off;
};

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Digit / key modes of one pass.
enum : int {
  KEY_PACK = 0,   // first pass packs the key columns (pack_row)
  KEY_HASH = 1,   // first pass hashes the key columns (hash_multi_columns)
  KEY_MODEL = 2,  // first pass: key = learned-model position of the uint64 key column
  DIG_BITS = 0,   // digit = (key >> shift) & mask
  DIG_MOD = 1,    // digit = key % modulus (hash partition)
  DIG_MODEL = 2,  // digit = (model position of key >> shift) & mask (learned sort)
};

// ---- learned-CDF model (fitted in learned.cuh), evaluated inside the passes
constexpr int kLeaves = 4096;

struct Leaf {
  u64 x0;        // first sampled key of the leaf
  double slope;  // positions per key unit (>= 0)
  double base;   // predicted position at x0
  u32 lo, hi;    // the leaf's position range [lo, hi)
};

static_assert(sizeof(Leaf) == 32, "model_pos loads a leaf as two 16-byte words");

struct ModelRef {
  double ra, rb;       // leaf coordinate = ra * feature(x) + rb
  const Leaf* leaves;  // [kLeaves]
};

// Monotone, log-like feature: the bit pattern of (double)x read as a number.
__device__ __forceinline__ double model_feature(u64 x) {
  return (double)__double_as_longlong((double)x);
}

__device__ __forceinline__ int model_leaf(const ModelRef& m, u64 x) {
  const double lf = m.ra * model_feature(x) + m.rb;
  if (!(lf > 0.0)) return 0;
  if (lf >= (double)(kLeaves - 1)) return kLeaves - 1;
  return (int)lf;
}

// Predicted output position of key x: monotone non-decreasing in x.
__device__ __forceinline__ u32 model_pos(const ModelRef& m, u64 x) {
  // the 32-byte leaf in two 16-byte loads (the leaf table is 256-byte aligned)
  const uint4* lp = reinterpret_cast<const uint4*>(m.leaves + model_leaf(m, x));
  const uint4 w0 = __ldg(lp), w1 = __ldg(lp + 1);
  const u64 x0 = (u64)w0.x | ((u64)w0.y << 32);
  const double slope = __longlong_as_double((long long)((u64)w0.z | ((u64)w0.w << 32)));
  const double base = __longlong_as_double((long long)((u64)w1.x | ((u64)w1.y << 32)));
  const u32 lo = w1.z, hi = w1.w;
  const double d = x >= x0 ? (double)(x - x0) : -(double)(x0 - x);
  const double p = base + slope * d;
  const u32 top = hi > lo ? hi - 1 : lo;
  if (!(p > (double)lo)) return lo;
  if (p >= (double)top) return top;
  return (u32)p;
}

struct PassArgs {
  const void* keys_in;   // K[n] (not read by the first pass)
  const u32* vin[kMaxWords];   // payload words u32[n] each (not read by the first pass)
  void* keys_out;        // K[n]
  u32* vout[kMaxWords];  // payload words out
  PayloadSrc pfirst[kMaxWords];  // first pass: payload word sources
  const u32* bin_base;   // [RADIX] exclusive global digit offsets of this pass
  u32* status;           // [tiles][RADIX] look-back words of this pass (zeroed)
  u32* status_next;      // [tiles][RADIX] to clear for the following pass, or null
  u32* tile_counter;     // zeroed counter for tile ids of this pass
  u32* err;              // device error word
  const u32* gather_idx; // first pass: rows are read through this index, or null
  u64 n;
  int shift, width;
  int key_mode, digit_mode;
  u32 modulus;
  int reverse;           // write position n-1-p (descending radix sort)
  void* raw_out;         // last pass: write the original integer key here instead of keys_out
  int raw_dtype;
  u32 raw_flags;
  u64 raw_tmin;
  const ModelRef* model; // DIG_MODEL / KEY_MODEL: device-resident model
  unsigned long long* vout64;  // last pass: payload words 0 and 1 written as one u64 here
  PackDesc pack;
  // two-phase pass: [RADIX][tiles] global position of each tile's first key
  // of each digit, computed beforehand (k_tile_count + k_tile_scan); the
  // pass then needs no look-back and takes tile ids from blockIdx
  const u32* tile_base;
  u64 ntiles;
  // two-phase pass: [RADIX] global start of each digit (tile_base holds the
  // prefix over earlier tiles only)
  const u32* digit_starts;
  u64 spin_ns;        // bound of each look-back wait
  u32 withhold_tile;  // failure injection: this look-back ticket publishes nothing (kNoTile: none)
};

__device__ __forceinline__ u32 fmix32(u32 h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

// Key column as the hash reads it (parallel_algorithms.py:89-93, 113-121).
__device__ __forceinline__ u32 hash_word(const ColDesc& c, size_t row, bool multi) {
  switch (c.dtype) {
    case JFX_F32: return __ldg((const u32*)c.ptr + row);
    case JFX_F64: {
      double x = __ldg((const double*)c.ptr + row);
      float f = (float)x;
      return __float_as_uint(f);
    }
    case JFX_I64: case JFX_U64: return (u32)__ldg((const u64*)c.ptr + row);
    case JFX_I32: case JFX_U32: return __ldg((const u32*)c.ptr + row);
    case JFX_I16: return (u32)(int)((const short*)c.ptr)[row];
    case JFX_I8: return (u32)(int)((const signed char*)c.ptr)[row];
    case JFX_U16: return ((const unsigned short*)c.ptr)[row];
    case JFX_U8: case JFX_BOOL: return ((const unsigned char*)c.ptr)[row];
  }
  return 0;
}

// hash_multi_columns (parallel_algorithms.py:69-136).
__device__ __forceinline__ u32 hash_row(const PackDesc& pd, size_t row) {
  if (pd.ncols == 1) return fmix32(hash_word(pd.c[0], row, false));
  u32 h = 0x1337u;
  for (int i = 0; i < pd.ncols; ++i) {
    u32 k = hash_word(pd.c[i], row, true);
    h ^= k * (0x9e3779b1u + (u32)i);
    h = (h << 13) | (h >> 19);
    h *= 0x85ebca6bu;
  }
  return fmix32(h);
}

__device__ __forceinline__ u32 fmix32_d(u32 h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

template <typename K>
__device__ __forceinline__ u32 digit_of(K key, int mode, int shift, u32 mask, u32 modulus, const ModelRef& m) {
  if (mode == DIG_MOD) return (u32)key % modulus;
  if (mode == DIG_MODEL) return (model_pos(m, (u64)key) >> shift) & mask;
  return (u32)(key >> shift) & mask;
}

// Exclusive scan of data[0..N) in shared memory by all THREADS threads.
template <int THREADS, int N>
__device__ __forceinline__ void block_exclusive_scan(u32* data, u32* scratch) {
  constexpr int PER = N >= THREADS ? N / THREADS : 1;
  constexpr int ACTIVE = N >= THREADS ? THREADS : N;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  u32 local[PER];
  u32 sum = 0;
  if (tid < ACTIVE) {
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      local[k] = data[tid * PER + k];
      sum += local[k];
    }
  }
  u32 x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    u32 y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scratch[warp] = x;
  __syncthreads();
  if (warp == 0) {
    u32 w = lane < THREADS / 32 ? scratch[lane] : 0u;
    u32 inc = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      u32 y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    scratch[lane] = inc - w;
  }
  __syncthreads();
  u32 ex = x - sum + scratch[warp];
  if (tid < ACTIVE) {
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      data[tid * PER + k] = ex;
      ex += local[k];
    }
  }
  __syncthreads();
}

// Bounded spin on a look-back word until its flag is set.  Returns the word, or
// ST_ERR after limit_ns or when another CTA already reported a timeout.
__device__ __forceinline__ u32 wait_status(const u32* p, u32* err, u64 limit_ns) {
  u32 v = ld_relaxed(p);
  if (v & 0xC0000000u) return v;
  u64 t0 = globaltimer_ns();
  for (u32 spins = 1;; ++spins) {
    v = ld_relaxed(p);
    if (v & 0xC0000000u) return v;
    if (spins > 128) __nanosleep(64);
    if ((spins & 255u) == 0) {
      if (ld_relaxed(err) & DERR_TIMEOUT) return ST_ERR;
      if (globaltimer_ns() - t0 > limit_ns) {
        atomicOr(err, DERR_TIMEOUT);
        return ST_ERR;
      }
    }
  }
}

// Exclusive prefix of digit d over tiles [0, tile): walks back from tile-1,
// reading W predecessors' words per round trip, summing aggregates until an
// inclusive word.  A word not yet published is waited on (bounded).
template <int W>
__device__ __forceinline__ u32 lookback_window(const u32* status, u32 tile, u32 tile0, u32 d, u32 radix,
                                               u32* err, u64 limit_ns, bool& bad) {
  u32 excl = 0;
  long k = (long)tile - 1;  // next predecessor to read; tile0 publishes inclusive sums
  while (true) {
    u32 v[W];
#pragma unroll
    for (int i = 0; i < W; ++i)
      v[i] = (k - i >= (long)tile0) ? ld_relaxed(status + (u64)(k - i) * radix + d) : ST_INC;
    int stop = W;
    bool found = false;
    u32 sum = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      const u32 f = v[i] & 0xC0000000u;
      if (!found && stop == W) {
        if (f == 0) {
          stop = i;
        } else if (f == ST_ERR) {
          bad = true;
          found = true;
        } else {
          sum += v[i] & ST_CNT;
          if (f == ST_INC) found = true;
        }
      }
    }
    excl += sum;
    if (found) return bad ? 0u : excl;
    if (stop < W) {
      const u32 w = wait_status(status + (u64)(k - stop) * radix + d, err, limit_ns);
      const u32 f = w & 0xC0000000u;
      if (f == ST_ERR) {
        bad = true;
        return 0u;
      }
      excl += w & ST_CNT;
      if (f == ST_INC) return excl;
      k = k - stop - 1;
    } else {
      k -= W;
    }
  }
}

// Packed key of two columns from their raw elements.
template <typename K>
__device__ __forceinline__ K pack2(const PackDesc& pd, u64 r0, u64 r1) {
  K k = 0;
  if (pd.c[0].bits) k |= (K)((transform_raw(pd.c[0], r0) - pd.c[0].tmin) << pd.c[0].shift);
  if (pd.c[1].bits) k |= (K)((transform_raw(pd.c[1], r1) - pd.c[1].tmin) << pd.c[1].shift);
  return k;
}

// FM: 0 = a later pass (keys and payload words from the previous pass);
// 1 = the first pass over one plain 32/64-bit integer key column (a lean
// instantiation: fewer registers, more CTAs per SM); 2 = any other first pass
// (packed or hashed columns, gathered rows, the learned position).
// TP: a two-phase pass over plain bit digits (PassArgs::tile_base set,
// DIG_BITS); otherwise the tile bases come from the look-back.
template <typename K, int RB, int FM, int NW, bool TP>
__global__ void __launch_bounds__(RadixCfg<RB, NW>::THREADS) k_onesweep(PassArgs a) {
  constexpr bool FIRST = FM != 0;
  using L = PassLayout<K, RB, NW>;
  constexpr int THREADS = L::THREADS, IPT = L::IPT, RADIX = L::RADIX, WARPS = L::WARPS,
                TILE = L::TILE;
  extern __shared__ __align__(16) unsigned char smem[];
  u32* whist = (u32*)smem;  // [WARPS][RADIX] during ranking
  K* skeys = (K*)smem;                // [TILE] after ranking (aliases whist)
  u32* spay = (u32*)(smem + L::A_BYTES);                 // [NW][TILE] payload, row order
  uint16_t* sidx = (uint16_t*)(smem + L::A_BYTES + L::PAY_BYTES);  // sorted slot -> row slot
  uint16_t* sdig = sidx + TILE;      // digit of each sorted slot
  u32* wmask = (u32*)sidx;           // [WARPS][RADIX] peer masks during the ranking (OR_RANK)
  u32* sexcl = (u32*)(smem + L::A_BYTES + L::PAY_BYTES + L::R_BYTES);  // tile digit counts, then the tile's exclusive prefix
  u32* sbase = sexcl + RADIX;        // global position of the tile's first key of each digit
  u32* sscan = sbase + RADIX;        // 32 words of block-scan scratch
  u32* sflag = sscan + 32;           // [0] tile id, [1] abort

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    sflag[0] = a.tile_base ? blockIdx.x : atomicAdd(a.tile_counter, 1u);
    sflag[1] = 0;
  }
  for (int i = tid; i < WARPS * RADIX; i += THREADS) whist[i] = 0u;
  if constexpr (L::OR_RANK)
    for (int i = tid; i < WARPS * RADIX; i += THREADS) wmask[i] = 0u;
  // two-phase pass: this tile's global digit bases do not depend on the
  // tile's keys; their loads go out now, ahead of the key loads' use
  constexpr int DPT = RADIX >= THREADS ? RADIX / THREADS : 1;  // digits per thread
  u32 tb_pre[DPT];
  if constexpr (TP) {
#pragma unroll
    for (int k = 0; k < DPT; ++k) {
      const int d = tid + k * THREADS;
      tb_pre[k] = d < RADIX ? __ldg(a.digit_starts + d) + __ldg(a.tile_base + (u64)d * a.ntiles + blockIdx.x) : 0u;
    }
  }
  __syncthreads();
  const u32 tile = sflag[0];
  const u32* bin_base = a.bin_base;
  const u64 base = (u64)tile * TILE;
  const u32 tile_n = (u32)min((u64)TILE, a.n - base);
  const bool first_tile = tile == 0;
  const u32 mask = a.width >= 32 ? 0xffffffffu : ((1u << a.width) - 1u);
  const bool full = tile_n == (u32)TILE;
  ModelRef model;
  if (a.digit_mode == DIG_MODEL || (FIRST && a.key_mode == KEY_MODEL)) model = *a.model;
  else model.leaves = nullptr;

  // Payload goes straight to shared memory (async copies, no registers),
  // staged in row order; only the row slot of each sorted position is kept.
  const bool two_first = FIRST && a.pack.ncols == 2 && a.key_mode == KEY_PACK && !a.gather_idx;
  const bool simple_first = FIRST && (a.pack.ncols == 1 || two_first) &&
                            (a.key_mode == KEY_PACK || a.key_mode == KEY_MODEL) && !a.gather_idx;
  // this thread's first slot in the tile; item i sits at toff + 32 i
  const u32 toff = warp * 32 * IPT + lane;
  // A later two-phase pass of 32-bit keys with one payload word moves each
  // full tile's (key, payload) pairs through shared memory as one 64-bit word
  // (PACK): the payload is loaded into registers instead of being staged, so
  // the tile costs one random shared-memory store per row instead of two
  // plus the staging writes and reads.
  constexpr bool PACK = TP && FM == 0 && sizeof(K) == 4 && NW == 1;
  static_assert(!PACK || L::A_BYTES + L::PAY_BYTES >= (size_t)TILE * 8, "packed tile fits");
  u32 pay_reg[PACK ? IPT : 1];
  if (PACK && full) {
    const u32* src = a.vin[0] + base + toff;
#pragma unroll
    for (int i = 0; i < (PACK ? IPT : 0); ++i) pay_reg[i] = __ldg(src + i * 32);
  } else if (!FIRST && full) {
    // later pass, full tile: per-thread base pointers, immediate offsets
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const u32* src = a.vin[w] + base + toff;
      u32* dst = spay + w * TILE + toff;
#pragma unroll
      for (int i = 0; i < IPT; ++i) cp_async4(dst + i * 32, src + i * 32);
    }
  } else if (!FIRST || simple_first) {
#pragma unroll
    for (int w = 0; w < NW; ++w) {
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const u32 off = toff + i * 32;
        if (full || off < tile_n) {
          const u64 idx = base + off;
          if (!FIRST) cp_async4(spay + w * TILE + off, a.vin[w] + idx);
          else if (a.pfirst[w].ptr) cp_async4(spay + w * TILE + off, a.pfirst[w].ptr + idx * a.pfirst[w].stride + a.pfirst[w].off);
          else spay[w * TILE + off] = (u32)idx;
        }
      }
    }
  }

  // rd[i]: the item's digit in bits [0, 12) (RADIX = not an item), and after
  // ranking its rank within the warp in bits [12, 32).  Every key load of the
  // tile is issued before any is used (one DRAM round trip per tile).
  K key[IPT];
  u32 rd[IPT];
  if (!FIRST && full && a.digit_mode == DIG_BITS) {
    const K* kin = (const K*)a.keys_in + base + toff;
#pragma unroll
    for (int i = 0; i < IPT; ++i) key[i] = kin[i * 32];
#pragma unroll
    for (int i = 0; i < IPT; ++i) rd[i] = (u32)(key[i] >> a.shift) & mask;
  } else if constexpr (FM == 1) {
    // first pass over one or two plain integer columns of one width: the
    // dtype is dispatched once per tile; each transform is the sign flip
    const int d0 = a.pack.c[0].dtype;
    const bool two = a.pack.ncols == 2;
    const u64 flip0 = d0 == JFX_I64 ? 0x8000000000000000ull : d0 == JFX_I32 ? 0x80000000ull : 0ull;
    const int d1 = two ? a.pack.c[1].dtype : d0;
    const u64 flip1 = d1 == JFX_I64 ? 0x8000000000000000ull : d1 == JFX_I32 ? 0x80000000ull : 0ull;
    const u64 tmin0 = a.pack.c[0].tmin, tmin1 = two ? a.pack.c[1].tmin : 0ull;
    const int sh0 = a.pack.c[0].shift, sh1 = two ? a.pack.c[1].shift : 0;
    const bool b1 = two && a.pack.c[1].bits;  // a constant second column adds nothing
    if (dtype_size(d0) == 8) {
      const u64* src = (const u64*)a.pack.c[0].ptr + base + toff;
      u64 raw[IPT];
#pragma unroll
      for (int i = 0; i < IPT; ++i) raw[i] = (full || toff + i * 32 < tile_n) ? __ldg(src + i * 32) : 0ull;
#pragma unroll
      for (int i = 0; i < IPT; ++i) key[i] = (K)(((raw[i] ^ flip0) - tmin0) << sh0);
      if (b1) {
        const u64* src1 = (const u64*)a.pack.c[1].ptr + base + toff;
#pragma unroll
        for (int i = 0; i < IPT; ++i) raw[i] = (full || toff + i * 32 < tile_n) ? __ldg(src1 + i * 32) : 0ull;
#pragma unroll
        for (int i = 0; i < IPT; ++i) key[i] |= (K)(((raw[i] ^ flip1) - tmin1) << sh1);
      }
    } else {
      const u32* src = (const u32*)a.pack.c[0].ptr + base + toff;
      const u32* src1 = (const u32*)(b1 ? a.pack.c[1].ptr : a.pack.c[0].ptr) + base + toff;
      u32 r0[IPT], r1[IPT];
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const bool in = full || toff + i * 32 < tile_n;
        r0[i] = in ? __ldg(src + i * 32) : 0u;
        r1[i] = (in && b1) ? __ldg(src1 + i * 32) : 0u;
      }
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        key[i] = (K)((((u64)r0[i] ^ flip0) - tmin0) << sh0);
        if (b1) key[i] |= (K)((((u64)r1[i] ^ flip1) - tmin1) << sh1);
      }
    }
    if (a.digit_mode == DIG_BITS) {
#pragma unroll
      for (int i = 0; i < IPT; ++i)
        rd[i] = (full || toff + i * 32 < tile_n) ? (u32)(key[i] >> a.shift) & mask : (u32)RADIX;
    } else {  // the batched partition pass: hash digit
#pragma unroll
      for (int i = 0; i < IPT; ++i)
        rd[i] = (full || toff + i * 32 < tile_n) ? digit_of<K>(key[i], a.digit_mode, a.shift, mask, a.modulus, model)
                                                 : (u32)RADIX;
    }
  } else if (two_first) {
    // two key columns: both columns' loads for 8 items, then pack
#pragma unroll
    for (int i0 = 0; i0 < IPT; i0 += 8) {
      u64 r0[8], r1[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const u32 off = warp * 32 * IPT + (i0 + i) * 32 + lane;
        const u64 idx = base + off;
        if (full || off < tile_n) {
          r0[i] = load_raw(a.pack.c[0].ptr, a.pack.c[0].dtype, idx);
          r1[i] = load_raw(a.pack.c[1].ptr, a.pack.c[1].dtype, idx);
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const u32 off = warp * 32 * IPT + (i0 + i) * 32 + lane;
        rd[i0 + i] = RADIX;
        if (full || off < tile_n) {
          key[i0 + i] = pack2<K>(a.pack, r0[i], r1[i]);
          rd[i0 + i] = digit_of<K>(key[i0 + i], a.digit_mode, a.shift, mask, a.modulus, model);
        }
      }
    }
  } else if (!FIRST || (simple_first && a.pack.ncols == 1)) {
    u64 raw[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 off = warp * 32 * IPT + i * 32 + lane;
      const u64 idx = base + off;
      if (full || off < tile_n) {
        if (FIRST) raw[i] = load_raw(a.pack.c[0].ptr, a.pack.c[0].dtype, idx);
        else key[i] = ((const K*)a.keys_in)[idx];
      }
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 off = warp * 32 * IPT + i * 32 + lane;
      rd[i] = RADIX;
      if (full || off < tile_n) {
        if (FIRST) {
          const u64 t = transform_raw(a.pack.c[0], raw[i]);
          key[i] = a.key_mode == KEY_MODEL ? (K)model_pos(model, t) : (K)(t - a.pack.c[0].tmin) << a.pack.c[0].shift;
        }
        rd[i] = digit_of<K>(key[i], a.digit_mode, a.shift, mask, a.modulus, model);
      }
    }
  } else {
    u64 rows[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 off = warp * 32 * IPT + i * 32 + lane;
      const u64 idx = base + off;
      rows[i] = (off < tile_n && a.gather_idx) ? (u64)a.gather_idx[idx] : idx;
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 off = warp * 32 * IPT + i * 32 + lane;
      if (off < tile_n) {
        key[i] = a.key_mode == KEY_HASH ? (K)hash_row(a.pack, rows[i]) : pack_row<K>(a.pack, rows[i]);
#pragma unroll
        for (int w = 0; w < NW; ++w) {
          if (a.pfirst[w].ptr) cp_async4(spay + w * TILE + off, a.pfirst[w].ptr + rows[i] * a.pfirst[w].stride + a.pfirst[w].off);
          else spay[w * TILE + off] = (u32)rows[i];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 off = warp * 32 * IPT + i * 32 + lane;
      rd[i] = off < tile_n ? digit_of<K>(key[i], a.digit_mode, a.shift, mask, a.modulus, model) : (u32)RADIX;
    }
  }

  if constexpr (TP) {
    // Two-phase pass over plain bit digits: the tile's global bases are
    // known, nothing is published, so the digit counts come out of the
    // ranking itself (warp-private counters from zero, then per-warp
    // prefixes), and the scatter recomputes each key's digit from the key and
    // reads the payload already moved to sorted order: no per-row count
    // atomics, digit or row-slot arrays in shared memory.
    u32* wh = whist + warp * RADIX;
    if constexpr (L::OR_RANK) {
      warp_rank_mixed<IPT, RADIX, RB>(rd, wh, wmask + warp * RADIX, lane);
#pragma unroll
      for (int i = 0; i < IPT; ++i)
        rd[i] = rd[i] != kNoRank ? 0x80000000u | ((rd[i] >> 16) << 13) | (rd[i] & 0xffffu) : 0u;
    } else {
      const u32 lt = lanemask_lt();
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const u32 d = rd[i];
        const bool valid = d < (u32)RADIX;
        u32 peers = __ballot_sync(0xffffffffu, valid);
        if (!valid) peers = ~peers;
#pragma unroll
        for (int b = 0; b < RB; ++b) {
          const u32 bit = (d >> b) & 1u;
          const u32 bb = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? bb : ~bb;
        }
        const int leader = 31 - __clz(peers);
        u32 prior = 0;
        if (valid && lane == leader) prior = atomicAdd(&wh[d], (u32)__popc(peers));
        prior = __shfl_sync(0xffffffffu, prior, leader);
        // bit 31 item present, bits [13, 24) digit, [0, 13) rank in the warp
        rd[i] = valid ? 0x80000000u | (d << 13) | (prior + __popc(peers & lt)) : 0u;
      }
    }
    __syncthreads();
    for (int d = tid; d < RADIX; d += THREADS) {
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
    block_exclusive_scan<THREADS, RADIX>(sexcl, sscan);  // tile-local start of each digit
#pragma unroll
    for (int k = 0; k < DPT; ++k) {
      const int d = tid + k * THREADS;
      if (d < RADIX) sbase[d] = tb_pre[k] - sexcl[d];
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      if (rd[i] & 0x80000000u) {
        const u32 d = (rd[i] >> 13) & 0x7ffu;
        rd[i] = 0x80000000u | (sexcl[d] + wh[d] + (rd[i] & 0x1fffu));  // tile-local sorted slot
      }
    }
    if constexpr (PACK) {
      if (full) {
        u64* skp = (u64*)smem;  // [TILE] key | payload << 32, over the histogram and staging bytes
        __syncthreads();        // every whist read is done
#pragma unroll
        for (int i = 0; i < IPT; ++i)
          if (rd[i] & 0x80000000u) skp[rd[i] & 0x1fffu] = (u64)(u32)key[i] | ((u64)pay_reg[i] << 32);
        __syncthreads();
        K* kout = (K*)a.keys_out;
        const u32 row0 = 0u, span = (u32)a.n;
        const int rsz = a.raw_out ? dtype_size(a.raw_dtype) : 0;
#pragma unroll
        for (int i0 = 0; i0 < IPT; i0 += 8) {
          u64 kp[8];
          u32 gg[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const u32 j = (i0 + i) * THREADS + tid;
            kp[i] = skp[j];
            gg[i] = sbase[((u32)kp[i] >> a.shift) & mask] + j;
          }
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            if (gg[i] - row0 >= span) {
              atomicOr(a.err, DERR_BOUNDS);
              continue;
            }
            const K k = (K)(u32)kp[i];
            const u64 g = a.reverse ? a.n - 1 - (u64)gg[i] : (u64)gg[i];
            if (rsz) store_raw(a.raw_out, a.raw_dtype, g, untransform_int(a.raw_dtype, a.raw_flags, (u64)k + a.raw_tmin));
            else kout[g] = k;
            a.vout[0][g] = (u32)(kp[i] >> 32);
          }
        }
        if (a.status_next)
          for (int d = tid; d < RADIX; d += THREADS) a.status_next[(u64)tile * RADIX + d] = 0u;
        return;
      }
    }
    cp_async_wait_all();
    __syncthreads();  // every whist read is done (skeys aliases it); the payload has landed
#pragma unroll
    for (int i = 0; i < IPT; ++i)
      if (rd[i] & 0x80000000u) skeys[rd[i] & 0x1fffu] = key[i];
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      u32 pv[IPT];
#pragma unroll
      for (int i = 0; i < IPT; ++i) pv[i] = spay[w * TILE + toff + i * 32];
      __syncthreads();  // this word's row-order slots are all read
#pragma unroll
      for (int i = 0; i < IPT; ++i)
        if (rd[i] & 0x80000000u) spay[w * TILE + (rd[i] & 0x1fffu)] = pv[i];
    }
    __syncthreads();

    K* kout = (K*)a.keys_out;
    const u32 row0 = 0u, span = (u32)a.n;
    const int rsz = a.raw_out ? dtype_size(a.raw_dtype) : 0;
    const bool plain = !a.raw_out && !a.reverse;
    if (full) {
#pragma unroll
      for (int i0 = 0; i0 < IPT; i0 += 8) {
        K kk[8];
        u32 gg[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const u32 j = (i0 + i) * THREADS + tid;
          kk[i] = skeys[j];
          gg[i] = sbase[(u32)(kk[i] >> a.shift) & mask] + j;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const u32 j = (i0 + i) * THREADS + tid;
          if (gg[i] - row0 >= span) {
            atomicOr(a.err, DERR_BOUNDS);
            continue;
          }
          u64 g = gg[i];
          if (plain) {
            kout[g] = kk[i];
          } else {
            if (a.reverse) g = a.n - 1 - g;
            if (rsz) {
              const u64 v = untransform_int(a.raw_dtype, a.raw_flags, (u64)kk[i] + a.raw_tmin);
              if (rsz == 4) ((u32*)a.raw_out)[g] = (u32)v;
              else if (rsz == 8) ((u64*)a.raw_out)[g] = v;
              else store_raw(a.raw_out, a.raw_dtype, g, v);
            } else {
              kout[g] = kk[i];
            }
          }
          if (NW >= 2 && a.vout64) {
            a.vout64[g] = (unsigned long long)spay[j] | ((unsigned long long)spay[TILE + j] << 32);
#pragma unroll
            for (int w = 2; w < NW; ++w) a.vout[w][g] = spay[w * TILE + j];
          } else {
#pragma unroll
            for (int w = 0; w < NW; ++w) a.vout[w][g] = spay[w * TILE + j];
          }
        }
      }
    } else {
      for (u32 j = tid; j < tile_n; j += THREADS) {
        const K k = skeys[j];
        const u32 g32 = sbase[(u32)(k >> a.shift) & mask] + j;
        if (g32 - row0 >= span) {
          atomicOr(a.err, DERR_BOUNDS);
          continue;
        }
        u64 g = g32;
        if (a.reverse) g = a.n - 1 - g;
        if (a.raw_out) store_raw(a.raw_out, a.raw_dtype, g, untransform_int(a.raw_dtype, a.raw_flags, (u64)k + a.raw_tmin));
        else kout[g] = k;
        if (NW >= 2 && a.vout64) {
          a.vout64[g] = (unsigned long long)spay[j] | ((unsigned long long)spay[TILE + j] << 32);
#pragma unroll
          for (int w = 2; w < NW; ++w) a.vout[w][g] = spay[w * TILE + j];
        } else {
#pragma unroll
          for (int w = 0; w < NW; ++w) a.vout[w][g] = spay[w * TILE + j];
        }
      }
    }
    if (a.status_next)
      for (int d = tid; d < RADIX; d += THREADS) a.status_next[(u64)tile * RADIX + d] = 0u;
    return;
  }

  // Digit counts first: per-warp histograms by shared-memory atomics (order
  // does not matter for a count), so the tile's counts are published and its
  // prefix over earlier tiles resolved before the ranking, which is the
  // longest phase.  Successors then find this tile's words early.
  u32* wh = whist + warp * RADIX;
#pragma unroll
  for (int i = 0; i < IPT; ++i)
    if (rd[i] < (u32)RADIX) atomicAdd(&wh[rd[i]], 1u);
  __syncthreads();

  // Per digit: exclusive prefix over warps (in place), the tile count, and
  // its publication (tile 0 of a segment: already inclusive).
  u32* st = a.status + (u64)tile * RADIX;
  for (int d = tid; d < RADIX; d += THREADS) {
    u32 run = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
      const u32 c = whist[w * RADIX + d];
      whist[w * RADIX + d] = run;
      run += c;
    }
    sexcl[d] = run;
    sbase[d] = run;
    if (!a.tile_base && tile != a.withhold_tile) st_relaxed(st + d, (first_tile ? ST_INC : ST_AGG) | run);
  }
  __syncthreads();
  block_exclusive_scan<THREADS, RADIX>(sexcl, sscan);  // tile-local start of each digit

  // Resolve each digit's prefix over the earlier tiles and publish it.
  constexpr int WIN = (RADIX / THREADS) >= 8 ? 4 : (RADIX / THREADS) >= 4 ? 8 : 16;
  for (int d = tid; d < RADIX; d += THREADS) {
    if (a.tile_base) {  // two-phase pass: the tile's digit bases are known
      sbase[d] = a.tile_base[(u64)d * a.ntiles + tile] - sexcl[d];
      continue;
    }
    const u32 c = sbase[d];
    u32 excl = 0;
    bool bad = false;
    if (!first_tile) {
      excl = lookback_window<WIN>(a.status, tile, 0u, (u32)d, (u32)RADIX, a.err, a.spin_ns, bad);
      if (tile != a.withhold_tile) st_relaxed(st + d, bad ? ST_ERR : (ST_INC | (excl + c)));
    }
    if (bad) sflag[1] = 1u;
    // global position of the tile's sorted index j is sbase[d] + j (mod 2^32)
    sbase[d] = bin_base[d] + excl - sexcl[d];
  }

  // Stable rank within the tile: lanes holding the same digit are ranked by
  // lane, items are visited in row order and warps in row order (the
  // per-warp counters start at the warp's exclusive prefix), so equal digits
  // keep row order.  Peers are found with one ballot per digit bit; the
  // lowest peer advances the warp's counter for the whole group.
  static_assert(TILE <= 8192 && RADIX <= 2048, "position/digit packing");
  if constexpr (L::OR_RANK) {
    warp_rank_or<IPT, RADIX>(rd, wh, wmask + warp * RADIX, lane);
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 d = rd[i] >> 16;
      // rd becomes: bit 31 item present, bits [13, 25) digit, [0, 13) tile-local position
      rd[i] = rd[i] != kNoRank ? 0x80000000u | (d << 13) | (sexcl[d] + (rd[i] & 0xffffu)) : 0u;
    }
  } else {
    const u32 lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 d = rd[i];
      const bool valid = d < (u32)RADIX;
      u32 peers = __ballot_sync(0xffffffffu, valid);
      if (!valid) peers = ~peers;
#pragma unroll
      for (int b = 0; b < RB; ++b) {
        const u32 bit = (d >> b) & 1u;
        const u32 bb = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bb : ~bb;
      }
      const int leader = 31 - __clz(peers);
      u32 prior = 0;
      if (valid && lane == leader) prior = atomicAdd(&wh[d], (u32)__popc(peers));
      prior = __shfl_sync(0xffffffffu, prior, leader);
      // rd becomes: bit 31 item present, bits [13, 25) digit, [0, 13) tile-local position
      rd[i] = valid ? 0x80000000u | (d << 13) | (sexcl[d] + prior + __popc(peers & lt)) : 0u;
    }
  }
  __syncthreads();  // whist reads above are done before skeys (aliased) is written
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    if (rd[i] & 0x80000000u) {
      const u32 p = rd[i] & 0x1fffu;
      skeys[p] = key[i];
      sidx[p] = (uint16_t)(warp * 32 * IPT + i * 32 + lane);
      sdig[p] = (uint16_t)((rd[i] >> 13) & 0xfffu);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if (sflag[1]) return;

  K* kout = (K*)a.keys_out;
  const bool plain_out = !a.raw_out && !a.reverse;
  if (full && plain_out) {
    const u32 row0 = 0u, span = (u32)a.n;
    // full tile: IPT independent slots per thread, loads before stores
#pragma unroll
    for (int i0 = 0; i0 < IPT; i0 += 8) {
      K kk[8];
      u32 gg[8], uu[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const u32 j = (i0 + i) * THREADS + tid;
        kk[i] = skeys[j];
        uu[i] = sidx[j];
        gg[i] = sbase[sdig[j]] + j;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const u32 g = gg[i];  // rows < 2^30: 32-bit positions
        if (g - row0 >= span) {
          atomicOr(a.err, DERR_BOUNDS);
          continue;
        }
        kout[g] = kk[i];
        if (NW >= 2 && a.vout64) {
          a.vout64[g] = (unsigned long long)spay[uu[i]] | ((unsigned long long)spay[TILE + uu[i]] << 32);
#pragma unroll
          for (int w = 2; w < NW; ++w) a.vout[w][g] = spay[w * TILE + uu[i]];
        } else {
#pragma unroll
          for (int w = 0; w < NW; ++w) a.vout[w][g] = spay[w * TILE + uu[i]];
        }
      }
    }
    if (a.status_next)
      for (int d = tid; d < RADIX; d += THREADS) a.status_next[(u64)tile * RADIX + d] = 0u;
    return;
  }
  if (full) {
    // full tile, other output forms (original-dtype keys, descending
    // positions, query-tagged keys): the same unrolled slots
    const u32 row0 = 0u, span = (u32)a.n;
    const int rsz = a.raw_out ? dtype_size(a.raw_dtype) : 0;
#pragma unroll
    for (int i0 = 0; i0 < IPT; i0 += 8) {
      K kk[8];
      u32 gg[8], uu[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const u32 j = (i0 + i) * THREADS + tid;
        kk[i] = skeys[j];
        uu[i] = sidx[j];
        gg[i] = sbase[sdig[j]] + j;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (gg[i] - row0 >= span) {
          atomicOr(a.err, DERR_BOUNDS);
          continue;
        }
        const u64 g = a.reverse ? a.n - 1 - (u64)gg[i] : (u64)gg[i];
        if (rsz) {
          const u64 v = untransform_int(a.raw_dtype, a.raw_flags, (u64)kk[i] + a.raw_tmin);
          if (rsz == 4) ((u32*)a.raw_out)[g] = (u32)v;
          else if (rsz == 8) ((u64*)a.raw_out)[g] = v;
          else store_raw(a.raw_out, a.raw_dtype, g, v);
        } else {
          kout[g] = kk[i];
        }
        if (NW >= 2 && a.vout64) {
          a.vout64[g] = (unsigned long long)spay[uu[i]] | ((unsigned long long)spay[TILE + uu[i]] << 32);
#pragma unroll
          for (int w = 2; w < NW; ++w) a.vout[w][g] = spay[w * TILE + uu[i]];
        } else {
#pragma unroll
          for (int w = 0; w < NW; ++w) a.vout[w][g] = spay[w * TILE + uu[i]];
        }
      }
    }
    if (a.status_next)
      for (int d = tid; d < RADIX; d += THREADS) a.status_next[(u64)tile * RADIX + d] = 0u;
    return;
  }
  for (u32 j = tid; j < tile_n; j += THREADS) {
    const K k = skeys[j];
    const u32 d = sdig[j];
    const u32 u = sidx[j];
    u64 g = (u64)(u32)(sbase[d] + j);
    if (g >= a.n) {  // only reachable if histogram and pass disagree
      atomicOr(a.err, DERR_BOUNDS);
      continue;
    }
    if (a.reverse) g = a.n - 1 - g;
    if (a.raw_out) store_raw(a.raw_out, a.raw_dtype, g, untransform_int(a.raw_dtype, a.raw_flags, (u64)k + a.raw_tmin));
    else kout[g] = k;
    if (NW >= 2 && a.vout64) {
      a.vout64[g] = (unsigned long long)spay[u] | ((unsigned long long)spay[TILE + u] << 32);
#pragma unroll
      for (int w = 2; w < NW; ++w) a.vout[w][g] = spay[w * TILE + u];
    } else {
#pragma unroll
      for (int w = 0; w < NW; ++w) a.vout[w][g] = spay[w * TILE + u];
    }
  }
  if (a.status_next)
    for (int d = tid; d < RADIX; d += THREADS) a.status_next[(u64)tile * RADIX + d] = 0u;
}

// ----------------------------------------------------------------- upsweep ---
struct HistArgs {
  PackDesc pack;
  u32* hist;       // [npass][RADIX], zeroed
  u32* targets;    // optional: digit of pass 0 per row (hash partition targets)
  u64 n;
  int npass;
  int key_mode, digit_mode;
  u32 modulus;
  int shift[8];
  int width[8];
  const ModelRef* model;
};

template <typename K, int RB>
__global__ void __launch_bounds__(256) k_hist(HistArgs a) {
  constexpr int RADIX = 1 << RB;
  extern __shared__ u32 sh[];
  const int total = a.npass * RADIX;
  for (int i = threadIdx.x; i < total; i += blockDim.x) sh[i] = 0u;
  __syncthreads();
  u32 mask[8];
#pragma unroll
  for (int p = 0; p < 8; ++p) mask[p] = a.width[p] >= 32 ? 0xffffffffu : ((1u << a.width[p]) - 1u);
  ModelRef model;
  if (a.digit_mode == DIG_MODEL || a.key_mode == KEY_MODEL) model = *a.model;
  else model.leaves = nullptr;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  constexpr int U = 8;  // rows per thread per step, loads issued together
  const bool simple = a.pack.ncols == 1 && a.key_mode == KEY_PACK;
  for (u64 r0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; r0 < a.n; r0 += stride * U) {
    K kk[U];
    if (a.key_mode == KEY_MODEL) {
      u64 raw[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 r = r0 + (u64)u * stride;
        raw[u] = r < a.n ? load_raw(a.pack.c[0].ptr, a.pack.c[0].dtype, r) : 0ull;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) kk[u] = (K)model_pos(model, transform_raw(a.pack.c[0], raw[u]));
    } else if (simple) {
      u64 raw[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 r = r0 + (u64)u * stride;
        raw[u] = r < a.n ? load_raw(a.pack.c[0].ptr, a.pack.c[0].dtype, r) : 0ull;
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        kk[u] = (K)(transform_raw(a.pack.c[0], raw[u]) - a.pack.c[0].tmin) << a.pack.c[0].shift;
    } else if (a.pack.ncols == 2 && a.key_mode == KEY_PACK) {
      u64 x0[U], x1[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 r = r0 + (u64)u * stride;
        x0[u] = r < a.n ? load_raw(a.pack.c[0].ptr, a.pack.c[0].dtype, r) : 0ull;
        x1[u] = r < a.n ? load_raw(a.pack.c[1].ptr, a.pack.c[1].dtype, r) : 0ull;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) kk[u] = pack2<K>(a.pack, x0[u], x1[u]);
    } else {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 r = r0 + (u64)u * stride;
        kk[u] = r < a.n ? (a.key_mode == KEY_HASH ? (K)hash_row(a.pack, r) : pack_row<K>(a.pack, r)) : (K)0;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
    const u64 r = r0 + (u64)u * stride;
    if (r >= a.n) break;
    const K k = kk[u];
    if (a.digit_mode == DIG_MODEL) {
      const u32 pos = model_pos(model, (u64)k);
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        if (p >= a.npass) break;
        atomicAdd(&sh[p * RADIX + ((pos >> a.shift[p]) & mask[p])], 1u);
      }
      continue;
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      if (p >= a.npass) break;
      const u32 d = digit_of<K>(k, a.digit_mode, a.shift[p], mask[p], a.modulus, model);
      atomicAdd(&sh[p * RADIX + d], 1u);
      if (p == 0 && a.targets) a.targets[r] = d;
    }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < total; i += blockDim.x)
    if (sh[i]) atomicAdd(&a.hist[i], sh[i]);
}

// k_hist for the common key: one plain 32/64-bit integer column, digits of
// its packed value.  T is the column's storage type.  The dtype dispatch and
// the transform are fixed per launch, so the loop body is a load, a sign flip,
// a subtraction and one shared-memory atomic per pass.
struct HistIntArgs {
  const void* col;
  const void* col2;  // optional second key column (same storage type), less significant
  u32* hist;  // [npass][RADIX], zeroed
  u64 n;
  u64 flip, tmin;
  u64 flip2, tmin2;
  int kshift, kshift2, npass;
  int shift[8];
  u32 mask[8];
  // optional: the first pass's digit counts of every radix tile, digit-major
  // [RADIX][tiles], so that pass can run in two phases as well
  u32* tile_counts;
  u64 tiles;
  u32 tile_rows;  // rows per tile of that pass
};

template <typename K, typename T, int RB>
__global__ void __launch_bounds__(256) k_hist_int(HistIntArgs a) {
  constexpr int RADIX = 1 << RB;
  extern __shared__ u32 sh[];
  const int total = a.npass * RADIX;
  const T* col = (const T*)a.col;
  const T* col2 = (const T*)a.col2;
  if (a.tile_counts) {
    // tile by tile (the radix pass's tiles): all passes' counts plus the
    // first pass's counts of this tile
    constexpr int CH = 8;  // rows per thread per chunk; a tile is 1 or 2 chunks
    const u32 TILE = a.tile_rows;
    u32* tsh = sh + total;
    for (int i = threadIdx.x; i < total + RADIX; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    for (u64 t = blockIdx.x; t < a.tiles; t += gridDim.x) {
      const u64 base = t * TILE;
      const u32 tn = (u32)min((u64)TILE, a.n - base);
      for (u32 c0 = 0; c0 < tn; c0 += 256 * CH) {
        T raw[CH], raw2[CH];
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          const u32 r = c0 + i * 256 + threadIdx.x;
          raw[i] = r < tn ? __ldg(col + base + r) : (T)0;
          raw2[i] = (col2 && r < tn) ? __ldg(col2 + base + r) : (T)0;
        }
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          if (c0 + i * 256 + threadIdx.x >= tn) break;
          K k = (K)((((u64)raw[i] ^ a.flip) - a.tmin) << a.kshift);
          if (col2) k |= (K)((((u64)raw2[i] ^ a.flip2) - a.tmin2) << a.kshift2);
          atomicAdd(&tsh[(u32)(k >> a.shift[0]) & a.mask[0]], 1u);
#pragma unroll
          for (int p = 0; p < 8; ++p) {
            if (p >= a.npass) break;
            atomicAdd(&sh[p * RADIX + ((u32)(k >> a.shift[p]) & a.mask[p])], 1u);
          }
        }
      }
      __syncthreads();
      for (int d = threadIdx.x; d < RADIX; d += blockDim.x) {
        a.tile_counts[(u64)d * a.tiles + t] = tsh[d];
        tsh[d] = 0u;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < total; i += blockDim.x)
      if (sh[i]) atomicAdd(&a.hist[i], sh[i]);
    return;
  }
  for (int i = threadIdx.x; i < total; i += blockDim.x) sh[i] = 0u;
  __syncthreads();
  const u64 stride = (u64)gridDim.x * blockDim.x;
  constexpr int U = 8;  // rows per thread per step, loads issued together
  for (u64 r0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; r0 < a.n; r0 += stride * U) {
    T raw[U], raw2[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 r = r0 + (u64)u * stride;
      raw[u] = r < a.n ? __ldg(col + r) : (T)0;
      raw2[u] = (col2 && r < a.n) ? __ldg(col2 + r) : (T)0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (r0 + (u64)u * stride >= a.n) break;
      K k = (K)((((u64)raw[u] ^ a.flip) - a.tmin) << a.kshift);
      if (col2) k |= (K)((((u64)raw2[u] ^ a.flip2) - a.tmin2) << a.kshift2);
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        if (p >= a.npass) break;
        atomicAdd(&sh[p * RADIX + ((u32)(k >> a.shift[p]) & a.mask[p])], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < total; i += blockDim.x)
    if (sh[i]) atomicAdd(&a.hist[i], sh[i]);
}

// Exclusive scan of each pass's histogram (one CTA per pass).
template <int RB>
__global__ void __launch_bounds__(1024) k_hist_scan(const u32* hist, u32* base) {
  constexpr int RADIX = 1 << RB;
  __shared__ u32 data[RADIX];
  __shared__ u32 scratch[32];
  const u32* h = hist + (u64)blockIdx.x * RADIX;
  for (int i = threadIdx.x; i < RADIX; i += 1024) data[i] = h[i];
  __syncthreads();
  block_exclusive_scan<1024, RADIX>(data, scratch);
  for (int i = threadIdx.x; i < RADIX; i += 1024) base[(u64)blockIdx.x * RADIX + i] = data[i];
}

// ------------------------------------------------------ two-phase passes ---
// A later pass can do without the decoupled look-back: k_tile_count counts
// each tile's digits, k_tile_scan turns the counts into every tile's global
// base per digit (column-wise exclusive scan plus the digit's global offset),
// and the pass reads its bases instead of waiting on earlier tiles.  That
// costs one more read of the keys, but no tile ever waits on another.

// counts[d][tile] (digit-major, so the scan reads rows) of digit
// (key >> shift) & mask; one CTA per tile.
template <typename K, int RB, int NW>
__global__ void __launch_bounds__(256) k_tile_count(const K* keys, u64 n, int shift, u32 mask, u32* counts,
                                                    u64 tiles) {
  constexpr int RADIX = 1 << RB, TILE = PassLayout<K, RB, NW>::TILE, IPT = TILE / 256;
  constexpr int NH = RB <= 9 ? 8 : RB == 10 ? 4 : 2;  // histogram copies (fewer same-address atomics)
  __shared__ u32 h[NH][RADIX];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < NH * RADIX; i += 256) (&h[0][0])[i] = 0u;
  const u64 base = (u64)blockIdx.x * TILE;
  const u32 tile_n = (u32)min((u64)TILE, n - base);
  const K* src = keys + base + warp * 32 * IPT + lane;
  K k[IPT];
  if (tile_n == (u32)TILE) {
#pragma unroll
    for (int i = 0; i < IPT; ++i) k[i] = src[i * 32];
  } else {
#pragma unroll
    for (int i = 0; i < IPT; ++i) k[i] = (warp * 32 * IPT + i * 32 + lane) < tile_n ? src[i * 32] : (K)0;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < IPT; ++i)
    if ((warp * 32 * IPT + i * 32 + lane) < tile_n) atomicAdd(&h[warp % NH][(u32)(k[i] >> shift) & mask], 1u);
  __syncthreads();
  for (int d = tid; d < RADIX; d += 256) {
    u32 c = 0;
#pragma unroll
    for (int w = 0; w < NH; ++w) c += h[w][d];
    counts[(u64)d * tiles + blockIdx.x] = c;
  }
}

// base[d][t] = bin_base[d] + sum over t' < t of counts[d][t'] (mod 2^32:
// rows < 2^30).  One CTA of T threads per digit row, 16 T tiles per round:
// coalesced loads into shared memory (padded one word in 32, so a thread's
// 16 consecutive entries sit in distinct banks across the warp), a block scan
// of the thread sums, and coalesced stores of the bases.  T = 1024 for long
// rows; T = 256 for short ones, where the small CTAs leave room for the other
// kernels in flight (the two sides of a join sort concurrently).
constexpr int kTileScanPer = 16;
template <int T>
constexpr size_t tile_scan_smem() { return (size_t)(T * kTileScanPer + T * kTileScanPer / 32) * sizeof(u32); }
__device__ __forceinline__ u32 tile_scan_slot(u32 i) { return i + (i >> 5); }

// With bin_base null the bases start at 0, the row's total goes to
// totals[d], and the last CTA to finish (counted on *done, which it resets)
// writes starts[d] = the sum of the totals below d: the two-phase passes add
// these digit starts themselves, so no histogram of the keys is needed.
// rot: digit d's counts are row (d + rot) mod RADIX of `counts` (first-pass
// counts taken from the min/max pass, rotated by the minimum's low byte).
template <int T>
__global__ void __launch_bounds__(T) k_tile_scan(const u32* counts, u64 tiles, const u32* bin_base, u32* base,
                                                 u32* totals, u32* starts, u32* done, u32 rot) {
  constexpr int PER = kTileScanPer, CH = T * PER;
  static_assert(T % 32 == 0 && T <= 1024, "warps of a block");
  extern __shared__ u32 buf[];  // [CH + CH / 32]
  __shared__ u32 wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32* row = counts + (u64)((blockIdx.x + rot) & (gridDim.x - 1)) * tiles;
  u32* out = base + (u64)blockIdx.x * tiles;
  u32 carry = bin_base ? bin_base[blockIdx.x] : 0u;
  for (u64 c0 = 0; c0 < tiles; c0 += CH) {
    const u32 m = (u32)min((u64)CH, tiles - c0);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const u32 i = k * T + tid;
      buf[tile_scan_slot(i)] = i < m ? row[c0 + i] : 0u;
    }
    __syncthreads();
    u32 v[PER];
    u32 sum = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      v[k] = buf[tile_scan_slot(tid * PER + k)];
      sum += v[k];
    }
    u32 x = sum;  // inclusive scan of the thread sums: warp, then across warps
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const u32 w = lane < T / 32 ? wsum[lane] : 0u;
      u32 z = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= o) z += y;
      }
      if (lane < T / 32) wsum[lane] = z - w;  // exclusive prefix of each warp
    }
    __syncthreads();
    u32 run = carry + wsum[warp] + x - sum;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      buf[tile_scan_slot(tid * PER + k)] = run;
      run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const u32 i = k * T + tid;
      if (i < m) out[c0 + i] = buf[tile_scan_slot(i)];
    }
    // the last thread's running value is carry + the round's total
    if (tid == T - 1) wsum[0] = run;
    __syncthreads();
    carry = wsum[0];
    __syncthreads();  // wsum and buf are rewritten next round
  }
  if (bin_base) return;
  __shared__ u32 s_last;
  if (tid == 0) {
    totals[blockIdx.x] = carry;
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // exclusive scan of the gridDim.x (<= 2048) totals: PER2 consecutive per thread
  const u32 R = gridDim.x, PER2 = (R + T - 1) / T;
  u32 sum = 0;
  for (u32 k = 0; k < PER2; ++k) {
    const u32 d = tid * PER2 + k;
    if (d < R) sum += __ldcg(totals + d);
  }
  u32 x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const u32 w = lane < T / 32 ? wsum[lane] : 0u;
    u32 z = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += y;
    }
    if (lane < T / 32) wsum[lane] = z - w;
  }
  __syncthreads();
  u32 run = wsum[warp] + x - sum;
  for (u32 k = 0; k < PER2; ++k) {
    const u32 d = tid * PER2 + k;
    if (d < R) {
      starts[d] = run;
      run += __ldcg(totals + d);
    }
  }
  if (tid == 0) *done = 0u;
}

// ---------------------------------------------------------------- min/max ---
// Min and max of every column's transformed value.  out[2j] = min, out[2j+1] = max.
__global__ void __launch_bounds__(256) k_minmax(PackDesc pd, u64 n, u64* out) {
  u64 mn[kMaxCols], mx[kMaxCols];
#pragma unroll
  for (int j = 0; j < kMaxCols; ++j) {
    mn[j] = ~0ull;
    mx[j] = 0ull;
  }
  const u64 stride = (u64)gridDim.x * blockDim.x;
  constexpr int U = 8;
  if (pd.ncols == 1) {
    for (u64 r0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += stride * U) {
      u64 raw[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const u64 r = r0 + (u64)u * stride;
        raw[u] = r < n ? load_raw(pd.c[0].ptr, pd.c[0].dtype, r) : 0ull;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (r0 + (u64)u * stride >= n) break;
        const u64 t = transform_raw(pd.c[0], raw[u]);
        mn[0] = t < mn[0] ? t : mn[0];
        mx[0] = t > mx[0] ? t : mx[0];
      }
    }
  } else {
    for (u64 r0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += stride * 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const u64 r = r0 + (u64)u * stride;
        if (r >= n) break;
#pragma unroll
        for (int j = 0; j < kMaxCols; ++j) {
          if (j >= pd.ncols) break;
          const u64 t = load_t(pd.c[j], r);
          mn[j] = t < mn[j] ? t : mn[j];
          mx[j] = t > mx[j] ? t : mx[j];
        }
      }
    }
  }
  // warp, then block reduction: one pair of global atomics per block and
  // column (every block hits the same two words, so they serialise in L2)
  __shared__ u64 smn[kMaxCols][8], smx[kMaxCols][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kMaxCols; ++j) {
    if (j >= pd.ncols) break;
    u64 a = mn[j], b = mx[j];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const u64 a2 = __shfl_xor_sync(0xffffffffu, a, o);
      const u64 b2 = __shfl_xor_sync(0xffffffffu, b, o);
      a = a2 < a ? a2 : a;
      b = b2 > b ? b2 : b;
    }
    if (lane == 0) {
      smn[j][warp] = a;
      smx[j][warp] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < pd.ncols) {
    const int j = threadIdx.x;
    u64 a = smn[j][0], b = smx[j][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      a = smn[j][w] < a ? smn[j][w] : a;
      b = smx[j][w] > b ? smx[j][w] : b;
    }
    atomicMin(&out[2 * j], a);
    atomicMax(&out[2 * j + 1], b);
  }
}

// Min/max of one plain 32/64-bit integer column's transformed value (the
// sign flip is the whole transform), T its storage type.
template <typename T>
__global__ void __launch_bounds__(256) k_minmax_int(const T* col, u64 n, u64 flip, u64* out) {
  u64 mn = ~0ull, mx = 0ull;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  constexpr int U = 8;
  for (u64 r0 = (u64)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += stride * U) {
    T raw[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const u64 r = r0 + (u64)u * stride;
      raw[u] = r < n ? __ldg(col + r) : (T)0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (r0 + (u64)u * stride >= n) break;
      const u64 t = (u64)raw[u] ^ flip;
      mn = t < mn ? t : mn;
      mx = t > mx ? t : mx;
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const u64 a2 = __shfl_xor_sync(0xffffffffu, mn, o);
    const u64 b2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mn = a2 < mn ? a2 : mn;
    mx = b2 > mx ? b2 : mx;
  }
  __shared__ u64 smn[8], smx[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smn[warp] = mn;
    smx[warp] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      mn = smn[w] < mn ? smn[w] : mn;
      mx = smx[w] > mx ? smx[w] : mx;
    }
    atomicMin(&out[0], mn);
    atomicMax(&out[1], mx);
  }
}

// k_minmax_int that also counts, per 2048-row tile, the low byte of every
// value (digit-major [256][tiles]).  Once the minimum is known, the first
// 8-bit radix pass's tile counts are these counts rotated by the minimum's
// low byte (the packed key is value - min, and the sign flip leaves the low
// byte alone), so that pass needs no separate counting read of the column.
constexpr int kPreTile = 2048;
template <typename T>
__global__ void __launch_bounds__(256) k_minmax_int_tiles(const T* col, u64 n, u64 flip, u64* out, u32* counts,
                                                          u64 tiles) {
  constexpr int NH = 8, IPT = kPreTile / 256;  // one histogram per warp
  __shared__ u32 h[NH][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < NH * 256; i += 256) (&h[0][0])[i] = 0u;
  __syncthreads();
  u64 mn = ~0ull, mx = 0ull;
  for (u64 t = blockIdx.x; t < tiles; t += gridDim.x) {
    const u64 base = t * kPreTile;
    const u32 tn = (u32)min((u64)kPreTile, n - base);
    T raw[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      const u32 r = i * 256 + tid;
      raw[i] = r < tn ? __ldg(col + base + r) : (T)0;
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
      if (i * 256 + tid >= tn) break;
      const u64 v = (u64)raw[i] ^ flip;
      mn = v < mn ? v : mn;
      mx = v > mx ? v : mx;
      atomicAdd(&h[warp][(u32)raw[i] & 255u], 1u);
    }
    __syncthreads();
    u32 c = 0;
#pragma unroll
    for (int q = 0; q < NH; ++q) {
      c += h[q][tid];
      h[q][tid] = 0u;
    }
    counts[(u64)tid * tiles + t] = c;
    __syncthreads();
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const u64 a2 = __shfl_xor_sync(0xffffffffu, mn, o);
    const u64 b2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mn = a2 < mn ? a2 : mn;
    mx = b2 > mx ? b2 : mx;
  }
  __shared__ u64 smn[8], smx[8];
  if (lane == 0) {
    smn[warp] = mn;
    smx[warp] = mx;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < 8; ++w) {
      mn = smn[w] < mn ? smn[w] : mn;
      mx = smx[w] > mx ? smx[w] : mx;
    }
    atomicMin((unsigned long long*)&out[0], (unsigned long long)mn);
    atomicMax((unsigned long long*)&out[1], (unsigned long long)mx);
  }
}

__global__ void k_init_minmax(u64* out, int ncols) {
  int j = threadIdx.x;
  if (j < ncols) {
    out[2 * j] = ~0ull;
    out[2 * j + 1] = 0ull;
  }
}

__global__ void k_iota(u32* out, u64 n, int reverse) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    out[i] = reverse ? (u32)(n - 1 - i) : (u32)i;
}

template <typename K>
__global__ void k_fill_keys(K* out, u64 n) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    out[i] = (K)0;
}

// ----------------------------------------------------------- host driver ---
// Thread-local tuning (jfx_set_tuning): widest radix digit of a pass.
struct Tuning {
  int max_digit_bits = 8;
  int two_phase = 1;  // later radix passes: counts + scan, no look-back
  int spin_limit_us = (int)(kSpinLimitNs / 1000);
};
extern thread_local Tuning g_tuning;

// Thread-local failure injection (jfx_set_fault).
struct Fault {
  int withhold_tile = 0;
  int learned_fallback = 0;
  int fail_workspace = 0;
  int withhold_order = 0;
};
extern thread_local Fault g_fault;

// The workspace check of every entry point (fail_workspace forces a failure).
inline int check_workspace(const Arena& ar, const void* workspace, size_t bytes) {
  if (ar.overflow || !workspace || g_fault.fail_workspace)
    return fail(JFX_ERR_ALLOC, "workspace of %zu bytes < %zu needed%s", bytes, ar.off,
                g_fault.fail_workspace ? " (failure injected by jfx_set_fault)" : "");
  // the carve hands out 256-byte offsets and kernels load 16-byte vectors
  // from them, so the base must be aligned as cudaMalloc returns it
  if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
    return fail(JFX_ERR_ARG, "workspace %p is not 256-byte aligned", workspace);
  return JFX_OK;
}

// Pinned host scratch for the few words an entry point reads back.
struct HostScratch {
  u64* p = nullptr;
  ~HostScratch() {
    if (p) cudaFreeHost(p);
  }
  u64* get() {
    if (!p && cudaMallocHost((void**)&p, 4096) != cudaSuccess) p = nullptr;
    return p;
  }
};
extern thread_local HostScratch g_host;

// Column ranges -> packing (shift/bits per column, most significant first).
struct KeyPlan {
  PackDesc pack;
  int total_bits = 0;
  u64 tmax[kMaxCols];
  const u32* pre_counts = nullptr;  // low-byte tile counts of the min/max pass, if written
};

// Fill `cols` from jfx_column descriptors (validates dtypes).
inline int build_pack(const jfx_column* in, int ncols, u32 extra_flags, bool allow_desc, PackDesc& pd) {
  if (ncols < 1 || ncols > kMaxCols) return fail(JFX_ERR_ARG, "1..%d key columns supported, got %d", kMaxCols, ncols);
  memset(&pd, 0, sizeof pd);
  pd.ncols = ncols;
  for (int j = 0; j < ncols; ++j) {
    if (!in[j].data) return fail(JFX_ERR_ARG, "key column %d has a null pointer", j);
    if (dtype_size(in[j].dtype) == 0) return fail(JFX_ERR_DTYPE, "key column %d: unsupported dtype %d", j, in[j].dtype);
    pd.c[j].ptr = in[j].data;
    pd.c[j].dtype = in[j].dtype;
    pd.c[j].flags = extra_flags | ((allow_desc && (in[j].flags & JFX_COL_DESC)) ? CF_DESC : 0u);
    if ((pd.c[j].flags & CF_DESC) && in[j].dtype == JFX_BOOL)
      return fail(JFX_ERR_DTYPE, "descending bool key (max(x) - x) is not defined for bool");
    if (dtype_is_float(in[j].dtype)) pd.nan_cols |= 1 << j;
  }
  return JFX_OK;
}

// tile_counts (optional, [256][ceil(n / 2048)] words): for one plain integer
// key column, also the low-byte counts of k_minmax_int_tiles; *counted says
// whether they were written.
inline int launch_minmax(const PackDesc& pd, u64 n, u64* dev_out, cudaStream_t s, u32* tile_counts = nullptr,
                         bool* counted = nullptr) {
  if (counted) *counted = false;
  k_init_minmax<<<1, 32, 0, s>>>(dev_out, pd.ncols), note_launch();
  if (n) {
    int grid = (int)std::min<u64>((n + 255) / 256, (u64)device_sm_count() * 8);
    const int d0 = pd.c[0].dtype;
    const bool int_key = pd.ncols == 1 && !(pd.c[0].flags & CF_DESC) &&
                         (d0 == JFX_I32 || d0 == JFX_I64 || d0 == JFX_U32 || d0 == JFX_U64);
    const u64 flip = d0 == JFX_I64 ? 0x8000000000000000ull : d0 == JFX_I32 ? 0x80000000ull : 0ull;
    bool all_int = true;  // every column a plain integer one: one specialised launch per column
    for (int j = 0; j < pd.ncols; ++j) {
      const int dt = pd.c[j].dtype;
      all_int &= !(pd.c[j].flags & CF_DESC) && (dt == JFX_I32 || dt == JFX_I64 || dt == JFX_U32 || dt == JFX_U64);
    }
    if (int_key && tile_counts) {
      const u64 tiles = (n + kPreTile - 1) / kPreTile;
      const int tg = (int)std::min<u64>(tiles, (u64)device_sm_count() * 8);
      if (d0 == JFX_I64 || d0 == JFX_U64)
        k_minmax_int_tiles<u64><<<tg, 256, 0, s>>>((const u64*)pd.c[0].ptr, n, flip, dev_out, tile_counts, tiles),
            note_launch();
      else
        k_minmax_int_tiles<u32><<<tg, 256, 0, s>>>((const u32*)pd.c[0].ptr, n, flip, dev_out, tile_counts, tiles),
            note_launch();
      if (counted) *counted = true;
    } else if (int_key && (d0 == JFX_I64 || d0 == JFX_U64))
      k_minmax_int<u64><<<grid, 256, 0, s>>>((const u64*)pd.c[0].ptr, n, flip, dev_out), note_launch();
    else if (int_key)
      k_minmax_int<u32><<<grid, 256, 0, s>>>((const u32*)pd.c[0].ptr, n, flip, dev_out), note_launch();
    else if (all_int && pd.ncols <= 4) {
      for (int j = 0; j < pd.ncols; ++j) {
        const int dt = pd.c[j].dtype;
        const u64 fj = dt == JFX_I64 ? 0x8000000000000000ull : dt == JFX_I32 ? 0x80000000ull : 0ull;
        if (dtype_size(dt) == 8)
          k_minmax_int<u64><<<grid, 256, 0, s>>>((const u64*)pd.c[j].ptr, n, fj, dev_out + 2 * j), note_launch();
        else
          k_minmax_int<u32><<<grid, 256, 0, s>>>((const u32*)pd.c[j].ptr, n, fj, dev_out + 2 * j), note_launch();
      }
    } else
      k_minmax<<<grid, 256, 0, s>>>(pd, n, dev_out), note_launch();
  }
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

// Computes min/max of every key column (two reductions when an integer column
// is descending: max(x) first, then the rewritten values) and assigns the bit
// fields.  One stream synchronisation.
// host: 2 * ncols words of host memory for the read-back (null: the pinned
// per-thread buffer).
// tile_counts: optional [256][ceil(n / 2048)] words for the low-byte tile
// counts of a plain integer key column (kp.pre_counts is set when written).
inline int plan_keys(KeyPlan& kp, u64 n, u64* dev_scratch, cudaStream_t s, u64* host = nullptr,
                     u32* tile_counts = nullptr) {
  PackDesc& pd = kp.pack;
  if (!host) host = g_host.get();
  if (!host) return fail(JFX_ERR_CUDA, "cudaMallocHost failed");
  bool need_raw_max = false;
  for (int j = 0; j < pd.ncols; ++j)
    if ((pd.c[j].flags & CF_DESC) && !dtype_is_float(pd.c[j].dtype)) need_raw_max = true;
  if (need_raw_max && n) {
    PackDesc raw = pd;
    for (int j = 0; j < raw.ncols; ++j) raw.c[j].flags &= ~(CF_DESC | CF_QUIRK);
    JFX_TRY(launch_minmax(raw, n, dev_scratch, s));
    JFX_CUDA(cudaMemcpyAsync(host, dev_scratch, 2 * pd.ncols * sizeof(u64), cudaMemcpyDeviceToHost, s));
    JFX_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < pd.ncols; ++j)
      if ((pd.c[j].flags & CF_DESC) && !dtype_is_float(pd.c[j].dtype)) {
        u64 raw_max = untransform_int(pd.c[j].dtype, 0, host[2 * j + 1]);
        // sign-extend narrow signed types so (short)desc_max is the max value
        pd.c[j].desc_max = raw_max;
      }
  }
  bool counted = false;
  JFX_TRY(launch_minmax(pd, n, dev_scratch, s, tile_counts, &counted));
  kp.pre_counts = counted ? tile_counts : nullptr;
  JFX_CUDA(cudaMemcpyAsync(host, dev_scratch, 2 * pd.ncols * sizeof(u64), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaStreamSynchronize(s));
  int shift = 0;
  kp.total_bits = 0;
  for (int j = pd.ncols - 1; j >= 0; --j) {
    ColDesc& c = pd.c[j];
    u64 mn = host[2 * j], mx = host[2 * j + 1];
    if (n == 0) mn = mx = 0;
    c.tmin = mn;
    kp.tmax[j] = mx;
    c.bits = bit_length(mx - mn);
    c.shift = shift;
    shift += c.bits;
  }
  kp.total_bits = shift;
  return JFX_OK;
}

// Workspace of one radix sort of n rows (worst case: 64-bit keys).
struct SortBuffers {
  void* keys[2];   // ping-pong packed keys
  u32* vals[2][kMaxWords];  // ping-pong payload words (word 0: row ids by default)
  int words = 1;
  u32* hist;       // [8][2048]
  u32* base;       // [8][2048]
  u32* counters;   // [8]
  u32* status[2];  // [tiles][RADIX] ping-pong look-back words
  u64 status_words;
  u32* totals;     // [2048] digit totals of the current two-phase pass
  u32* starts;     // [2048] their exclusive scan: global start of each digit
};

inline u64 max_status_words(u64 n) {
  // the largest tiles x RADIX over the kernel configurations used
  u64 w8 = (u64)ceil_div(n ? n : 1, PassLayout<u64, 8>::TILE) * 256;
  u64 w9 = (u64)ceil_div(n ? n : 1, PassLayout<u64, 9>::TILE) * 512;
  u64 w10 = (u64)ceil_div(n ? n : 1, PassLayout<u64, 10>::TILE) * 1024;
  u64 w11 = (u64)ceil_div(n ? n : 1, PassLayout<u64, 11>::TILE) * 2048;
  return std::max(std::max(w8, w9), std::max(w10, w11));
}

inline int launch_tile_scan(int radix, const u32* counts, u64 tiles, const u32* bin_base, u32* base, u32* totals,
                            u32* starts, u32* done, cudaStream_t s, u32 rot = 0) {
  static SmemAttr attr;
  if (tiles >= 32768) JFX_TRY(ensure_smem(attr, k_tile_scan<1024>, tile_scan_smem<1024>()));
  if (tiles >= 32768)
    k_tile_scan<1024><<<radix, 1024, tile_scan_smem<1024>(), s>>>(counts, tiles, bin_base, base, totals, starts, done,
                                                                rot), note_launch();
  else
    k_tile_scan<256><<<radix, 256, tile_scan_smem<256>(), s>>>(counts, tiles, bin_base, base, totals, starts, done,
                                                              rot), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

inline void take_sort_buffers(Arena& ar, u64 n, SortBuffers& b, int words = 1) {
  b.keys[0] = ar.take<u64>(n ? n : 1);
  b.keys[1] = ar.take<u64>(n ? n : 1);
  b.words = words;
  for (int w = 0; w < kMaxWords; ++w) {
    b.vals[0][w] = w < words ? ar.take<u32>(n ? n : 1) : nullptr;
    b.vals[1][w] = w < words ? ar.take<u32>(n ? n : 1) : nullptr;
  }
  b.hist = ar.take<u32>(8 * 2048);
  b.base = ar.take<u32>(8 * 2048);
  b.counters = ar.take<u32>(64);
  b.status_words = max_status_words(n);
  b.status[0] = ar.take<u32>(b.status_words);
  b.status[1] = ar.take<u32>(b.status_words);
  b.totals = ar.take<u32>(2048);
  b.starts = ar.take<u32>(2048);
}

template <typename K, int RB, int FM, int NW = 1, bool TP = false>
inline int launch_pass(const PassArgs& a, u64 n, cudaStream_t s, u64 grid_tiles = 0) {
  constexpr bool FIRST = FM != 0;
  using L = PassLayout<K, RB, NW>;
  if (TP && (!a.tile_base || a.digit_mode != DIG_BITS))
    return fail(JFX_ERR_ARG, "two-phase pass without tile bases or with non-bit digits");
  static SmemAttr attr;  // per instantiation
  JFX_TRY(ensure_smem(attr, k_onesweep<K, RB, FM, NW, TP>, L::SMEM));
  int tiles = grid_tiles ? (int)grid_tiles : ceil_div(n, L::TILE);
  PassArgs pa = a;
  pa.spin_ns = (u64)g_tuning.spin_limit_us * 1000ull;
  pa.withhold_tile = g_fault.withhold_tile > 0 ? (u32)g_fault.withhold_tile : kNoTile;
  const long t = timing_begin(s);
  k_onesweep<K, RB, FM, NW, TP><<<tiles, L::THREADS, L::SMEM, s>>>(pa), note_launch();
  if (t >= 0) {
    // algorithmic bytes: the first pass reads the key columns and writes
    // key + row id; later passes read and write key + row id
    double kraw = 0;
    if (FIRST) {
      for (int j = 0; j < a.pack.ncols; ++j) kraw += dtype_size(a.pack.c[j].dtype);
      if (a.gather_idx) kraw += 4;
    }
    const double per = FIRST ? kraw + sizeof(K) + 4.0 * NW : 2.0 * (sizeof(K) + 4.0 * NW);
    timing_end(t, s, per * (double)n);
  }
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

struct RadixRequest {
  PackDesc pack;
  int key_mode = KEY_PACK;
  int digit_mode = DIG_BITS;
  u32 modulus = 0;
  int total_bits = 0;        // packed key width (DIG_BITS)
  int max_digit_bits = g_tuning.max_digit_bits;  // widest digit allowed
  bool reverse = false;      // descending: write n-1-p in the last pass
  const u32* gather_idx = nullptr;
  u32* targets = nullptr;    // hash partition: digit of each row (row order)
  u32* perm_out = nullptr;   // sorted row ids (payload word 0 unless vout_final is set)
  int nwords = 1;            // payload words carried (1..4)
  PayloadSrc pfirst[kMaxWords] = {};  // first-pass payload sources (null ptr: row id)
  u32* vout_final[kMaxWords] = {};    // sorted payload words (word 0 defaults to perm_out)
  void* keys_out = nullptr;  // sorted packed keys (K), may be null -> internal buffer
  bool key64 = false;        // packed key type
  void* keys_result = nullptr; // filled: where the sorted packed keys ended up
  int npass = 0;               // filled: passes run
  // optional: the last pass writes the original integer key (single column)
  // instead of the packed key
  void* raw_out = nullptr;
  int raw_dtype = 0;
  u32 raw_flags = 0;
  u64 raw_tmin = 0;
  const ModelRef* model = nullptr;  // DIG_MODEL / KEY_MODEL
  unsigned long long* vout64 = nullptr;  // last pass: words 0 and 1 as one u64
  // optional: low-byte counts of the single integer key column per 2048-row
  // tile (k_minmax_int_tiles), used for the first pass when it has 8-bit
  // digits over 2048-row tiles instead of counting the column again
  const u32* pre_counts = nullptr;
};

template <typename K, int RB, int NW>
inline int run_radix(RadixRequest& rq, u64 n, SortBuffers& b, u32* err, cudaStream_t s) {
  constexpr int RADIX = 1 << RB;
  if (NW > b.words) return fail(JFX_ERR_ARG, "sort buffers hold %d payload words, %d requested", b.words, NW);
  int npass;
  int shift[8] = {0}, width[8] = {0};
  if (rq.digit_mode == DIG_MOD) {
    npass = 1;
    width[0] = RB;
  } else {
    npass = ceil_div(rq.total_bits, rq.max_digit_bits);
    if (npass > 8) return fail(JFX_ERR_ARG, "too many radix passes");
    int base_w = rq.total_bits / npass, rem = rq.total_bits % npass, at = 0;
    for (int p = 0; p < npass; ++p) {
      width[p] = base_w + (p < rem ? 1 : 0);
      shift[p] = at;
      at += width[p];
    }
  }
  rq.npass = npass;
  JFX_CUDA(cudaMemsetAsync(b.hist, 0, (size_t)npass * RADIX * sizeof(u32), s));
  JFX_CUDA(cudaMemsetAsync(b.counters, 0, 64 * sizeof(u32), s));
  const u64 tiles = (u64)ceil_div(n, PassLayout<K, RB, NW>::TILE);
  JFX_CUDA(cudaMemsetAsync(b.status[0], 0, tiles * RADIX * sizeof(u32), s));

  // the passes after the first of a plain digit sort run in two phases (no
  // look-back); the first pass too when the histogram kernel can count its
  // tiles (one plain integer key column)
  const bool two_phase = rq.digit_mode == DIG_BITS && g_tuning.two_phase && tiles >= 2;
  const int d0 = rq.pack.c[0].dtype, d1 = rq.pack.ncols > 1 ? rq.pack.c[1].dtype : 0;
  auto plain_int = [](int dt) { return dt == JFX_I32 || dt == JFX_I64 || dt == JFX_U32 || dt == JFX_U64; };
  // one plain integer key column, or two of the same width
  const bool int_key = (rq.pack.ncols == 1 || (rq.pack.ncols == 2 && plain_int(d1) && dtype_size(d1) == dtype_size(d0) &&
                                               !(rq.pack.c[1].flags & CF_DESC))) &&
                       rq.key_mode == KEY_PACK && rq.digit_mode == DIG_BITS && !rq.targets &&
                       !(rq.pack.c[0].flags & CF_DESC) && plain_int(d0);
  // (a gathered first pass reads its tiles in another order than the column)
  const bool first_two_phase = two_phase && int_key && !rq.gather_idx;
  // the first pass's tile counts from the min/max pass (one column, 8-bit
  // first digit at bit 0, 2048-row tiles): no counting kernel at all
  const bool pre = rq.pre_counts && first_two_phase && RB == 8 && (int)PassLayout<K, RB, NW>::TILE == kPreTile &&
                   rq.pack.ncols == 1 && rq.pack.c[0].shift == 0 && npass >= 1 && width[0] == 8;
  // the first pass's lean instantiation: one or two plain integer columns of
  // one width, read in order
  const bool int1 = int_key && !rq.gather_idx;

  HistArgs h;
  memset(&h, 0, sizeof h);
  h.pack = rq.pack;
  h.hist = b.hist;
  h.targets = rq.targets;
  h.n = n;
  h.npass = npass;
  h.key_mode = rq.key_mode;
  h.digit_mode = rq.digit_mode;
  h.modulus = rq.modulus;
  h.model = rq.model;
  for (int p = 0; p < 8; ++p) {
    h.shift[p] = shift[p];
    h.width[p] = width[p];
  }
  {
    int grid = (int)std::min<u64>((n + 1023) / 1024, (u64)device_sm_count() * 4);
    size_t smem = (size_t)npass * RADIX * sizeof(u32);
    static SmemAttr a_hist, a_hist64, a_hist32;
    JFX_TRY(ensure_smem(a_hist, k_hist<K, RB>, 8 * 2048 * 4));
    JFX_TRY(ensure_smem(a_hist64, k_hist_int<K, u64, RB>, 9 * 2048 * 4));
    JFX_TRY(ensure_smem(a_hist32, k_hist_int<K, u32, RB>, 9 * 2048 * 4));
    if (int_key) {
      HistIntArgs hi;
      memset(&hi, 0, sizeof hi);
      hi.col = rq.pack.c[0].ptr;
      hi.hist = b.hist;
      hi.n = n;
      hi.flip = d0 == JFX_I64 ? 0x8000000000000000ull : d0 == JFX_I32 ? 0x80000000ull : 0ull;
      hi.tmin = rq.pack.c[0].tmin;
      hi.kshift = rq.pack.c[0].shift;
      if (rq.pack.ncols == 2) {
        hi.col2 = rq.pack.c[1].ptr;
        hi.flip2 = d1 == JFX_I64 ? 0x8000000000000000ull : d1 == JFX_I32 ? 0x80000000ull : 0ull;
        hi.tmin2 = rq.pack.c[1].tmin;
        hi.kshift2 = rq.pack.c[1].shift;
      }
      hi.npass = first_two_phase ? 0 : npass;  // two-phase passes take their digit starts from the tile counts
      for (int p = 0; p < 8; ++p) {
        hi.shift[p] = shift[p];
        hi.mask[p] = width[p] >= 32 ? 0xffffffffu : ((1u << width[p]) - 1u);
      }
      int g = std::max(grid, 1);
      size_t sm = smem;
      if (first_two_phase) {
        hi.tile_counts = b.status[1];
        hi.tiles = tiles;
        hi.tile_rows = (u32)PassLayout<K, RB, NW>::TILE;
        g = (int)std::min<u64>(tiles, (u64)device_sm_count() * 8);
        sm += (size_t)RADIX * sizeof(u32);
      }
      if (pre) {
        // counted by the min/max pass
      } else if (d0 == JFX_I64 || d0 == JFX_U64)
        k_hist_int<K, u64, RB><<<g, 256, sm, s>>>(hi), note_launch();
      else
        k_hist_int<K, u32, RB><<<g, 256, sm, s>>>(hi), note_launch();
    } else {
      k_hist<K, RB><<<std::max(grid, 1), 256, smem, s>>>(h), note_launch();
    }
    JFX_CUDA(cudaGetLastError());
  }
  if (!first_two_phase) {
    k_hist_scan<RB><<<npass, 1024, 0, s>>>(b.hist, b.base), note_launch();
    JFX_CUDA(cudaGetLastError());
  }

  if (first_two_phase) {
    if (pre)
      JFX_TRY(launch_tile_scan(RADIX, rq.pre_counts, tiles, nullptr, b.status[0], b.totals, b.starts, b.counters + 63, s,
                               (u32)(rq.pack.c[0].tmin & 255u)));
    else
      JFX_TRY(launch_tile_scan(RADIX, b.status[1], tiles, nullptr, b.status[0], b.totals, b.starts, b.counters + 63, s));
    JFX_CUDA(cudaGetLastError());
  }
  u32* out_vals[kMaxWords];
  for (int w = 0; w < kMaxWords; ++w) out_vals[w] = rq.vout_final[w];
  if (!out_vals[0]) out_vals[0] = rq.perm_out;
  void* out_keys = rq.keys_out ? rq.keys_out : b.keys[(npass - 1) & 1];
  for (int p = 0; p < npass; ++p) {
    PassArgs a;
    memset(&a, 0, sizeof a);
    const bool last = p == npass - 1;
    a.keys_in = p ? b.keys[(p - 1) & 1] : nullptr;
    a.keys_out = last ? out_keys : b.keys[p & 1];
    for (int w = 0; w < NW; ++w) {
      a.vin[w] = p ? b.vals[(p - 1) & 1][w] : nullptr;
      a.vout[w] = last ? out_vals[w] : b.vals[p & 1][w];
      a.pfirst[w] = rq.pfirst[w];
    }
    a.bin_base = b.base + (u64)p * RADIX;
    a.status = b.status[p & 1];
    a.status_next = last ? nullptr : b.status[(p + 1) & 1];
    a.tile_counter = b.counters + p;
    a.err = err;
    a.gather_idx = rq.gather_idx;
    a.n = n;
    a.shift = shift[p];
    a.width = width[p];
    a.key_mode = rq.key_mode;
    a.digit_mode = rq.digit_mode;
    a.modulus = rq.modulus;
    a.model = rq.model;
    a.vout64 = last ? rq.vout64 : nullptr;
    a.reverse = last && rq.reverse;
    if (last && rq.raw_out) {
      a.raw_out = rq.raw_out;
      a.raw_dtype = rq.raw_dtype;
      a.raw_flags = rq.raw_flags;
      a.raw_tmin = rq.raw_tmin;
    }
    a.pack = rq.pack;
    if (two_phase && p > 0) {
      // status[1] holds this pass's tile counts, status[0] its tile bases
      // (pass 0, the only look-back pass, is done with both by now)
      const u32 mask_p = width[p] >= 32 ? 0xffffffffu : ((1u << width[p]) - 1u);
      k_tile_count<K, RB, NW><<<(unsigned)tiles, 256, 0, s>>>((const K*)a.keys_in, n, shift[p], mask_p, b.status[1],
                                                           tiles), note_launch();
      JFX_TRY(launch_tile_scan(RADIX, b.status[1], tiles, nullptr, b.status[0], b.totals, b.starts, b.counters + 63,
                               s));
      JFX_CUDA(cudaGetLastError());
      a.tile_base = b.status[0];
      a.digit_starts = b.starts;
      a.ntiles = tiles;
      a.status = nullptr;
      a.status_next = nullptr;
    }
    if (two_phase && p == 0) a.status_next = nullptr;
    if (first_two_phase && p == 0) {
      a.tile_base = b.status[0];
      a.digit_starts = b.starts;
      a.ntiles = tiles;
      a.status = nullptr;
    }
    const bool tp = a.tile_base != nullptr;  // two-phase (plain bit digits)
    if (p == 0 && int1) {
      JFX_TRY(tp ? (launch_pass<K, RB, 1, NW, true>(a, n, s)) : (launch_pass<K, RB, 1, NW, false>(a, n, s)));
    } else if (p == 0) {
      JFX_TRY(tp ? (launch_pass<K, RB, 2, NW, true>(a, n, s)) : (launch_pass<K, RB, 2, NW, false>(a, n, s)));
    } else {
      JFX_TRY(tp ? (launch_pass<K, RB, 0, NW, true>(a, n, s)) : (launch_pass<K, RB, 0, NW, false>(a, n, s)));
    }
  }
  rq.keys_result = out_keys;
  return JFX_OK;
}

template <typename K>
inline int run_radix_k(RadixRequest& rq, u64 n, SortBuffers& b, u32* err, cudaStream_t s) {
  // payload-carrying sorts use 8- to 10-bit digits (shared memory for the
  // staged words leaves no room for wider histograms); 9 and 10 save a pass
  // for keys of 25..30 bits
  if (rq.nwords > 1 && rq.digit_mode == DIG_BITS) rq.max_digit_bits = 10;
  int rb;
  if (rq.digit_mode == DIG_MOD) {
    rb = rq.modulus <= 256 ? 8 : rq.modulus <= 512 ? 9 : rq.modulus <= 1024 ? 10 : 11;
  } else {
    int npass = ceil_div(rq.total_bits, rq.max_digit_bits);
    int w = ceil_div(rq.total_bits, npass);
    rb = w <= 8 ? 8 : w;
  }
  if (rq.nwords > 1) {
    if (rb > 10) return fail(JFX_ERR_ARG, "digit width %d with payload words unsupported", rb);
    switch (rq.nwords * 16 + rb) {
      case 2 * 16 + 8: return run_radix<K, 8, 2>(rq, n, b, err, s);
      case 3 * 16 + 8: return run_radix<K, 8, 3>(rq, n, b, err, s);
      case 4 * 16 + 8: return run_radix<K, 8, 4>(rq, n, b, err, s);
      case 2 * 16 + 9: return run_radix<K, 9, 2>(rq, n, b, err, s);
      case 3 * 16 + 9: return run_radix<K, 9, 3>(rq, n, b, err, s);
      case 4 * 16 + 9: return run_radix<K, 9, 4>(rq, n, b, err, s);
      case 2 * 16 + 10: return run_radix<K, 10, 2>(rq, n, b, err, s);
      case 3 * 16 + 10: return run_radix<K, 10, 3>(rq, n, b, err, s);
      case 4 * 16 + 10: return run_radix<K, 10, 4>(rq, n, b, err, s);
    }
    return fail(JFX_ERR_ARG, "1..4 payload words supported");
  }
  switch (rb) {
    case 8: return run_radix<K, 8, 1>(rq, n, b, err, s);
    case 9: return run_radix<K, 9, 1>(rq, n, b, err, s);
    case 10: return run_radix<K, 10, 1>(rq, n, b, err, s);
    case 11: return run_radix<K, 11, 1>(rq, n, b, err, s);
  }
  return fail(JFX_ERR_ARG, "digit width %d unsupported", rb);
}

// Sorts rows by the packed key (or hash digit).  n >= 1.  With total_bits == 0
// (every key equal) the stable order is the identity.
inline int radix_sort(RadixRequest& rq, u64 n, SortBuffers& b, u32* err, cudaStream_t s) {
  if (n > (u64)kMaxRows) return fail(JFX_ERR_CAPACITY, "%llu rows exceed the %lld-row limit", n, (long long)kMaxRows);
  if (rq.digit_mode == DIG_BITS && rq.total_bits == 0) {
    int grid = (int)std::min<u64>((n + 255) / 256, 4096);
    if (rq.nwords > 1 || rq.pfirst[0].ptr || rq.reverse && rq.nwords > 1)
      return fail(JFX_ERR_ARG, "constant keys with a payload: carry it with total_bits >= 1");
    k_iota<<<std::max(grid, 1), 256, 0, s>>>(rq.perm_out, n, rq.reverse ? 1 : 0), note_launch();
    void* out_keys = rq.keys_out ? rq.keys_out : b.keys[0];
    if (rq.key64) k_fill_keys<u64><<<std::max(grid, 1), 256, 0, s>>>((u64*)out_keys, n), note_launch();
    else k_fill_keys<u32><<<std::max(grid, 1), 256, 0, s>>>((u32*)out_keys, n), note_launch();
    JFX_CUDA(cudaGetLastError());
    rq.keys_result = out_keys;
    rq.npass = 0;
    return JFX_OK;
  }
  if (rq.key64) return run_radix_k<u64>(rq, n, b, err, s);
  return run_radix_k<u32>(rq, n, b, err, s);
}

}  // namespace jfx
