// api.cu -- extern "C" entry points of libjfx (declared in include/jfx.h).
#include "join.cuh"
#include "learned.cuh"
#include "batch.cuh"

namespace jfx {

thread_local std::string g_last_error;
thread_local HostScratch g_host;
std::atomic<unsigned long long> g_launches{0};
thread_local Tuning g_tuning;
thread_local Fault g_fault;
Timing g_timing;

int device_sm_count() {
  static int cache[128] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 128) return 148;
  if (!cache[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cache[dev] = v;
  }
  return cache[dev];
}

static inline cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

static inline int grid_for(u64 n, int threads) {
  u64 g = (n + threads - 1) / threads;
  u64 cap = (u64)device_sm_count() * 16;
  return (int)std::max<u64>(1, std::min(g, cap));
}

// Copies the device error word (and up to 3 more words) back, synchronising
// the stream once, and converts device error bits into a status.
static int read_back(const void* dev, size_t bytes, u64* host, cudaStream_t s) {
  JFX_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaStreamSynchronize(s));
  return JFX_OK;
}

static int check_err_word(u32 e) {
  if (e & DERR_TIMEOUT)
    return fail(JFX_ERR_TIMEOUT, "a device-side wait exceeded its limit (decoupled look-back)");
  if (e & DERR_BOUNDS) return fail(JFX_ERR_ARG, "a device-side bounds check failed");
  return JFX_OK;
}

// Header shared by every entry point: error word + min/max scratch + readback.
struct Common {
  u32* err;
  u64* mm;    // [4 * kMaxCols]
  u64* words; // [8] values read back by the host
};
static void take_common(Arena& ar, Common& c) {
  c.err = ar.take<u32>(64);
  c.mm = ar.take<u64>(4 * kMaxCols);
  c.words = ar.take<u64>(8);
}

template <typename K>
__global__ void k_unpack(const K* sk, u64 n, int dtype, u32 flags, u64 tmin, void* out) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    store_raw(out, dtype, i, untransform_int(dtype, flags, (u64)sk[i] + tmin));
}

// out[i] = src[idx[i]] over one array of n rows.  An index outside [0, n)
// (only after a failed pass, which the call reports) reads nothing.
__global__ void k_gather_same(const void* src, int dt, const u32* idx, u64 n, void* out) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u32 r = idx[i];
    store_raw(out, dt, i, r < n ? load_raw(src, dt, r) : 0ull);
  }
}

// ------------------------------------------------------------------ sort ---
static void carve_sort(Arena& ar, u64 n, Common& c, SortBuffers& b) {
  take_common(ar, c);
  take_sort_buffers(ar, n, b);
}

// ---------------------------------------------------------------- lexsort ---
static void carve_lexsort(Arena& ar, u64 n, Common& c, SortBuffers& b, u32** tmp) {
  carve_sort(ar, n, c, b);
  *tmp = ar.take<u32>(n ? n : 1);
}

// ---------------------------------------------------------------- groupby ---
struct GroupBuffers {
  void* sk;
  u32* perm;
  u32* words[kMaxWords];  // sorted payload words when values are carried
  u32* warp_count;
  u32* warp_base;
  u32* partial;
  u32* total;
  u32* slot_gid;
  u32* slot_started;
  u64* slot_state;
  u64 nwarps;
};
static void take_group_buffers(Arena& ar, u64 n, int nvals, GroupBuffers& g) {
  g.nwarps = (n + 32 * kGroupIPT - 1) / (32 * kGroupIPT);
  g.warp_count = ar.take<u32>(g.nwarps + 1);
  g.warp_base = ar.take<u32>(g.nwarps + 1);
  g.partial = ar.take<u32>(scan_partials_count(g.nwarps));
  g.total = ar.take<u32>(4);
  g.slot_gid = ar.take<u32>(2 * g.nwarps + 1);
  g.slot_started = ar.take<u32>(2 * g.nwarps + 1);
  g.slot_state = ar.take<u64>((u64)std::max(nvals, 1) * 4 * (2 * g.nwarps + 1));
}
static void carve_groupby(Arena& ar, u64 n, int nvals, Common& c, SortBuffers& b, GroupBuffers& g) {
  take_common(ar, c);
  take_sort_buffers(ar, n, b, kMaxWords);
  g.sk = ar.take<u64>(n ? n : 1);
  g.perm = ar.take<u32>(n ? n : 1);
  for (int w = 0; w < kMaxWords; ++w) g.words[w] = ar.take<u32>(n ? n : 1);
  take_group_buffers(ar, n, nvals, g);
}

// Group boundaries and counts, the scan of the per-warp counts, the
// lane-sequential segmented reduction and the fix-up of groups that span
// warps (groupby.cuh).  n >= 1.
template <typename K>
static int launch_group_reduce(GroupArgs& ga, GroupBuffers& g, u64 n, cudaStream_t s) {
  ga.slot_gid = g.slot_gid;
  ga.slot_started = g.slot_started;
  ga.slot_state = g.slot_state;
  ga.nslots = 2 * g.nwarps;
  const unsigned blocks = (unsigned)((g.nwarps * 32 + 255) / 256);
  k_group_count<K><<<blocks, 256, 0, s>>>(ga, g.nwarps), note_launch();
  JFX_CUDA(cudaGetLastError());
  JFX_TRY(device_exclusive_scan<u32>(g.warp_count, g.nwarps, g.warp_base, g.total, g.partial, s));
  JFX_CUDA(cudaMemsetAsync(g.slot_gid, 0xff, ga.nslots * sizeof(u32), s));
  k_group_reduce<K><<<blocks, 256, 0, s>>>(ga, g.nwarps), note_launch();
  JFX_CUDA(cudaGetLastError());
  const u64 fix_blocks = std::min<u64>((ga.nslots + 255) / 256, (u64)device_sm_count() * 16);
  k_group_fixup<<<(unsigned)std::max<u64>(fix_blocks, 1), 256, 0, s>>>(ga), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

// ------------------------------------------------------------------- join ---
struct JoinPlan {
  u64 magic;
  int how;
  int key64;
  int ncols;
  int reverse_counted;  // counts with the sides swapped exist (lo2/cnt2)
  int unique;           // inner join, every A row matches exactly once: output i = sorted A row i
  int carried[2];       // words carried through the left / right sort (0: that side sorted row ids)
  u32* cw[2][kMaxWords];
  int npay;             // payload list given to prepare: side, dtype and first carried word
  int pay_side[kMaxJoinPayloads], pay_dtype[kMaxJoinPayloads], pay_word[kMaxJoinPayloads];
  u64 nl, nr, m;
  u64 unmatched[2];     // rows without a match: [0] left, [1] right
  void* skL;
  void* skR;
  u32* pL;
  u32* pR;
  u32* lo;
  u32* cnt;
  u32* lo2;
  u32* cnt2;
  u64* off;
  u32* flag;
  u32* foff;
  u32* fpart;
  u32* ftotal;
  u64* win;
  u64 win_cap;  // tiles the window buffer holds
  ColDesc lc[kMaxCols];
  ColDesc rc[kMaxCols];
};
static_assert(sizeof(JoinPlan) <= sizeof(jfx_join_plan), "join plan does not fit");
constexpr u64 kJoinMagic = 0x6a66786a6f696e32ull;

struct JoinBuffers {
  void *skL, *skR;
  u32 *pL, *pR, *lo, *cnt, *lo2, *cnt2, *flag, *foff, *fpart, *ftotal;
  u64 *off, *partial, *total, *win, *stats;
  u32* cw[2][kMaxWords];  // carried payload words of each side, sorted order
};
// b: the left side's sort buffers, br the right side's (the two sorts run
// on two streams at once).
static void carve_join(Arena& ar, u64 nl, u64 nr, Common& c, SortBuffers& b, SortBuffers& br, JoinBuffers& j) {
  take_common(ar, c);
  u64 nmax = std::max(nl, nr);
  take_sort_buffers(ar, nl, b, kMaxWords);
  take_sort_buffers(ar, nr, br, kMaxWords);
  j.skL = ar.take<u64>(nl ? nl : 1);
  j.skR = ar.take<u64>(nr ? nr : 1);
  j.pL = ar.take<u32>(nl ? nl : 1);
  j.pR = ar.take<u32>(nr ? nr : 1);
  j.lo = ar.take<u32>(nmax ? nmax : 1);
  j.cnt = ar.take<u32>(nmax ? nmax : 1);
  j.lo2 = ar.take<u32>(nmax ? nmax : 1);
  j.cnt2 = ar.take<u32>(nmax ? nmax : 1);
  j.off = ar.take<u64>(nmax ? nmax : 1);
  j.partial = ar.take<u64>(scan_partials_count(nmax));
  j.total = ar.take<u64>(4);
  j.flag = ar.take<u32>(nmax ? nmax : 1);
  j.foff = ar.take<u32>(nmax ? nmax : 1);
  j.fpart = ar.take<u32>(scan_partials_count(nmax));
  j.ftotal = ar.take<u32>(4);
  j.win = ar.take<u64>(2 * ((nmax + kJoinTile - 1) / kJoinTile + 1));
  j.stats = ar.take<u64>(2 * kJoinStatSlots);
  for (int w = 0; w < kMaxWords; ++w) {
    j.cw[0][w] = ar.take<u32>(nl ? nl : 1);
    j.cw[1][w] = ar.take<u32>(nr ? nr : 1);
  }
}

template <typename K>
// stats (optional): kJoinStatSlots (sum, max) pairs of the counts; zeroed here.
static int launch_join_count(const void* A, u64 na, const void* B, u64 nb, u32* lo, u32* cnt, const PackDesc& pd,
                             u64* win, cudaStream_t s, unsigned long long* stats = nullptr) {
  if (stats) JFX_CUDA(cudaMemsetAsync(stats, 0, 2 * kJoinStatSlots * sizeof(unsigned long long), s));
  if (!na) return JFX_OK;
  if (!nb) {
    JFX_CUDA(cudaMemsetAsync(cnt, 0, na * sizeof(u32), s));
    JFX_CUDA(cudaMemsetAsync(lo, 0, na * sizeof(u32), s));
    return JFX_OK;
  }
  const unsigned blocks = (unsigned)((na + kJoinTile - 1) / kJoinTile);
  k_join_windows<K><<<(blocks + 7) / 8, 256, 0, s>>>((const K*)A, na, (const K*)B, nb, blocks, win), note_launch();
  k_join_count<K><<<blocks, kJoinThreads, 0, s>>>((const K*)A, na, (const K*)B, nb, win, lo, cnt, pd, stats), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

// ---------------------------------------------------------------- learned ---
struct LearnedBuffers {
  u32* pos;   // bucket of each key (predicted position >> kBucketShift), in row order
  u32* spos;  // the buckets in sorted order
  u64* sample;
  u64* ssorted;
  u32* sperm;
  double* acc;
  ModelRef* model;
  Leaf* leaves;
  u32* first;
  u32* last;
  double* fit;
  u32* flags;   // [0] model check passed
  u32* starts;  // [buckets + 1]
  u32* large;   // [kBucketLargeMax][2]
  u32* bcounts; // [0] large buckets
  u32* chunks;  // [cap_chunks][3] min/max chunks of the large buckets
  u64* mm;      // [kBucketLargeMax][2] their min and max
  u32* cspans;  // [kBucketLargeMax][2] large buckets for k_bucket_sort_large
  u64* cmins;
  u32* cbits;
  u64 cap_chunks;
  u64* tkeys;   // scratch of the large-bucket sorts
  u32* tids;
  u64 s, nb;
};
static void carve_learned(Arena& ar, u64 n, Common& c, SortBuffers& b, LearnedBuffers& l) {
  take_common(ar, c);
  take_sort_buffers(ar, n, b, 3);
  l.pos = ar.take<u32>(n ? n : 1);
  l.spos = ar.take<u32>(n ? n : 1);
  l.s = n / kSampleStride;
  l.sample = ar.take<u64>(l.s + 1);
  l.ssorted = ar.take<u64>(l.s + 1);
  l.sperm = ar.take<u32>(l.s + 1);
  l.acc = ar.take<double>(8);
  l.model = ar.take<ModelRef>(1);
  l.leaves = ar.take<Leaf>(kLeaves);
  l.first = ar.take<u32>(kLeaves);
  l.last = ar.take<u32>(kLeaves);
  l.fit = ar.take<double>(2 * kLeaves);
  l.flags = ar.take<u32>(8);
  l.nb = n ? ((4 * n - 1) >> kBucketShift) + 1 : 1;  // positions lie in [0, 4n)
  l.starts = ar.take<u32>(l.nb + 1);
  l.large = ar.take<u32>(2 * kBucketLargeMax);
  l.cap_chunks = n / kLargeChunk + kBucketLargeMax + 1;
  l.chunks = ar.take<u32>(3 * l.cap_chunks);
  l.mm = ar.take<u64>(2 * kBucketLargeMax);
  l.cspans = ar.take<u32>(2 * kBucketLargeMax);
  l.cmins = ar.take<u64>(kBucketLargeMax);
  l.cbits = ar.take<u32>(kBucketLargeMax);
  l.bcounts = ar.take<u32>(8);
  l.tkeys = ar.take<u64>(n ? n : 1);
  l.tids = ar.take<u32>(n ? n : 1);
}

// Plain radix sort of raw uint64 keys: sorted keys and row ids.
static int plain_sort_u64(const u64* keys, u64 n, u64* sorted_out, u32* perm_out, SortBuffers& b, Common& c,
                          cudaStream_t s) {
  jfx_column col{keys, JFX_U64, 0u};
  PackDesc pd;
  JFX_TRY(build_pack(&col, 1, 0u, false, pd));
  KeyPlan kp;
  kp.pack = pd;
  JFX_TRY(plan_keys(kp, n, c.mm, s, nullptr, b.status[1]));
  RadixRequest rq;
  rq.pack = kp.pack;
  rq.total_bits = kp.total_bits;
  rq.key64 = kp.total_bits > 32;
  rq.perm_out = perm_out;
  rq.pre_counts = kp.pre_counts;
  if (kp.total_bits > 0) {
    rq.raw_out = sorted_out;
    rq.raw_dtype = JFX_U64;
    rq.raw_tmin = kp.pack.c[0].tmin;
  }
  JFX_TRY(radix_sort(rq, n, b, c.err, s));
  if (kp.total_bits == 0) JFX_CUDA(cudaMemcpyAsync(sorted_out, keys, n * 8, cudaMemcpyDeviceToDevice, s));
  return JFX_OK;
}

// Stable sort of the rows [0, m) of (keys, ids) by key (one large bucket of
// the learned sort): the plain radix sort over the rows' key range, the ids
// carried as the payload, through the scratch arrays and back.
static int sort_rows_u64(u64* keys, u32* ids, u64 m, u64 kmin, int bits, u64* tkeys, u32* tids, SortBuffers& b,
                         Common& c, cudaStream_t s) {
  jfx_column col{keys, JFX_U64, 0u};
  KeyPlan kp;
  JFX_TRY(build_pack(&col, 1, 0u, false, kp.pack));
  kp.pack.c[0].tmin = kmin;  // the rows' key range is known
  kp.pack.c[0].bits = bits;
  kp.pack.c[0].shift = 0;
  kp.total_bits = bits;
  if (kp.total_bits == 0) return JFX_OK;  // one key: the rows are in row order already
  RadixRequest rq;
  rq.pack = kp.pack;
  rq.total_bits = kp.total_bits;
  rq.key64 = kp.total_bits > 32;
  rq.nwords = 1;
  rq.pfirst[0] = PayloadSrc{(const unsigned char*)ids, 4u, 0u};
  rq.vout_final[0] = tids;
  rq.raw_out = tkeys;
  rq.raw_dtype = JFX_U64;
  rq.raw_tmin = kp.pack.c[0].tmin;
  JFX_TRY(radix_sort(rq, m, b, c.err, s));
  JFX_CUDA(cudaMemcpyAsync(keys, tkeys, m * 8, cudaMemcpyDeviceToDevice, s));
  JFX_CUDA(cudaMemcpyAsync(ids, tids, m * 4, cudaMemcpyDeviceToDevice, s));
  return JFX_OK;
}

// ------------------------------------------------------------------ batch ---
struct BatchBuffers {
  u32* sk[2];
  u32* sv[2];
  u32* tkeys;
  double* tsums;
  u32* tcnts;
  u32* qgroups;
  u32* order;
  u32* ctl;
};

static void carve_batch(Arena& ar, u64 n, u64 nq, Common& c, BatchBuffers& b) {
  take_common(ar, c);  // the error word opens the workspace (jfx_batch_status)
  const u64 nn = n ? n : 1;
  for (int i = 0; i < 2; ++i) {
    b.sk[i] = ar.take<u32>(nn);
    b.sv[i] = ar.take<u32>(nn);
  }
  b.tkeys = ar.take<u32>(nn);
  b.tsums = ar.take<double>(nn);
  b.tcnts = ar.take<u32>(nn);
  b.qgroups = ar.take<u32>(nq + 1);
  b.order = ar.take<u32>(nq + 1);
  b.ctl = ar.take<u32>(64);
}

// -------------------------------------------------------------- partition ---
static void carve_partition(Arena& ar, u64 n, Common& c, SortBuffers& b) { carve_sort(ar, n, c, b); }

static int check_n(int64_t n) {
  if (n < 0) return fail(JFX_ERR_ARG, "negative row count %lld", (long long)n);
  if (n > kMaxRows) return fail(JFX_ERR_CAPACITY, "%lld rows exceed the %lld-row limit", (long long)n, (long long)kMaxRows);
  return JFX_OK;
}


// A second stream (and two events) per host thread and device, created on
// first use, so that independent sorts of one call can overlap.
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
static int side_stream(SideStream** out) {
  thread_local SideStream per_dev[128];
  int dev = -1;
  JFX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(JFX_ERR_ARG, "device ordinal %d out of range", dev);
  SideStream& ss = per_dev[dev];
  if (!ss.stream) {
    JFX_CUDA(cudaStreamCreateWithFlags(&ss.stream, cudaStreamNonBlocking));
    JFX_CUDA(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming));
    JFX_CUDA(cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming));
  }
  *out = &ss;
  return JFX_OK;
}

// ------------------------------------------------ sort without allocation ---
// Scratch of jfx_sort_static: a fixed device array in this library instead of
// a caller workspace.  Every device that loads the library holds it until the
// process exits.  It is sized for the sort buffers of kStaticSortMaxRows rows
// (64-bit keys, the widest digit configuration); jfx_sort_static checks that
// the carve fits before it launches anything.
constexpr int64_t kStaticSortMaxRows = JFX_SORT_STATIC_MAX_ROWS;
constexpr size_t kStaticSortScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_static_sort_scratch[kStaticSortScratchBytes];

// Device address of g_static_sort_scratch on the current device.  In host
// code the array's name is only a host-side stand-in for the symbol, so the
// address is looked up once per device (with that device current) and
// cached; the lookup may load this library's device code on that device.
static int static_sort_scratch(void** out) {
  static std::mutex mu;
  static void* addr[128] = {nullptr};
  int dev = -1;
  JFX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(JFX_ERR_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_sort_scratch);
    if (e != cudaSuccess || !p)
      return fail(JFX_ERR_CUDA, "cudaGetSymbolAddress of the static sort scratch failed on device %d: %s", dev,
                  cudaGetErrorString(e));
    addr[dev] = p;
  }
  *out = addr[dev];
  return JFX_OK;
}

}  // namespace jfx

using namespace jfx;

extern "C" {

const char* jfx_last_error(void) { return g_last_error.c_str(); }

uint64_t jfx_launch_count(void) { return g_launches.load(); }

int jfx_set_tuning(const jfx_tuning* t) {
  if (!t) {
    g_tuning = Tuning();
    return JFX_OK;
  }
  if (t->max_digit_bits < 8 || t->max_digit_bits > 11)
    return fail(JFX_ERR_ARG, "max_digit_bits must be in [8, 11], got %d", t->max_digit_bits);
  if (t->two_phase != 0 && t->two_phase != 1) return fail(JFX_ERR_ARG, "two_phase must be 0 or 1, got %d", t->two_phase);
  if (t->spin_limit_us < 1 || t->spin_limit_us > 10000000)
    return fail(JFX_ERR_ARG, "spin_limit_us must be in [1, 10^7], got %d", t->spin_limit_us);
  g_tuning.max_digit_bits = t->max_digit_bits;
  g_tuning.two_phase = t->two_phase;
  g_tuning.spin_limit_us = t->spin_limit_us;
  return JFX_OK;
}

int jfx_get_tuning(jfx_tuning* t) {
  if (!t) return fail(JFX_ERR_ARG, "null pointer");
  t->max_digit_bits = g_tuning.max_digit_bits;
  t->two_phase = g_tuning.two_phase;
  t->spin_limit_us = g_tuning.spin_limit_us;
  t->reserved = 0;
  return JFX_OK;
}

int jfx_set_fault(const jfx_fault* f) {
  if (!f) {
    g_fault = Fault();
    return JFX_OK;
  }
  if (f->withhold_tile < 0) return fail(JFX_ERR_ARG, "withhold_tile must be >= 0, got %d", f->withhold_tile);
  if (f->learned_fallback != 0 && f->learned_fallback != -1 && f->learned_fallback != -3)
    return fail(JFX_ERR_ARG, "learned_fallback must be 0, -1 or -3, got %d", f->learned_fallback);
  if (f->fail_workspace != 0 && f->fail_workspace != 1)
    return fail(JFX_ERR_ARG, "fail_workspace must be 0 or 1, got %d", f->fail_workspace);
  if (f->withhold_order != 0 && f->withhold_order != 1)
    return fail(JFX_ERR_ARG, "withhold_order must be 0 or 1, got %d", f->withhold_order);
  g_fault.withhold_tile = f->withhold_tile;
  g_fault.learned_fallback = f->learned_fallback;
  g_fault.fail_workspace = f->fail_workspace;
  g_fault.withhold_order = f->withhold_order;
  return JFX_OK;
}

int jfx_timing_enable(int enable) {
  std::lock_guard<std::mutex> lk(g_timing.mu);
  for (auto& r : g_timing.recs) {
    g_timing.pool.push_back(r.start);
    g_timing.pool.push_back(r.stop);
  }
  g_timing.recs.clear();
  g_timing.on = enable != 0;
  return JFX_OK;
}

int jfx_timing_read(double* total_ms, int64_t* launches, double* algo_bytes) {
  std::lock_guard<std::mutex> lk(g_timing.mu);
  double ms = 0, bytes = 0;
  for (auto& r : g_timing.recs) {
    JFX_CUDA(cudaEventSynchronize(r.stop));
    float e = 0;
    JFX_CUDA(cudaEventElapsedTime(&e, r.start, r.stop));
    ms += e;
    bytes += r.bytes;
  }
  if (total_ms) *total_ms = ms;
  if (launches) *launches = (int64_t)g_timing.recs.size();
  if (algo_bytes) *algo_bytes = bytes;
  return JFX_OK;
}
int jfx_version(void) { return 2; }
int jfx_max_rows(void) { return (int)kMaxRows; }

size_t jfx_workspace_size(int kind, int64_t n1, int64_t n2) {
  Arena ar(nullptr, ~size_t(0));
  Common c;
  SortBuffers b;
  u64 a = n1 > 0 ? (u64)n1 : 0, bn = n2 > 0 ? (u64)n2 : 0;
  switch (kind) {
    case JFX_WS_SORT: {
      u32* tmp;
      carve_lexsort(ar, a, c, b, &tmp);
      break;
    }
    case JFX_WS_GROUPBY: {
      GroupBuffers g;
      carve_groupby(ar, a, kMaxVals, c, b, g);
      break;
    }
    case JFX_WS_JOIN: {
      JoinBuffers j;
      SortBuffers br;
      carve_join(ar, a, bn, c, b, br, j);
      break;
    }
    case JFX_WS_PARTITION:
      carve_partition(ar, a, c, b);
      break;
    case JFX_WS_LEARNED: {
      LearnedBuffers l;
      carve_learned(ar, a, c, b, l);
      break;
    }
    case JFX_WS_BATCH: {
      BatchBuffers bb;
      carve_batch(ar, a, bn, c, bb);
      break;
    }
    default:
      return 0;
  }
  return ar.off + 256;
}

int jfx_sort(const jfx_column* key, int64_t n, int ascending, int32_t* perm_out, void* sorted_keys_out,
             void* workspace, size_t workspace_bytes, void* stream) {
  JFX_TRY(check_n(n));
  if (!key || !perm_out) return fail(JFX_ERR_ARG, "null key or permutation pointer");
  if (n == 0) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  PackDesc pd;
  JFX_TRY(build_pack(key, 1, CF_QUIRK, false, pd));
  if (key->dtype == JFX_BOOL) return fail(JFX_ERR_DTYPE, "ParallelRadixSort cannot shift a bool key");
  Arena ar(workspace, workspace_bytes);
  Common c;
  SortBuffers b;
  carve_sort(ar, (u64)n, c, b);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  KeyPlan kp;
  kp.pack = pd;
  JFX_TRY(plan_keys(kp, (u64)n, c.mm, s, nullptr, b.status[1]));
  RadixRequest rq;
  rq.pack = kp.pack;
  rq.total_bits = kp.total_bits;
  rq.key64 = kp.total_bits > 32;
  rq.reverse = !ascending;
  rq.perm_out = (u32*)perm_out;
  rq.pre_counts = kp.pre_counts;
  const bool int_keys = !dtype_is_float(key->dtype);
  if (sorted_keys_out && int_keys && kp.total_bits > 0) {
    rq.raw_out = sorted_keys_out;
    rq.raw_dtype = key->dtype;
    rq.raw_flags = CF_QUIRK;
    rq.raw_tmin = kp.pack.c[0].tmin;
  }
  JFX_TRY(radix_sort(rq, (u64)n, b, c.err, s));
  if (sorted_keys_out && !(int_keys && kp.total_bits > 0)) {
    const int g = grid_for((u64)n, 256);
    if (dtype_is_float(key->dtype)) {
      k_gather_same<<<g, 256, 0, s>>>(key->data, key->dtype, (const u32*)perm_out, (u64)n, sorted_keys_out), note_launch();
    } else if (rq.key64) {
      k_unpack<u64><<<g, 256, 0, s>>>((const u64*)rq.keys_result, (u64)n, key->dtype, CF_QUIRK, kp.pack.c[0].tmin, sorted_keys_out), note_launch();
    } else {
      k_unpack<u32><<<g, 256, 0, s>>>((const u32*)rq.keys_result, (u64)n, key->dtype, CF_QUIRK, kp.pack.c[0].tmin, sorted_keys_out), note_launch();
    }
    JFX_CUDA(cudaGetLastError());
  }
  u64* host = g_host.get();
  JFX_TRY(read_back(c.err, sizeof(u32), host, s));
  return check_err_word((u32)host[0]);
}

// jfx_sort without a workspace argument: the scratch is g_static_sort_scratch.
// Callers that cannot allocate device memory use it: code that runs inside a
// memory-pool or allocator callback (allocating there would re-enter the
// allocator), loops that must not take cudaMalloc's implicit device-wide
// synchronisation, and host frameworks that own all device memory and hand a
// plugin only its input and output buffers.  Nothing here allocates: no
// cudaMalloc / cudaFree, no pinned host buffer (read-backs go to the stack),
// no library allocator.  The first call on a device looks up the scratch
// address (static_sort_scratch), so make it before any stream capture.  Every
// call shares the one array and finds the previous call's data there: the
// error word, the digit histograms, the tile counter and the first pass's
// look-back words are cleared on the stream before use (the rest is written
// before it is read).  Calls whose work overlaps on the GPU -- two streams, or
// two host threads -- race on the array and must be serialised by the caller.
int jfx_sort_static(const jfx_column* key, int64_t n, int ascending, int32_t* perm_out, void* sorted_keys_out,
                    void* stream) {
  JFX_TRY(check_n(n));
  if (n > kStaticSortMaxRows)
    return fail(JFX_ERR_CAPACITY, "jfx_sort_static takes at most %lld rows (got %lld): its scratch is a fixed "
                "%zu-byte device array; use jfx_sort with a workspace for more", (long long)kStaticSortMaxRows,
                (long long)n, kStaticSortScratchBytes);
  if (!key || !perm_out) return fail(JFX_ERR_ARG, "null key or permutation pointer");
  if (n == 0) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  PackDesc pd;
  JFX_TRY(build_pack(key, 1, CF_QUIRK, false, pd));
  if (key->dtype == JFX_BOOL) return fail(JFX_ERR_DTYPE, "ParallelRadixSort cannot shift a bool key");
  void* scratch = nullptr;
  JFX_TRY(static_sort_scratch(&scratch));
  Arena ar(scratch, kStaticSortScratchBytes);
  Common c;
  SortBuffers b;
  carve_sort(ar, (u64)n, c, b);
  if (ar.overflow) return fail(JFX_ERR_ALLOC, "static sort scratch of %zu bytes < %zu needed", kStaticSortScratchBytes, ar.off);
  u64 host[2 * kMaxCols];  // read-back words (pageable: no pinned buffer is allocated)
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  KeyPlan kp;
  kp.pack = pd;
  JFX_TRY(plan_keys(kp, (u64)n, c.mm, s, host));
  RadixRequest rq;
  rq.pack = kp.pack;
  rq.total_bits = kp.total_bits;
  rq.key64 = kp.total_bits > 32;
  rq.reverse = !ascending;
  rq.perm_out = (u32*)perm_out;
  const bool int_keys = !dtype_is_float(key->dtype);
  if (sorted_keys_out && int_keys && kp.total_bits > 0) {
    rq.raw_out = sorted_keys_out;
    rq.raw_dtype = key->dtype;
    rq.raw_flags = CF_QUIRK;
    rq.raw_tmin = kp.pack.c[0].tmin;
  }
  JFX_TRY(radix_sort(rq, (u64)n, b, c.err, s));
  if (sorted_keys_out && !(int_keys && kp.total_bits > 0)) {
    const int g = grid_for((u64)n, 256);
    if (dtype_is_float(key->dtype)) {
      k_gather_same<<<g, 256, 0, s>>>(key->data, key->dtype, (const u32*)perm_out, (u64)n, sorted_keys_out), note_launch();
    } else if (rq.key64) {
      k_unpack<u64><<<g, 256, 0, s>>>((const u64*)rq.keys_result, (u64)n, key->dtype, CF_QUIRK, kp.pack.c[0].tmin, sorted_keys_out), note_launch();
    } else {
      k_unpack<u32><<<g, 256, 0, s>>>((const u32*)rq.keys_result, (u64)n, key->dtype, CF_QUIRK, kp.pack.c[0].tmin, sorted_keys_out), note_launch();
    }
    JFX_CUDA(cudaGetLastError());
  }
  JFX_TRY(read_back(c.err, sizeof(u32), host, s));
  return check_err_word((u32)host[0]);
}

int jfx_lexsort(const jfx_column* keys, int ncols, int64_t n, int32_t* perm_out, void* workspace,
                size_t workspace_bytes, void* stream) {
  JFX_TRY(check_n(n));
  if (!keys || !perm_out) return fail(JFX_ERR_ARG, "null keys or permutation pointer");
  if (n == 0) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  PackDesc pd;
  // one key: plain stable ascending argsort, `ascending` ignored (line 44-45)
  JFX_TRY(build_pack(keys, ncols, 0u, ncols > 1, pd));
  Arena ar(workspace, workspace_bytes);
  Common c;
  SortBuffers b;
  u32* tmp;
  carve_lexsort(ar, (u64)n, c, b, &tmp);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  KeyPlan kp;
  kp.pack = pd;
  JFX_TRY(plan_keys(kp, (u64)n, c.mm, s));
  if (kp.total_bits <= 64) {
    RadixRequest rq;
    rq.pack = kp.pack;
    rq.total_bits = kp.total_bits;
    rq.key64 = kp.total_bits > 32;
    rq.perm_out = (u32*)perm_out;
    JFX_TRY(radix_sort(rq, (u64)n, b, c.err, s));
  } else {
    // LSD over groups of columns whose packed width fits 64 bits, last group
    // first; later rounds read their columns through the current order.
    int groups[kMaxCols + 1], ng = 0;
    int end = pd.ncols;
    while (end > 0) {
      int bits = 0, start = end;
      while (start > 0 && bits + kp.pack.c[start - 1].bits <= 64) {
        bits += kp.pack.c[start - 1].bits;
        --start;
      }
      groups[ng++] = start;
      end = start;
    }
    // groups[r] = first column of round r; round r covers [groups[r], prev_end)
    u32* bufs[2] = {(u32*)perm_out, tmp};
    int prev_end = pd.ncols;
    const u32* gather = nullptr;
    for (int r = 0; r < ng; ++r) {
      int start = groups[r];
      RadixRequest rq;
      memset(&rq.pack, 0, sizeof rq.pack);
      rq.pack.ncols = prev_end - start;
      int shift = 0;
      for (int j = prev_end - 1; j >= start; --j) {
        ColDesc cd = kp.pack.c[j];
        cd.shift = shift;
        shift += cd.bits;
        rq.pack.c[j - start] = cd;
      }
      rq.total_bits = shift;
      rq.key64 = shift > 32;
      rq.gather_idx = gather;
      u32* out = bufs[(ng - 1 - r) & 1];
      rq.perm_out = out;
      if (shift == 0) {
        if (!gather) {
          k_iota<<<grid_for((u64)n, 256), 256, 0, s>>>(out, (u64)n, 0), note_launch();
        } else {
          JFX_CUDA(cudaMemcpyAsync(out, gather, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
        }
      } else {
        JFX_TRY(radix_sort(rq, (u64)n, b, c.err, s));
      }
      gather = out;
      prev_end = start;
    }
  }
  u64* host = g_host.get();
  JFX_TRY(read_back(c.err, sizeof(u32), host, s));
  return check_err_word((u32)host[0]);
}

int jfx_groupby(const jfx_column* keys, int ncols, int64_t n, int multi_key, const jfx_agg_column* values,
                int nvalues, void* const* unique_out, int64_t* num_groups, void* workspace, size_t workspace_bytes,
                void* stream) {
  JFX_TRY(check_n(n));
  if (!keys || !num_groups) return fail(JFX_ERR_ARG, "null keys or num_groups pointer");
  if (nvalues < 0 || nvalues > kMaxVals) return fail(JFX_ERR_ARG, "0..%d value columns supported", kMaxVals);
  if (!multi_key && ncols != 1) return fail(JFX_ERR_ARG, "single-key groupby takes one key column");
  *num_groups = 0;
  if (n == 0) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  PackDesc pd;
  JFX_TRY(build_pack(keys, ncols, multi_key ? 0u : CF_QUIRK, false, pd));
  if (!multi_key && keys[0].dtype == JFX_BOOL) return fail(JFX_ERR_DTYPE, "ParallelRadixSort cannot shift a bool key");
  GroupArgs ga;
  memset(&ga, 0, sizeof ga);
  ga.nvals = nvalues;
  for (int i = 0; i < nvalues; ++i) {
    const jfx_agg_column& v = values[i];
    ValDesc& d = ga.v[i];
    if (!v.data) return fail(JFX_ERR_ARG, "value column %d has a null pointer", i);
    if (dtype_size(v.dtype) == 0) return fail(JFX_ERR_DTYPE, "value column %d: unsupported dtype", i);
    if (v.aggs & ~31u) return fail(JFX_ERR_ARG, "value column %d: unknown aggregation bits 0x%x", i, v.aggs);
    d.ptr = v.data;
    d.dtype = v.dtype;
    d.kind = dtype_is_float(v.dtype) ? VK_F : dtype_is_signed_int(v.dtype) ? VK_I : VK_U;
    d.aggs = v.aggs;
    d.mean_dtype = v.mean_dtype;
    d.count_dtype = v.count_dtype;
    d.count_via_f32 = multi_key ? 1 : 0;
    d.out_sum = v.out_sum;
    d.out_mean = v.out_mean;
    d.out_count = v.out_count;
    d.out_min = v.out_min;
    d.out_max = v.out_max;
    if (((v.aggs & JFX_AGG_SUM) && !v.out_sum) || ((v.aggs & JFX_AGG_MEAN) && !v.out_mean) ||
        ((v.aggs & JFX_AGG_COUNT) && !v.out_count) || ((v.aggs & JFX_AGG_MIN) && !v.out_min) ||
        ((v.aggs & JFX_AGG_MAX) && !v.out_max))
      return fail(JFX_ERR_ARG, "value column %d: missing output pointer", i);
    if ((v.aggs & JFX_AGG_MEAN) && v.mean_dtype != JFX_F32 && v.mean_dtype != JFX_F64)
      return fail(JFX_ERR_DTYPE, "value column %d: mean dtype must be float32 or float64", i);
    if ((v.aggs & JFX_AGG_COUNT) && dtype_size(v.count_dtype) == 0)
      return fail(JFX_ERR_DTYPE, "value column %d: bad count dtype", i);
  }
  Arena ar(workspace, workspace_bytes);
  Common c;
  SortBuffers b;
  GroupBuffers g;
  carve_groupby(ar, (u64)n, nvalues, c, b, g);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  KeyPlan kp;
  kp.pack = pd;
  JFX_TRY(plan_keys(kp, (u64)n, c.mm, s));
  if (kp.total_bits > 64)
    return fail(JFX_ERR_CAPACITY, "group keys need %d packed bits; at most 64 are supported", kp.total_bits);
  // Carry the value columns through the sort when they fit in the payload
  // words (4- and 8-byte values, plus the row id when a key is a float):
  // the reduce then reads them in sorted order instead of gathering.
  int words = kp.pack.nan_cols ? 1 : 0;
  bool carry = true;
  for (int i = 0; i < nvalues; ++i) {
    const int sz = dtype_size(values[i].dtype);
    if (sz < 4) carry = false;
    words += sz == 8 ? 2 : 1;
  }
  if (words > kMaxWords || nvalues == 0) carry = false;
  RadixRequest rq;
  rq.pack = kp.pack;
  rq.total_bits = kp.total_bits;
  rq.key64 = kp.total_bits > 32;
  rq.perm_out = g.perm;
  rq.keys_out = g.sk;
  int rowid_word = -1;
  if (carry) {
    rq.total_bits = std::max(1, kp.total_bits);  // one pass even for constant keys
    int w = 0;
    for (int i = 0; i < nvalues; ++i) {
      const int sz = dtype_size(values[i].dtype);
      ValDesc& d = ga.v[i];
      d.carried = 1;
      rq.pfirst[w] = PayloadSrc{(const unsigned char*)values[i].data, (u32)sz, 0u};
      rq.vout_final[w] = g.words[w];
      d.ptr = g.words[w++];
      if (sz == 8) {
        rq.pfirst[w] = PayloadSrc{(const unsigned char*)values[i].data, 8u, 4u};
        rq.vout_final[w] = g.words[w];
        d.ptr_hi = g.words[w++];
      }
    }
    if (kp.pack.nan_cols) {
      rowid_word = w;
      rq.pfirst[w] = PayloadSrc{nullptr, 0u, 0u};
      rq.vout_final[w] = g.words[w];
      ++w;
    }
    rq.nwords = w;
  }
  JFX_TRY(radix_sort(rq, (u64)n, b, c.err, s));

  ga.skeys = g.sk;
  ga.perm = carry ? (rowid_word >= 0 ? g.words[rowid_word] : nullptr) : g.perm;
  ga.values_sorted = carry ? 1 : 0;
  ga.n = (u64)n;
  ga.warp_count = g.warp_count;
  ga.warp_base = g.warp_base;
  ga.pack = kp.pack;
  for (int j = 0; j < ncols; ++j) ga.uniq_out[j] = unique_out ? unique_out[j] : nullptr;
  if (rq.key64) JFX_TRY(launch_group_reduce<u64>(ga, g, (u64)n, s));
  else JFX_TRY(launch_group_reduce<u32>(ga, g, (u64)n, s));
  u64* host = g_host.get();
  JFX_CUDA(cudaMemcpyAsync(host, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaMemcpyAsync(host + 1, g.total, sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaStreamSynchronize(s));
  JFX_TRY(check_err_word((u32)host[0]));
  *num_groups = (int64_t)(u32)host[1];
  return JFX_OK;
}

}  // extern "C"

// Shared body of jfx_join_prepare (no payloads) and jfx_join_prepare_payloads.
static int join_prepare(const jfx_column* left_keys, int64_t nl, const jfx_column* right_keys, int64_t nr,
                        int ncols, int how, const jfx_join_payload* payloads, int npayloads, jfx_join_plan* plan_out,
                        int64_t* num_out, void* workspace, size_t workspace_bytes, void* stream) {
  JFX_TRY(check_n(nl));
  JFX_TRY(check_n(nr));
  if (!left_keys || !right_keys || !plan_out || !num_out) return fail(JFX_ERR_ARG, "null argument");
  if (ncols < 1 || ncols > kMaxCols) return fail(JFX_ERR_ARG, "1..%d join key columns supported", kMaxCols);
  for (int c = 0; c < ncols; ++c) {
    if (left_keys[c].dtype != right_keys[c].dtype)
      return fail(JFX_ERR_DTYPE, "join key %d: left and right dtypes differ (%d, %d)", c, left_keys[c].dtype,
                  right_keys[c].dtype);
    if (ncols == 1 && left_keys[c].dtype == JFX_BOOL)
      return fail(JFX_ERR_DTYPE, "ParallelRadixSort cannot shift a bool key");
  }
  if (how < JFX_JOIN_INNER || how > JFX_JOIN_OUTER) return fail(JFX_ERR_ARG, "unknown join kind %d", how);
  cudaStream_t s = as_stream(stream);
  Arena ar(workspace, workspace_bytes);
  Common c;
  SortBuffers b, br;
  JoinBuffers j;
  carve_join(ar, (u64)nl, (u64)nr, c, b, br, j);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  // a single key is sorted by ParallelRadixSort (narrow ints keep the
  // reference's unsigned order); several keys are compared for equality only
  const u32 flags = ncols == 1 ? CF_QUIRK : 0u;
  PackDesc pl, pr;
  JFX_TRY(build_pack(left_keys, ncols, flags, false, pl));
  JFX_TRY(build_pack(right_keys, ncols, flags, false, pr));
  // shared packing: min and max of every column over both sides
  // (the sides' first-pass tile counts are left to their sorts, which run on
  // two streams: counting them here, before the fork, lengthened the join)
  // the right side's min/max runs on the side stream beside the left's
  SideStream* mss = nullptr;
  cudaStream_t sm2 = s;
  if (nl && nr) {
    JFX_TRY(side_stream(&mss));
    sm2 = mss->stream;
    JFX_CUDA(cudaEventRecord(mss->fork, s));
    JFX_CUDA(cudaStreamWaitEvent(sm2, mss->fork, 0));
  }
  JFX_TRY(launch_minmax(pl, (u64)nl, c.mm, s));
  JFX_TRY(launch_minmax(pr, (u64)nr, c.mm + 2 * kMaxCols, sm2));
  if (mss) {
    JFX_CUDA(cudaEventRecord(mss->join, sm2));
    JFX_CUDA(cudaStreamWaitEvent(s, mss->join, 0));
  }
  u64* host = g_host.get();
  JFX_TRY(read_back(c.mm, 4 * kMaxCols * sizeof(u64), host, s));
  int shift = 0;
  for (int k = ncols - 1; k >= 0; --k) {
    u64 mn = ~0ull, mx = 0;
    if (nl) { mn = std::min(mn, host[2 * k]); mx = std::max(mx, host[2 * k + 1]); }
    if (nr) { mn = std::min(mn, host[2 * kMaxCols + 2 * k]); mx = std::max(mx, host[2 * kMaxCols + 2 * k + 1]); }
    if (!nl && !nr) mn = mx = 0;
    const int bits = bit_length(mx - mn);
    pl.c[k].tmin = pr.c[k].tmin = mn;
    pl.c[k].bits = pr.c[k].bits = bits;
    pl.c[k].shift = pr.c[k].shift = shift;
    shift += bits;
  }
  if (shift > 64) return fail(JFX_ERR_CAPACITY, "join keys need %d packed bits; at most 64 are supported", shift);
  const int total_bits = shift;
  const bool key64 = total_bits > 32;
  // Payload columns of a side ride through that side's sort as 32-bit words
  // (4- and 8-byte dtypes, at most kMaxWords words) instead of being gathered
  // by row id afterwards; then the side's row ids are not kept.  Not with a
  // float key (its output is re-read by row id) nor for outer joins (their
  // unmatched rows are found by row id).
  int carried[2] = {0, 0};
  int pay_word[kMaxJoinPayloads];
  PayloadSrc psrc[2][kMaxWords];
  memset(psrc, 0, sizeof psrc);
  bool float_key = false;
  for (int k = 0; k < ncols; ++k) float_key |= dtype_is_float(left_keys[k].dtype);
  for (int side = 0; side < 2 && npayloads; ++side) {
    int words = 0;
    bool fits = how != JFX_JOIN_OUTER && !float_key;
    for (int k = 0; k < npayloads; ++k) {
      if (payloads[k].side != side) continue;
      const int sz = dtype_size(payloads[k].dtype);
      if (sz != 4 && sz != 8) fits = false;
      words += sz / 4;
    }
    if (!fits || words == 0 || words > kMaxWords) continue;
    int w = 0;
    for (int k = 0; k < npayloads; ++k) {
      if (payloads[k].side != side) continue;
      const int sz = dtype_size(payloads[k].dtype);
      pay_word[k] = w;
      for (int h = 0; h < sz / 4; ++h) psrc[side][w++] = PayloadSrc{(const unsigned char*)payloads[k].data, (u32)sz, (u32)(4 * h)};
    }
    carried[side] = words;
  }
  // the right side sorts on a second stream while the left side sorts on s
  cudaStream_t s2 = s;
  SideStream* ss = nullptr;
  if (nl && nr) {
    JFX_TRY(side_stream(&ss));
    s2 = ss->stream;
    JFX_CUDA(cudaEventRecord(ss->fork, s));
    JFX_CUDA(cudaStreamWaitEvent(s2, ss->fork, 0));
  }
  for (int side = 0; side < 2; ++side) {
    const u64 ns = side ? (u64)nr : (u64)nl;
    if (!ns) continue;
    const cudaStream_t st = side ? s2 : s;
    RadixRequest rq;
    rq.pack = side ? pr : pl;
    rq.total_bits = total_bits;
    rq.key64 = key64;
    rq.keys_out = side ? j.skR : j.skL;
    if (carried[side]) {
      rq.total_bits = std::max(total_bits, 1);  // constant keys still run one pass to move the words
      rq.nwords = carried[side];
      for (int w = 0; w < carried[side]; ++w) {
        rq.pfirst[w] = psrc[side][w];
        rq.vout_final[w] = j.cw[side][w];
      }
    } else {
      rq.perm_out = side ? j.pR : j.pL;
    }
    JFX_TRY(radix_sort(rq, ns, side ? br : b, c.err, st));
  }
  if (ss) {
    JFX_CUDA(cudaEventRecord(ss->join, s2));
    JFX_CUDA(cudaStreamWaitEvent(s, ss->join, 0));
  }
  // forward counts drive inner/left joins, swapped counts right joins; the
  // unmatched rows of a side need that side's counts
  const bool swap = how == JFX_JOIN_RIGHT;
  const u64 na = swap ? nr : nl, nb = swap ? nl : nr;
  const void* A = swap ? j.skR : j.skL;
  const void* B = swap ? j.skL : j.skR;
  unsigned long long* stats = (unsigned long long*)j.stats;
  if (key64) JFX_TRY(launch_join_count<u64>(A, na, B, nb, j.lo, j.cnt, pl, j.win, s, stats));
  else JFX_TRY(launch_join_count<u32>(A, na, B, nb, j.lo, j.cnt, pl, j.win, s, stats));
  const bool rev = how == JFX_JOIN_OUTER;
  if (rev) {
    if (key64) JFX_TRY(launch_join_count<u64>(j.skR, nr, j.skL, nl, j.lo2, j.cnt2, pl, j.win, s));
    else JFX_TRY(launch_join_count<u32>(j.skR, nr, j.skL, nl, j.lo2, j.cnt2, pl, j.win, s));
  }
  // one synchronisation: error word, sum of the counts (= inner pairs) and
  // the largest count
  JFX_CUDA(cudaMemcpyAsync(host + 8, stats, 2 * kJoinStatSlots * sizeof(u64), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaMemcpyAsync(host, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaStreamSynchronize(s));
  JFX_TRY(check_err_word((u32)host[0]));
  host[1] = host[2] = 0;
  for (int k = 0; k < kJoinStatSlots; ++k) {
    host[1] += host[8 + 2 * k];
    host[2] = std::max(host[2], host[8 + 2 * k + 1]);
  }
  const u64 inner = (na && nb) ? host[1] : 0;
  // many-to-one inner join with every row matched: no offsets are needed
  const bool unique = how == JFX_JOIN_INNER && na && nb && host[2] <= 1 && inner == na;
  if ((how == JFX_JOIN_INNER || how == JFX_JOIN_OUTER) && !unique && na && nb)
    JFX_TRY(device_exclusive_scan<u64>(j.cnt, na, j.off, j.total, j.partial, s));
  u64 m = how == JFX_JOIN_INNER || how == JFX_JOIN_OUTER ? inner : na;
  if (m > (u64)0x7fffffffull) return fail(JFX_ERR_CAPACITY, "join produces %llu rows; at most 2^31-1 are supported", m);
  JoinPlan* jp = (JoinPlan*)plan_out;
  memset(plan_out, 0, sizeof *plan_out);
  jp->magic = kJoinMagic;
  jp->how = how;
  jp->key64 = key64;
  jp->ncols = ncols;
  jp->reverse_counted = rev;
  jp->unique = unique;
  jp->npay = npayloads;
  for (int side = 0; side < 2; ++side) {
    jp->carried[side] = carried[side];
    for (int w = 0; w < kMaxWords; ++w) jp->cw[side][w] = carried[side] ? j.cw[side][w] : nullptr;
  }
  for (int k = 0; k < npayloads; ++k) {
    jp->pay_side[k] = payloads[k].side;
    jp->pay_dtype[k] = payloads[k].dtype;
    jp->pay_word[k] = carried[payloads[k].side] ? pay_word[k] : -1;
  }
  jp->nl = (u64)nl;
  jp->nr = (u64)nr;
  jp->m = m;
  jp->skL = j.skL;
  jp->skR = j.skR;
  jp->pL = j.pL;
  jp->pR = j.pR;
  jp->lo = j.lo;
  jp->cnt = j.cnt;
  jp->lo2 = j.lo2;
  jp->cnt2 = j.cnt2;
  jp->off = j.off;
  jp->flag = j.flag;
  jp->foff = j.foff;
  jp->fpart = j.fpart;
  jp->win = j.win;
  jp->win_cap = (std::max(jp->nl, jp->nr) + kJoinTile - 1) / kJoinTile + 1;
  jp->ftotal = j.ftotal;
  for (int k = 0; k < ncols; ++k) {
    jp->lc[k] = pl.c[k];
    jp->rc[k] = pr.c[k];
  }
  *num_out = (int64_t)m;
  return JFX_OK;
}

extern "C" {

int jfx_join_prepare(const jfx_column* left_keys, int64_t nl, const jfx_column* right_keys, int64_t nr, int ncols,
                     int how, jfx_join_plan* plan_out, int64_t* num_out, void* workspace, size_t workspace_bytes,
                     void* stream) {
  return join_prepare(left_keys, nl, right_keys, nr, ncols, how, nullptr, 0, plan_out, num_out, workspace,
                      workspace_bytes, stream);
}

int jfx_join_prepare_payloads(const jfx_column* left_keys, int64_t nl, const jfx_column* right_keys, int64_t nr,
                              int ncols, int how, const jfx_join_payload* payloads, int npayloads,
                              jfx_join_plan* plan_out, int64_t* num_out, void* workspace, size_t workspace_bytes,
                              void* stream) {
  if (npayloads < 0 || npayloads > kMaxJoinPayloads)
    return fail(JFX_ERR_ARG, "0..%d payload columns per call, got %d", kMaxJoinPayloads, npayloads);
  if (npayloads && !payloads) return fail(JFX_ERR_ARG, "null payload array");
  for (int k = 0; k < npayloads; ++k) {
    const jfx_join_payload& q = payloads[k];
    if (q.side != 0 && q.side != 1) return fail(JFX_ERR_ARG, "payload %d: side must be 0 (left) or 1 (right)", k);
    if (dtype_size(q.dtype) == 0) return fail(JFX_ERR_DTYPE, "payload %d: unsupported dtype", k);
    if (q.n != (q.side ? nr : nl)) return fail(JFX_ERR_ARG, "payload %d has %lld rows, its table %lld", k,
                                               (long long)q.n, (long long)(q.side ? nr : nl));
    if (!q.data && q.n) return fail(JFX_ERR_ARG, "payload %d: null pointer", k);
  }
  return join_prepare(left_keys, nl, right_keys, nr, ncols, how, payloads, npayloads, plan_out, num_out, workspace,
                      workspace_bytes, stream);
}

}  // extern "C"

// Shared body of jfx_join_expand and jfx_join_expand_gather.
static int join_expand(const JoinPlan* jp, int32_t* left_idx_out, int32_t* right_idx_out, void* const* keys_out,
                       const JoinPayloads& pay, cudaStream_t s) {
  const bool swap = jp->how == JFX_JOIN_RIGHT;
  JoinKeyOut ko;
  memset(&ko, 0, sizeof ko);
  ko.ncols = jp->ncols;
  for (int k = 0; k < jp->ncols; ++k) {
    ko.out[k] = keys_out ? keys_out[k] : nullptr;
    ko.c[k] = swap ? jp->rc[k] : jp->lc[k];
    if (ko.out[k] && dtype_is_float(ko.c[k].dtype)) ko.float_key = 1;
  }
  {
    const int dt = ko.c[0].dtype;
    if (jp->ncols == 1 && ko.out[0] && (dt == JFX_I32 || dt == JFX_I64 || dt == JFX_U32 || dt == JFX_U64)) {
      ko.fast_size = dtype_size(dt);
      ko.fast_flip = dt == JFX_I64 ? 0x8000000000000000ull : dt == JFX_I32 ? 0x80000000ull : 0ull;
    }
  }
  const u64 na = swap ? jp->nr : jp->nl;
  const void* skA = swap ? jp->skR : jp->skL;
  const u32* pA = swap ? jp->pR : jp->pL;
  const u32* pB = swap ? jp->pL : jp->pR;
  int32_t* a_out = swap ? right_idx_out : left_idx_out;
  int32_t* b_out = swap ? left_idx_out : right_idx_out;
  bool carried_only = pay.n > 0 && !pay.gathered && ko.fast_size && !a_out && !b_out;
  for (int k = 0; k < pay.n && carried_only; ++k)
    carried_only = pay.cw0[k] && pay.kind[k] >= PK_SAME4 && pay.kind[k] <= PK_U64_F32;
  if (jp->unique && carried_only) {
    const int g = grid_for(na, 256);
    if (jp->key64)
      k_join_expand_unique_carried<u64><<<g, 256, 0, s>>>(na, jp->lo, (const u64*)skA, ko, pay), note_launch();
    else
      k_join_expand_unique_carried<u32><<<g, 256, 0, s>>>(na, jp->lo, (const u32*)skA, ko, pay), note_launch();
  } else if (jp->unique) {
    const int g = grid_for(na, 256);
    if (jp->key64)
      k_join_expand_unique<u64><<<g, 256, 0, s>>>(na, jp->lo, pA, pB, (const u64*)skA, a_out, b_out, ko, pay), note_launch();
    else
      k_join_expand_unique<u32><<<g, 256, 0, s>>>(na, jp->lo, pA, pB, (const u32*)skA, a_out, b_out, ko, pay), note_launch();
  } else if (jp->how == JFX_JOIN_INNER || jp->how == JFX_JOIN_OUTER) {
    // output tiles in chunks of the window buffer's capacity
    const u64 tiles = (jp->m + kJoinTile - 1) / kJoinTile;
    for (u64 t0 = 0; t0 < tiles; t0 += jp->win_cap) {
      const unsigned blocks = (unsigned)std::min<u64>(jp->win_cap, tiles - t0);
      k_expand_windows<<<(blocks + 7) / 8, 256, 0, s>>>(jp->off, na, jp->m, t0, blocks, jp->win), note_launch();
      if (jp->key64)
        k_join_expand_inner<u64><<<blocks, kJoinThreads, 0, s>>>(jp->off, na, jp->m, jp->win, jp->lo, pA, pB, (const u64*)skA, a_out, b_out, ko, pay, t0), note_launch();
      else
        k_join_expand_inner<u32><<<blocks, kJoinThreads, 0, s>>>(jp->off, na, jp->m, jp->win, jp->lo, pA, pB, (const u32*)skA, a_out, b_out, ko, pay, t0), note_launch();
    }
  } else {
    const int g = grid_for(na, 256);
    if (jp->key64)
      k_join_expand_first<u64><<<g, 256, 0, s>>>(na, jp->lo, jp->cnt, pA, pB, (const u64*)skA, a_out, b_out, ko, pay), note_launch();
    else
      k_join_expand_first<u32><<<g, 256, 0, s>>>(na, jp->lo, jp->cnt, pA, pB, (const u32*)skA, a_out, b_out, ko, pay), note_launch();
  }
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

extern "C" {

int jfx_join_expand(const jfx_join_plan* plan, int32_t* left_idx_out, int32_t* right_idx_out, void* const* keys_out,
                    void* stream) {
  if (!plan) return fail(JFX_ERR_ARG, "null plan");
  const JoinPlan* jp = (const JoinPlan*)plan;
  if (jp->magic != kJoinMagic) return fail(JFX_ERR_ARG, "plan was not filled by jfx_join_prepare");
  if (jp->m == 0) return JFX_OK;
  if (!left_idx_out || !right_idx_out) return fail(JFX_ERR_ARG, "null index output");
  if (jp->carried[0] || jp->carried[1])
    return fail(JFX_ERR_ARG, "this plan carried payloads through the sorts and kept no row ids: use jfx_join_expand_gather");
  JoinPayloads pay;
  memset(&pay, 0, sizeof pay);
  return join_expand(jp, left_idx_out, right_idx_out, keys_out, pay, as_stream(stream));
}

int jfx_join_expand_gather(const jfx_join_plan* plan, int32_t* left_idx_out, int32_t* right_idx_out,
                           void* const* keys_out, const jfx_join_payload* payloads, int npayloads, void* stream) {
  if (!plan) return fail(JFX_ERR_ARG, "null plan");
  const JoinPlan* jp = (const JoinPlan*)plan;
  if (jp->magic != kJoinMagic) return fail(JFX_ERR_ARG, "plan was not filled by jfx_join_prepare");
  if (npayloads < 0 || npayloads > kMaxJoinPayloads)
    return fail(JFX_ERR_ARG, "0..%d payload columns per call, got %d", kMaxJoinPayloads, npayloads);
  if (npayloads && !payloads) return fail(JFX_ERR_ARG, "null payload array");
  if (jp->how == JFX_JOIN_OUTER) return fail(JFX_ERR_ARG, "outer joins gather their payloads with jfx_gather");
  JoinPayloads pay;
  memset(&pay, 0, sizeof pay);
  pay.n = npayloads;
  pay.swap = jp->how == JFX_JOIN_RIGHT;
  for (int k = 0; k < npayloads; ++k) {
    const jfx_join_payload& q = payloads[k];
    if (q.side != 0 && q.side != 1) return fail(JFX_ERR_ARG, "payload %d: side must be 0 (left) or 1 (right)", k);
    if (dtype_size(q.dtype) == 0 || dtype_size(q.out_dtype) == 0) return fail(JFX_ERR_DTYPE, "payload %d: unsupported dtype", k);
    const u64 rows = q.side ? jp->nr : jp->nl;
    if (q.n != (int64_t)rows) return fail(JFX_ERR_ARG, "payload %d has %lld rows, its table %llu", k, (long long)q.n, rows);
    if ((!q.data && rows) || (!q.out && jp->m)) return fail(JFX_ERR_ARG, "payload %d: null pointer", k);
    pay.src[k] = q.data;
    pay.out[k] = q.out;
    pay.n_src[k] = rows;
    pay.sdt[k] = q.dtype;
    pay.odt[k] = q.out_dtype;
    pay.side[k] = q.side;
    pay.kind[k] = payload_kind(q.dtype, q.out_dtype);
    if (jp->carried[q.side]) {
      // the side's payloads were carried: this list must be the one given to prepare
      if (npayloads != jp->npay || jp->pay_side[k] != q.side || jp->pay_dtype[k] != q.dtype || jp->pay_word[k] < 0)
        return fail(JFX_ERR_ARG, "payload %d does not match the list given to jfx_join_prepare_payloads", k);
      pay.cw0[k] = jp->cw[q.side][jp->pay_word[k]];
      pay.cw1[k] = dtype_size(q.dtype) == 8 ? jp->cw[q.side][jp->pay_word[k] + 1] : nullptr;
    } else {
      pay.gathered = 1;
    }
  }
  bool need_rows[2] = {left_idx_out != nullptr, right_idx_out != nullptr};
  for (int k = 0; k < npayloads; ++k)
    if (!pay.cw0[k]) need_rows[payloads[k].side] = true;
  if ((need_rows[0] && jp->carried[0]) || (need_rows[1] && jp->carried[1]))
    return fail(JFX_ERR_ARG, "row ids were not kept for a side whose payloads were carried; pass null index outputs");
  if (jp->m == 0) return JFX_OK;
  return join_expand(jp, left_idx_out, right_idx_out, keys_out, pay, as_stream(stream));
}

int jfx_join_unmatched(const jfx_join_plan* plan, int side, int32_t* rows_out, int64_t capacity, int64_t* count,
                       void* stream) {
  if (!plan || !count) return fail(JFX_ERR_ARG, "null argument");
  const JoinPlan* jp = (const JoinPlan*)plan;
  if (jp->magic != kJoinMagic) return fail(JFX_ERR_ARG, "plan was not filled by jfx_join_prepare");
  if (side != 0 && side != 1) return fail(JFX_ERR_ARG, "side must be 0 (left) or 1 (right)");
  if (jp->carried[0] || jp->carried[1]) return fail(JFX_ERR_ARG, "this plan kept no row ids (payloads were carried)");
  const u32 *cnt, *pA;
  u64 na;
  if (side == 0) {
    if (jp->how == JFX_JOIN_RIGHT) return fail(JFX_ERR_ARG, "a right-join plan holds no counts for left rows");
    cnt = jp->cnt;
    pA = jp->pL;
    na = jp->nl;
  } else if (jp->how == JFX_JOIN_RIGHT) {
    cnt = jp->cnt;
    pA = jp->pR;
    na = jp->nr;
  } else if (jp->reverse_counted) {
    cnt = jp->cnt2;
    pA = jp->pR;
    na = jp->nr;
  } else {
    return fail(JFX_ERR_ARG, "right rows' counts exist only for right/outer plans");
  }
  *count = 0;
  if (!na) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  const int g = grid_for(na, 256);
  k_mark_unmatched<<<g, 256, 0, s>>>(cnt, pA, na, jp->flag), note_launch();
  JFX_CUDA(cudaGetLastError());
  JFX_TRY(device_exclusive_scan<u32>(jp->flag, na, jp->foff, jp->ftotal, jp->fpart, s));
  u64* host = g_host.get();
  JFX_CUDA(cudaMemcpyAsync(host, jp->ftotal, sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaStreamSynchronize(s));
  const u64 k = (u32)host[0];
  *count = (int64_t)k;
  if (k > (u64)capacity || (!rows_out && k)) return fail(JFX_ERR_CAPACITY, "%llu unmatched rows exceed capacity %lld", k, (long long)capacity);
  if (k) {
    k_compact_rows<<<g, 256, 0, s>>>(jp->flag, jp->foff, na, rows_out), note_launch();
    JFX_CUDA(cudaGetLastError());
  }
  return JFX_OK;
}

int jfx_coalesce(const void* left, const int32_t* left_idx, int64_t nl, const void* right, const int32_t* right_idx,
                 int64_t nr, int64_t n, int32_t dtype, void* out, void* stream) {
  if (n < 0 || nl < 0 || nr < 0) return fail(JFX_ERR_ARG, "negative count");
  if (n == 0) return JFX_OK;
  if (!left_idx || !right_idx || !out) return fail(JFX_ERR_ARG, "null pointer");
  if (dtype_size(dtype) == 0) return fail(JFX_ERR_DTYPE, "unsupported dtype");
  cudaStream_t s = as_stream(stream);
  k_coalesce<<<grid_for((u64)n, 256), 256, 0, s>>>(left, left_idx, (u64)nl, right, right_idx, (u64)nr, (u64)n, dtype, out), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

int jfx_gather(const void* src, int32_t src_dtype, int64_t n_src, const int32_t* idx, int64_t n, void* out,
               int32_t out_dtype, void* stream) {
  if (n < 0 || n_src < 0) return fail(JFX_ERR_ARG, "negative count");
  if (n == 0) return JFX_OK;
  if (!idx || !out || (!src && n_src)) return fail(JFX_ERR_ARG, "null pointer");
  if (dtype_size(src_dtype) == 0 || dtype_size(out_dtype) == 0) return fail(JFX_ERR_DTYPE, "unsupported dtype");
  cudaStream_t s = as_stream(stream);
  k_gather<<<grid_for((u64)n, 256), 256, 0, s>>>(src, src_dtype, (u64)n_src, idx, (u64)n, out, out_dtype), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

int jfx_hash_columns(const jfx_column* keys, int ncols, int64_t n, uint32_t* hash_out, void* stream) {
  if (n < 0) return fail(JFX_ERR_ARG, "negative count");
  if (!hash_out) return fail(JFX_ERR_ARG, "null output");
  PackDesc pd;
  JFX_TRY(build_pack(keys, ncols, 0u, false, pd));
  if (ncols == 1 && keys[0].dtype == JFX_F64)
    return fail(JFX_ERR_DTYPE, "a single float64 key hashes to two words per row in the reference; not a row hash");
  if (n == 0) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  k_hash<<<grid_for((u64)n, 256), 256, 0, s>>>(pd, (u64)n, hash_out), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

int jfx_hash_partition(const jfx_column* keys, int ncols, int64_t n, int num_partitions, int32_t* targets_out,
                       int32_t* perm_out, int64_t* offsets_out, void* workspace, size_t workspace_bytes,
                       void* stream) {
  JFX_TRY(check_n(n));
  if (num_partitions < 1 || num_partitions > 2048) return fail(JFX_ERR_ARG, "num_partitions must be in [1, 2048]");
  if (!perm_out || !offsets_out) return fail(JFX_ERR_ARG, "null output");
  PackDesc pd;
  JFX_TRY(build_pack(keys, ncols, 0u, false, pd));
  if (ncols == 1 && keys[0].dtype == JFX_F64)
    return fail(JFX_ERR_DTYPE, "a single float64 key hashes to two words per row in the reference; not a row hash");
  cudaStream_t s = as_stream(stream);
  if (n == 0) {
    JFX_CUDA(cudaMemsetAsync(offsets_out, 0, (num_partitions + 1) * sizeof(int64_t), s));
    return JFX_OK;
  }
  Arena ar(workspace, workspace_bytes);
  Common c;
  SortBuffers b;
  carve_partition(ar, (u64)n, c, b);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  RadixRequest rq;
  rq.pack = pd;
  rq.key_mode = KEY_HASH;
  rq.digit_mode = DIG_MOD;
  rq.modulus = (u32)num_partitions;
  rq.key64 = false;
  rq.targets = (u32*)targets_out;
  rq.perm_out = (u32*)perm_out;
  JFX_TRY(radix_sort(rq, (u64)n, b, c.err, s));
  k_offsets_from_base<<<1, 256, 0, s>>>(b.base, num_partitions, (u64)n, offsets_out), note_launch();
  JFX_CUDA(cudaGetLastError());
  u64* host = g_host.get();
  JFX_TRY(read_back(c.err, sizeof(u32), host, s));
  return check_err_word((u32)host[0]);
}

int jfx_learned_sort(const uint64_t* keys_in, int64_t n, uint64_t* sorted_out_in, int32_t* perm_out, int mode,
                     int32_t* learned_used, void* workspace, size_t workspace_bytes, void* stream) {
  JFX_TRY(check_n(n));
  if (!keys_in || !sorted_out_in || !perm_out) return fail(JFX_ERR_ARG, "null pointer");
  const u64* keys = (const u64*)keys_in;
  u64* sorted_keys_out = (u64*)sorted_out_in;
  if (mode < 0 || mode > 1) return fail(JFX_ERR_ARG, "mode must be 0 (learned, plain fallback) or 1 (plain)");
  if (learned_used) *learned_used = 0;
  if (n == 0) return JFX_OK;
  cudaStream_t s = as_stream(stream);
  Arena ar(workspace, workspace_bytes);
  Common c;
  SortBuffers b;
  LearnedBuffers l;
  carve_learned(ar, (u64)n, c, b, l);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  const u64 N = (u64)n;
  u64* host = g_host.get();
  if (mode == 1 || N < (1u << 17) || l.s < 4096) {
    JFX_TRY(plain_sort_u64(keys, N, sorted_keys_out, (u32*)perm_out, b, c, s));
    JFX_TRY(read_back(c.err, sizeof(u32), host, s));
    return check_err_word((u32)host[0]);
  }
  const int g = grid_for(l.s, 256);
  // 1. sample and its plain sort (the labels are the sample ranks)
  k_sample<<<g, 256, 0, s>>>(keys, kSampleStride, l.s, l.sample), note_launch();
  {
    jfx_column col{l.sample, JFX_U64, 0u};
    RadixRequest rq;
    JFX_TRY(build_pack(&col, 1, 0u, false, rq.pack));
    rq.pack.c[0].bits = 64;
    rq.total_bits = 64;
    rq.key64 = true;
    rq.perm_out = l.sperm;
    rq.raw_out = l.ssorted;
    rq.raw_dtype = JFX_U64;
    JFX_TRY(radix_sort(rq, l.s, b, c.err, s));
  }
  // 2. least-squares fit and the monotonicity check
  JFX_CUDA(cudaMemsetAsync(l.acc, 0, 8 * sizeof(double), s));
  k_root_sum<<<g, 256, 0, s>>>(l.ssorted, l.s, l.acc), note_launch();
  k_root_cov<<<g, 256, 0, s>>>(l.ssorted, l.s, l.acc), note_launch();
  k_root_solve<<<1, 1, 0, s>>>(l.acc, l.s, l.model, l.leaves), note_launch();
  JFX_CUDA(cudaMemsetAsync(l.first, 0xff, kLeaves * sizeof(u32), s));
  JFX_CUDA(cudaMemsetAsync(l.last, 0, kLeaves * sizeof(u32), s));
  JFX_CUDA(cudaMemsetAsync(l.flags, 0x01, 8 * sizeof(u32), s));
  k_leaf_bounds<<<g, 256, 0, s>>>(l.ssorted, l.s, l.model, l.first, l.last), note_launch();
  k_leaf_fit<<<kLeaves, 256, 0, s>>>(l.ssorted, l.first, l.last, l.fit), note_launch();
  // predicted positions range over [0, 4n): finer than one slot per row, so
  // distinct keys share a position less often
  const u64 npos = 4 * N;
  k_leaf_finalize<<<1, 1024, 0, s>>>(l.ssorted, l.s, npos, l.first, l.last, l.fit, l.leaves, l.flags), note_launch();
  JFX_CUDA(cudaGetLastError());
  // 3. bucket of every key (the predicted position's top bits), then a
  // plain stable radix sort of that uint32 column carrying the key's two
  // words and the row id: rows in bucket order, row order inside a bucket
  {
    k_model_positions<<<grid_for(N, 256), 256, 0, s>>>(keys, N, l.model, kBucketShift, l.pos), note_launch();
    JFX_CUDA(cudaGetLastError());
    jfx_column col{l.pos, JFX_U32, 0u};
    RadixRequest rq;
    JFX_TRY(build_pack(&col, 1, 0u, false, rq.pack));
    rq.total_bits = std::max(1, bit_length(l.nb - 1));
    rq.pack.c[0].tmin = 0;
    rq.pack.c[0].bits = rq.total_bits;
    rq.pack.c[0].shift = 0;
    rq.key_mode = KEY_PACK;
    rq.digit_mode = DIG_BITS;
    rq.key64 = false;
    rq.max_digit_bits = 9;  // 17 bucket bits at 2^28 rows: two passes of 9 + 8 bits
    rq.nwords = 3;
    rq.pfirst[0] = PayloadSrc{(const unsigned char*)keys, 8u, 0u};
    rq.pfirst[1] = PayloadSrc{(const unsigned char*)keys, 8u, 4u};
    rq.pfirst[2] = PayloadSrc{nullptr, 0u, 0u};
    rq.vout64 = sorted_keys_out;
    rq.vout_final[2] = (u32*)perm_out;
    rq.keys_out = l.spos;
    JFX_TRY(radix_sort(rq, N, b, c.err, s));
  }
  // 4. sort inside every bucket: most by k_bucket_sort<8>, those of 2049 to
  // 4096 rows by k_bucket_sort<16>, which lists the larger ones
  JFX_CUDA(cudaMemsetAsync(l.bcounts, 0, 8 * sizeof(u32), s));
  k_bucket_starts<<<grid_for(N / 4 + 1, 256), 256, 0, s>>>(l.spos, N, (u32)l.nb, l.starts), note_launch();
  {
    static SmemAttr attr8, attr16;
    JFX_TRY(ensure_smem(attr8, k_bucket_sort<8>, bucket_smem<8>()));
    JFX_TRY(ensure_smem(attr16, k_bucket_sort<16>, bucket_smem<16>()));
    BucketArgs ba;
    ba.keys = sorted_keys_out;
    ba.ids = (u32*)perm_out;
    ba.starts = l.starts;
    ba.nb = (u32)l.nb;
    ba.counts = l.bcounts;
    ba.large = nullptr;
    ba.min_rows = 0;
    const int grid = (int)std::min<u64>(l.nb, (u64)device_sm_count() * 12);
    k_bucket_sort<8><<<grid, kBucketThreads, bucket_smem<8>(), s>>>(ba), note_launch();
    ba.large = l.large;
    ba.min_rows = kBucketSmallCap;
    k_bucket_sort<16><<<grid, kBucketThreads, bucket_smem<16>(), s>>>(ba), note_launch();
  }
  JFX_CUDA(cudaGetLastError());
  JFX_CUDA(cudaMemcpyAsync(host, c.err, sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaMemcpyAsync(host + 1, l.flags, sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaMemcpyAsync(host + 2, l.bcounts, sizeof(u32), cudaMemcpyDeviceToHost, s));
  std::vector<u32> spans(2 * (size_t)kBucketLargeMax);
  JFX_CUDA(cudaMemcpyAsync(spans.data(), l.large, spans.size() * sizeof(u32), cudaMemcpyDeviceToHost, s));
  JFX_CUDA(cudaStreamSynchronize(s));
  JFX_TRY(check_err_word((u32)host[0]));
  const u32 ok = (u32)host[1];
  const u32 nlarge = (u32)host[2];
  if (!ok || nlarge > kBucketLargeMax || g_fault.learned_fallback) {
    // model not monotone, or more large buckets than listed: plain radix
    // sort.  *learned_used reports why: -1 model check, -3 list full (or the
    // fallback jfx_set_fault asked for)
    const int why = g_fault.learned_fallback ? g_fault.learned_fallback : !ok ? -1 : -3;
    JFX_TRY(plain_sort_u64(keys, N, sorted_keys_out, (u32*)perm_out, b, c, s));
    JFX_TRY(read_back(c.err, sizeof(u32), host, s));
    if (learned_used) *learned_used = why;
    return check_err_word((u32)host[0]);
  }
  if (nlarge) {
    // buckets of more than 4096 rows (many rows of a few heavy keys, or a
    // region the model under-predicts): min and max of each by chunks of
    // kLargeChunk rows over many CTAs; a bucket of one key is in row order
    // already; the others are sorted by one CTA each (up to kLargeCtaMax
    // rows) or by the multi-CTA radix sort over their rows
    std::vector<u32> chunks;
    for (u32 r = 0; r < nlarge; ++r)
      for (u32 c0 = spans[2 * r]; c0 < spans[2 * r + 1]; c0 += kLargeChunk) {
        chunks.push_back(r);
        chunks.push_back(c0);
        chunks.push_back(std::min(spans[2 * r + 1], c0 + kLargeChunk));
      }
    const u32 nchunks = (u32)(chunks.size() / 3);
    if (nchunks > l.cap_chunks) return fail(JFX_ERR_CUDA, "internal: %u min/max chunks exceed %llu", nchunks, l.cap_chunks);
    JFX_CUDA(cudaMemcpyAsync(l.chunks, chunks.data(), chunks.size() * sizeof(u32), cudaMemcpyHostToDevice, s));
    k_init_pairs<<<grid_for(nlarge, 256), 256, 0, s>>>(l.mm, nlarge), note_launch();
    k_large_minmax<<<(unsigned)std::min<u64>(nchunks, (u64)device_sm_count() * 8), 256, 0, s>>>(
        sorted_keys_out, l.chunks, nchunks, l.mm), note_launch();
    JFX_CUDA(cudaGetLastError());
    std::vector<u64> mm(2 * (size_t)nlarge);
    JFX_CUDA(cudaMemcpyAsync(mm.data(), l.mm, mm.size() * sizeof(u64), cudaMemcpyDeviceToHost, s));
    JFX_CUDA(cudaStreamSynchronize(s));
    std::vector<u32> cspans, cbits;
    std::vector<u64> cmins;
    bool any = false;
    for (u32 r = 0; r < nlarge; ++r) {
      const u64 b0 = spans[2 * r], b1 = spans[2 * r + 1];
      if (mm[2 * r] == mm[2 * r + 1]) continue;  // one key
      const int bits = bit_length(mm[2 * r + 1] - mm[2 * r]);
      if (b1 - b0 <= kLargeCtaMax) {
        cspans.push_back((u32)b0);
        cspans.push_back((u32)b1);
        cmins.push_back(mm[2 * r]);
        cbits.push_back((u32)bits);
      } else {
        JFX_TRY(sort_rows_u64(sorted_keys_out + b0, (u32*)perm_out + b0, b1 - b0, mm[2 * r], bits, l.tkeys, l.tids, b,
                              c, s));
      }
      any = true;
    }
    if (!cmins.empty()) {
      JFX_CUDA(cudaMemcpyAsync(l.cspans, cspans.data(), cspans.size() * sizeof(u32), cudaMemcpyHostToDevice, s));
      JFX_CUDA(cudaMemcpyAsync(l.cmins, cmins.data(), cmins.size() * sizeof(u64), cudaMemcpyHostToDevice, s));
      JFX_CUDA(cudaMemcpyAsync(l.cbits, cbits.data(), cbits.size() * sizeof(u32), cudaMemcpyHostToDevice, s));
      LargeArgs la;
      la.keys = sorted_keys_out;
      la.ids = (u32*)perm_out;
      la.tkeys = l.tkeys;
      la.tids = l.tids;
      la.spans = l.cspans;
      la.mins = l.cmins;
      la.bits = l.cbits;
      la.count = (u32)cmins.size();
      k_bucket_sort_large<<<(unsigned)std::min<u64>(cmins.size(), (u64)device_sm_count() * 2), kBucketThreads, 0, s>>>(
          la), note_launch();
      JFX_CUDA(cudaGetLastError());
    }
    if (any) {
      JFX_TRY(read_back(c.err, sizeof(u32), host, s));
      JFX_TRY(check_err_word((u32)host[0]));
    }
  }
  if (learned_used) *learned_used = 1;
  return JFX_OK;
}

int jfx_batch_partition_groupby(const int32_t* keys, const float* values, const int64_t* query_offsets, int nq,
                                int64_t n, int num_partitions, int key_bits, int32_t* part_keys_out,
                                float* part_values_out, int64_t* part_offsets_out, int32_t* group_keys_out,
                                float* group_sums_out, float* group_counts_out, int64_t* group_offsets_out,
                                void* workspace, size_t workspace_bytes, void* stream) {
  JFX_TRY(check_n(n));
  if (nq < 1) return fail(JFX_ERR_ARG, "need at least one query");
  if (num_partitions < 1 || num_partitions > 256) return fail(JFX_ERR_ARG, "num_partitions must be in [1, 256]");
  if (key_bits < 1 || key_bits > 30) return fail(JFX_ERR_ARG, "key_bits must be in [1, 30]");
  if (!keys || !values || !query_offsets || !part_keys_out || !part_values_out || !part_offsets_out ||
      !group_keys_out || !group_sums_out || !group_counts_out || !group_offsets_out)
    return fail(JFX_ERR_ARG, "null pointer");
  cudaStream_t s = as_stream(stream);
  Arena ar(workspace, workspace_bytes);
  Common c;
  BatchBuffers bb;
  carve_batch(ar, (u64)n, (u64)nq, c, bb);
  JFX_TRY(check_workspace(ar, workspace, workspace_bytes));
  // one persistent launch: as many CTAs as are resident at once
  static SmemAttr attr;
  const size_t smem = sizeof(QueueShared);
  JFX_TRY(ensure_smem(attr, k_batch_queue, smem));
  int per_sm = 0;
  JFX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_queue, kQueueThreads, smem));
  const int grid = std::max(1, std::min(per_sm * device_sm_count(), nq));
  JFX_CUDA(cudaMemsetAsync(c.err, 0, sizeof(u32), s));
  JFX_CUDA(cudaMemsetAsync(bb.ctl, 0, 64 * sizeof(u32), s));
  QueueArgs qa;
  qa.keys = keys;
  qa.values = values;
  qa.qoff = query_offsets;
  qa.n = (u64)n;
  qa.nq = (u32)nq;
  qa.P = (u32)num_partitions;
  qa.key_bits = key_bits;
  qa.part_keys = part_keys_out;
  qa.part_values = part_values_out;
  qa.part_offsets = part_offsets_out;
  qa.group_keys = group_keys_out;
  qa.group_sums = group_sums_out;
  qa.group_counts = group_counts_out;
  qa.group_offsets = group_offsets_out;
  for (int i = 0; i < 2; ++i) {
    qa.sk[i] = bb.sk[i];
    qa.sv[i] = bb.sv[i];
  }
  qa.tkeys = bb.tkeys;
  qa.tsums = bb.tsums;
  qa.tcnts = bb.tcnts;
  qa.qgroups = bb.qgroups;
  qa.order = bb.order;
  qa.ctl = bb.ctl;
  qa.err = c.err;
  qa.spin_ns = (u64)g_tuning.spin_limit_us * 1000ull;
  qa.withhold_order = g_fault.withhold_order ? 1u : 0u;
  k_batch_queue<<<grid, kQueueThreads, smem, s>>>(qa), note_launch();
  JFX_CUDA(cudaGetLastError());
  return JFX_OK;
}

int jfx_batch_status(void* workspace, size_t workspace_bytes, void* stream) {
  if (!workspace || workspace_bytes < 256) return fail(JFX_ERR_ARG, "null or small workspace");
  cudaStream_t s = as_stream(stream);
  u64* host = g_host.get();
  JFX_TRY(read_back(workspace, sizeof(u32), host, s));  // the error word opens every workspace
  const u32 e = (u32)host[0];
  if (e & DERR_BOUNDS) return fail(JFX_ERR_ARG, "a key is outside [0, 2^key_bits) or a query offset decreases");
  return check_err_word(e);
}

}  // extern "C"
