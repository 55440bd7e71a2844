// common.cuh -- shared device/host utilities for the jfx kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/jfx.h"

namespace jfx {

typedef unsigned long long u64;
typedef uint32_t u32;

// ---------------------------------------------------------------- errors ---
// Thread-local last error message returned by jfx_last_error().
extern thread_local std::string g_last_error;

inline int fail(int status, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
inline int fail(int status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

#define JFX_CUDA(call)                                                                \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return ::jfx::fail(JFX_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,     \
                         cudaGetErrorString(e_));                                     \
  } while (0)

#define JFX_TRY(expr)           \
  do {                          \
    int s_ = (expr);            \
    if (s_ != JFX_OK) return s_; \
  } while (0)

// Device-side error bits, OR-ed into a status word in the workspace.  The host
// copies the word back once per entry point and turns bits into jfx_status.
enum : u32 { DERR_TIMEOUT = 1u, DERR_BOUNDS = 2u };

// Row limit: lookback status words hold a 30-bit count.
constexpr int64_t kMaxRows = (int64_t(1) << 30) - 1;

// ---------------------------------------------------------------- dtypes ---
__host__ __device__ inline int dtype_size(int dt) {
  switch (dt) {
    case JFX_I8: case JFX_U8: case JFX_BOOL: return 1;
    case JFX_I16: case JFX_U16: return 2;
    case JFX_I32: case JFX_U32: case JFX_F32: return 4;
    case JFX_I64: case JFX_U64: case JFX_F64: return 8;
    default: return 0;
  }
}
__host__ __device__ inline bool dtype_is_float(int dt) { return dt == JFX_F32 || dt == JFX_F64; }
__host__ __device__ inline bool dtype_is_signed_int(int dt) {
  return dt == JFX_I8 || dt == JFX_I16 || dt == JFX_I32 || dt == JFX_I64;
}
__host__ __device__ inline int dtype_bits(int dt) { return dtype_size(dt) * 8; }

// ------------------------------------------------------- column transforms ---
// Column descriptor used by the kernels that read key columns.
enum : u32 {
  CF_DESC = 1u,    // multi_column_lexsort descending rewrite (-x or max(x)-x)
  CF_QUIRK = 2u,   // ParallelRadixSort: int8/int16 are not sign-flipped
};

constexpr int kMaxCols = 8;

struct ColDesc {
  const void* ptr;
  int dtype;
  u32 flags;
  u64 desc_max;  // raw max bits (sign-extended) for an integer CF_DESC column
  u64 tmin;      // min of the transformed value
  int shift;     // bit position in the packed key
  int bits;      // bit width in the packed key (0: constant column, skipped)
};

struct PackDesc {
  int ncols;
  int nan_cols;  // bit j set: column j is float (a NaN in it starts a new group)
  ColDesc c[kMaxCols];
};

// Canonical sortable bits of a float (parallel_algorithms.py:583-603 plus JAX's
// sort comparator): -0.0 -> +0.0, any NaN -> one NaN that sorts after +inf.
__host__ __device__ __forceinline__ u32 f32_sortable(float x) {
  u32 b;
  memcpy(&b, &x, 4);
  if (x == 0.0f) b = 0u;
  if (x != x) b = 0x7fc00000u;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ u64 f64_sortable(double x) {
  u64 b;
  memcpy(&b, &x, 8);
  if (x == 0.0) b = 0ull;
  if (x != x) b = 0x7ff8000000000000ull;
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
constexpr u32 kF32NanT = 0xffc00000u;             // f32_sortable(NaN)
constexpr u64 kF64NanT = 0xfff8000000000000ull;   // f64_sortable(NaN)

// Transformed (order-preserving unsigned) value of row `row` of column `c`.
__device__ __forceinline__ u64 load_t(const ColDesc& c, size_t row) {
  const bool desc = c.flags & CF_DESC;
  switch (c.dtype) {
    case JFX_I32: {
      u32 x = (u32)__ldg((const int*)c.ptr + row);
      if (desc) x = (u32)c.desc_max - x;
      return x ^ 0x80000000u;
    }
    case JFX_I64: {
      u64 x = (u64)__ldg((const long long*)c.ptr + row);
      if (desc) x = c.desc_max - x;
      return x ^ 0x8000000000000000ull;
    }
    case JFX_U32: {
      u32 x = __ldg((const unsigned*)c.ptr + row);
      if (desc) x = (u32)c.desc_max - x;
      return x;
    }
    case JFX_U64: {
      u64 x = __ldg((const unsigned long long*)c.ptr + row);
      if (desc) x = c.desc_max - x;
      return x;
    }
    case JFX_F32: {
      float x = __ldg((const float*)c.ptr + row);
      if (desc) x = -x;
      return f32_sortable(x);
    }
    case JFX_F64: {
      double x = __ldg((const double*)c.ptr + row);
      if (desc) x = -x;
      return f64_sortable(x);
    }
    case JFX_I16: {
      short x = ((const short*)c.ptr)[row];
      if (desc) x = (short)((short)c.desc_max - x);
      return (c.flags & CF_QUIRK) ? (u64)(u32)(int)x : (u64)((u32)(int)x ^ 0x80000000u);
    }
    case JFX_I8: {
      signed char x = ((const signed char*)c.ptr)[row];
      if (desc) x = (signed char)((signed char)c.desc_max - x);
      return (c.flags & CF_QUIRK) ? (u64)(u32)(int)x : (u64)((u32)(int)x ^ 0x80000000u);
    }
    case JFX_U16: {
      unsigned short x = ((const unsigned short*)c.ptr)[row];
      if (desc) x = (unsigned short)((unsigned short)c.desc_max - x);
      return x;
    }
    case JFX_U8: {
      unsigned char x = ((const unsigned char*)c.ptr)[row];
      if (desc) x = (unsigned char)((unsigned char)c.desc_max - x);
      return x;
    }
    case JFX_BOOL: {
      unsigned char x = ((const unsigned char*)c.ptr)[row];
      return x ? 1u : 0u;
    }
  }
  return 0;
}

// load_t split in two: the transform of a raw element (read with load_raw).
__device__ __forceinline__ u64 transform_raw(const ColDesc& c, u64 raw) {
  const bool desc = c.flags & CF_DESC;
  switch (c.dtype) {
    case JFX_I32: {
      u32 x = (u32)raw;
      if (desc) x = (u32)c.desc_max - x;
      return x ^ 0x80000000u;
    }
    case JFX_I64: {
      u64 x = raw;
      if (desc) x = c.desc_max - x;
      return x ^ 0x8000000000000000ull;
    }
    case JFX_U32: {
      u32 x = (u32)raw;
      if (desc) x = (u32)c.desc_max - x;
      return x;
    }
    case JFX_U64: return desc ? c.desc_max - raw : raw;
    case JFX_F32: {
      float x = __uint_as_float((u32)raw);
      if (desc) x = -x;
      return f32_sortable(x);
    }
    case JFX_F64: {
      double x = __longlong_as_double((long long)raw);
      if (desc) x = -x;
      return f64_sortable(x);
    }
    case JFX_I16: {
      short x = (short)raw;
      if (desc) x = (short)((short)c.desc_max - x);
      return (c.flags & CF_QUIRK) ? (u64)(u32)(int)x : (u64)((u32)(int)x ^ 0x80000000u);
    }
    case JFX_I8: {
      signed char x = (signed char)raw;
      if (desc) x = (signed char)((signed char)c.desc_max - x);
      return (c.flags & CF_QUIRK) ? (u64)(u32)(int)x : (u64)((u32)(int)x ^ 0x80000000u);
    }
    case JFX_U16: {
      unsigned short x = (unsigned short)raw;
      if (desc) x = (unsigned short)((unsigned short)c.desc_max - x);
      return x;
    }
    case JFX_U8: {
      unsigned char x = (unsigned char)raw;
      if (desc) x = (unsigned char)((unsigned char)c.desc_max - x);
      return x;
    }
    case JFX_BOOL: return raw ? 1u : 0u;
  }
  return 0;
}

// Inverse of load_t (without CF_DESC) for integer columns: raw bits of the
// original value, written with the column's element size.
__host__ __device__ __forceinline__ u64 untransform_int(int dtype, u32 flags, u64 t) {
  switch (dtype) {
    case JFX_I32: return (u64)(u32)((u32)t ^ 0x80000000u);
    case JFX_I64: return t ^ 0x8000000000000000ull;
    case JFX_I16:
    case JFX_I8: return (flags & CF_QUIRK) ? t : (u64)((u32)t ^ 0x80000000u);
    default: return t;
  }
}

__device__ __forceinline__ void store_raw(void* base, int dtype, size_t i, u64 bits) {
  switch (dtype_size(dtype)) {
    case 1: ((unsigned char*)base)[i] = (unsigned char)bits; break;
    case 2: ((unsigned short*)base)[i] = (unsigned short)bits; break;
    case 4: ((u32*)base)[i] = (u32)bits; break;
    case 8: ((u64*)base)[i] = bits; break;
  }
}
__device__ __forceinline__ u64 load_raw(const void* base, int dtype, size_t i) {
  switch (dtype_size(dtype)) {
    case 1: return ((const unsigned char*)base)[i];
    case 2: return ((const unsigned short*)base)[i];
    case 4: return __ldg((const u32*)base + i);
    case 8: return __ldg((const u64*)base + i);
  }
  return 0;
}

template <typename K>
__device__ __forceinline__ K pack_row(const PackDesc& pd, size_t row) {
  K k = 0;
#pragma unroll 1
  for (int j = 0; j < pd.ncols; ++j) {
    const ColDesc& c = pd.c[j];
    if (c.bits == 0) continue;
    u64 t = load_t(c, row) - c.tmin;
    k |= (K)(t << c.shift);
  }
  return k;
}

// True when row `row` has a NaN in one of the float key columns: the
// reference's `!=` boundary test makes such a row a group of its own.
__device__ __forceinline__ bool row_has_nan(const PackDesc& pd, size_t row) {
  if (!pd.nan_cols) return false;
  for (int j = 0; j < pd.ncols; ++j) {
    if (!((pd.nan_cols >> j) & 1)) continue;
    const ColDesc& c = pd.c[j];
    if (c.dtype == JFX_F32) {
      float x = __ldg((const float*)c.ptr + row);
      if (x != x) return true;
    } else {
      double x = __ldg((const double*)c.ptr + row);
      if (x != x) return true;
    }
  }
  return false;
}

// ------------------------------------------------------- memory ordering ---
__device__ __forceinline__ u32 ld_relaxed(const u32* p) {
  u32 v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(u32* p, u32 v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ u64 globaltimer_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ u32 lanemask_gt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_gt;" : "=r"(m));
  return m;
}

// Default upper bound on any device-side spin (decoupled look-back); the
// bound a launch uses comes from the tuning (jfx_tuning.spin_limit_us).
constexpr u64 kSpinLimitNs = 1000000000ull;  // 1 s

// ---------------------------------------------------------------- arena ---
// Bump allocator over the caller's workspace.  With base == nullptr it only
// measures, which is how jfx_workspace_size is computed.
struct Arena {
  char* base;
  size_t cap;
  size_t off = 0;
  bool overflow = false;
  Arena(void* b, size_t c) : base((char*)b), cap(c) {}
  template <typename T>
  T* take(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    size_t at = off;
    off += bytes;
    if (off > cap) overflow = true;
    return base ? (T*)(base + at) : (T*)nullptr;
  }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
__host__ __device__ inline int bit_length(u64 v) {
#ifdef __CUDA_ARCH__
  return v ? 64 - __clzll((long long)v) : 0;
#else
  return v ? 64 - __builtin_clzll(v) : 0;
#endif
}

// Number of SMs of the current device (cached per device).
int device_sm_count();

// One-time raise of a kernel's dynamic shared-memory limit on each device.
// CUDA keeps the attribute per device, so a process that calls the library on
// several devices needs it set on every one; each call site owns one
// SmemAttr (bit d of `done`: set on device d).  Two threads that race here
// both set the same value, which is harmless.
struct SmemAttr {
  std::atomic<unsigned long long> done[2];
};
template <typename Kernel>
inline int ensure_smem(SmemAttr& a, Kernel* kernel, size_t bytes) {
  int dev = -1;
  JFX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(JFX_ERR_ARG, "device ordinal %d out of range", dev);
  const unsigned long long bit = 1ull << (dev & 63);
  std::atomic<unsigned long long>& w = a.done[dev >> 6];
  if (w.load(std::memory_order_acquire) & bit) return JFX_OK;
  JFX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  w.fetch_or(bit, std::memory_order_release);
  return JFX_OK;
}

// ------------------------------------------------------------ accounting ---
// Every kernel launch of the library bumps this counter (jfx_launch_count).
extern std::atomic<unsigned long long> g_launches;
inline void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Optional CUDA-event timing of the radix pass kernels (jfx_timing_enable /
// jfx_timing_read): each record is one launch with its algorithmic bytes.
struct TimedLaunch {
  cudaEvent_t start, stop;
  double bytes;
};
struct Timing {
  std::mutex mu;
  bool on = false;
  std::vector<TimedLaunch> recs;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
};
extern Timing g_timing;

// Starts a timed launch if timing is on; returns an index or -1.
inline long timing_begin(cudaStream_t s) {
  if (!g_timing.on) return -1;
  std::lock_guard<std::mutex> lk(g_timing.mu);
  TimedLaunch t;
  t.start = g_timing.get();
  t.stop = g_timing.get();
  t.bytes = 0;
  cudaEventRecord(t.start, s);
  g_timing.recs.push_back(t);
  return (long)g_timing.recs.size() - 1;
}
inline void timing_end(long idx, cudaStream_t s, double bytes) {
  if (idx < 0) return;
  std::lock_guard<std::mutex> lk(g_timing.mu);
  g_timing.recs[idx].bytes = bytes;
  cudaEventRecord(g_timing.recs[idx].stop, s);
}

}  // namespace jfx
