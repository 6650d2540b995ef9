// Shared helpers for the ofb200 kernels (sm_100a).
//
// The library is compiled with -fmad=false: every float/double multiply-add that the
// kernels fuse is written as an explicit __fmaf_rn / __fma_rn, so the arithmetic order is
// fixed by the source and matches the CPU oracle bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>

#include "../../include/ofb200.h"

namespace ofb {

int set_error(int code, const char* fmt, ...);
// Reports the first launch error of an entry point; `nlaunch` kernel launches are added
// to the process-wide counter behind of_launch_count().
int check_launch(const char* what, long long nlaunch = 1);
// *dst |= *src on the device (status words), one launch.
int status_or(const int* src, int* dst, cudaStream_t stream);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__host__ __device__ inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// scipy.ndimage 'mirror' / OpenCV reflect-101 index for |i| < n (one reflection).
__host__ __device__ inline int mirror1(int i, int n) {
  if (n == 1) return 0;
  if (i < 0) i = -i;
  if (i >= n) i = 2 * n - 2 - i;
  return i;
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Carves typed sub-buffers out of a caller workspace.
struct Carver {
  char* base;
  size_t cap, off;
  Carver(void* b, size_t c) : base(static_cast<char*>(b)), cap(c), off(0) {}
  template <class T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
  bool ok() const { return off <= cap; }
};

// Size bookkeeping with the same alignment rule as Carver.
struct Sizer {
  size_t off = 0;
  template <class T>
  void take(size_t count) {
    off = align_up(off, 256);
    off += count * sizeof(T);
  }
};

inline bool bad_plane(const void* p, int H, int W, int pitch) { return !p || H <= 0 || W <= 0 || pitch < W; }

constexpr int kNumSMs = 148;

// The dynamic shared-memory opt-in (cudaFuncAttributeMaxDynamicSharedMemorySize) is a
// per-device attribute of a kernel.  Each call site keeps the size it has set on each
// device (ordinals 0-63; others set the attribute on every call), so a solve on a second
// GPU of the process opts in there too.  Concurrent first calls both set it: harmless.
struct SmemOptIn {
  std::atomic<int> bytes[64];
};

template <class K>
inline cudaError_t smem_opt_in(SmemOptIn& s, K* kernel, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool cached = dev >= 0 && dev < 64;
  if (cached && s.bytes[dev].load(std::memory_order_acquire) >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && cached) {
    int cur = s.bytes[dev].load(std::memory_order_relaxed);
    while (cur < bytes && !s.bytes[dev].compare_exchange_weak(cur, bytes, std::memory_order_release)) {
    }
  }
  return e;
}

}  // namespace ofb

// smem_opt_in with a call-site-local record (one per template instantiation).
#define OF_SMEM_OPT_IN(kernel, bytes)                                       \
  ([&]() {                                                                  \
    static ::ofb::SmemOptIn of_smem_record_;                                \
    return ::ofb::smem_opt_in(of_smem_record_, kernel, (int)(bytes));       \
  }())

#define OF_REQUIRE(cond, ...)                                        \
  do {                                                               \
    if (!(cond)) return ::ofb::set_error(OF_ERR_INVALID, __VA_ARGS__); \
  } while (0)
