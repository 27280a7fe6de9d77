// Shared helpers of the sm_100a kernels: error plumbing, device-wide barrier
// with a bounded wait, timers and exact-rounding arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/ks_b200.h"

namespace ks {

// Message of the last failure on the calling host thread.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define KS_CUDA(call)                                        \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return ::ks::cuda_fail(_e, #call); \
  } while (0)

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Per-device properties cached on first use.
struct DeviceInfo {
  int device = -1;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  size_t smem_optin = 0;
};
int device_info(DeviceInfo* out);

// Simple bump allocator over a caller workspace.
struct Carve {
  char* base;
  size_t used = 0;
  explicit Carve(void* p) : base(static_cast<char*>(p)) {}
  template <typename T>
  T* take(size_t n) {
    T* p = reinterpret_cast<T*>(base ? base + used : nullptr);
    used = align256(used + n * sizeof(T));
    return p;
  }
};

// Default limit of every device-side wait (ns of %globaltimer).
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
// kWaitLimitNs, or KS_B200_WAIT_LIMIT_NS from the environment when set.
unsigned long long wait_limit_ns();
// Stage marks of ks_trace_stages: record the calling thread's event `slot`
// on the stream when tracing is on (no-op otherwise).
constexpr int kTraceMarks = 5;
void trace_mark(int slot, cudaStream_t stream);

}  // namespace ks

// ---------------------------------------------------------------- device side

__device__ __forceinline__ unsigned long long ks_globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ks_ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ks_ld_volatile(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}

// Device-wide barrier for a cooperative (co-resident) grid.  *count starts
// at zero and only grows: barrier number `epoch` (1, 2, ...) completes when it
// reaches epoch * nblocks, so arriving is a single atomic and there is no reset
// to order.  Every block passes the same sequence of barriers and keeps its own
// epoch.  A wait that exceeds limit_ns records KS_ERR_TIMEOUT in *err and
// returns; every caller then sees the error flag and leaves its loop, so no
// block waits without bound.  Returns true when no error is recorded; the
// answer is the same for every thread of the block (thread 0 reads the flag
// and the closing barrier broadcasts it), so callers may branch on it around
// further block barriers.
__device__ __forceinline__ bool ks_grid_sync(unsigned* count, unsigned nblocks,
                                             unsigned& epoch, int* err,
                                             unsigned long long limit_ns) {
  __syncthreads();
  ++epoch;
  int bad = 0;
  if (threadIdx.x == 0) {
    const unsigned target = epoch * nblocks;
    __threadfence();
    atomicAdd(count, 1u);
    if (ks_ld_acquire(count) < target) {
      const unsigned long long t0 = ks_globaltimer();
      while (ks_ld_acquire(count) < target) {
        __nanosleep(20);
        if (ks_globaltimer() - t0 > limit_ns) {
          atomicCAS(err, 0, KS_ERR_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
    bad = ks_ld_volatile(err) != 0;
  }
  return __syncthreads_or(bad) == 0;
}
