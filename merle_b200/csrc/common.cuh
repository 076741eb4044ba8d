// common.cuh - shared host/device helpers of the merle_b200 CUDA library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <nvtx3/nvToolsExt.h>
#include "merle_b200.h"

namespace mb {

// An NVTX range over a scope (engine phases show up by name in Nsight
// Systems; without a profiler attached the calls do nothing).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------------- errors
// Thread-local message of the last failing call (mb_last_error()).
void set_error(const char *fmt, ...);
mb_status fail(mb_status st, const char *fmt, ...);
mb_status cuda_fail(cudaError_t e, const char *what);

#define MB_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return ::mb::cuda_fail(e_, #call);                \
  } while (0)

#define MB_CHECK(st)                                                         \
  do {                                                                       \
    mb_status s_ = (st);                                                     \
    if (s_ != MB_OK) return s_;                                              \
  } while (0)

// Launch check: reports configuration errors of the last launch.
#define MB_LAUNCH_CHECK(what)                                                \
  do {                                                                       \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess) return ::mb::cuda_fail(e_, what);                 \
  } while (0)

// ---------------------------------------------------------------- device info
struct DevInfo {
  int device = -1;
  int sms = 148;
  int max_smem_optin = 227 * 1024;
  int max_threads_sm = 2048;
};
// Properties of the current device (cached per device).
const DevInfo &dev_info();

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// A stream-ordered memory pool per device for short-lived scratch, which
// keeps what it was given (release threshold: unlimited) so that repeated
// calls reuse it instead of mapping fresh memory each time.
cudaMemPool_t scratch_pool();

// Device scratch from that pool, freed on scope exit (stream-ordered: after
// the work enqueued on `st` before the exit).
struct Scratch {
  cudaStream_t st;
  void *ptrs[16];
  int n = 0;
  explicit Scratch(cudaStream_t s) : st(s) {}
  ~Scratch() {
    for (int i = 0; i < n; ++i) cudaFreeAsync(ptrs[i], st);
  }
  Scratch(const Scratch &) = delete;
  Scratch &operator=(const Scratch &) = delete;
  template <typename T>
  mb_status get(T **p, uint64_t count) {
    cudaMemPool_t pool = scratch_pool();
    if (!pool || n == 16) return fail(MB_ERR_CUDA, "scratch: no memory pool or too many buffers");
    void *q = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&q, count ? count * sizeof(T) : sizeof(T), pool, st);
    if (e != cudaSuccess) return cuda_fail(e, "scratch allocation");
    ptrs[n++] = q;
    *p = static_cast<T *>(q);
    return MB_OK;
  }
};

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
inline uint64_t round_up(uint64_t a, uint64_t b) { return ceil_div(a, b) * b; }

// ---------------------------------------------------------------- device
// Error word written by kernels whose bounded waits ran out.  Index 0 is a
// flag, index 1 a code (which wait), index 2 the block that gave up.
// MB_DEVERR_TMA_WAIT: copies into a shared-memory stage did not arrive;
// MB_DEVERR_IDLE_WAIT: a stage was not released by the warps reading it.
// A kernel that gave up has left its outputs partial: the host treats the
// whole launch's results as lost (and zeroes what it hands back).
enum { MB_DEVERR_NONE = 0, MB_DEVERR_TMA_WAIT = 1, MB_DEVERR_IDLE_WAIT = 2 };
uint32_t *device_error_word();   // per-device, allocated on first use
mb_status check_device_error(cudaStream_t s);

// mb_bitmap_create_levels over a foreign key that also writes every row's
// dimension value to dout (dimension width; 0 where the key leaves the
// dimension) and counts such rows in *bad (either may be NULL): the
// denormalised column comes out of the same pass.  MB_ERR_INVALID when the
// levels need more than one pass.
mb_status bitmap_create_levels_join(const mb_src *src, uint64_t nrows, const mb_level *levels, uint32_t nlevels,
                                    uint64_t stride_words, void *stream, void *dout, unsigned long long *bad);

// Unsigned 32-bit division by an invariant divisor d >= 1 as a multiply-high
// and shifts (Granlund and Montgomery, "Division by Invariant Integers using
// Multiplication", PLDI 1994, figure 4.1): with l = ceil(log2 d),
// m = floor(2^32 * (2^l - d) / d) + 1, sh1 = min(l, 1), sh2 = max(l - 1, 0),
// x / d = (t + ((x - t) >> sh1)) >> sh2 where t = mulhi(m, x).
struct DivMagic {
  uint32_t m, sh1, sh2;
};
inline DivMagic div_magic(uint32_t d) {
  uint32_t l = 0;
  while (l < 32 && (1ull << l) < d) ++l;
  DivMagic r;
  r.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
  r.sh1 = l < 1 ? l : 1;
  r.sh2 = l > 0 ? l - 1 : 0;
  return r;
}
__host__ __device__ inline uint32_t div_by_magic(uint32_t x, uint32_t m, uint32_t sh1, uint32_t sh2) {
#ifdef __CUDA_ARCH__
  const uint32_t t = __umulhi(m, x);
#else
  const uint32_t t = (uint32_t)(((uint64_t)m * x) >> 32);
#endif
  return (t + ((x - t) >> sh1)) >> sh2;
}

// ssbDateToYear (ssb/ssbdemo.h:28-39): day 0 = 1992-01-01.
__host__ __device__ inline uint32_t date_to_year(uint32_t d) {
  // the year starts 0, 366, 731, 1096, 1461, 1827, 2192 (1992 and 1996 leap)
  // are exactly the d with 4d / 1461 stepping: the same result as comparing
  // with each start, in one multiply-high instead of six compares
  return d >= 2557 ? 6u : (4u * d) / 1461u;
}

__device__ __forceinline__ uint64_t load_width(const void *p, uint64_t i, uint32_t w) {
  switch (w) {
  case 1: return __ldg(reinterpret_cast<const uint8_t *>(p) + i);
  case 2: return __ldg(reinterpret_cast<const uint16_t *>(p) + i);
  case 4: return __ldg(reinterpret_cast<const uint32_t *>(p) + i);
  default: return __ldg(reinterpret_cast<const unsigned long long *>(p) + i);
  }
}

// Streaming 128-bit load of 4 bitmap words (read once: evict-first in L1).
__device__ __forceinline__ uint4 ld_stream4(const uint32_t *p) {
  return __ldcs(reinterpret_cast<const uint4 *>(p));
}

}  // namespace mb
