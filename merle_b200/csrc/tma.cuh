// tma.cuh - TMA bulk and tensor copies (cp.async.bulk, cp.async.bulk.tensor)
// global -> shared with mbarrier completion, and a bounded mbarrier wait.
// Every copy lands in the issuing CTA's own shared memory, from this GPU's
// memory.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace mb {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive on `bar` announcing `bytes` of transaction to come.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// 2-D tiled tensor copy global -> shared of the box at (x, y) (x the inner
// coordinate; x * element size a multiple of 16 bytes), completing on `bar`.
// Elements outside the tensor read as zero.  `map` is the generic address of
// a kernel-parameter (__grid_constant__) tensor map.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// 16-byte asynchronous copy global -> shared (both addresses 16-byte
// aligned), bypassing L1.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

// Makes `bar` receive one arrival once every cp.async this thread issued so
// far has landed (the arrival is not pre-counted: the barrier's expected
// count includes it).
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Waits for every cp.async this thread issued.
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Bulk prefetch of `bytes` (multiple of 16; address 16-byte aligned) of
// global memory into L2; no completion to wait for.
__device__ __forceinline__ void prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// One arrival on `bar` (release semantics: this thread's earlier shared
// memory writes are visible to threads that see the phase complete).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of `bar` with the given parity.  Each try_wait
// may suspend the thread for a hardware-chosen interval; after `limit` tries
// the wait gives up, records (code, block) in errw and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t *errw,
                                                  uint32_t code, uint32_t limit = (1u << 20)) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (errw) {
    if (atomicCAS(errw, 0u, 1u) == 0u) {
      errw[1] = code;
      errw[2] = blockIdx.x;
    }
  }
  return false;
}

}  // namespace mb
