// Bulk asynchronous copies (the TMA engine's non-tensor form) from this GPU's
// global memory into the executing CTA's shared memory, completed through an
// mbarrier transaction count.  No multicast: every copy lands in the issuing
// CTA only.  Addresses must be 16-byte aligned and sizes multiples of 16.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "spoc_tc.cuh"

namespace spoc {
namespace bulk {

// polls of an mbarrier before a wait gives up (far beyond any copy's time)
constexpr uint32_t kWaitLimit = 1u << 26;
constexpr uint32_t kChunk = 32768;  // bytes per copy instruction

__device__ __forceinline__ void arrive_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mbar)),
               "r"(bytes)
               : "memory");
}

// expect_tx without arriving (several lanes announce their own copies)
__device__ __forceinline__ void expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(tc::smem_u32(mbar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tc::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tc::smem_u32(mbar))
      : "memory");
}

// Whole-block staging of `bytes` (a multiple of 16) from src to dst through
// the block's mbarrier `mbar` (phase 0): thread 0 initialises the barrier,
// announces the bytes and issues the copies; every thread waits.  Returns
// false on every thread of the block when the wait limit ran out: then bit 2
// of *flag is set and the block waits once more (bounded) for its copies
// before the caller returns.  Must be called by all threads of the block,
// once per barrier.
__device__ __forceinline__ bool stage_block(void *dst, const void *src, uint32_t bytes,
                                            uint64_t *mbar, int *flag) {
  if (threadIdx.x == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    arrive_expect_tx(mbar, bytes);
    for (uint32_t off = 0; off < bytes; off += kChunk) {
      const uint32_t n = bytes - off < kChunk ? bytes - off : kChunk;
      copy_g2s(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, n, mbar);
    }
  }
  const bool ok = tc::mbar_wait(mbar, 0, kWaitLimit);
  const bool any_failed = __syncthreads_or(!ok);
  if (any_failed) {
    if (threadIdx.x == 0 && flag) atomicOr(flag, 2);
    // give the copies in flight (bounded) time to land before the block exits
    tc::mbar_wait(mbar, 0, kWaitLimit);
    __syncthreads();
  }
  return !any_failed;
}

}  // namespace bulk
}  // namespace spoc
