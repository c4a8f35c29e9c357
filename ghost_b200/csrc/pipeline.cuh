// pipeline.cuh -- asynchronous tile pipeline for the FFT passes.
//
// Tiles move HBM -> shared memory with TMA bulk copies (cp.async.bulk,
// plain global-to-shared form, no multicast) that complete on an mbarrier
// per stage.  A persistent CTA keeps STAGES-1 tiles in flight while it
// transforms the current one, so the copy engine, not warp occupancy,
// hides the HBM latency.
//
// Every wait is bounded: after `cap` unsuccessful polls the CTA agrees (by
// __syncthreads_or) to give up, records GHOST_ERR_TIMEOUT in the context's
// device status word, drains its own copies still in flight (with a fixed
// generous bound) and returns.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Make the initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Order this thread's earlier generic shared-memory accesses before later
// async-proxy writes into the same buffer.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// bytes must be a multiple of 16; both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// TMA tensor load of one box of a 3D tensor map (coordinates innermost
// first, in elements of the map's data type) into shared memory.  The
// innermost coordinate times the element size is a multiple of 16 bytes
// at every call site; dst is 128-byte aligned.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// TMA tensor store of one box from shared memory (bulk-group completion).
// Coordinates are never negative at the call sites; boxes that overrun the
// tensor are clipped by the hardware.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// this thread's committed bulk stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// ... and have completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// Hint: bring the 32-byte sector holding p into L2.
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of bar; false after cap polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t cap) {
  for (uint32_t n = 0; n < cap; ++n)
    if (mbar_test(bar, parity)) return true;
  return false;
}

constexpr uint32_t kDrainPolls = 1u << 24;

// With PipeCtl::stall set (fault-injection testing), a pass first waits on a
// barrier that nothing ever completes, so its bounded wait runs out.
__device__ __forceinline__ bool injected_stall_wait(uint64_t *never, uint32_t cap) {
  return mbar_wait(never, 0u, cap);
}

// Status word written on a timeout (GHOST_ERR_TIMEOUT).
__device__ __forceinline__ void record_timeout(int *status) {
  if (status) atomicExch(status, 5);
}

}  // namespace gb
