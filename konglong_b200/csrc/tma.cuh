// tma.cuh - Tensor Memory Accelerator and mbarrier helpers (sm_100a inline PTX)
// for the plane pipelines of the FD8 kernels.  Loads are plain (non-multicast)
// cp.async.bulk.tensor copies into this CTA's own shared memory; every wait on
// an mbarrier is bounded.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace rtm {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// producer: announce `bytes` of TMA traffic on this phase and arrive
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// try_wait with a suspend-time hint: a waiting warp sleeps (up to ~1 us)
// until the phase completes instead of spinning on the issue slots
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
      : "memory");
  return ok != 0;
}

// plain arrive (count 1, no transaction bytes)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase of `parity`.  Gives up after 2^16 polls, or as
// soon as another CTA has raised *err, sets *err and returns false (the caller
// then skips its compute; the copies it waited for are its own).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err) {
  for (uint32_t it = 0; it < (1u << 16); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63) == 63 && err && *(volatile int *)err) return false;
  }
  if (err) atomicExch(err, 1);
  return false;
}

// Bounded wait used on an error path before a CTA exits: polls the phase of
// `parity` up to 2^16 times whatever *err says (its own copies must land
// before the shared memory is released).
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 16); it++)
    if (mbar_try_wait(bar, parity)) return;
}

// 3-D tiled load (coordinates innermost first: z, x, y) completing on `bar`.
// The proxy fence orders earlier generic writes of this stage before the copy.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int cz, int cx, int cy) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(cz), "r"(cx), "r"(cy), "r"(smem_u32(bar))
      : "memory");
}

// 4-D tiled load (coordinates innermost first) completing on `bar`
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// 3-D tiled store of a shared-memory box (bulk-group completion); elements
// outside the tensor are not written
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int cz, int cx, int cy) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"((uint64_t)map),
               "r"(smem_u32(src)), "r"(cz), "r"(cx), "r"(cy)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// wait until every committed bulk store has finished reading shared memory
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// order this thread's generic shared-memory writes before later async-proxy reads
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 4-byte asynchronous global -> shared copy (no register staging)
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

}  // namespace rtm
