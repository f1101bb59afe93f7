// tma.cuh -- the Tensor Memory Accelerator (TMA) and mbarrier operations the
// tiled line solves use, as inline PTX (sm_90 and later; built for sm_100a):
//
//   * a tiled tensor load, global -> shared, completing on an mbarrier
//     (cp.async.bulk.tensor ... mbarrier::complete_tx::bytes), and a tiled
//     tensor store, shared -> global, tracked by a bulk group;
//   * mbarrier init / arrive.expect_tx / try_wait.parity, with every wait
//     bounded: a wait that runs out records A3G_ERR_TIMEOUT in the device
//     error word and returns false, so the kernel can leave instead of
//     spinning;
//   * the proxy fences between the threads' own shared-memory accesses and
//     the asynchronous (TMA) proxy.
//
// Every load here copies from this GPU's own memory into the shared memory
// of the CTA that issues it alone; each CTA fetches its own tiles.
//
// Host side: tensor maps are encoded with the driver's cuTensorMapEncodeTiled,
// reached through cudaGetDriverEntryPoint so the library links no libcuda.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace a3g {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes the barrier initialisation visible to the asynchronous proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.b32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.  Each
// try_wait may itself suspend the thread for a hardware-chosen interval;
// 2^22 attempts is seconds, far beyond any tile copy.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 22); it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Tiled 4-D tensor load of one box into shared memory; completes
// box-bytes of transaction count on bar.  Coordinates are element indices
// (x innermost); elements outside the tensor read as zero.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y,
                                            int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

// Tiled 2-D tensor load of one box into shared memory (as tma_load_4d).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Tiled 4-D tensor store of one box from shared memory; elements outside the
// tensor are not written.  Tracked by the issuing thread's bulk groups.
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, const void *src, int x, int y, int z,
                                             int w) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z), "r"(w)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// the issuing thread's committed stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read0() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// the issuing thread's committed stores are complete
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// orders this thread's generic-proxy shared-memory accesses before later
// asynchronous-proxy (TMA) accesses of the same memory
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// orders this thread's generic-proxy accesses of every state space (global
// memory included) before its later asynchronous-proxy (TMA) accesses
__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace a3g
