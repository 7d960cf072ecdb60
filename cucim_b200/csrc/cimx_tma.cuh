// cimx_tma.cuh — tensor-memory-accelerator (TMA) tile loads and mbarrier
// waits for sm_100a, written as inline PTX.
//
// Every wait is bounded: after kWaitLimit polls the kernel records an error
// code in the per-device status word it was given (read back with
// cimx_device_status()) and gives up instead of spinning forever. No load
// here uses cluster multicast.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cimx {

constexpr long long kWaitLimit = 1ll << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses to shared memory before
// later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait for `phase` of an mbarrier. Returns false (and records
// CIMX_E_TIMEOUT in *status) if the barrier did not complete within `limit`
// polls (kWaitLimit in the kernels; cimx_wait_selftest passes a small one).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int* status,
                                          long long limit = kWaitLimit) {
  for (long long i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, phase)) return true;
  if (status) atomicExch(status, -6 /* CIMX_E_TIMEOUT */);
  return false;
}

// 3-D tiled TMA load of box {x, y, z} starting at the given coordinates into
// shared memory, completing on `bar`. x * sizeof(T) must be a multiple of 16.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// Host: encode a 3-D tiled tensor map over a C-contiguous (Z, Y, X) array.
// Returns false when the layout is not TMA-eligible (alignment, extents).
// swizzle128 selects the 128-byte shared-memory swizzle (box_x * element
// size must then be at most 128 bytes and the destination 1024-byte aligned).
bool make_tensor_map_3d(CUtensorMap* map, const void* base, int dtype, long long X, long long Y,
                        long long Z, int box_x, int box_y, bool swizzle128 = false);

// Host: the current device's status word (device memory, allocated once).
int* device_status_word();

}  // namespace cimx
