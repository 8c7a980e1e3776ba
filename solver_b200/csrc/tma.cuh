// Tensor-memory-accelerator (TMA) plane loads and mbarrier waits for the
// plane-pipelined stencil kernels, plus the host-side tensor-map encoding.
//
// Every load here is a plain 3-D tiled cp.async.bulk.tensor into this CTA's
// shared memory from this GPU's own memory (no multicast, no cluster), and
// every wait is bounded: a wait that gives up records a fault code and the
// kernel finishes its remaining work on whatever is in shared memory, so the
// host sees an error instead of a hang.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace ofb {
namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the barrier initialisation visible to the async proxy (the TMA unit).
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses to shared memory before
// later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Plain arrival (no transaction bytes): a consumer warp releasing a slot.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                        int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for phase `parity` of the barrier; gives up after `limit` polls
// (each try_wait itself suspends for a while), records `code` in *fault and
// returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* fault, int code,
                                          int limit = 1 << 22) {
  for(int it = 0; it < limit; ++it)
    if(mbar_try_wait(bar, parity)) return true;
  if(fault != nullptr) atomicOr(fault, code);
  return false;
}

// Host: a 3-D tiled tensor map over a compact array (nx, ny, nz) of 4- or
// 8-byte elements with box (bx, by, 1).  Checks the rules the TMA unit relies
// on: 16-byte aligned base, row pitch a multiple of 16 bytes, inner box extent
// a multiple of 16 bytes.
CUtensorMap make_map_3d(const void* base, int elem_bytes, int nx, int ny, int nz, int bx, int by);

}  // namespace tma
}  // namespace ofb
