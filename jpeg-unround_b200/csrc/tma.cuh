// Helpers of the TMA-fed kernels (sm_100a): mbarriers and tiled bulk-tensor loads of a 3D box
// into shared memory (no cluster multicast: every load is of this GPU's own memory into this
// CTA's shared memory). Waits are bounded (kWaitLimit tries).
#pragma once

#include <cstdint>

#include <cuda.h>

namespace urb {

constexpr long long kWaitLimit = 1LL << 22;

__device__ __forceinline__ unsigned smem_address(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void barrier_init(std::uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_address(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void barrier_expect(std::uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_address(bar)), "r"(bytes)
               : "memory");
}

// One arrival (release: the thread's earlier writes are seen by whoever sees the phase end).
__device__ __forceinline__ void barrier_arrive(std::uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_address(bar)) : "memory");
}

__device__ __forceinline__ bool barrier_try(std::uint64_t* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_address(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for a phase of a barrier, at most `limit` tries; false where it ran out.
__device__ __forceinline__ bool barrier_wait(std::uint64_t* bar, unsigned parity, long long limit = kWaitLimit) {
  for (long long k = 0; k < limit; ++k) {
    if (barrier_try(bar, parity)) return true;
  }
  return false;
}

__device__ __forceinline__ void load_box(float* to, const CUtensorMap* map, std::uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_address(to)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_address(bar))
      : "memory");
}

// A contiguous bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// global into shared memory, completing on `bar`.
__device__ __forceinline__ void load_bulk(void* to, const void* from, unsigned bytes, std::uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_address(to)),
      "l"(from), "r"(bytes), "r"(smem_address(bar))
      : "memory");
}

}  // namespace urb
