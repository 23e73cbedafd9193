// mbar.cuh -- shared-memory mbarrier helpers (sm_100a) of the TMA-fed and
// tensor-core kernels.  Every wait is bounded.
#pragma once

#include <cstdint>

namespace ofg {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
   return (uint32_t)__cvta_generic_to_shared(p);
}

constexpr long long kMbarSpin = 1LL << 26;

// waits for the given phase of an mbarrier, at most kMbarSpin polls
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase)
{
   for (long long spins = 0; spins < kMbarSpin; ++spins) {
      uint32_t done;
      asm volatile(
         "{\n\t.reg .pred P1;\n\t"
         "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
         "selp.b32 %0, 1, 0, P1;\n\t}\n"
         : "=r"(done)
         : "r"(addr), "r"(phase)
         : "memory");
      if (done) return true;
   }
   return false;
}

// one arrival that also announces `bytes` of transactions on the barrier
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes)
                : "memory");
}

}  // namespace
}  // namespace ofg
