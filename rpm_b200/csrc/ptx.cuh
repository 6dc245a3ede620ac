// Shared PTX helpers of the TMA / mbarrier pipelines (persistent Lanczos
// kernel, tensor-core Gram): shared-memory addresses, mbarriers with bounded
// waits, bulk global -> shared copies.
#pragma once

namespace rpm {
namespace ptx {

constexpr long long kWaitCycles = 4000000000LL;  // about 2 s at 1.965 GHz

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for phase `parity` of `bar` to complete; false after the time limit
// or when another thread already raised the status word.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* status) {
  const long long t0 = clock64();
  for (int spin = 0;; ++spin) {
    if (mbar_test(bar, parity)) return true;
    if ((spin & 63) == 63) {
      if (*reinterpret_cast<volatile int*>(status)) return false;
      if (clock64() - t0 > kWaitCycles) {
        atomicExch(status, 1);
        return false;
      }
    }
  }
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace ptx
}  // namespace rpm
