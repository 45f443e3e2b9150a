// Time-bounded mbarrier waits shared by the tcgen05 kernels.
//
// A wait polls mbarrier.try_wait and gives up after OA_WAIT_NS nanoseconds
// of %globaltimer (200 ms, far above any legitimate stage wait, which is
// microseconds).  The caller then takes its error path: set the device error
// flag, wait (again bounded) for the bulk copies it issued, free its TMEM
// and return, so the context stays usable and oa_gpu_check reports the
// failure.
#pragma once
#include <stdint.h>

#ifndef OA_WAIT_NS
#define OA_WAIT_NS 200000000ull
#endif

__device__ __forceinline__ uint64_t oa_globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// true once phase `phase` of the mbarrier at shared address `a` completed;
// false after OA_WAIT_NS
__device__ __forceinline__ bool oa_mbar_wait_bounded(uint32_t a, uint32_t phase) {
  const uint64_t t0 = oa_globaltimer();
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(phase) : "memory");
    if (ok) return true;
    if ((it & 63u) == 63u && oa_globaltimer() - t0 > OA_WAIT_NS) return false;
  }
}
