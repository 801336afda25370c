// pipe.cuh — shared-memory producer/consumer rings on mbarriers, with bounded waits.
//
// A ring of S stages: full[s] completes when the producers have filled stage s (their
// arrivals plus every cp.async they issued for it), empty[s] when the consumer warps
// have released it. Every wait is bounded by a %globaltimer limit; a thread that gives
// up sets the CTA's abort flag and the plan's error word (reported by
// shtb_plan_status as SHTB_ERR_TIMEOUT), and every other waiter of the CTA returns as
// soon as it sees the flag.
#pragma once

#include <cuda_runtime.h>

namespace shtb {

constexpr unsigned long long kPipeWaitNs = 2000000000ull;   // 2 s

__device__ __forceinline__ unsigned pipe_smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long pipe_gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void pipe_bar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(pipe_smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void pipe_bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Release-arrive: the thread's earlier shared-memory writes are visible to threads that
// observe the phase completion.
__device__ __forceinline__ void pipe_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(pipe_smem_u32(bar)) : "memory");
}
// The barrier's current phase also waits for every cp.async this thread issued before.
__device__ __forceinline__ void pipe_arrive_cp_async(unsigned long long* bar) {
  asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(pipe_smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool pipe_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(pipe_smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of the given parity: false after the limit or once another
// thread of the CTA gave up.
__device__ __forceinline__ bool pipe_wait(unsigned long long* bar, unsigned parity, volatile int* abort_flag,
                                          int* err) {
  if (pipe_test(bar, parity)) return true;
  const unsigned long long t0 = pipe_gtimer();
  while (!pipe_test(bar, parity)) {
    if (*abort_flag) return false;
    if (pipe_gtimer() - t0 > kPipeWaitNs) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// 16-byte cp.async global -> shared; src_bytes = 0 writes zeros without reading src.
__device__ __forceinline__ void pipe_cp16(void* smem, const void* gmem, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(pipe_smem_u32(smem)), "l"(gmem),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void pipe_cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace shtb
