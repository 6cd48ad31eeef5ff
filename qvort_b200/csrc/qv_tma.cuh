// qv_tma.cuh -- 1-D TMA bulk copies into a block's own shared memory and the
// mbarriers they complete, with bounded waits (the direct sums' source tiles).
// No cluster multicast: every copy reads this GPU's own global memory into the
// issuing block's shared memory.
#pragma once
#include "qv_internal.cuh"

// A wait gives up after QV_STAGE_WAIT_NS of wall time (and an iteration cap);
// the caller then sets QV_STAT_STAGE and stops, so a copy that never lands
// ends the launch with an error, not a hang.
#define QV_STAGE_WAIT_NS 1000000000ull  // 1 s

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

// make the initialised barriers visible to the copy engine before first use
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// one thread: arm the barrier for `bytes` and start the copy
__device__ __forceinline__ void stage_copy(unsigned dst, const void *src, unsigned bytes,
                                           unsigned bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ unsigned long long wall_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait for the barrier's phase of parity `parity` to complete, giving up
// after QV_STAGE_WAIT_NS or 2^30 polls
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = wall_ns();
  for (unsigned it = 0; it < (1u << 30); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (wall_ns() - t0 > QV_STAGE_WAIT_NS) break;
  }
  return false;
}

