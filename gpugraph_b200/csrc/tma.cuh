// Bulk (TMA, non-tensor) global -> shared copies completed on an mbarrier,
// for staging contiguous tiles (row/column offsets) into shared memory.
// Rules kept by every caller: source and destination 16-byte aligned, size a
// multiple of 16 bytes, source inside the allocation, no cluster multicast.
// Waits are bounded: a wait that runs out reports failure instead of hanging.
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace mg {

MG_DEVINL uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

MG_DEVINL void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before the
// async-proxy (bulk copy) writes issued after it.
MG_DEVINL void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

MG_DEVINL void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

MG_DEVINL void bulk_copy_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

MG_DEVINL bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of the barrier; false if the limit ran out.
MG_DEVINL bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, unsigned long long limit) {
  for (unsigned long long i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(32);
  }
  return false;
}

}  // namespace mg
