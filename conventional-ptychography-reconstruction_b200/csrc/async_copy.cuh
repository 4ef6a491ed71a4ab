// async_copy.cuh -- TMA bulk copies, L2 prefetch and mbarrier waits (sm_90+/sm_100a PTX).
//
// Every wait is bounded: after kMaxWaitIters unsuccessful try_wait polls the
// caller gets `false` and must record PTYCHO_ERR_TIMEOUT and leave.
#pragma once
#include "common.cuh"

namespace pty {

constexpr int kMaxWaitIters = 1 << 22;

PTY_DEVI uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

PTY_DEVI void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

PTY_DEVI void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// arrive (count 1) and announce `bytes` of incoming transaction
PTY_DEVI void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

PTY_DEVI bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for the phase with the given parity to complete
PTY_DEVI bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < kMaxWaitIters; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// global -> shared bulk copy (both addresses 16-byte aligned, bytes % 16 == 0)
PTY_DEVI void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// hint: bring [p, p + bytes) into L2 (p 16-byte aligned, bytes % 16 == 0)
PTY_DEVI void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// prefetch the byte range [lo, hi) clipped to [base, end) with 16-byte rounding
PTY_DEVI void prefetch_l2_range(const char* lo, const char* hi, const char* base, const char* end) {
  const uintptr_t b = reinterpret_cast<uintptr_t>(base), e = reinterpret_cast<uintptr_t>(end);
  uintptr_t a = reinterpret_cast<uintptr_t>(lo) & ~uintptr_t(15);
  uintptr_t z = (reinterpret_cast<uintptr_t>(hi) + 15) & ~uintptr_t(15);
  if (a < ((b + 15) & ~uintptr_t(15))) a = (b + 15) & ~uintptr_t(15);
  if (z > (e & ~uintptr_t(15))) z = e & ~uintptr_t(15);
  if (z > a) prefetch_l2(reinterpret_cast<const void*>(a), static_cast<uint32_t>(z - a));
}

}  // namespace pty
