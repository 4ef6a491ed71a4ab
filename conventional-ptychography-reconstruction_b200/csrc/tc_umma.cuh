// tc_umma.cuh -- thin wrappers over the sm_100a 5th-generation tensor core
// instructions (tcgen05.*) used by the complex-MLP kernels.
//
// Shared-memory operands use the SWIZZLE_NONE canonical layout: 8 x 16-byte
// core matrices; a descriptor gives the start address, the leading-dimension
// byte offset (LBO) and stride-dimension byte offset (SBO).  For a K-major
// operand element (row r, k) sits at (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2;
// for an MN-major operand element (mn, k) sits at (mn/8)*SBO + (k/8)*LBO +
// (k%8)*16 + (mn%8)*2.  Accumulators live in tensor memory (TMEM): row i of
// an M = 128 tile is TMEM lane i, one fp32 column per output column.
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace pty {
namespace tc {

PTY_DEVI uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// shared-memory matrix descriptor (sm100 version field = 1, no swizzle)
PTY_DEVI uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// instruction descriptor, kind::f16: BF16 x BF16 -> FP32, dense
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// D (+)= A * B^T on the tensor core; issued by a single thread
PTY_DEVI void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// arrive on an mbarrier when all previously issued tcgen05.mma of this thread complete
PTY_DEVI void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

PTY_DEVI void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
PTY_DEVI void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make generic-proxy shared-memory writes visible to the tensor core (async proxy)
PTY_DEVI void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// warp-wide: allocate / free `ncols` TMEM columns; the base address is written to *dst
PTY_DEVI void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
               "r"(ncols)
               : "memory");
}
PTY_DEVI void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
PTY_DEVI void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// warp-wide: 16 consecutive fp32 columns of this thread's TMEM lane.  The
// wait is tied to the destination registers ("+r") so no use of them can be
// scheduled before the load has completed.
PTY_DEVI void ld16(uint32_t taddr, float (&r)[16]) {
  uint32_t u[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
        "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(u[0]), "+r"(u[1]), "+r"(u[2]), "+r"(u[3]), "+r"(u[4]), "+r"(u[5]), "+r"(u[6]), "+r"(u[7]),
                 "+r"(u[8]), "+r"(u[9]), "+r"(u[10]), "+r"(u[11]), "+r"(u[12]), "+r"(u[13]), "+r"(u[14]),
                 "+r"(u[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(u[i]);
}

}  // namespace tc
}  // namespace pty
