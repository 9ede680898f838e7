// tc.cuh -- 5th-generation tensor-core (tcgen05) building blocks for sm_100a.
//
// The split-precision DFT stages issue tcgen05.mma (kind::f16, FP16 operands
// from shared memory, FP32 accumulators in tensor memory) from one thread
// and read the accumulators back with tcgen05.ld.  This header holds the
// PTX wrappers and the descriptor encodings they need:
//
//  * shared-memory matrix descriptor (64 bit): start address >> 4 in bits
//    [0,14), leading-dimension byte offset >> 4 in [16,30), stride-dimension
//    byte offset >> 4 in [32,46), descriptor version 1 in [46,48), layout
//    (swizzle) type in [61,64); only the unswizzled layout is used here.
//    Unswizzled operands are tiled in 8 x 16-byte core matrices (128
//    contiguous bytes).  K-major: a core matrix is 8 rows (M or N) of 8
//    consecutive K values; LBO = byte distance between core matrices along
//    K, SBO = along M/N.  MN-major: a core matrix is 8 K-rows of 8
//    consecutive M values; again LBO steps along K and SBO along M/N.
//  * instruction descriptor (32 bit) of kind::f16: D format F32 (bits 4-5 =
//    1), A/B format F16 (0), A major in bit 15 (1 = MN-major), B major in
//    bit 16, N >> 3 in bits [17,23), M >> 4 in bits [24,29).
//
// Every wait on an mbarrier is bounded; a wait that gives up returns false
// and the caller reports it through the launch's status word.
#pragma once

#include <cstdint>

namespace sws {
namespace tc {

__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool a_mn, bool b_mn)
{
   return (1u << 4) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
          ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
   return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
          ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Tensor-memory allocation by one full warp; the base address lands in *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_saddr, uint32_t ncols)
{
   asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_saddr),
                "r"(ncols)
                : "memory");
   asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
   asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]; issued by a single thread.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate)
{
   asm volatile(
       "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
       " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
       "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
       : "memory");
}

// Arrive (once) on an mbarrier of this CTA when all earlier tcgen05 ops of
// the issuing thread have completed.
__device__ __forceinline__ void commit(uint32_t mbar_saddr)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                    mbar_saddr)
                : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core's (async proxy) reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 16 consecutive 32-bit columns of this warp's 32 lanes (thread i <- lane base+i).
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16])
{
   uint32_t r[16];
   asm volatile(
       "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
       : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
         "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
       : "r"(taddr));
#pragma unroll
   for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init_cta(uint32_t mbar, int count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
   asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Bounded wait for the completion of phase `parity`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
   for (int it = 0; it < (1 << 20); it++) {
      uint32_t done;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                   " selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done)
                   : "r"(mbar), "r"(parity)
                   : "memory");
      if (done) return true;
      if (it > 32) __nanosleep(32);
   }
   return false;
}

// Byte offset of element (m, k) in an unswizzled FP16 operand.
__host__ __device__ constexpr uint32_t kmajor_off(int m, int k, uint32_t lbo, uint32_t sbo)
{
   return (uint32_t)(m >> 3) * sbo + (uint32_t)(k >> 3) * lbo + (uint32_t)(m & 7) * 16u + (uint32_t)(k & 7) * 2u;
}
__host__ __device__ constexpr uint32_t mnmajor_off(int m, int k, uint32_t lbo, uint32_t sbo)
{
   return (uint32_t)(m >> 3) * sbo + (uint32_t)(k >> 3) * lbo + (uint32_t)(k & 7) * 16u + (uint32_t)(m & 7) * 2u;
}

}  // namespace tc
}  // namespace sws
