// tcdft.cuh -- radix-16 DFT levels on the 5th-generation tensor cores:
// FP16 hi/lo split operands in shared memory, FP32 accumulators in tensor
// memory, one operand row per thread.  Used by the cluster kernel's
// tensor-core forms (Q = 4096 per CTA) and by the four-step row pass of
// 4096-point rows.
#pragma once

#include <cuda_fp16.h>

#include "tc.cuh"

namespace sws {

// ---------------------------------------------------------------------------
// Tensor-core split-precision stages (tcgen05.mma, FP16 x FP16 -> FP32 in TMEM)
// ---------------------------------------------------------------------------
// The CTA's Q = 4096-point transform is three radix-16 levels,
// q = q0 + 16 q1 + 256 q2 and kappa = k0 + 16 k1 + 256 k2:
//   level 1: DFT16 over q2 for each row r1 = q0 + 16 q1, then W_4096^{r1 k0};
//   level 2: DFT16 over q1 for each row (k0, q0), then W_256^{q0 k1};
//   level 3: DFT16 over q0 for each row (k1, k0) -> F[k0 + 16 k1 + 256 k2].
// Each level is the real GEMM  D[row][n] = sum_k A[row][k] B[k][n]  with
// 256 rows (two M = 128 tiles), K = 64 and N = 64:
//   A = [Re x hi | Im x hi | Re x lo | Im x lo]          (16 values each)
//   B = [[Mh | Ml]; [Mh | 0]],  M = s * [[C, -S]; [S, C]]-form of the DFT16
// so that D[:, n] + D[:, n + 32] = Ah Mh + Al Mh + Ah Ml (n < 32): the
// three products of an FP16 hi/lo split (hi = rn(x), lo = rn(x - hi)),
// about 22 significant bits, accumulated in FP32.  s = 1/4 keeps the FP16
// operands in range; the push multiplies the powers of 4 back (exact).
// The accumulators land in tensor memory, one TMEM lane per row, which is
// the thread's own row in the epilogue (warp w reads lanes 32 (w % 4) + i of
// tile w / 4, so row = threadIdx.x).  The epilogue loads its row's 16
// complex outputs, applies the next level's FP32 twiddle, splits them and
// stores them as the next level's operand in MN-major order: the level's
// output digit d = d0 + 8 d1 becomes the row digits of the next level, row
// (d0, g, d1) = d0 + 8 g + 128 d1 for the thread's remaining digit g < 16,
// so the thread's values d < 8 and d >= 8 are the 8 rows of row groups g
// and 16 + g of one K column (two 16-byte core-matrix rows per K value and
// part), and the 8 lanes of a shared-memory wavefront, which differ in g,
// write 8 distinct 16-byte bank groups (144-byte group stride).
// Level 1 is either on the tensor cores (operand = decoded, windowed
// samples, K-major rows) or an FP32 radix-16 in registers fused with the
// decode (PREC 1).

// hi/lo split of two floats into f16x2 words (lower half = first value)
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
   const __half2 h = __floats2half2_rn(a, b);
   const float2 hf = __half22float2(h);
   const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
   hi = *reinterpret_cast<const uint32_t *>(&h);
   lo = *reinterpret_cast<const uint32_t *>(&l);
}

__device__ __forceinline__ void st_shared_v4(uint32_t saddr, const uint32_t (&v)[4])
{
   asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(saddr), "r"(v[0]), "r"(v[1]), "r"(v[2]),
                "r"(v[3])
                : "memory");
}

// Operand geometry: 256 rows x 64 K values of FP16.
// MN-major (levels 2, 3): core matrices 8 K x 8 rows; rows step by SBO =
// 144 bytes (16 bytes of padding per core matrix), K groups by LBO = 32 x 144.
// K-major (level 1 on tensor cores): core matrices 8 rows x 8 K; K groups
// step by 128 bytes, row groups by 1024.
constexpr uint32_t TC_MN_SBO = 144, TC_MN_LBO = 32 * TC_MN_SBO;
constexpr uint32_t TC_K_LBO = 128, TC_K_SBO = 1024;
constexpr uint32_t TC_OPND_BYTES = 8 * TC_MN_LBO;  // 36864 >= 32768 (K-major)
constexpr uint32_t TC_BMAT_BYTES = 64 * 64 * 2;
constexpr uint32_t TC_TMEM_COLS = 128;             // two M = 128 tiles x N = 64 FP32 columns
// up to four resident CTAs of a tensor-core form share an SM's 512 columns,
// so no CTA's allocation ever waits for another's release
static_assert(4 * TC_TMEM_COLS <= 512, "tensor memory of the resident CTAs of one SM");

// 16 complex values into an MN-major operand: values 0-7 as the 8 rows of
// row group g0, values 8-15 as row group g1, K column kq of the real part
// and kq + 16 of the imaginary part (hi parts; lo parts at +32).
__device__ __forceinline__ void store_mn16(uint32_t opnd, int g0, int g1, int kq, const float2 (&v)[16])
{
#pragma unroll
   for (int c = 0; c < 2; c++) {
#pragma unroll
      for (int g = 0; g < 2; g++) {
         uint32_t hi[4], lo[4];
#pragma unroll
         for (int e = 0; e < 4; e++) {
            const float2 x = v[8 * g + 2 * e], y = v[8 * g + 2 * e + 1];
            split2(c ? x.y : x.x, c ? y.y : y.x, hi[e], lo[e]);
         }
         const int m = 8 * (g ? g1 : g0);
         st_shared_v4(opnd + tc::mnmajor_off(m, 16 * c + kq, TC_MN_LBO, TC_MN_SBO), hi);
         st_shared_v4(opnd + tc::mnmajor_off(m, 32 + 16 * c + kq, TC_MN_LBO, TC_MN_SBO), lo);
      }
   }
}

// Row `row` of the K-major level-1 operand from its 16 complex samples.
__device__ __forceinline__ void store_k16(uint32_t opnd, int row, const float2 (&v)[16])
{
#pragma unroll
   for (int c = 0; c < 2; c++) {
#pragma unroll
      for (int g = 0; g < 2; g++) {
         uint32_t hi[4], lo[4];
#pragma unroll
         for (int e = 0; e < 4; e++) {
            const float2 x = v[8 * g + 2 * e], y = v[8 * g + 2 * e + 1];
            split2(c ? x.y : x.x, c ? y.y : y.x, hi[e], lo[e]);
         }
         st_shared_v4(opnd + tc::kmajor_off(row, 16 * c + 8 * g, TC_K_LBO, TC_K_SBO), hi);
         st_shared_v4(opnd + tc::kmajor_off(row, 32 + 16 * c + 8 * g, TC_K_LBO, TC_K_SBO), lo);
      }
   }
}

// The B operand (K-major: 64 rows n of 64 K values) of the DFT16 scaled by
// `scale` (a power of two, so the scaling is exact).
__device__ __forceinline__ void fill_dft16_bmat(uint32_t bmat, int T, double scale = 0.25)
{
   for (int i = threadIdx.x; i < 64 * 64; i += T) {
      const int n = i >> 6, k = i & 63;
      const int part = k >> 5, cin = (k >> 4) & 1, j = k & 15;
      const int half = n >> 5, cout = (n >> 4) & 1, kk = n & 15;
      double sn, cs;
      sincospi(-2.0 * (double)((j * kk) & 15) / 16.0, &sn, &cs);  // W_16^{j kk} = cs + i sn
      // y = x W: Re y = Re x cs - Im x sn, Im y = Re x sn + Im x cs
      const double m = scale * ((cin == cout) ? cs : (cin == 0 ? sn : -sn));
      const __half h = __double2half(m);
      const __half l = __double2half(m - (double)__half2float(h));
      const __half val = (part == 0) ? (half == 0 ? h : l) : (half == 0 ? h : __double2half(0.0));
      asm volatile("st.shared.b16 [%0], %1;\n" ::"r"(bmat + tc::kmajor_off(n, k, 128, 1024)),
                   "h"(*reinterpret_cast<const unsigned short *>(&val))
                   : "memory");
   }
}

// Issue one level: two M = 128 tiles x four K = 16 steps into TMEM columns
// [0, 64) and [64, 128); one thread.
__device__ __forceinline__ void tc_issue_level(uint32_t tmem, uint32_t opnd, uint32_t bmat, bool kmajor,
                                               uint32_t mbar)
{
   tc::fence_after();
   const uint32_t id = tc::idesc_f16(128, 64, !kmajor, false);
#pragma unroll
   for (int t = 0; t < 2; t++) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
         const uint32_t a0 = kmajor ? opnd + (uint32_t)t * 16u * TC_K_SBO + (uint32_t)kk * 2u * TC_K_LBO
                                    : opnd + (uint32_t)t * 16u * TC_MN_SBO + (uint32_t)kk * 2u * TC_MN_LBO;
         const uint64_t ad = kmajor ? tc::smem_desc(a0, TC_K_LBO, TC_K_SBO) : tc::smem_desc(a0, TC_MN_LBO, TC_MN_SBO);
         const uint64_t bd = tc::smem_desc(bmat + (uint32_t)kk * 256u, 128u, 1024u);
         tc::mma_f16(tmem + 64u * (uint32_t)t, ad, bd, id, kk > 0);
      }
   }
   tc::commit(mbar);
}

// The calling thread's row (= threadIdx.x) of a level's output: 16 complex values.
__device__ __forceinline__ void tc_load_row(uint32_t tmem, float2 (&y)[16])
{
   const int w = threadIdx.x >> 5;
   const uint32_t ta = tmem + ((uint32_t)(32 * (w & 3)) << 16) + 64u * (uint32_t)(w >> 2);
   float a[16], b[16];
   tc::ld16(ta, a);
   tc::ld16(ta + 32, b);
   tc::ld_wait();
#pragma unroll
   for (int i = 0; i < 16; i++) y[i].x = a[i] + b[i];
   tc::ld16(ta + 16, a);
   tc::ld16(ta + 48, b);
   tc::ld_wait();
#pragma unroll
   for (int i = 0; i < 16; i++) y[i].y = a[i] + b[i];
}

}  // namespace sws
