// bins.cuh -- sample decode and per-bin products shared by the FFT kernels.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace sws {

// Level of one NBIT-bit code: 8-bit offset binary (2b - 255)/256
// (format_vdif.c:117); 2-bit and 1-bit through the format's level table
// lv = {code 0, 1, 2, 3} (mark5_format_mark5b.c:59-96, format_vdif.c:69-73).
template <int NBIT>
__device__ __forceinline__ float decode_level(uint32_t code, float4 lv)
{
   if constexpr (NBIT == 8) {
      return fmaf(lv.x, (float)(code ^ __float_as_uint(lv.z)), lv.y);
   } else if constexpr (NBIT == 2) {
      float lo = (code & 1u) ? lv.y : lv.x;
      float hi = (code & 1u) ? lv.w : lv.z;
      return (code & 2u) ? hi : lo;
   } else {
      return (code & 1u) ? lv.y : lv.x;
   }
}

// Accumulate the products of one bin from Z_k (zk) and Z_{N-k} (zm).
// A' = 2A, B' = 2B; the reduction applies the 1/4.
__device__ __forceinline__ void acc_bin(float *acc4, int mode, float2 zk, float2 zm)
{
   float2 A = make_float2(zk.x + zm.x, zk.y - zm.y);
   if (mode == MODE_XPOL) {
      float2 B = make_float2(zk.y + zm.y, zm.x - zk.x);
      acc4[0] = fmaf(A.x, A.x, fmaf(A.y, A.y, acc4[0]));
      acc4[1] = fmaf(B.x, B.x, fmaf(B.y, B.y, acc4[1]));
      acc4[2] = fmaf(A.x, B.x, fmaf(A.y, B.y, acc4[2]));
      acc4[3] = fmaf(A.y, B.x, fmaf(-A.x, B.y, acc4[3]));
   } else if (mode == MODE_AUTOSUM) {
      float s = fmaf(zk.x, zk.x, fmaf(zk.y, zk.y, fmaf(zm.x, zm.x, zm.y * zm.y)));
      acc4[0] = fmaf(2.0f, s, acc4[0]);
   } else {
      acc4[0] = fmaf(A.x, A.x, fmaf(A.y, A.y, acc4[0]));
   }
}

}  // namespace sws
