// spectra.cuh -- K2: windowed real FFT of frame pairs + spectral accumulation.
//
// Replaces the hot loop of TaskCoreIPP::doMaths (src/IA-32/TaskCoreIPP.cpp:
// 401-487): unpack -> window multiply (:427) -> forward real DFT (:430) ->
// |X|^2 accumulate with separate DC/Nyquist handling (:437-447) -> cross
// product X_i conj(X_j) (:456-487).
//
// Design (B200):
//  * Two real frames a, b of N samples are packed as z = w*(a + i b) and
//    transformed by ONE complex FFT of N points; A_k = (Z_k + conj Z_{N-k})/2
//    and B_k = (Z_k - conj Z_{N-k})/(2i) recover both real spectra, and
//    |A|^2, |B|^2, A conj(B) follow.  A dual-pol pair (X, Y) is one job; an
//    auto-only channel pairs two consecutive frames of itself.
//  * The N-point FFT is split N = P*Q over a thread-block cluster of P CTAs
//    (decimation in time): CTA p decodes, windows and transforms the
//    subsequence z[p + P q] (q < Q) in its shared memory (Stockham passes,
//    radices R1 R2 R3), then, after a cluster barrier, each thread gathers
//    F_p[k1] and F_p[Q-k1] from all P CTAs through distributed shared memory,
//    applies W_N^{p k1}, finishes a P-point DFT and holds both Z_k and Z_{N-k}
//    for its bins in registers.
//  * Spectra of consecutive jobs of a work item accumulate in registers (the
//    thread-to-bin map is fixed) and are written once per item; a reduction
//    kernel adds items with compensated FP32 sums and applies the
//    1/core_overlapped_ffts scale.
//  * The first Stockham pass is fused with decode and window: samples come
//    straight from the packed per-channel codes written by K1.
#pragma once

#include <cooperative_groups.h>

#include "dft.cuh"
#include "kernels.cuh"

namespace sws {

namespace cg = cooperative_groups;

__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }  // 1 pad per 16 float2

template <int NBIT>
__device__ __forceinline__ float decode_level(uint32_t code, float4 lv)
{
   if constexpr (NBIT == 8) {
      return (float)((int)code * 2 - 255) * (1.0f / 256.0f);
   } else if constexpr (NBIT == 2) {
      float lo = (code & 1u) ? lv.y : lv.x;
      float hi = (code & 1u) ? lv.w : lv.z;
      return (code & 2u) ? hi : lo;
   } else {
      return (code & 1u) ? lv.y : lv.x;
   }
}

template <int NBIT>
__device__ __forceinline__ float sample_at(const SpecArgs &a, int src, long long s, bool chk_blank,
                                           int stream)
{
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT >= 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   uint32_t word = __ldg(a.codes + (long long)src * a.code_words + s / SPW);
   uint32_t code = (word >> (NBIT * (int)(s % SPW))) & MASK;
   float v = decode_level<NBIT>(code, a.levels);
   if (chk_blank) {
      uint32_t bw = __ldg(a.blank + (long long)stream * a.blank_words + (s >> 5));
      if ((bw >> (s & 31)) & 1u) v = 0.0f;
   }
   return v;
}

// One in-place Stockham pass over the padded shared buffer.
template <int Q, int T, int R, int Ns>
__device__ __forceinline__ void smem_pass(float2 *buf, const float2 *__restrict__ twQ)
{
   constexpr int nb = Q / R;
   constexpr int BPT = (nb + T - 1) / T;
   const int tid = threadIdx.x;
   float2 v[BPT][R];
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
         const int k = j % Ns;
#pragma unroll
         for (int r = 0; r < R; r++) {
            float2 x = buf[pidx(j + r * nb)];
            if (r > 0 && Ns > 1) x = cmul(x, __ldg(twQ + k * r * (Q / (Ns * R))));
            v[b][r] = x;
         }
         DFT<R>::run(v[b]);
      }
   }
   __syncthreads();
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
         const int k = j % Ns;
         const int d = (j / Ns) * Ns * R + k;
#pragma unroll
         for (int r = 0; r < R; r++) buf[pidx(d + r * Ns)] = v[b][r];
      }
   }
   __syncthreads();
}

// First pass (Ns = 1) fused with decode + window + pair packing.
template <int P, int Q, int T, int R, int NBIT>
__device__ __forceinline__ void first_pass(float2 *buf, const float *wsl, const SpecArgs &a,
                                           int rank, int src_a, long long sa, int src_b,
                                           long long sb, bool has_b, bool blank_a, bool blank_b,
                                           int stream_a, int stream_b)
{
   constexpr int nb = Q / R;
   constexpr int BPT = (nb + T - 1) / T;
   const int tid = threadIdx.x;
   float2 v[BPT][R];
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
#pragma unroll
         for (int r = 0; r < R; r++) {
            const int q = j + r * nb;
            const long long n = rank + (long long)P * q;
            const float w = wsl[q];
            float xa = sample_at<NBIT>(a, src_a, sa + n, blank_a, stream_a);
            float xb = has_b ? sample_at<NBIT>(a, src_b, sb + n, blank_b, stream_b) : 0.0f;
            v[b][r] = make_float2(xa * w, xb * w);
         }
         DFT<R>::run(v[b]);
      }
   }
   // writes go to locations no other thread reads in this pass (out of place
   // w.r.t. the code stream), so no barrier before the stores
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
#pragma unroll
         for (int r = 0; r < R; r++) buf[pidx(j * R + r)] = v[b][r];
      }
   }
   __syncthreads();
}

// Bins handled per k1-pair slot.
template <int P>
__host__ __device__ constexpr int slots_per_pair() { return P == 1 ? 2 : P + 1; }

template <int NBIT_>
struct NbitTag { static constexpr int value = NBIT_; };

// Accumulate the products of one bin from Z_k (zk) and Z_{N-k} (zm).
__device__ __forceinline__ void acc_bin(float *acc4, int mode, float2 zk, float2 zm)
{
   // A' = 2A, B' = 2B (the reduction applies the 1/4)
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

template <int P, int Q, int T, int R1, int R2, int R3, int NBIT>
__global__ void __launch_bounds__(T, 1) k_spectra(SpecArgs a)
{
   static_assert(R1 * R2 * R3 == Q, "radix plan must multiply to Q");
   constexpr int UC = Q / (2 * P);            // k1-pairs per CTA
   constexpr int UPT = (UC + T - 1) / T;      // k1-pairs per thread
   constexpr int NS = slots_per_pair<P>();
   extern __shared__ float4 smem_raw[];
   float2 *buf = reinterpret_cast<float2 *>(smem_raw);
   float *wsl = reinterpret_cast<float *>(buf + (Q + Q / 16));

   cg::cluster_group cluster = cg::this_cluster();
   const int rank = (int)cluster.block_rank();
   const int cid = blockIdx.x / P;
   const int ncl = gridDim.x / P;
   const int tid = threadIdx.x;
   const int N = a.N, S = a.S;

   // window slice w[rank + P q]
   for (int q = tid; q < Q; q += T) wsl[q] = __ldg(a.window + rank + (long long)P * q);
   __syncthreads();

   float2 *remote[P];
#pragma unroll
   for (int p = 0; p < P; p++) remote[p] = cluster.map_shared_rank(buf, p);

   for (int it = cid; it < a.nitems; it += ncl) {
      const Item item = a.items[it];
      const int mode = item.mode;
      const bool has_b = mode != MODE_SINGLE;
      const int src_b = (mode == MODE_AUTOSUM) ? item.src_a : item.src_b;
      const int stream_a = a.code_stream[item.src_a];
      const int stream_b = has_b ? a.code_stream[src_b] : 0;
      const bool blank_a = a.blank_any[stream_a] != 0;
      const bool blank_b = has_b && a.blank_any[stream_b] != 0;
      float acc[UPT][NS][4];
#pragma unroll
      for (int u = 0; u < UPT; u++)
#pragma unroll
         for (int s = 0; s < NS; s++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[u][s][c] = 0.0f;

      for (int j = 0; j < item.nfr; j++) {
         const long long sa = item.start + (long long)j * item.step;
         const long long sb = (mode == MODE_AUTOSUM) ? sa + item.offset_b : sa;
         first_pass<P, Q, T, R1, NBIT>(buf, wsl, a, rank, item.src_a, sa, src_b, sb, has_b,
                                       blank_a, blank_b, stream_a, stream_b);
         if constexpr (R2 > 1) smem_pass<Q, T, R2, R1>(buf, a.twQ);
         if constexpr (R3 > 1) smem_pass<Q, T, R3, R1 * R2>(buf, a.twQ);
         cluster.sync();
         // ---- final radix-P stage across the cluster + pair separation ----
#pragma unroll
         for (int ui = 0; ui < UPT; ui++) {
            const int u = rank * UC + tid + ui * T;
            if (UC % T != 0 && tid + ui * T >= UC) continue;
            float2 lo[P], hi[P];
            if (u == 0) {
#pragma unroll
               for (int p = 0; p < P; p++) {
                  lo[p] = remote[p][pidx(0)];
                  hi[p] = remote[p][pidx(Q / 2)];
               }
               // W_N^{p Q/2} = W_{2P}^p
               static_for<0, P>([&](auto I) {
                  constexpr int p = decltype(I)::value;
                  hi[p] = twmul<p, 2 * P>(hi[p]);
               });
               DFT<P>::run(lo);
               DFT<P>::run(hi);
               if constexpr (P == 1) {
                  acc_bin(acc[ui][0], mode, lo[0], lo[0]);
                  acc_bin(acc[ui][1], mode, hi[0], hi[0]);
               } else {
#pragma unroll
                  for (int k2 = 0; k2 <= P / 2; k2++) acc_bin(acc[ui][k2], mode, lo[k2], lo[(P - k2) % P]);
#pragma unroll
                  for (int k2 = 0; k2 < P / 2; k2++)
                     acc_bin(acc[ui][P / 2 + 1 + k2], mode, hi[k2], hi[P - 1 - k2]);
               }
            } else {
#pragma unroll
               for (int p = 0; p < P; p++) {
                  float2 fl = remote[p][pidx(u)];
                  float2 fh = remote[p][pidx(Q - u)];
                  if (p == 0) {
                     lo[p] = fl;
                     hi[p] = fh;
                  } else {
                     float2 w = __ldg(a.twN + (long long)p * u);
                     lo[p] = cmul(fl, w);
                     hi[p] = cmulconj(fh, w);  // W_N^{p(Q-u)} = W_P^p conj(W_N^{p u})
                  }
               }
               static_for<1, P>([&](auto I) {
                  constexpr int p = decltype(I)::value;
                  hi[p] = twmul<p, P>(hi[p]);
               });
               DFT<P>::run(lo);
               DFT<P>::run(hi);
               if constexpr (P == 1) {
                  acc_bin(acc[ui][0], mode, lo[0], hi[0]);
               } else {
#pragma unroll
                  for (int k2 = 0; k2 < P / 2; k2++) {
                     acc_bin(acc[ui][k2], mode, lo[k2], hi[P - 1 - k2]);
                     acc_bin(acc[ui][P / 2 + k2], mode, hi[k2], lo[P - 1 - k2]);
                  }
               }
            }
         }
         cluster.sync();
      }
      // ---- write this item's partial sums: partial[it][prod][bin] ----
      float *part = a.partial + (long long)it * 4 * S;
      const int nprod = (mode == MODE_XPOL) ? 4 : 1;
#pragma unroll
      for (int ui = 0; ui < UPT; ui++) {
         const int u = rank * UC + tid + ui * T;
         if (UC % T != 0 && tid + ui * T >= UC) continue;
         for (int c = 0; c < nprod; c++) {
            float *pc = part + (long long)c * S;
            if (u == 0) {
               if constexpr (P == 1) {
                  pc[0] = acc[ui][0][c];
                  pc[Q / 2] = acc[ui][1][c];
               } else {
#pragma unroll
                  for (int k2 = 0; k2 <= P / 2; k2++) pc[Q * k2] = acc[ui][k2][c];
#pragma unroll
                  for (int k2 = 0; k2 < P / 2; k2++) pc[Q / 2 + Q * k2] = acc[ui][P / 2 + 1 + k2][c];
               }
            } else {
               if constexpr (P == 1) {
                  pc[u] = acc[ui][0][c];
               } else {
#pragma unroll
                  for (int k2 = 0; k2 < P / 2; k2++) {
                     pc[u + Q * k2] = acc[ui][k2][c];
                     pc[(Q - u) + Q * k2] = acc[ui][P / 2 + k2][c];
                  }
               }
            }
         }
      }
      (void)N;
   }
   // keep every CTA's shared memory alive until the whole cluster is done
   cluster.sync();
}

// K3: out[o][k] = sum over entries of scale * partial[item][prod][k], Kahan.
__global__ void k_reduce(const float *__restrict__ partial, int S, const RedEntry *__restrict__ ent,
                         const OutVec *__restrict__ ov)
{
   const int k = blockIdx.x * blockDim.x + threadIdx.x;
   const OutVec o = ov[blockIdx.y];
   if (k >= S) return;
   float sum = 0.0f, comp = 0.0f;
   for (int e = o.first; e < o.first + o.count; e++) {
      const RedEntry r = ent[e];
      float x = __ldg(partial + ((long long)r.item * 4 + r.prod) * S + k) * r.scale - comp;
      float t = sum + x;
      comp = (t - sum) - x;
      sum = t;
   }
   if (o.acc_mode == 0) {
      o.dst[(long long)k * o.stride] = sum;
   } else if (o.acc_mode == 1) {
      o.acc[k] = (double)sum;
   } else {
      double t = o.acc[k] + (double)sum;
      o.acc[k] = t;
      if (o.acc_mode == 3) o.dst[(long long)k * o.stride] = (float)t;
   }
}

}  // namespace sws
