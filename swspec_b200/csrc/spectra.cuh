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
//  * N = P*Q over a thread-block cluster of P CTAs (decimation in time):
//    CTA p decodes, windows and transforms z[p + P q] (q < Q) in shared
//    memory with Stockham passes of radix R1, R2, R3 -- one butterfly per
//    thread per pass when Q/R = T -- then, after a cluster barrier, threads
//    gather F_p[k1] (lo side) or F_p[Q-k1] (hi side) from all P CTAs through
//    distributed shared memory, apply W_N^{p k1}, finish the P-point DFT and
//    swap half of their outputs with the partner lane, so each lane holds
//    Z_k and Z_{N-k} for its bins.
//  * Per-pass twiddles live in thread-major shared tables [r][k] (k = the
//    butterfly's index mod Ns), filled once per CTA, so every twiddle read is
//    bank-conflict free; the cluster-stage twiddles W_N^{p k1} likewise.
//  * Spectra of consecutive jobs of a work item accumulate in registers (the
//    thread-to-bin map is fixed) and are written once per item; a reduction
//    kernel adds items with compensated sums and applies the scaling.
//  * The cluster barrier that protects a CTA's buffer from the previous
//    job's remote readers is split (arrive after the gathers, wait just
//    before the next job's first stores), so decode and the first radix-R1
//    butterflies of the next job overlap it.
#pragma once

#include <cooperative_groups.h>
#include <cuda_fp16.h>

#include "dft.cuh"
#include "tcdft.cuh"
#include "kernels.cuh"
#include "bins.cuh"

namespace sws {

namespace cg = cooperative_groups;

__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }  // 1 pad per 16 float2

// Distributed shared memory: 32-bit shared::cluster address of the same
// offset in CTA `rank` of the cluster, and a 64-bit load from it.
__device__ __forceinline__ uint32_t dsmem_addr(uint32_t local_addr, uint32_t rank)
{
   uint32_t r;
   asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(local_addr), "r"(rank));
   return r;
}
__device__ __forceinline__ float2 dsmem_ld2(uint32_t addr)
{
   float2 v;
   asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
   return v;
}

__device__ __forceinline__ void cluster_arrive()
{
   asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait()
{
   asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Asynchronous 4-byte global -> shared copies (cp.async), for prefetching
// the next job's codes while the current job computes.
__device__ __forceinline__ void cp_async4(uint32_t smem_addr, const void *gptr)
{
   asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr), "l"(gptr) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void dsmem_st2(uint32_t addr, float2 v)
{
   asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};\n" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}

// Asynchronous remote store whose 8 bytes are counted on the destination
// CTA's mbarrier (both addresses shared::cluster): the receiver learns of
// the data from its own barrier, the sender neither waits nor fences.
__device__ __forceinline__ void dsmem_st2_async(uint32_t addr, float2 v, uint32_t mbar)
{
   asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];\n"
                ::"r"(addr), "f"(v.x), "f"(v.y), "r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar, int count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
   asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint32_t mbar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}
// Waits for the completion of phase `parity` with a bounded number of
// polls; returns false when it gave up (the caller reports it and goes on,
// so that every cluster barrier is still reached).
__device__ __forceinline__ bool mbar_wait_parity(uint32_t mbar, uint32_t parity)
{
   for (int it = 0; it < (1 << 18); it++) {
      uint32_t done;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
                   " selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
      if (done) return true;
      if (it > 64) __nanosleep(64);
   }
   return false;
}

// Twiddle table of a pass: tw[(r-1)*Ns + k] = W_{Ns R}^{k r}, k < Ns, 0 < r < R.
template <int Q, int R, int Ns>
__device__ __forceinline__ void fill_pass_twiddles(float2 *tw, const float2 *__restrict__ twQ, int T)
{
   for (int i = threadIdx.x; i < (R - 1) * Ns; i += T) {
      const int r = i / Ns + 1, k = i % Ns;
      tw[i] = __ldg(twQ + k * r * (Q / (Ns * R)));
   }
}

// Two-level twiddles for a wide pass: W^{k r} = TA[r][k/16] * TB[r][k%16]
// with TA = W^{16 (k/16) r}, TB = W^{(k%16) r} (one extra rounding).
template <int Ns>
__host__ __device__ constexpr bool two_level_tw() { return Ns >= 64 && Ns % 16 == 0; }

template <int Q, int R, int Ns>
__host__ __device__ constexpr int pass_tw_entries()
{
   return two_level_tw<Ns>() ? (R - 1) * (Ns / 16 + 16) : (R - 1) * Ns;
}

template <int Q, int R, int Ns>
__device__ __forceinline__ void fill_pass_twiddles2(float2 *tw, const float2 *__restrict__ twQ, int T)
{
   if constexpr (two_level_tw<Ns>()) {
      constexpr int NA = Ns / 16;
      for (int i = threadIdx.x; i < (R - 1) * (NA + 16); i += T) {
         const int r = i / (NA + 16) + 1, x = i % (NA + 16);
         const int k = x < NA ? 16 * x : x - NA;
         tw[i] = __ldg(twQ + k * r * (Q / (Ns * R)));
      }
   } else {
      fill_pass_twiddles<Q, R, Ns>(tw, twQ, T);
   }
}

template <int R, int Ns>
__device__ __forceinline__ float2 pass_tw(const float2 *tw, int r, int k)
{
   if constexpr (two_level_tw<Ns>()) {
      constexpr int NA = Ns / 16;
      const float2 *row = tw + (r - 1) * (NA + 16);
      return cmul(row[k >> 4], row[NA + (k & 15)]);
   } else {
      return tw[(r - 1) * Ns + k];
   }
}

// Twiddles by powers: with base[i] = W^{2^i k} (i < log2 R), x[r] *= W^{r k}
// where W^{r k} is built from the bases of r's set bits (at most
// popcount(r) - 1 products, one rounding each).
__host__ __device__ constexpr int hibit(int r) { return r >= 16 ? 16 : r >= 8 ? 8 : r >= 4 ? 4 : r >= 2 ? 2 : 1; }
__host__ __device__ constexpr int ilog2c(int r) { return r >= 16 ? 4 : r >= 8 ? 3 : r >= 4 ? 2 : r >= 2 ? 1 : 0; }
__host__ __device__ constexpr int nbases(int R) { return ilog2c(R - 1) + 1; }

template <int R>
__device__ __forceinline__ void twiddle_by_powers(float2 *x, const float2 *base)
{
   float2 w[R];
   static_for<1, R>([&](auto I) {
      constexpr int r = decltype(I)::value;
      constexpr int hb = hibit(r);
      if constexpr (r == hb) w[r] = base[ilog2c(hb)];
      else w[r] = cmul(w[r - hb], base[ilog2c(hb)]);
      x[r] = cmul(x[r], w[r]);
   });
}

// Base table of a pass: tb[i*Ns + k] = W_{Ns R}^{2^i k}.
template <int Q, int R, int Ns>
__device__ __forceinline__ void fill_pass_bases(float2 *tb, const float2 *__restrict__ twQ, int T)
{
   constexpr int NBASE = nbases(R);
   for (int idx = threadIdx.x; idx < NBASE * Ns; idx += T) {
      const int i = idx / Ns, k = idx % Ns;
      tb[idx] = __ldg(twQ + ((long long)k << i) % (Ns * R) * (Q / (Ns * R)));
   }
}

// Load + twiddle (by powers) + radix-R DFT of one Stockham pass into registers.
template <int Q, int T, int R, int Ns, int BPT>
__device__ __forceinline__ void pass_compute_pw(const float2 *buf, const float2 *tb, float2 (&v)[BPT][R])
{
   constexpr int nb = Q / R;
   constexpr int NBASE = nbases(R);
   const int tid = threadIdx.x;
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
         const int k = j % Ns;
         if constexpr (nb % 16 == 0) {
            const int pj = pidx(j);
#pragma unroll
            for (int r = 0; r < R; r++) v[b][r] = buf[pj + r * (nb + nb / 16)];
         } else {
#pragma unroll
            for (int r = 0; r < R; r++) v[b][r] = buf[pidx(j + r * nb)];
         }
         float2 base[NBASE];
#pragma unroll
         for (int i = 0; i < NBASE; i++) base[i] = tb[i * Ns + k];
         twiddle_by_powers<R>(v[b], base);
         DFT<R>::run(v[b]);
      }
   }
}

// Load + twiddle + radix-R DFT of one Stockham pass into registers.
template <int Q, int T, int R, int Ns, int BPT>
__device__ __forceinline__ void pass_compute(const float2 *buf, const float2 *tw, float2 (&v)[BPT][R])
{
   constexpr int nb = Q / R;
   const int tid = threadIdx.x;
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
         const int k = j % Ns;
         const int pj = pidx(j);
#pragma unroll
         for (int r = 0; r < R; r++) {
            float2 x = (nb % 16 == 0) ? buf[pj + r * (nb + nb / 16)] : buf[pidx(j + r * nb)];
            if (r > 0) x = cmul(x, pass_tw<R, Ns>(tw, r, k));
            v[b][r] = x;
         }
         DFT<R>::run(v[b]);
      }
   }
}

// One in-place Stockham pass over the padded shared buffer (FP32).
template <int Q, int T, int R, int Ns>
__device__ __forceinline__ void smem_pass(float2 *buf, const float2 *tw)
{
   constexpr int nb = Q / R;
   constexpr int BPT = (nb + T - 1) / T;
   const int tid = threadIdx.x;
   float2 v[BPT][R];
   pass_compute<Q, T, R, Ns, BPT>(buf, tw, v);
   __syncthreads();
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int j = tid + b * T;
      if (nb % T == 0 || j < nb) {
         const int k = j % Ns;
         const int d = (j / Ns) * Ns * R + k;
         const int pd = pidx(d);
#pragma unroll
         for (int r = 0; r < R; r++) buf[(Ns % 16 == 0) ? pd + r * (Ns + Ns / 16) : pidx(d + r * Ns)] = v[b][r];
      }
   }
   __syncthreads();
}

// Staged code words per source and job (see PERM in k_spectra); 256-thread
// plans use the permuted layout whenever Q/R1 <= 256.
template <int Q, int R1, int NBIT>
__host__ __device__ constexpr int stage_slots()
{
   constexpr int SPW = 32 / NBIT, NW = Q / SPW + 2, nb1 = Q / R1;
   constexpr int ST = (nb1 % SPW == 0) ? nb1 / SPW : 1;
   return (nb1 % SPW == 0) ? ST * ((((NW + ST - 1) / ST) + 3) / 4) * 4 : NW;
}

// Receive buffer of the cluster exchange, [p][hi][u]: one row of
// rx_stride float2 per side.  The cluster stage's warp reads, for one p,
// sides (u, hi) of 16 consecutive threads: u over 8 values, hi alternating;
// rx_stride = 8 (mod 16) puts the hi row 16 banks away from the lo row, so
// the 16 eight-byte reads of a wavefront hit distinct banks.
template <int P, int Q, int PREC>
__host__ __device__ constexpr int rx_stride()
{
   constexpr int UC = Q / (2 * P);
   return UC + (24 - UC % 16) % 16;
}

// The FP32 form's hi-side cluster bases start TWC_HI_PAD float2 after the
// lo-side ones: the lanes of a half-warp read the lo and hi bases of the same
// 8 pairs, and the 64-byte offset puts the two halves in different banks.
constexpr int TWC_HI_PAD = 8;

// Shared memory layout of a plan: byte offsets of every region, used both
// for the kernel's pointers and for the host-side launch size.
template <int P, int Q, int R1, int R2, int R3, int NBIT, int PREC>
struct SmemLayout {
   static constexpr size_t BUFB = PREC ? (size_t)TC_OPND_BYTES : (size_t)(Q + Q / 16) * 8;
   static constexpr size_t buf = 0;                                             // FFT buffer / operand
   static constexpr size_t bmat = buf + BUFB;                                   // DFT16 B operand
   static constexpr size_t rbuf = bmat + (PREC ? TC_BMAT_BYTES : 0);            // receive [P][hi][u]
   static constexpr size_t wsl = rbuf + (size_t)P * 2 * rx_stride<P, Q, PREC>() * 8;  // window slice (float)
   static constexpr size_t tw2 = wsl + (size_t)Q * 4;                           // pass-2 twiddles
   static constexpr size_t tw3 = tw2 + (size_t)(PREC ? 0 : pass_tw_entries<Q, R2, R1>()) * 8;
   static constexpr size_t twc = tw3 + (size_t)nbases(R3) * R1 * R2 * 8;        // pass-3 bases
   // cluster-stage bases: lo sides, and (FP32 form) hi sides
   static constexpr size_t stage =
       ((twc + ((size_t)(PREC ? 1 : 2) * nbases(P) * (Q / (2 * P)) + (PREC ? 0 : TWC_HI_PAD)) * 8) + 15) / 16 * 16;
   static constexpr size_t total = stage + (size_t)2 * 2 * stage_slots<Q, R1, NBIT>() * 4;
};

template <int P, int Q, int R1, int R2, int R3, int NBIT, int PREC>
__host__ __device__ constexpr size_t spectra_smem()
{
   return SmemLayout<P, Q, R1, R2, R3, NBIT, PREC>::total;
}

template <int P, int Q, int T, int R1, int R2, int R3, int NBIT, int MINB, int PREC>
__global__ void __launch_bounds__(T, MINB) k_spectra(SpecArgs a)
{
   // PREC 1: levels 2 and 3 of the CTA's 4096-point transform on tensor
   // cores (tcgen05), level 1 in FP32 registers fused with the decode;
   // PREC 2: all three levels on tensor cores.  One operand row per thread.
   static_assert(PREC == 0 || (Q == 4096 && R1 == 16 && R2 == 16 && R3 == 16 && T == 256),
                 "tensor-core form plan");
   static_assert(R1 * R2 * R3 == Q, "radix plan must multiply to Q");
   static_assert(R3 > 1, "three passes");
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT >= 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   constexpr int UC = Q / (2 * P);          // k1-pairs per CTA
   constexpr int SIDES = 2 * UC;            // lo/hi sides per CTA
   constexpr int RX = rx_stride<P, Q, PREC>();  // receive row stride (float2)
   constexpr int SPT = (SIDES + T - 1) / T; // sides per thread
   constexpr int HB = (P == 1) ? 1 : P / 2; // bins per side (regular)
   constexpr int NB = HB + 1;               // + the lo special's extra bin
   constexpr int NX = (P == 1) ? 1 : P / 2; // values exchanged with the partner lane
   constexpr int NW = Q / SPW + 2;          // staged code words per source and job
   // Pass 1 thread jj needs code words g + r*ST (g = (off + jj)/SPW, r < R1,
   // ST = (Q/R1)/SPW).  With PERM the prefetch stores word w at slot
   // (w % ST)*GS + w/ST, so those R1 words are contiguous (128-bit loads).
   constexpr int nb1c = Q / R1;
   constexpr bool PERM = (nb1c % SPW == 0) && (R1 % 4 == 0) && (nb1c <= T);
   constexpr int ST = PERM ? nb1c / SPW : 1;
   constexpr int GS = PERM ? (((NW + ST - 1) / ST + 3) / 4) * 4 : NW;
   constexpr int NSLOT = PERM ? ST * GS : NW;  // staged words per source and job
   static_assert(NSLOT <= stage_slots<Q, R1, NBIT>(), "code staging exceeds its shared-memory region");
   constexpr int NS3 = R1 * R2;             // span of the last pass
   constexpr int nb3 = Q / R3;
   constexpr int BPT3 = (nb3 + T - 1) / T;
   extern __shared__ float4 smem_raw[];
   using L = SmemLayout<P, Q, R1, R2, R3, NBIT, PREC>;
   char *smem = reinterpret_cast<char *>(smem_raw);
   float2 *buf = reinterpret_cast<float2 *>(smem + L::buf);
   float2 *rbuf = reinterpret_cast<float2 *>(smem + L::rbuf);
   float *wsl = reinterpret_cast<float *>(smem + L::wsl);
   float2 *tw2 = reinterpret_cast<float2 *>(smem + L::tw2);
   float2 *tw3 = reinterpret_cast<float2 *>(smem + L::tw3);
   float2 *twc = reinterpret_cast<float2 *>(smem + L::twc);  // cluster bases [i][u_local] = W_N^{2^i u}
   uint32_t *stage = reinterpret_cast<uint32_t *>(smem + L::stage);

   cg::cluster_group cluster = cg::this_cluster();
   const int rank = (int)cluster.block_rank();
   const int cid = blockIdx.x / P;
   const int ncl = gridDim.x / P;
   const int tid = threadIdx.x;
   const int S = a.S;

   // ---- per-CTA constant tables ----
   for (int q = tid; q < Q; q += T) wsl[q] = __ldg(a.window + rank + (long long)P * q);
   if constexpr (PREC == 0) fill_pass_twiddles2<Q, R2, R1>(tw2, a.twQ, T);
   fill_pass_bases<Q, R3, NS3>(tw3, a.twQ, T);
   const uint32_t opnd_addr = (uint32_t)__cvta_generic_to_shared(smem + L::buf);
   const uint32_t bmat_addr = (uint32_t)__cvta_generic_to_shared(smem + L::bmat);
   __shared__ uint32_t tmem_holder;
   __shared__ __align__(8) unsigned long long mma_bar;
   const uint32_t mma_bar_addr = (uint32_t)__cvta_generic_to_shared(&mma_bar);
   if constexpr (PREC >= 1) {
      fill_dft16_bmat(bmat_addr, T);
      tc::fence_async_smem();
      if (tid < 32) tc::tmem_alloc((uint32_t)__cvta_generic_to_shared(&tmem_holder), TC_TMEM_COLS);
      if (tid == 0) tc::mbar_init_cta(mma_bar_addr, 1);
   }
   // twc[i*UC + u_local] = W_N^{2^i u} (lo side of pair u); the FP32 form
   // adds twc[(NBASE + i)*UC + TWC_HI_PAD + u_local] = W_N^{2^i (Q - u)} for the hi side
   // (index <= N/2, inside the W_N table), so that neither side needs a
   // conjugation or a further rotation; the tensor-core forms, short of
   // shared memory, derive the hi side's from the lo side's
   for (int idx = tid; idx < nbases(P) * UC; idx += T) {
      const int i = idx / UC, uu = idx % UC, u = rank * UC + uu;
      twc[idx] = __ldg(a.twN + ((long long)u << i));
      if constexpr (PREC == 0)
         twc[nbases(P) * UC + TWC_HI_PAD + idx] = __ldg(a.twN + ((long long)(u ? Q - u : 0) << i));
   }

   const uint32_t rbuf_addr = (uint32_t)__cvta_generic_to_shared(rbuf);
   const uint32_t stage_addr = (uint32_t)__cvta_generic_to_shared(stage);
   // levels of a (code_a, code_b) pair, and every CTA's receive buffer as a
   // shared::cluster address (mapped once instead of per pushed value)
   __shared__ float2 pair_lut[NBIT <= 2 ? (1 << (2 * NBIT)) : 1];
   __shared__ uint32_t rbase[P];
   __shared__ uint32_t rbar[P];                   // every CTA's receive barrier (shared::cluster)
   __shared__ __align__(8) unsigned long long rx_bar;  // this CTA's: Q values received per job
   const uint32_t rx_bar_addr = (uint32_t)__cvta_generic_to_shared(&rx_bar);
   if (tid == 0) mbar_init(rx_bar_addr, 1);
   if constexpr (NBIT <= 2)
      for (int i = tid; i < (1 << (2 * NBIT)); i += T)
         pair_lut[i] = make_float2(decode_level<NBIT>((uint32_t)i & MASK, a.levels),
                                   decode_level<NBIT>((uint32_t)i >> NBIT, a.levels));
   for (int i = tid; i < P; i += T) {
      rbase[i] = dsmem_addr(rbuf_addr, (uint32_t)i);
      rbar[i] = dsmem_addr(rx_bar_addr, (uint32_t)i);
   }

   // ---- job sequence of this cluster: its items in order, jobs 0..nfr-1 of each ----
   struct JobPos {
      int it, j;
   };
   // this cluster's items: the contiguous range [cl_first[cid], cl_first[cid + 1])
   // when the schedule balanced jobs across clusters, else every ncl-th item
   const int it_end = a.cl_first ? a.cl_first[cid + 1] : a.nitems;
   const int it_step = a.cl_first ? 1 : ncl;
   auto job_valid = [&](const JobPos &jp) { return jp.it < it_end; };
   auto next_job = [&](JobPos jp) {
      if (jp.j + 1 < a.items[jp.it].nfr) return JobPos{jp.it, jp.j + 1};
      return JobPos{jp.it + it_step, 0};
   };
   // prefetch the codes of job jp into staging slot `slot`
   auto prefetch = [&](const JobPos &jp, int slot) {
      const Item item = a.items[jp.it];
      const bool has_b = item.mode != MODE_SINGLE;
      const long long sa = item.start + (long long)jp.j * item.step;
      const long long sb = (item.mode == MODE_AUTOSUM) ? sa + item.offset_b : sa;
#pragma unroll
      for (int src = 0; src < 2; src++) {
         if (src == 1 && !has_b) break;
         const int code = src == 0 ? item.src_a : (item.mode == MODE_AUTOSUM ? item.src_a : item.src_b);
         const long long s0 = (src == 0 ? sa : sb) + rank;
         const long long i0 = s0 / P;
         const int ph = (int)(s0 - i0 * P);
         const uint32_t *g = a.codes + (long long)code * a.code_words + (long long)ph * a.wpp + i0 / SPW;
         const int nw = (int)(((i0 % SPW) + Q - 1) / SPW) + 1;
         const uint32_t dst = stage_addr + 4u * (uint32_t)((slot * 2 + src) * NSLOT);
         for (int w = tid; w < nw; w += T) {
            const int sl = PERM ? (w % ST) * GS + w / ST : w;
            cp_async4(dst + 4u * sl, g + w);
         }
      }
   };

   // pass 1 (Ns = 1) of job jp from staging slot `slot`: decode + window + radix-R1
   auto pass1 = [&](const JobPos &jp, int slot) {
      const Item item = a.items[jp.it];
      const int mode = item.mode;
      const bool has_b = mode != MODE_SINGLE;
      const long long sa = item.start + (long long)jp.j * item.step;
      const long long sb = (mode == MODE_AUTOSUM) ? sa + item.offset_b : sa;
      const int offa = (int)(((sa + rank) / P) % SPW);
      const int offb = (int)(((sb + rank) / P) % SPW);
      const uint32_t *sta = stage + slot * 2 * NSLOT;
      const uint32_t *stb = sta + NSLOT;
      const int stream_a = a.code_stream[item.src_a];
      const int src_b = (mode == MODE_AUTOSUM) ? item.src_a : item.src_b;
      const int stream_b = has_b ? a.code_stream[src_b] : 0;
      const uint32_t *blank_a = a.blank_any[stream_a] ? a.blank + (long long)stream_a * a.blank_words : nullptr;
      const uint32_t *blank_b = (has_b && a.blank_any[stream_b]) ? a.blank + (long long)stream_b * a.blank_words : nullptr;
      constexpr int nb1 = Q / R1;
      constexpr int BPT1 = (nb1 + T - 1) / T;
      float2 v[BPT1][R1];
#pragma unroll
      for (int b = 0; b < BPT1; b++) {
         const int jj = tid + b * T;
         if (nb1 % T == 0 || jj < nb1) {
            uint32_t wa[R1], wb[R1];
            if constexpr (PERM) {
               // this thread's R1 words of each source, contiguous after the permutation
               const int ga = (offa + jj) / SPW, gb = (offb + jj) / SPW;
               const int sa0 = (ga % ST) * GS + ga / ST, sb0 = (gb % ST) * GS + gb / ST;
               if ((sa0 & 3) == 0) {
#pragma unroll
                  for (int r = 0; r < R1; r += 4) {
                     const uint4 t4 = *reinterpret_cast<const uint4 *>(sta + sa0 + r);
                     wa[r] = t4.x; wa[r + 1] = t4.y; wa[r + 2] = t4.z; wa[r + 3] = t4.w;
                  }
               } else {
#pragma unroll
                  for (int r = 0; r < R1; r++) wa[r] = sta[sa0 + r];
               }
               if (has_b) {
                  if ((sb0 & 3) == 0) {
#pragma unroll
                     for (int r = 0; r < R1; r += 4) {
                        const uint4 t4 = *reinterpret_cast<const uint4 *>(stb + sb0 + r);
                        wb[r] = t4.x; wb[r + 1] = t4.y; wb[r + 2] = t4.z; wb[r + 3] = t4.w;
                     }
                  } else {
#pragma unroll
                     for (int r = 0; r < R1; r++) wb[r] = stb[sb0 + r];
                  }
               }
            }
            if constexpr (PERM && NBIT <= 2) {
               if (has_b) {
                  // both sources' codes of sample q index one table entry
                  // holding both levels; nb1 % SPW == 0, so the bit offset
                  // within the word is the same for all r
                  const int sha = NBIT * ((offa + jj) % SPW), shb = NBIT * ((offb + jj) % SPW);
#pragma unroll
                  for (int r = 0; r < R1; r++) {
                     const int q = jj + r * nb1;
                     const float w = wsl[q];
                     const uint32_t ca = (wa[r] >> sha) & MASK, cb = (wb[r] >> shb) & MASK;
                     float2 lv = pair_lut[(cb << NBIT) | ca];
                     if (blank_a) {
                        const long long smp = sa + rank + (long long)P * q;
                        if ((__ldg(blank_a + (smp >> 5)) >> (smp & 31)) & 1u) lv.x = 0.0f;
                     }
                     if (blank_b) {
                        const long long smp = sb + rank + (long long)P * q;
                        if ((__ldg(blank_b + (smp >> 5)) >> (smp & 31)) & 1u) lv.y = 0.0f;
                     }
                     v[b][r] = make_float2(lv.x * w, lv.y * w);
                  }
                  if constexpr (PREC != 2) DFT<R1>::run(v[b]);
                  continue;
               }
            }
#pragma unroll
            for (int r = 0; r < R1; r++) {
               const int q = jj + r * nb1;
               const float w = wsl[q];
               const int ia = offa + q;
               const uint32_t worda = PERM ? wa[r] : sta[ia / SPW];
               float xa = decode_level<NBIT>((worda >> (NBIT * (ia % SPW))) & MASK, a.levels);
               if (blank_a) {
                  const long long smp = sa + rank + (long long)P * q;
                  if ((__ldg(blank_a + (smp >> 5)) >> (smp & 31)) & 1u) xa = 0.0f;
               }
               float xb = 0.0f;
               if (has_b) {
                  const int ib = offb + q;
                  const uint32_t wordb = PERM ? wb[r] : stb[ib / SPW];
                  xb = decode_level<NBIT>((wordb >> (NBIT * (ib % SPW))) & MASK, a.levels);
                  if (blank_b) {
                     const long long smp = sb + rank + (long long)P * q;
                     if ((__ldg(blank_b + (smp >> 5)) >> (smp & 31)) & 1u) xb = 0.0f;
                  }
               }
               v[b][r] = make_float2(xa * w, xb * w);
            }
            if constexpr (PREC != 2) DFT<R1>::run(v[b]);
         }
      }
      if constexpr (PREC == 0) {
#pragma unroll
         for (int b = 0; b < BPT1; b++) {
            const int jj = tid + b * T;
            if (nb1 % T == 0 || jj < nb1) {
#pragma unroll
               for (int r = 0; r < R1; r++)
                  buf[(R1 == 16) ? jj * 17 + r : pidx(jj * R1 + r)] = v[b][r];  // pidx(16 jj + r), r < 16
            }
         }
      } else if constexpr (PREC == 1) {
         // level 1 done in registers: row r1 = tid holds k0 = r; twiddle
         // W_4096^{r1 k0} (tw3 holds W_Q^{2^i r1}, the bases the FP32 form's
         // last pass uses) and store as level 2's operand, rows k0 + 16 q0,
         // K column q1 (r1 = q0 + 16 q1)
         float2 base[nbases(R3)];
#pragma unroll
         for (int i = 0; i < nbases(R3); i++) base[i] = tw3[i * NS3 + tid];
         twiddle_by_powers<R1>(v[0], base);
         store_mn16(opnd_addr, tid & 15, 16 + (tid & 15), tid >> 4, v[0]);
         tc::fence_async_smem();
      } else {
         // the decoded, windowed samples z[r1 + 256 q2] as row r1 = tid of
         // level 1's K-major operand
         store_k16(opnd_addr, tid, v[0]);
         tc::fence_async_smem();
      }
   };

   JobPos cur{a.cl_first ? a.cl_first[cid] : cid, 0};
   if (job_valid(cur)) prefetch(cur, 0);
   cp_async_commit();
   if (job_valid(cur) && job_valid(next_job(cur))) prefetch(next_job(cur), 1);
   cp_async_commit();
   if constexpr (PREC >= 1) tc::fence_before();
   __syncthreads();      // tables visible
   uint32_t tmem_base = 0, mma_par = 0;
   bool tc_gave_up = false;
   if constexpr (PREC >= 1) {
      tc::fence_after();
      tmem_base = tmem_holder;
   }
   cluster_arrive();     // pairs with the wait before the first job's pushes

   float acc[SPT][NB][4];
#pragma unroll
   for (int u = 0; u < SPT; u++)
#pragma unroll
      for (int x = 0; x < NB; x++)
#pragma unroll
         for (int c = 0; c < 4; c++) acc[u][x][c] = 0.0f;

   int n = 0;  // job counter (staging slot parity, receive-barrier phase)
   bool gave_up = false;
   if (job_valid(cur)) {
      cp_async_wait1();  // the first job's codes have landed
      __syncthreads();
      pass1(cur, 0);
   }
   while (job_valid(cur)) {
      const Item item = a.items[cur.it];
      const int mode = item.mode;
      const bool has_b = mode != MODE_SINGLE;
      (void)has_b;
      const JobPos nxt = next_job(cur);
      // fault injection (tests): the cluster's last job sends nothing, so
      // every receiver's bounded wait for it runs out
      const bool send = !(a.drop_last_exchange && !job_valid(nxt));
      __syncthreads();  // this job's pass-1 output is visible
      // push F_rank[k1] to the CTA that owns pair min(k1, Q-k1); receive layout
      // [p][hi][u], rows of RX float2
      auto push = [&](int k1, float2 val) {
         int u, hi;
         if (k1 == 0) { u = 0; hi = 0; }
         else if (2 * k1 == Q) { u = 0; hi = 1; }
         else if (2 * k1 < Q) { u = k1; hi = 0; }
         else { u = Q - k1; hi = 1; }
         const int owner = u / UC;
         const int slot = hi * RX + (u - owner * UC);
         dsmem_st2_async(rbase[owner] + 8u * (uint32_t)(rank * 2 * RX + slot), val, rbar[owner]);
      };
      if constexpr (PREC == 0) {
         // ---- pass 2 in shared memory, pass 3 into registers ----
         smem_pass<Q, T, R2, R1>(buf, tw2);
         float2 v3[BPT3][R3];
         pass_compute_pw<Q, T, R3, NS3, BPT3>(buf, tw3, v3);
         cluster_wait();  // owners have finished reading their receive buffers
         // k1 = j + r NS3 with j < NS3 and Q = R3 NS3: for even R3 the side
         // (lo: k1 < Q/2, hi otherwise) is fixed by r, and with power-of-two
         // Q and UC the owner and slot are shifts and masks
         constexpr bool FASTPUSH = (R3 % 2 == 0) && ((Q & (Q - 1)) == 0) && ((UC & (UC - 1)) == 0);
#pragma unroll
         for (int b = 0; b < BPT3; b++) {
            const int j = tid + b * T;
            if ((nb3 % T == 0 || j < nb3) && send) {
               if constexpr (FASTPUSH) {
                  const uint32_t self = 8u * (uint32_t)(rank * 2 * RX);
#pragma unroll
                  for (int r = 0; r < R3; r++) {
                     const int k1 = j + r * NS3;
                     const int uu = (r < R3 / 2) ? k1 : ((Q - k1) & (Q / 2 - 1));
                     const int slot = ((r < R3 / 2) ? 0 : RX) + (uu & (UC - 1));
                     dsmem_st2_async(rbase[uu / UC] + self + 8u * (uint32_t)slot, v3[b][r], rbar[uu / UC]);
                  }
               } else {
#pragma unroll
                  for (int r = 0; r < R3; r++) push(j + r * NS3, v3[b][r]);
               }
            }
         }
      } else {
         // ---- levels (1,) 2 and 3 on tensor cores; this thread owns row tid ----
         // the operand was stored and fenced by pass 1; the barrier at the top
         // of the loop made it visible to the issuing thread
         constexpr float COMP = (PREC == 2) ? 64.0f : 16.0f;  // (1/s)^levels, exact
         auto level = [&](bool kmajor) {
            if (tid == 0) tc_issue_level(tmem_base, opnd_addr, bmat_addr, kmajor, mma_bar_addr);
            if (!tc_gave_up && !tc::mbar_wait(mma_bar_addr, mma_par)) {
               tc_gave_up = true;  // report once; later levels do not wait again
               if (a.status) atomicExch(a.status, 1);
            }
            mma_par ^= 1u;
            tc::fence_after();
         };
         // hand the next operand to the tensor core: loads of TMEM done,
         // generic stores visible to the async proxy, then one barrier.
         // Overwriting the operand needs no barrier before it: every thread
         // has seen the level's commit arrive on mma_bar, and the commit
         // arrives only after the MMAs, their operand reads included, have
         // completed; no thread reads the operand through the generic proxy.
         auto handoff = [&]() {
            tc::fence_before();
            tc::fence_async_smem();
            __syncthreads();
         };
         float2 y[16];
         if constexpr (PREC == 2) {
            // level 1: row r1 = tid = q0 + 16 q1, outputs k0; twiddle W_4096^{r1 k0}
            level(true);
            tc_load_row(tmem_base, y);
            float2 base[nbases(R3)];
#pragma unroll
            for (int i = 0; i < nbases(R3); i++) base[i] = tw3[i * NS3 + tid];
            twiddle_by_powers<16>(y, base);
            store_mn16(opnd_addr, tid & 15, 16 + (tid & 15), tid >> 4, y);
            handoff();
         }
         // level 2: row tid = (k0 & 7) + 8 q0 + 128 (k0 >> 3), outputs k1;
         // twiddle W_256^{q0 k1}; level 3's operand rows (k1 & 7) + 8 k0 +
         // 128 (k1 >> 3), K column q0
         level(false);
         tc_load_row(tmem_base, y);
         const int k0 = (tid & 7) + 8 * (tid >> 7);
         {
            const int q0 = (tid >> 3) & 15;
#pragma unroll
            for (int k1 = 1; k1 < 16; k1++) {
               // W_256^m = W_4096^(16 m): the last pass's base table holds
               // W_4096^(8 k), k < 256, so W_256^m = +-tw3[768 + 2 (m mod 128)]
               const int m = (q0 * k1) & 255;
               float2 w = tw3[3 * NS3 + 2 * (m & 127)];
               if (m & 128) w = make_float2(-w.x, -w.y);
               y[k1] = cmul(y[k1], w);
            }
            store_mn16(opnd_addr, k0, 16 + k0, q0, y);
            handoff();
         }
         // level 3: row tid = (k1 & 7) + 8 k0 + 128 (k1 >> 3), outputs k2:
         // F[k0 + 16 k1 + 256 k2]
         level(false);
         tc_load_row(tmem_base, y);
         tc::fence_before();
         cluster_wait();  // owners have finished reading their receive buffers
         if (send) {
            const int kap = ((tid >> 3) & 15) + 16 * ((tid & 7) + 8 * (tid >> 7));
#pragma unroll
            for (int k2 = 0; k2 < 16; k2++)
               push(kap + 256 * k2, make_float2(y[k2].x * COMP, y[k2].y * COMP));
         }
      }
      // ---- the next job's pass 1 while this job's values are in flight ----
      if (job_valid(nxt)) {
         cp_async_wait0();  // its codes have landed
         __syncthreads();   // and this job's last reads of buf are done
         pass1(nxt, (n + 1) & 1);
         const JobPos nn = next_job(nxt);
         if (job_valid(nn)) prefetch(nn, n & 1);  // the slot this job's codes used
         cp_async_commit();
      }
      // this CTA's Q values of the job have landed (counted in bytes on
      // its barrier; one arrival per phase, from thread 0)
      if (tid == 0) mbar_arrive_expect(rx_bar_addr, (uint32_t)(Q * 8));
      if (!gave_up && !mbar_wait_parity(rx_bar_addr, (uint32_t)(n & 1))) {
         gave_up = true;  // report once; later jobs do not wait again
         if (a.status) atomicExch(a.status, 1);
      }

      // ---- radix-P stage across the cluster + pair separation ----
#pragma unroll
      for (int si = 0; si < SPT; si++) {
         const int s = tid + si * T;  // side index within the CTA
         const bool active = (SIDES % T == 0) || s < SIDES;
         const bool hi = (s & 1) != 0;
         const int u = rank * UC + (s >> 1);
         float2 z[P];
         if (active) {
#pragma unroll
            for (int p = 0; p < P; p++) z[p] = rbuf[p * 2 * RX + (hi ? RX : 0) + (s >> 1)];
            if (u == 0) {
               // lo: k1 = 0 (no twiddle); hi: k1 = Q/2, W_N^{p Q/2} = W_{2P}^p
               if (hi) {
                  static_for<1, P>([&](auto I) {
                     constexpr int p = decltype(I)::value;
                     z[p] = twmul<p, 2 * P>(z[p]);
                  });
               }
            } else {
               // z[p] *= W_N^{p u} (lo) or W_N^{p (Q - u)} (hi), from the power bases
               float2 base[nbases(P)];
               if constexpr (PREC == 0) {
                  const float2 *tb = twc + (hi ? nbases(P) * UC + TWC_HI_PAD : 0) + (s >> 1);
#pragma unroll
                  for (int i = 0; i < nbases(P); i++) base[i] = tb[i * UC];
                  twiddle_by_powers<P>(z, base);
               } else {
#pragma unroll
                  for (int i = 0; i < nbases(P); i++) {
                     const float2 w = twc[i * UC + (s >> 1)];
                     base[i] = hi ? make_float2(w.x, -w.y) : w;
                  }
                  twiddle_by_powers<P>(z, base);
                  if (hi) {
                     // W_N^{p(Q-u)} = W_P^p conj(W_N^{p u})
                     static_for<1, P>([&](auto I) {
                        constexpr int p = decltype(I)::value;
                        z[p] = twmul<p, P>(z[p]);
                     });
                  }
               }
            }
            DFT<P>::run(z);
         } else {
#pragma unroll
            for (int p = 0; p < P; p++) z[p] = make_float2(0.0f, 0.0f);
         }
         // swap the upper half with the partner side (lane ^ 1)
         float2 rv[NX];
#pragma unroll
         for (int i = 0; i < NX; i++) {
            const int src = (P == 1) ? 0 : P / 2 + i;
            rv[i].x = __shfl_xor_sync(0xffffffffu, z[src].x, 1);
            rv[i].y = __shfl_xor_sync(0xffffffffu, z[src].y, 1);
         }
         if (active) {
            if (u == 0) {
               if constexpr (P == 1) {
                  acc_bin(acc[si][0], mode, z[0], z[0]);
               } else if (!hi) {
#pragma unroll
                  for (int k2 = 0; k2 <= P / 2; k2++) acc_bin(acc[si][k2], mode, z[k2], z[(P - k2) % P]);
               } else {
#pragma unroll
                  for (int k2 = 0; k2 < P / 2; k2++) acc_bin(acc[si][k2], mode, z[k2], z[P - 1 - k2]);
               }
            } else {
               if constexpr (P == 1) {
                  if (!hi) acc_bin(acc[si][0], mode, z[0], rv[0]);
               } else {
#pragma unroll
                  for (int k2 = 0; k2 < P / 2; k2++) acc_bin(acc[si][k2], mode, z[k2], rv[P / 2 - 1 - k2]);
               }
            }
         }
      }
      cluster_arrive();  // this CTA has finished reading its receive buffer

      // ---- end of a work item: write partial sums, reset accumulators ----
      if (cur.j + 1 == item.nfr) {
         float *part = a.partial + (long long)cur.it * 4 * S;
         const int nprod = (mode == MODE_XPOL) ? 4 : 1;
#pragma unroll
         for (int si = 0; si < SPT; si++) {
            const int s = tid + si * T;
            if ((SIDES % T == 0) || s < SIDES) {
               const bool hi = (s & 1) != 0;
               const int u = rank * UC + (s >> 1);
               for (int c = 0; c < nprod; c++) {
                  float *pc = part + (long long)c * S;
                  if (u == 0) {
                     if constexpr (P == 1) {
                        pc[hi ? Q / 2 : 0] = acc[si][0][c];
                     } else if (!hi) {
#pragma unroll
                        for (int k2 = 0; k2 <= P / 2; k2++) pc[Q * k2] = acc[si][k2][c];
                     } else {
#pragma unroll
                        for (int k2 = 0; k2 < P / 2; k2++) pc[Q / 2 + Q * k2] = acc[si][k2][c];
                     }
                  } else {
                     if constexpr (P == 1) {
                        if (!hi) pc[u] = acc[si][0][c];
                     } else {
                        const int k1 = hi ? Q - u : u;
#pragma unroll
                        for (int k2 = 0; k2 < P / 2; k2++) pc[k1 + Q * k2] = acc[si][k2][c];
                     }
                  }
               }
            }
#pragma unroll
            for (int x = 0; x < NB; x++)
#pragma unroll
               for (int c = 0; c < 4; c++) acc[si][x][c] = 0.0f;
         }
      }
      cur = nxt;
      n++;
   }
   cp_async_wait0();
   cluster_wait();  // pairs with the last arrive: no one still reads a receive buffer
   if constexpr (PREC >= 1) {
      tc::fence_before();
      __syncthreads();
      if (tid < 32) {
         tc::fence_after();
         tc::tmem_dealloc(tmem_base, TC_TMEM_COLS);
      }
   }
}

// K3: out[o][k] = sum over entries of scale * partial[item][prod][k], Kahan.
__global__ void k_reduce(const float *__restrict__ partial, int S, const RedEntry *__restrict__ ent,
                         const OutVec *__restrict__ ov)
{
   const int k = blockIdx.x * blockDim.x + threadIdx.x;
   const OutVec o = ov[blockIdx.y];
   if (k >= S) return;
   float sum = 0.0f, comp = 0.0f;
   auto add = [&](float v) {
      const float x = v - comp;
      const float t = sum + x;
      comp = (t - sum) - x;
      sum = t;
   };
   // eight entries' partials in flight, then their Kahan updates in order
   const int end = o.first + o.count;
   int e = o.first;
   for (; e + 8 <= end; e += 8) {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
         const RedEntry r = ent[e + u];
         v[u] = __ldg(partial + ((long long)r.item * 4 + r.prod) * S + k) * r.scale;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) add(v[u]);
   }
   for (; e < end; e++) {
      const RedEntry r = ent[e];
      add(__ldg(partial + ((long long)r.item * 4 + r.prod) * S + k) * r.scale);
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
