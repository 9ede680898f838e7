// bigfft.cu -- four-step FFT of the long transforms (N = N1 * N2).
//
// The same spectra as the cluster kernel -- window, real FFT of every frame,
// |X|^2 and X.Y* accumulated per spectrum (TaskCoreIPP.cpp:427-487) -- for
// lengths whose working set (8N bytes per pair FFT) exceeds a cluster's
// shared memory.  Two real frames are packed into one complex transform
// z = w (a + i b) as in the cluster kernel; the transform is split four-step
// (Bailey) with the intermediate in HBM:
//
//   column pass  X1[k1][n2] = W_N^(n2 k1) sum_n1 z[n1 N2 + n2] W_N1^(n1 k1)
//     a persistent grid over units of C adjacent columns n2 of one pair job.
//     With codes decimated by N2 (the column layout) a column is one
//     contiguous code run, staged by cp.async one unit ahead; decode +
//     window + first radix fused, the N1-point Stockham FFT in shared
//     memory, and the last pass applies the four-step twiddle (two small
//     tables of FP64 values, W_N^(2048 h) W_N^l, multiplied in FP64 and
//     rounded once to FP32) in registers
//     and writes 32-byte row segments of scratch.
//   row pass     X[k1 + N1 k2] = sum_n2 X1[k1][n2] W_N2^(n2 k2)
//     a persistent grid over units (row pair (k1, N1 - k1), work item), the
//     next job's rows prefetched by cp.async: both rows' N2-point FFTs, the
//     pair separation Z_k / Z_(N-k) -- bin N-k of row k1 sits in row N1 - k1
//     at column N2 - 1 - k2 -- and the products of every job of the item
//     accumulated in registers, written once per bin into the partial rows
//     the reduction kernel scales and combines.
//
// Traffic per pair job: the packed codes once, 8N bytes written and read
// back; the window and twiddle tables stay in L2.
#include "bigfft.cuh"
#include "bins.cuh"
#include "dft.cuh"
#include "tcdft.cuh"

namespace sws {

__host__ __device__ constexpr int big_col_stride(int M, int C)
{
   // column stride in float2: one pad per 16 entries, rounded to 16, plus
   // 16 / min(C, 16): the 16 lanes of a half-warp (one shared-memory
   // wavefront of 8-byte accesses) cover min(C, 16) columns at 16 / min(C, 16)
   // consecutive points each, which this offset puts in distinct banks
   return ((M + M / 16 + 15) / 16) * 16 + 16 / (C < 16 ? C : 16);
}
__device__ __forceinline__ int bpad(int i) { return i + (i >> 4); }

// Staged code words per column in the column pass: N1 samples from an
// arbitrary position within their first word.
template <int N1, int NBIT>
__host__ __device__ constexpr int big_col_words()
{
   return (N1 + 32 / NBIT - 1) / (32 / NBIT) + 1;
}
// Their shared-memory region: the run is copied from the 16-byte boundary
// at or below its first word, in whole 16-byte units.
template <int N1, int NBIT>
__host__ __device__ constexpr int big_col_region()
{
   return (big_col_words<N1, NBIT>() + 3 + 3) / 4 * 4;
}

// One Stockham pass (radix R, span NS) over C columns of M points held in
// shared memory, in place through registers.  Butterfly j of column c reads
// x[j + i M/R], twiddles by W_(NS R)^(k i) (k = j mod NS) from the pass's
// table tw[(i - 1) NS + k] and writes d + i NS, d = (j / NS) NS R + k.
template <int M, int C, int T, int R, int NS>
__device__ __forceinline__ void big_pass(float2 *buf, const float2 *tw)
{
   constexpr int CS = big_col_stride(M, C);
   constexpr int NB = M / R, TOT = C * NB, BPT = (TOT + T - 1) / T;
   const int tid = threadIdx.x;
   float2 v[BPT][R];
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int idx = tid + b * T;
      if (TOT % T == 0 || idx < TOT) {
         const int c = idx % C, j = idx / C, k = j % NS;
#pragma unroll
         for (int i = 0; i < R; i++) {
            float2 x = buf[c * CS + bpad(j + i * NB)];
            if (NS > 1 && i > 0) x = cmul(x, tw[(i - 1) * NS + k]);
            v[b][i] = x;
         }
         DFT<R>::run(v[b]);
      }
   }
   __syncthreads();
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int idx = tid + b * T;
      if (TOT % T == 0 || idx < TOT) {
         const int c = idx % C, j = idx / C, k = j % NS;
         const int d = (j / NS) * NS * R + k;
#pragma unroll
         for (int i = 0; i < R; i++) buf[c * CS + bpad(d + i * NS)] = v[b][i];
      }
   }
   __syncthreads();
}

// The column pass's last Stockham pass, with the four-step twiddle applied
// in registers: output k1 = d + i NS of column c goes straight to scratch
// row k1 as x W_N^((c0 + c) k1), W_N^m = W_N^(2048 (m >> 11)) W_N^(m & 2047).
template <int M, int C, int T, int R, int NS>
__device__ __forceinline__ void big_pass_out(const float2 *buf, const float2 *tw, float2 *dst, int N2, int c0,
                                             const double2 *twA, const double2 *twB)
{
   constexpr int CS = big_col_stride(M, C);
   constexpr int NB = M / R, TOT = C * NB, BPT = (TOT + T - 1) / T;
   const int tid = threadIdx.x;
#pragma unroll
   for (int b = 0; b < BPT; b++) {
      const int idx = tid + b * T;
      if (TOT % T == 0 || idx < TOT) {
         const int c = idx % C, j = idx / C, k = j % NS;
         float2 v[R];
#pragma unroll
         for (int i = 0; i < R; i++) {
            float2 x = buf[c * CS + bpad(j + i * NB)];
            if (NS > 1 && i > 0) x = cmul(x, tw[(i - 1) * NS + k]);
            v[i] = x;
         }
         DFT<R>::run(v);
         const int d = (j / NS) * NS * R + k;
#pragma unroll
         for (int i = 0; i < R; i++) {
            const int k1 = d + i * NS;
            const int m = (c0 + c) * k1;  // < N
            // W_N^m = W_N^(2048 (m >> 11)) W_N^(m & 2047): the product of the two
            // FP64 table entries, rounded once to FP32
            const double2 A = __ldg(twA + (m >> 11)), B = __ldg(twB + (m & 2047));
            const float2 w = make_float2((float)fma(A.x, B.x, -A.y * B.y), (float)fma(A.x, B.y, A.y * B.x));
            dst[(long long)k1 * N2 + c] = cmul(v[i], w);
         }
      }
   }
}

// Twiddle tables of the passes of span R1 (radix R2) and R1 R2 (radix R3),
// laid out [i - 1][k] so that the lanes of a warp (consecutive k) read
// consecutive entries: W_M^(k i M / (R1 R2)) then W_M^(k i), from the W_M
// table wm in global memory.  M - R1 entries.
template <int M, int T, int R1, int R2, int R3>
__device__ __forceinline__ void load_pass_twiddles(float2 *tab, const float2 *wm)
{
   constexpr int NA = (R2 - 1) * R1, NBT = (R3 - 1) * R1 * R2;
   for (int e = threadIdx.x; e < NA + NBT; e += T) {
      if (e < NA) {
         const int i = e / R1 + 1, k = e % R1;
         tab[e] = wm[k * i * (M / (R1 * R2))];
      } else {
         const int f = e - NA, i = f / (R1 * R2) + 1, k = f % (R1 * R2);
         tab[e] = wm[k * i];
      }
   }
}

template <int NBIT>
__device__ __forceinline__ float big_sample(const BigArgs &a, int code, long long s, const uint32_t *blank)
{
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT == 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   const uint32_t w = __ldg(a.codes + (long long)code * a.code_words + s / SPW);
   float x = decode_level<NBIT>((w >> (NBIT * (int)(s % SPW))) & MASK, a.levels);
   if (blank && ((__ldg(blank + (s >> 5)) >> (s & 31)) & 1u)) x = 0.0f;
   return x;
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
   const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
   asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
   const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
   asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
   const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Bulk copy global -> shared by the TMA engine (addresses 16-byte aligned,
// size a multiple of 16), its bytes counted on an mbarrier of this CTA.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                "l"(src), "r"(bytes), "r"(mbar)
                : "memory");
}
__device__ __forceinline__ void big_mbar_init(uint32_t mbar, int count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
   asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void big_mbar_expect(uint32_t mbar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}
// Bounded wait for phase `parity`; false when it gave up.
__device__ __forceinline__ bool big_mbar_wait(uint32_t mbar, uint32_t parity)
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
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared memory of the column pass: C columns, the W_N1 table and `slots`
// staging slots of code words (both frames of the pair).
template <int N1, int C, int NBIT>
__host__ __device__ constexpr size_t big_cols_smem_slots(int slots)
{
   return sizeof(float2) * ((size_t)C * big_col_stride(N1, C) + N1 + 1) +
          sizeof(uint32_t) * (size_t)slots * 2 * C * big_col_region<N1, NBIT>();
}
template <int N1, int C, int NBIT>
__host__ __device__ constexpr int big_cols_slots()
{
   return big_cols_smem_slots<N1, C, NBIT>(2) <= 227 * 1024 ? 2 : 1;
}

// Column pass: a persistent grid over the units u = job * (N2 / C) + g of
// the batch (columns gC .. gC + C - 1 of one pair job).  With the column
// layout -- column n2 of a frame starting at sample s0 is the run idx0 ..
// idx0 + N1 - 1 of phase array (s0 + n2) % N2, idx0 = (s0 + n2) / N2 -- the
// unit's code runs (the 16-byte aligned span around the WPC words per
// column and frame from the word holding idx0) are staged in shared memory
// by bulk copies of the TMA engine, one per run, issued by warp 0 and
// counted on the slot's mbarrier; the next unit's go into a second slot
// while the current one is transformed.  The W_N1 table is loaded once per
// CTA.
template <int N1, int N2, int C, int T, int R1, int R2, int R3, int NBIT>
__global__ void __launch_bounds__(T, 65536 / (T * 128)) k_big_cols(BigArgs a)
{
   static_assert(R1 * R2 * R3 == N1, "radices must multiply to N1");
   static_assert(N2 % C == 0, "columns per CTA must divide N2");
   constexpr int CS = big_col_stride(N1, C);
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT == 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   constexpr int WPC = big_col_region<N1, NBIT>();  // staged words per run (16-byte multiple)
   constexpr int SLOT = 2 * C * WPC;
   constexpr int NIW = (2 * C + 31) / 32;  // warps issuing the bulk copies, one per run
   static_assert(NIW * 32 <= T, "issuing warps within the block");
   constexpr int NS = big_cols_slots<N1, C, NBIT>();
   constexpr int NG = N2 / C;
   extern __shared__ float2 smf[];
   float2 *buf = smf;
   float2 *tw1 = smf + C * CS;
   // [NS][2][C][WPC], 16-byte aligned for the bulk copies
   uint32_t *stg = reinterpret_cast<uint32_t *>(tw1 + N1 + ((C * CS + N1) & 1));
   __shared__ int soff[2][2][C];
   __shared__ __align__(8) unsigned long long sbar[2];  // one per staging slot: its bulk copies' bytes
   const int tid = threadIdx.x;
   const int nunits = NG * a.nbjobs;
   int u = blockIdx.x;
   if (u >= nunits) return;
   load_pass_twiddles<N1, T, R1, R2, R3>(tw1, a.tw1);
   const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(&sbar[0]);
   const uint32_t stg_addr = (uint32_t)__cvta_generic_to_shared(stg);
   if (tid == 0) {
      big_mbar_init(bar0, NIW);
      big_mbar_init(bar0 + 8, NIW);
   }
   __syncthreads();
   uint32_t par = 0u;  // bit s: the phase of slot s's barrier to wait for
   bool gave_up = false;

   // warps 0 .. NIW-1: thread l < nside*C copies run l (side l / C, column
   // l % C) from the 16-byte boundary at or below its first word; each
   // warp's lane 0 arrives on the slot's barrier announcing its warp's bytes
   // before they are copied
   auto stage = [&](int uu, int sl) {
      if (tid >= 32 * NIW) return;
      const BigJob sj = a.jobs[uu / NG];
      const int sc0 = (uu % NG) * C;
      const int nside = sj.mode != MODE_SINGLE ? 2 : 1;
      uint32_t bytes = 0;
      const uint32_t *src = nullptr;
      if (tid < nside * C) {
         const int side = tid / C, c = tid % C;
         const long long s = (side ? sj.sb : sj.sa) + sc0 + c;
         const long long wi = (s / N2) / SPW;
         const long long w0 = wi & ~3ll;
         const int extra = (int)(wi - w0);
         const long long nw = min((long long)WPC, a.wpp - w0);  // wpp is a multiple of 4 words
         src = a.codes + (long long)(side ? sj.code_b : sj.code_a) * a.code_words + (s % N2) * a.wpp + w0;
         bytes = (uint32_t)(nw > 0 ? nw : 0) * 4u;
         soff[sl][side][c] = extra * SPW + (int)((s / N2) % SPW);
      }
      uint32_t total = bytes;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      if ((tid & 31) == 0) big_mbar_expect(bar0 + 8u * (uint32_t)sl, total);
      __syncwarp();
      if (bytes)
         bulk_g2s(stg_addr + 4u * (uint32_t)(sl * SLOT + tid * WPC), src, bytes, bar0 + 8u * (uint32_t)sl);
   };
   auto wait_slot = [&](int sl) {
      if (!gave_up && !big_mbar_wait(bar0 + 8u * (uint32_t)sl, (par >> sl) & 1u)) {
         gave_up = true;  // report once; the data of this unit are invalid
         if (a.status) atomicExch(a.status, 1);
      }
      par ^= 1u << sl;
   };

   int slot = 0;
   if (a.col_layout) stage(u, 0);
   while (true) {
      const int un = u + gridDim.x;
      const bool more = un < nunits;
      if constexpr (NS == 2) {
         if (a.col_layout && more) stage(un, slot ^ 1);
      }
      if (a.col_layout) wait_slot(slot);
      __syncthreads();

      const int job = u / NG, c0 = (u % NG) * C;
      const BigJob jb = a.jobs[job];
      const bool has_b = jb.mode != MODE_SINGLE;
      const int sta = a.code_stream[jb.code_a];
      const uint32_t *blank_a = a.blank_any[sta] ? a.blank + (long long)sta * a.blank_words : nullptr;
      const uint32_t *blank_b = nullptr;
      if (has_b) {
         const int stb = a.code_stream[jb.code_b];
         blank_b = a.blank_any[stb] ? a.blank + (long long)stb * a.blank_words : nullptr;
      }
      const uint32_t *sg = stg + slot * SLOT;

      // pass 1 (span 1): decode + window + radix R1
      {
         constexpr int NB = N1 / R1, TOT = C * NB, BPT = (TOT + T - 1) / T;
#pragma unroll
         for (int b = 0; b < BPT; b++) {
            const int idx = tid + b * T;
            if (TOT % T == 0 || idx < TOT) {
               const int c = idx % C, j = idx / C;
               float2 v[R1];
               if (a.col_layout) {
                  const int oa = soff[slot][0][c] + j, ob = has_b ? soff[slot][1][c] + j : 0;
#pragma unroll
                  for (int i = 0; i < R1; i++) {
                     const long long n = (long long)(j + i * NB) * N2 + c0 + c;
                     const float w = __ldg(a.window + n);
                     const int pa = oa + i * NB, pb = ob + i * NB;
                     float xa = decode_level<NBIT>((sg[c * WPC + pa / SPW] >> (NBIT * (pa % SPW))) & MASK, a.levels);
                     float xb = 0.0f;
                     if (has_b)
                        xb = decode_level<NBIT>((sg[(C + c) * WPC + pb / SPW] >> (NBIT * (pb % SPW))) & MASK,
                                                a.levels);
                     if (blank_a && ((__ldg(blank_a + ((jb.sa + n) >> 5)) >> ((jb.sa + n) & 31)) & 1u)) xa = 0.0f;
                     if (blank_b && ((__ldg(blank_b + ((jb.sb + n) >> 5)) >> ((jb.sb + n) & 31)) & 1u)) xb = 0.0f;
                     v[i] = make_float2(xa * w, xb * w);
                  }
               } else {
#pragma unroll
                  for (int i = 0; i < R1; i++) {
                     const long long n = (long long)(j + i * NB) * N2 + c0 + c;
                     const float w = __ldg(a.window + n);
                     const float xa = big_sample<NBIT>(a, jb.code_a, jb.sa + n, blank_a);
                     const float xb = has_b ? big_sample<NBIT>(a, jb.code_b, jb.sb + n, blank_b) : 0.0f;
                     v[i] = make_float2(xa * w, xb * w);
                  }
               }
               DFT<R1>::run(v);
#pragma unroll
               for (int i = 0; i < R1; i++) buf[c * CS + bpad(j * R1 + i)] = v[i];
            }
         }
      }
      __syncthreads();
      // remaining passes; the last writes the twiddled 32-byte row segments
      // of scratch itself
      float2 *dst = a.scratch + (long long)job * N1 * N2 + c0;
      if constexpr (R3 > 1) {
         big_pass<N1, C, T, R2, R1>(buf, tw1);
         big_pass_out<N1, C, T, R3, R1 * R2>(buf, tw1 + (R2 - 1) * R1, dst, N2, c0, a.twA, a.twB);
      } else {
         big_pass_out<N1, C, T, R2, R1>(buf, tw1, dst, N2, c0, a.twA, a.twB);
      }
      if (!more) break;
      __syncthreads();  // the columns and this staging slot are reused
      u = un;
      if constexpr (NS == 2) {
         slot ^= 1;
      } else {
         if (a.col_layout) stage(u, 0);
      }
   }
   // a unit staged but never waited for cannot exist: every stage is
   // followed by the wait of the iteration that transforms it
}

// Row pass: a persistent grid over the units u = item * NP + rp of the
// batch (row pair rp = (k1, N1 - k1), NP = N1 / 2 + 1).  A CTA walks its
// units' jobs in order; while it transforms one job's row pair, the next
// one streams into the other shared-memory slot (cp.async), and the W_N2
// table is loaded once per CTA.
template <int N1, int N2, int T, int R1, int R2, int R3>
__global__ void __launch_bounds__(T, 65536 / (T * 128)) k_big_rows(BigArgs a)
{
   static_assert(R1 * R2 * R3 == N2, "radices must multiply to N2");
   static_assert(N1 % 2 == 0, "row pairs need an even N1");
   constexpr int CS = big_col_stride(N2, 2);
   constexpr int KPT = (N2 + T - 1) / T;
   constexpr int NP = N1 / 2 + 1;
   extern __shared__ float2 smf[];
   float2 *tw2 = smf + 4 * CS;  // two slots of two rows, then the table
   const int tid = threadIdx.x;
   const int nunits = NP * a.nbitems;
   int u = blockIdx.x;
   if (u >= nunits) return;
   load_pass_twiddles<N2, T, R1, R2, R3>(tw2, a.tw2);
   const long long N = (long long)N1 * N2;

   auto stage = [&](int uu, int jj, int sl) {
      const BigItem si = a.bitems[uu / NP];
      const int rp = uu % NP;
      const int k1b = (N1 - rp) % N1;
      const float2 *ra = a.scratch + ((long long)(si.job0 + jj) * N1 + rp) * N2;
      const float2 *rb = a.scratch + ((long long)(si.job0 + jj) * N1 + k1b) * N2;
      float2 *dst = smf + sl * 2 * CS;
      for (int i = tid; i < N2; i += T) {
         cp_async8(dst + bpad(i), ra + i);
         if (k1b != rp) cp_async8(dst + CS + bpad(i), rb + i);
      }
   };

   float acc[KPT][4];
#pragma unroll
   for (int q = 0; q < KPT; q++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[q][c] = 0.0f;

   int j = 0, slot = 0;
   BigItem bi = a.bitems[u / NP];
   stage(u, 0, 0);
   cp_async_commit();
   while (true) {
      int un = u, jn = j + 1;
      if (jn >= bi.nfr) {
         un = u + gridDim.x;
         jn = 0;
      }
      const bool more = un < nunits;
      if (more) stage(un, jn, slot ^ 1);
      cp_async_commit();
      cp_async_wait1();
      __syncthreads();

      float2 *buf = smf + slot * 2 * CS;
      const int rp = u % NP;
      const bool two = rp != (N1 - rp) % N1;
      big_pass<N2, 2, T, R1, 1>(buf, tw2);
      big_pass<N2, 2, T, R2, R1>(buf, tw2);
      if constexpr (R3 > 1) big_pass<N2, 2, T, R3, R1 * R2>(buf, tw2 + (R2 - 1) * R1);
#pragma unroll
      for (int q = 0; q < KPT; q++) {
         const int k2 = tid + q * T;
         if (N2 % T == 0 || k2 < N2) {
            const float2 zk = buf[bpad(k2)];
            float2 zm;
            if (rp == 0) zm = buf[bpad((N2 - k2) % N2)];
            else if (two) zm = buf[CS + bpad(N2 - 1 - k2)];
            else zm = buf[bpad(N2 - 1 - k2)];
            acc_bin(acc[q], bi.mode, zk, zm);
         }
      }

      if (j == bi.nfr - 1) {
         // bin k = k1 + N1 k2 of row k1, or its mirror N - k (conjugate cross
         // product) when k lies above N/2; self-paired rows keep k <= N/2 only
         float *part = a.partial + (long long)bi.item * 4 * a.S;
         const int nprod = (bi.mode == MODE_XPOL) ? 4 : 1;
#pragma unroll
         for (int q = 0; q < KPT; q++) {
            const int k2 = tid + q * T;
            if (N2 % T == 0 || k2 < N2) {
               const long long k = rp + (long long)N1 * k2;
               if (k <= N / 2 || two) {
                  const bool conj = k > N / 2;
                  const long long bin = conj ? N - k : k;
                  for (int c = 0; c < nprod; c++)
                     part[(long long)c * a.S + bin] = (c == 3 && conj) ? -acc[q][c] : acc[q][c];
               }
            }
#pragma unroll
            for (int c = 0; c < 4; c++) acc[q][c] = 0.0f;
         }
      }
      __syncthreads();  // this slot is restaged two iterations on
      if (!more) break;
      if (un != u) bi = a.bitems[un / NP];
      u = un;
      j = jn;
      slot ^= 1;
   }
}

// Row pass of 4096-point rows on the tensor cores (the tensor-core split
// form of the four-step path).  Each row's DFT is three radix-16 levels,
// n2 = q0 + 16 q1 + 256 q2 and k2 = k0 + 16 k1 + 256 kk, on tcgen05 exactly
// as the cluster kernel's all-levels form: level 1 over q2 for operand row
// r1 = q0 + 16 q1 = threadIdx.x, twiddle W_4096^(r1 k0); level 2 over q1,
// twiddle W_256^(q0 k1); level 3 over q0.  Scaling: the DFT16 operand
// carries 1/4, so a level's outputs are at most 4x its inputs (16 terms of
// modulus 1/4) and noise keeps its level; each row enters multiplied by the
// power of two 2^(8 - e) that puts its largest component m (2^e <= m <
// 2^(e+1)) below 2^9, so no FP16 operand of any level can exceed 2^15
// (a carrier concentrating 4096-fold included), while noise stays well
// inside the FP16 normal range where the hi/lo split keeps about 22 bits.
// The outputs are multiplied back by 64 / 2^(8 - e), exact.  Both rows of
// the pair land in shared memory for the pair separation, which with the
// accumulation and the partial write is the FP32 row pass's.  The next
// unit's rows stream into a staging slot by cp.async as soon as every
// thread has taken this unit's last row into its registers.  One unit at a
// time per CTA, one CTA per SM (208 KB of shared memory).
constexpr int kTcRowThreads = 256;

template <int N1>
__global__ void __launch_bounds__(kTcRowThreads, 1) k_big_rows_tc(BigArgs a)
{
   constexpr int N2 = 4096, T = kTcRowThreads, KPT = N2 / T;
   static_assert(N1 % 2 == 0, "row pairs need an even N1");
   constexpr int NP = N1 / 2 + 1;
   constexpr int FS = N2 + N2 / 16;  // padded row in float2
   extern __shared__ __align__(1024) unsigned char smb[];
   float2 *w4096 = reinterpret_cast<float2 *>(smb + TC_OPND_BYTES + TC_BMAT_BYTES);
   float2 *fa = w4096 + N2;
   float2 *fb = fa + FS;
   float2 *sa = fb + FS;        // staged rows of the unit in hand
   float2 *sb = sa + N2;
   __shared__ uint32_t tmem_holder;
   __shared__ __align__(8) unsigned long long mma_bar;
   __shared__ float wmax[T / 32];
   const int tid = threadIdx.x;
   const int nunits = NP * a.nbitems;
   int u = blockIdx.x;
   if (u >= nunits) return;  // the whole CTA, before any barrier
   const uint32_t opnd = (uint32_t)__cvta_generic_to_shared(smb);
   const uint32_t bmat = opnd + TC_OPND_BYTES;
   const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&mma_bar);
   for (int i = tid; i < N2; i += T) w4096[i] = a.tw2[i];
   fill_dft16_bmat(bmat, T);
   tc::fence_async_smem();
   if (tid < 32) tc::tmem_alloc((uint32_t)__cvta_generic_to_shared(&tmem_holder), TC_TMEM_COLS);
   if (tid == 0) tc::mbar_init_cta(mbar, 1);
   tc::fence_before();
   __syncthreads();
   tc::fence_after();
   const uint32_t tmem = tmem_holder;
   uint32_t par = 0;
   bool gave_up = false;
   const long long N = (long long)N1 * N2;

   auto level = [&](bool kmajor) {
      if (tid == 0) tc_issue_level(tmem, opnd, bmat, kmajor, mbar);
      if (!gave_up && !tc::mbar_wait(mbar, par)) {
         gave_up = true;  // report once; later levels do not wait again
         if (a.status) atomicExch(a.status, 1);
      }
      par ^= 1u;
      tc::fence_after();
   };
   auto handoff = [&]() {
      tc::fence_before();
      tc::fence_async_smem();
      __syncthreads();
   };
   // stage the rows of unit uu, job jj (16-byte cp.async, 8 per thread and row)
   auto stage = [&](int uu, int jj) {
      const BigItem si = a.bitems[uu / NP];
      const int rp = uu % NP;
      const int k1b = (N1 - rp) % N1;
      const float2 *ra = a.scratch + ((long long)(si.job0 + jj) * N1 + rp) * N2;
      const float2 *rb = a.scratch + ((long long)(si.job0 + jj) * N1 + k1b) * N2;
      for (int i = tid; i < N2 / 2; i += T) {
         cp_async16(sa + 2 * i, ra + 2 * i);
         if (k1b != rp) cp_async16(sb + 2 * i, rb + 2 * i);
      }
      cp_async_commit();
   };
   // the 4096-point DFT of one staged row into out[bpad(k)]; on_read runs
   // once every thread holds the row in registers
   auto transform = [&](const float2 *row, float2 *out, auto &&on_read) {
      float2 y[16];
      float m = 0.0f;
#pragma unroll
      for (int q2 = 0; q2 < 16; q2++) {
         y[q2] = row[tid + 256 * q2];
         m = fmaxf(m, fmaxf(fabsf(y[q2].x), fabsf(y[q2].y)));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if ((tid & 31) == 0) wmax[tid >> 5] = m;
      __syncthreads();
#pragma unroll
      for (int w = 0; w < T / 32; w++) m = fmaxf(m, wmax[w]);
      const int ex = (m > 0.0f) ? ilogbf(m) : 0;
      const float in_scale = ldexpf(1.0f, 8 - ex), comp = ldexpf(64.0f, ex - 8);
#pragma unroll
      for (int q2 = 0; q2 < 16; q2++) y[q2] = make_float2(y[q2].x * in_scale, y[q2].y * in_scale);
      store_k16(opnd, tid, y);
      handoff();
      on_read();
      level(true);
      tc_load_row(tmem, y);
#pragma unroll
      for (int k0 = 1; k0 < 16; k0++) y[k0] = cmul(y[k0], w4096[(tid * k0) & (N2 - 1)]);
      store_mn16(opnd, tid & 15, 16 + (tid & 15), tid >> 4, y);
      handoff();
      level(false);
      tc_load_row(tmem, y);
      const int k0 = (tid & 7) + 8 * (tid >> 7), q0 = (tid >> 3) & 15;
#pragma unroll
      for (int k1 = 1; k1 < 16; k1++) y[k1] = cmul(y[k1], w4096[16 * ((q0 * k1) & 255)]);
      store_mn16(opnd, k0, 16 + k0, q0, y);
      handoff();
      level(false);
      tc_load_row(tmem, y);
      const int kap = ((tid >> 3) & 15) + 16 * ((tid & 7) + 8 * (tid >> 7));
#pragma unroll
      for (int kk = 0; kk < 16; kk++) out[bpad(kap + 256 * kk)] = make_float2(y[kk].x * comp, y[kk].y * comp);
   };

   float acc[KPT][4];
#pragma unroll
   for (int q = 0; q < KPT; q++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[q][c] = 0.0f;
   int j = 0;
   BigItem bi = a.bitems[u / NP];
   stage(u, 0);
   while (true) {
      const int rp = u % NP;
      const int k1b = (N1 - rp) % N1;
      const bool two = rp != k1b;
      int un = u, jn = j + 1;
      if (jn >= bi.nfr) {
         un = u + gridDim.x;
         jn = 0;
      }
      const bool more = un < nunits;
      cp_async_wait0();
      __syncthreads();  // this unit's staged rows are visible
      auto next = [&]() {
         if (more) stage(un, jn);
      };
      auto none = []() {};
      if (two) {
         transform(sa, fa, none);
         transform(sb, fb, next);
      } else {
         transform(sa, fa, next);
      }
      tc::fence_before();
      __syncthreads();  // both rows' spectra visible
#pragma unroll
      for (int q = 0; q < KPT; q++) {
         const int k2 = tid + q * T;
         const float2 zk = fa[bpad(k2)];
         float2 zm;
         if (rp == 0) zm = fa[bpad((N2 - k2) % N2)];
         else if (two) zm = fb[bpad(N2 - 1 - k2)];
         else zm = fa[bpad(N2 - 1 - k2)];
         acc_bin(acc[q], bi.mode, zk, zm);
      }
      if (j == bi.nfr - 1) {
         // bin k = k1 + N1 k2 of row k1, or its mirror N - k (conjugate
         // cross product) above N/2; self-paired rows keep k <= N/2 only
         float *part = a.partial + (long long)bi.item * 4 * a.S;
         const int nprod = (bi.mode == MODE_XPOL) ? 4 : 1;
#pragma unroll
         for (int q = 0; q < KPT; q++) {
            const int k2 = tid + q * T;
            const long long k = rp + (long long)N1 * k2;
            if (k <= N / 2 || two) {
               const bool conj = k > N / 2;
               const long long bin = conj ? N - k : k;
               for (int c = 0; c < nprod; c++)
                  part[(long long)c * a.S + bin] = (c == 3 && conj) ? -acc[q][c] : acc[q][c];
            }
#pragma unroll
            for (int c = 0; c < 4; c++) acc[q][c] = 0.0f;
         }
      }
      __syncthreads();  // the row spectra are read before the next unit writes them
      if (!more) break;
      if (un != u) bi = a.bitems[un / NP];
      u = un;
      j = jn;
   }
   tc::fence_before();
   __syncthreads();
   if (tid < 32) {
      tc::fence_after();
      tc::tmem_dealloc(tmem, TC_TMEM_COLS);
   }
}

constexpr size_t big_rows_tc_smem()
{
   // operand, DFT16 matrix, W_4096 table, two padded row spectra, two staged rows
   return (size_t)TC_OPND_BYTES + TC_BMAT_BYTES + sizeof(float2) * (4096 + 2 * (4096 + 4096 / 16) + 2 * 4096);
}

// The tensor-core row pass of a split, or null where rows are not 4096 points.
template <int N1, int N2>
constexpr BigRowsKernel big_rows_tc_kernel()
{
   if constexpr (N2 == 4096) return k_big_rows_tc<N1>;
   else return nullptr;
}

template <int N2>
constexpr size_t big_rows_smem()
{
   // two slots of a row pair, then the W_N2 table
   return sizeof(float2) * ((size_t)4 * big_col_stride(N2, 2) + N2);
}

#define SWS_BIG_C(N1_, C_, TA_, A1, A2, A3, N2_, TB_, B1, B2, B3)                                 \
   {N1_ * N2_, N1_, N2_, C_, TA_, TB_,                                                            \
    {k_big_cols<N1_, N2_, C_, TA_, A1, A2, A3, 1>, k_big_cols<N1_, N2_, C_, TA_, A1, A2, A3, 2>,  \
     k_big_cols<N1_, N2_, C_, TA_, A1, A2, A3, 8>},                                               \
    k_big_rows<N1_, N2_, TB_, B1, B2, B3>,                                                        \
    {big_cols_smem_slots<N1_, C_, 1>(big_cols_slots<N1_, C_, 1>()),                               \
     big_cols_smem_slots<N1_, C_, 2>(big_cols_slots<N1_, C_, 2>()),                               \
     big_cols_smem_slots<N1_, C_, 8>(big_cols_slots<N1_, C_, 8>())},                              \
    big_rows_smem<N2_>(), big_rows_tc_kernel<N1_, N2_>(), big_rows_tc_smem(), kTcRowThreads}
#define SWS_BIG(N1_, TA_, A1, A2, A3, N2_, TB_, B1, B2, B3) SWS_BIG_C(N1_, 4, TA_, A1, A2, A3, N2_, TB_, B1, B2, B3)

// Candidate splits per length; the first of each length is the default,
// the others are timed by the autotuner (swsgpu_autotune).
static const BigPlan kBigPlans[] = {
    SWS_BIG_C(256, 16, 256, 16, 16, 1, 256, 128, 16, 16, 1),  // 2^16 (the cluster kernel is the default)
    SWS_BIG_C(256, 32, 512, 16, 16, 1, 256, 128, 16, 16, 1),
    SWS_BIG_C(128, 32, 256, 16, 8, 1, 512, 256, 16, 16, 2),
    SWS_BIG(512, 256, 16, 16, 2, 512, 256, 16, 16, 2),        // 2^18
    SWS_BIG(256, 256, 16, 16, 1, 1024, 128, 16, 16, 4),
    SWS_BIG(1024, 256, 16, 16, 4, 256, 256, 16, 16, 1),
    SWS_BIG(512, 256, 16, 16, 2, 1024, 128, 16, 16, 4),       // 2^19
    SWS_BIG(1024, 256, 16, 16, 4, 512, 256, 16, 16, 2),
    SWS_BIG(1024, 256, 16, 16, 4, 1024, 128, 16, 16, 4),      // 2^20
    SWS_BIG_C(1024, 8, 512, 16, 16, 4, 1024, 128, 16, 16, 4),
    SWS_BIG(512, 256, 16, 16, 2, 2048, 256, 16, 16, 8),
    SWS_BIG(2048, 512, 16, 16, 8, 512, 256, 16, 16, 2),
    SWS_BIG(1024, 256, 16, 16, 4, 2048, 256, 16, 16, 8),      // 2^21
    SWS_BIG(2048, 512, 16, 16, 8, 1024, 128, 16, 16, 4),
    SWS_BIG(2048, 512, 16, 16, 8, 2048, 256, 16, 16, 8),      // 2^22
    SWS_BIG(1024, 256, 16, 16, 4, 4096, 512, 16, 16, 16),
    SWS_BIG(4096, 512, 16, 16, 16, 1024, 128, 16, 16, 4),
    SWS_BIG(3200, 512, 16, 8, 25, 1000, 256, 8, 5, 25),       // 3,200,000 = 2^10 5^5
    SWS_BIG(1600, 512, 16, 4, 25, 2000, 256, 16, 5, 25),
    SWS_BIG(2000, 512, 16, 5, 25, 1600, 256, 16, 4, 25),
    SWS_BIG(1280, 512, 16, 16, 5, 2500, 256, 4, 25, 25),
};

bool find_big_plan(int N, BigPlan *out)
{
   for (const BigPlan &p : kBigPlans)
      if (p.N == N) {
         *out = p;
         return true;
      }
   return false;
}

int big_plan_candidates(int N, BigPlan *out, int max)
{
   int n = 0;
   for (const BigPlan &p : kBigPlans)
      if (p.N == N && n < max) out[n++] = p;
   return n;
}

}  // namespace sws
