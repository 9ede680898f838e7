// pcal.cu -- K4: phase-cal folding with an FP64 rotator.
//
// Restates TaskCoreIPP::extract_PCal (src/IA-32/TaskCoreIPP.cpp:633-693):
// every block of rotatorlen samples of an FFT's (unwindowed) input is
// multiplied by exp(i dphi n), n = 0..rotatorlen-1 counted from the FFT start,
// dphi = 2 pi (-f_offset / fs) (prepare, :129-136), and folded modulo
// tonebins; only the first (rotatorlen / tonebins) * tonebins samples of each
// block are folded (the reference's integer division).  The rotator phase is
// evaluated in FP64 from the integer position in the period, and products and
// sums are FP64 (the word-wise fold first adds at most 64 samples of a
// position in FP32), so folding 1e5 samples per bin per FFT loses nothing;
// the folded bins are rounded to FP32 once, at the output.
#include "pcal.cuh"
#include "bins.cuh"
#include "dft.cuh"

namespace sws {

template <int NBIT>
__device__ __forceinline__ float pc_sample(const PcalArgs &a, int src, long long s, bool chk)
{
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT >= 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   const long long i = s / a.D;
   uint32_t word = __ldg(a.codes + (long long)src * a.code_words + (s % a.D) * a.wpp + i / SPW);
   uint32_t code = (word >> (NBIT * (int)(i % SPW))) & MASK;
   float v;
   if (NBIT == 8) v = (float)((int)code * 2 - 255) * (1.0f / 256.0f);
   else if (NBIT == 2) v = (code == 0) ? a.levels.x : (code == 1) ? a.levels.y : (code == 2) ? a.levels.z : a.levels.w;
   else v = code ? a.levels.y : a.levels.x;
   if (chk) {
      int st = a.code_stream[src];
      uint32_t bw = __ldg(a.blank + (long long)st * a.blank_words + (s >> 5));
      if ((bw >> (s & 31)) & 1u) v = 0.0f;
   }
   return v;
}

// grid.x: blocks per job, grid.y: job.  Each block folds a contiguous range
// of rotator periods; thread t visits in-period positions t, t+T, ...
template <int NBIT>
__global__ void k_pcal_fold(PcalArgs a)
{
   extern __shared__ double pc_smem[];  // [tonebins][2]
   const PcalJob job = a.jobs[blockIdx.y];
   const int T = blockDim.x;
   for (int i = threadIdx.x; i < 2 * a.tonebins; i += T) pc_smem[i] = 0.0;
   __syncthreads();
   const int nper = a.N / a.rotatorlen;
   const int p0 = (int)((long long)nper * blockIdx.x / gridDim.x);
   const int p1 = (int)((long long)nper * (blockIdx.x + 1) / gridDim.x);
   const bool chk = a.blank_any[a.code_stream[job.src]] != 0;
   for (int i = threadIdx.x; i < a.used; i += T) {
      double sr = 0.0, si = 0.0;
      for (int p = p0; p < p1; p++) {
         long long s = job.start + (long long)p * a.rotatorlen + i;
         double x = (double)pc_sample<NBIT>(a, job.src, s, chk);
         sr += x;
         (void)si;
      }
      // all samples of this thread share the in-period position i, so the
      // rotator factor is common: sum(x) * exp(i dphi i)
      double sn, cs;
      sincos(a.dphi * (double)i, &sn, &cs);
      const int b = i % a.tonebins;
      atomicAdd(&pc_smem[2 * b], sr * cs);
      atomicAdd(&pc_smem[2 * b + 1], sr * sn);
   }
   __syncthreads();
   double *dst = a.acc + (long long)job.out * 2 * a.tonebins;
   for (int i = threadIdx.x; i < 2 * a.tonebins; i += T) atomicAdd(&dst[i], pc_smem[i]);
   if (threadIdx.x == 0)
      atomicAdd(a.acc + (long long)a.nout * 2 * a.tonebins + job.out, (double)(p1 - p0) * (double)a.used);
}

// Tone phasors of the folded bins: tone k (frequency k * spacing + offset,
// moved to k * spacing by the rotator) is DFT bin k of the tonebins folded
// sums, divided by the number of samples folded -- the final step of the
// PCal library's extractors (src/IA-32/PhaseCal/PCal.cpp:654-678: forward DFT
// normalised by the length, bins picked per tone), in FP64 throughout.
__global__ void k_pcal_tones(PcalArgs a)
{
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= (long long)a.nout * a.ntones) return;
   const int o = (int)(t / a.ntones), k = (int)(t % a.ntones);
   const double *bins = a.acc + (long long)o * 2 * a.tonebins;
   const double cnt = a.acc[(long long)a.nout * 2 * a.tonebins + o];
   double sr = 0.0, si = 0.0;
   for (int b = 0; b < a.tonebins; b++) {
      // exp(-2 pi i k b / tonebins), the angle reduced exactly in integers
      const int m = (int)(((long long)k * b) % a.tonebins);
      double s, c;
      sincospi(-2.0 * (double)m / (double)a.tonebins, &s, &c);
      const double re = bins[2 * b], im = bins[2 * b + 1];
      sr += re * c - im * s;
      si += re * s + im * c;
   }
   const double inv = cnt > 0.0 ? 1.0 / cnt : 0.0;
   a.tones[2 * t] = sr * inv;
   a.tones[2 * t + 1] = si * inv;
}

// Word-wise fold, for rotator periods and job starts that are multiples of
// SPW * D: thread t of a job owns code word wi = t mod wpd of phase array
// ph = t / wpd in every period, i.e. the SPW sample positions
// i_k = (wi SPW + k) D + ph of the period, and sums them over its block's
// periods -- one coalesced load per code word (four periods in flight), two
// codes per pair-table lookup and packed FP32 add, FP32 partial sums
// flushed every 64 periods into FP64 sums held in shared memory; the FP64
// rotator is applied once per position at the end.
template <int NBIT>
__global__ void __launch_bounds__(256, 4) k_pcal_fold_words(PcalArgs a)
{
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT >= 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   constexpr int NPAIR = SPW / 2;                 // code pairs per word
   constexpr int PB = 2 * NBIT;                   // bits per pair
   constexpr int NLUT = NBIT < 8 ? 1 << PB : 1;   // pair table (1/2-bit codes)
   extern __shared__ double pc_smem[];  // [tonebins][2], then the FP64 sums [SPW][blockDim.x]
   __shared__ float lut[4];
   __shared__ float2 plut[NLUT];
   const PcalJob job = a.jobs[blockIdx.y];
   for (int i = threadIdx.x; i < 2 * a.tonebins; i += blockDim.x) pc_smem[i] = 0.0;
   if (threadIdx.x < 4) {
      const float lv[4] = {a.levels.x, a.levels.y, a.levels.z, a.levels.w};
      lut[threadIdx.x] = lv[threadIdx.x];
   }
   if (NBIT < 8)
      for (int i = threadIdx.x; i < NLUT; i += blockDim.x)
         plut[i] = make_float2(decode_level<NBIT>(i & MASK, a.levels), decode_level<NBIT>((i >> NBIT) & MASK, a.levels));
   __syncthreads();
   const int D = a.D, rot = a.rotatorlen;
   const int wpd = rot / (SPW * D);
   const int nper = a.N / rot;
   const int p0 = (int)((long long)nper * blockIdx.x / gridDim.x);
   const int p1 = (int)((long long)nper * (blockIdx.x + 1) / gridDim.x);
   const bool chk = a.blank_any[a.code_stream[job.src]] != 0;
   const uint32_t *blank = a.blank + (long long)a.code_stream[job.src] * a.blank_words;
   for (int t = threadIdx.x; t < wpd * D; t += blockDim.x) {
      const int ph = t / wpd, wi = t % wpd;
      const uint32_t *base = a.codes + (long long)job.src * a.code_words + (long long)ph * a.wpp +
                             job.start / ((long long)D * SPW) + wi;
      // per-position FP64 sums in shared memory ([k][thread]: a warp's
      // accesses are consecutive), leaving the registers to the FP32 sums
      double *sd = pc_smem + 2 * a.tonebins + threadIdx.x;
      float s[SPW];
#pragma unroll
      for (int k = 0; k < SPW; k++) {
         s[k] = 0.0f;
         sd[k * blockDim.x] = 0.0;
      }
      if (!chk) {
         // four periods' words in flight, two codes per table lookup and
         // packed add; the FP32 sums of each position run in period order
         // and are flushed after the same 64-period groups as below
         float2 s2[NPAIR];
#pragma unroll
         for (int q = 0; q < NPAIR; q++) s2[q] = make_float2(0.0f, 0.0f);
         for (int p = p0; p < p1; p += 4) {
            uint32_t w[4];
#pragma unroll
            for (int v = 0; v < 4; v++) w[v] = p + v < p1 ? __ldg(base + (long long)(p + v) * wpd) : 0u;
#pragma unroll
            for (int v = 0; v < 4; v++) {
               if (p + v < p1) {
#pragma unroll
                  for (int q = 0; q < NPAIR; q++) {
                     float2 x;
                     if constexpr (NBIT == 8)
                        x = make_float2(decode_level<8>((w[v] >> (PB * q)) & 0xffu, a.levels),
                                        decode_level<8>((w[v] >> (PB * q + 8)) & 0xffu, a.levels));
                     else
                        x = plut[(w[v] >> (PB * q)) & ((1u << PB) - 1u)];
                     s2[q] = padd(s2[q], x);
                  }
               }
            }
            if (((p - p0) & 63) == 60) {
#pragma unroll
               for (int q = 0; q < NPAIR; q++) {
                  sd[2 * q * blockDim.x] += (double)s2[q].x;
                  sd[(2 * q + 1) * blockDim.x] += (double)s2[q].y;
                  s2[q] = make_float2(0.0f, 0.0f);
               }
            }
         }
#pragma unroll
         for (int q = 0; q < NPAIR; q++) {
            s[2 * q] = s2[q].x;
            s[2 * q + 1] = s2[q].y;
         }
      } else {
         for (int p = p0; p < p1; p++) {
            const uint32_t w = __ldg(base + (long long)p * wpd);
#pragma unroll
            for (int k = 0; k < SPW; k++) {
               const uint32_t code = (w >> (NBIT * k)) & MASK;
               float v = (NBIT == 8) ? (float)((int)code * 2 - 255) * (1.0f / 256.0f) : lut[code & 3];
               const long long smp = job.start + (long long)p * rot + (long long)(wi * SPW + k) * D + ph;
               if ((__ldg(blank + (smp >> 5)) >> (smp & 31)) & 1u) v = 0.0f;
               s[k] += v;
            }
            if (((p - p0) & 63) == 63) {
#pragma unroll
               for (int k = 0; k < SPW; k++) {
                  sd[k * blockDim.x] += (double)s[k];
                  s[k] = 0.0f;
               }
            }
         }
      }
#pragma unroll
      for (int k = 0; k < SPW; k++) {
         const double tot = sd[k * blockDim.x] + (double)s[k];
         const int i = (wi * SPW + k) * D + ph;  // position within the period
         if (i < a.used) {
            double sn, cs;
            sincos(a.dphi * (double)i, &sn, &cs);
            const int b = i % a.tonebins;
            atomicAdd(&pc_smem[2 * b], tot * cs);
            atomicAdd(&pc_smem[2 * b + 1], tot * sn);
         }
      }
   }
   __syncthreads();
   double *dst = a.acc + (long long)job.out * 2 * a.tonebins;
   for (int i = threadIdx.x; i < 2 * a.tonebins; i += blockDim.x) atomicAdd(&dst[i], pc_smem[i]);
   if (threadIdx.x == 0)
      atomicAdd(a.acc + (long long)a.nout * 2 * a.tonebins + job.out, (double)(p1 - p0) * (double)a.used);
}

__global__ void k_pcal_out(PcalArgs a)
{
   long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (i < (long long)a.nout * 2 * a.tonebins) a.out[i] = (float)a.acc[i];
}

int launch_pcal(PcalArgs a, int nbit, cudaStream_t st)
{
   const size_t n = (size_t)a.nout * 2 * a.tonebins;
   if (a.zero_acc) cudaMemsetAsync(a.acc, 0, sizeof(double) * (n + a.nout), st);
   const int nper = a.N / a.rotatorlen;
   int bpj = nper < 8 ? nper : 8;
   dim3 grid(bpj, a.njobs);
   size_t sm = sizeof(double) * 2 * a.tonebins;
   const int spw = 32 / nbit;
   if (a.word_fold) {
      const int nw = a.rotatorlen / spw;  // threads' words per job (all phases)
      const int T = nw >= 256 ? 256 : ((nw + 31) / 32) * 32;
      sm += sizeof(double) * (size_t)spw * T;  // per-thread FP64 sums
      const void *kf = nbit == 1 ? (const void *)k_pcal_fold_words<1>
                                 : nbit == 2 ? (const void *)k_pcal_fold_words<2> : (const void *)k_pcal_fold_words<8>;
      if (sm > 48 * 1024 && cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
         return 1;
      if (nbit == 1) k_pcal_fold_words<1><<<grid, T, sm, st>>>(a);
      else if (nbit == 2) k_pcal_fold_words<2><<<grid, T, sm, st>>>(a);
      else k_pcal_fold_words<8><<<grid, T, sm, st>>>(a);
   } else {
      const int T = 256;
      if (nbit == 1) k_pcal_fold<1><<<grid, T, sm, st>>>(a);
      else if (nbit == 2) k_pcal_fold<2><<<grid, T, sm, st>>>(a);
      else k_pcal_fold<8><<<grid, T, sm, st>>>(a);
   }
   if (a.write_out) {
      k_pcal_out<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
      if (a.tones && a.ntones > 0) {
         const long long nt = (long long)a.nout * a.ntones;
         k_pcal_tones<<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(a);
      }
   }
   return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace sws
