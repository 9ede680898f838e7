// pcallib.cu -- the reference's phase-cal extractor library on the GPU.
//
// Restates the three extractor classes of src/IA-32/PhaseCal/PCal.cpp and
// the factory that picks one (PCal::getNew, :92-112):
//   Trivial       (offset 0, :183-318): real samples folded into
//                 N = fs / gcd(spacing, fs) bins;
//   ImplicitShift (the offset's period a multiple of N, :521-678): real
//                 samples folded into N = fs / gcd(offset, fs) bins, the
//                 offset removed by picking DFT bins offset + n step;
//   Shifting      (otherwise, :321-517): samples rotated by exp(-i 2 pi
//                 offset t) from an FP32 oscillator table of period R and
//                 folded into N = fs / gcd(spacing, fs) bins, only the
//                 first floor(R / N) N samples of every full period.
// getFinalPCal folds the 2N-slot accumulator, takes the forward DFT scaled
// by 1/N and returns the tone bins.  Here every sum is FP64 (the reference
// adds in FP32) and the DFT is direct in FP64; the slot bookkeeping --
// pcal_index and rotator_index advanced only by the samples past the last
// whole period of a call, reset by adjustSampleOffset -- is the reference's.
//
// GPU layout: one extract call is a fold kernel over positions j of the
// period (one thread per j, summing x[k R + j] over a range of periods k,
// coalesced across j, then one FP64 atomic add per (thread, slot)) and a
// small kernel for the samples past the last whole period.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <string>

#include "../../include/swsgpu.h"

namespace sws {
void record_create_error(const std::string &msg);
}

namespace {

__global__ void k_pcallib_fold(const float *__restrict__ x, long long nper, int R, int N, int P, int kind,
                               long long pi, long long ri, const float2 *__restrict__ rot, double2 *acc,
                               int per_chunk)
{
   const int j = blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= R) return;
   if (kind == SWSGPU_PCAL_SHIFTING && j >= P * N) return;  // past the last whole pulse of a period
   const long long k0 = (long long)blockIdx.y * per_chunk;
   const long long k1 = min(nper, k0 + per_chunk);
   double s = 0.0;
   for (long long k = k0; k < k1; k++) s += (double)__ldg(x + k * R + j);
   const long long slot = pi + (j % N);
   if (kind == SWSGPU_PCAL_SHIFTING) {
      const float2 w = rot[ri + j];
      atomicAdd(&acc[slot].x, s * (double)w.x);
      atomicAdd(&acc[slot].y, s * (double)w.y);
   } else {
      atomicAdd(&acc[slot].x, s);
   }
}

// The samples past the last whole period: sample m at slot pi + m mod N,
// rotated by the oscillator at ri + m (Shifting), every sample added.
__global__ void k_pcallib_tail(const float *__restrict__ x, int tail, int N, int kind, long long pi, long long ri,
                               const float2 *__restrict__ rot, double2 *acc)
{
   const int m = blockIdx.x * blockDim.x + threadIdx.x;
   if (m >= tail) return;
   const double v = (double)x[m];
   const long long slot = pi + (m % N);
   if (kind == SWSGPU_PCAL_SHIFTING) {
      const float2 w = rot[ri + m];
      atomicAdd(&acc[slot].x, v * (double)w.x);
      atomicAdd(&acc[slot].y, v * (double)w.y);
   } else {
      atomicAdd(&acc[slot].x, v);
   }
}

// One tone per thread: fold the two halves, forward DFT bin idx scaled by 1/N.
__global__ void k_pcallib_final(const double2 *__restrict__ acc, int N, int ntones, int kind, long long step,
                                long long off, double2 *out)
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= ntones) return;
   const long long idx = (kind == SWSGPU_PCAL_TRIVIAL) ? t : off + (long long)t * step;
   double sr = 0.0, si = 0.0;
   if (idx < N) {
      for (int k = 0; k < N; k++) {
         const double2 a = acc[k], b = acc[k + N];
         const double re = a.x + b.x, im = a.y + b.y;
         double s, c;
         sincospi(-2.0 * (double)((idx * (long long)k) % N) / (double)N, &s, &c);
         sr += re * c - im * s;
         si += re * s + im * c;
      }
      sr /= N;
      si /= N;
   }
   out[t] = make_double2(sr, si);
}

long long gcdll(long long a, long long b)
{
   while (b) {
      const long long t = a % b;
      a = b;
      b = t;
   }
   return a < 0 ? -a : a;
}

}  // namespace

struct swsgpu_pcal {
   int device = 0;
   int kind = 0;
   double fs = 0, spacing = 0, offset = 0;
   int nbins = 0, ntones = 0, rotlen = 0;
   long long pcal_index = 0, rotator_index = 0;
   uint64_t samplecount = 0;
   bool finalized = false;
   double2 *d_acc = nullptr;  // [2 nbins]
   float2 *d_rot = nullptr;   // [2 rotlen], Shifting only
   double2 *d_out = nullptr;  // [ntones]
};

extern "C" {

int swsgpu_pcal_create(double bandwidth_hz, double spacing_hz, int offset_hz, int64_t sampleoffset, int kind,
                       int device, swsgpu_pcal **out)
{
   if (!out) return SWSGPU_EINVAL;
   *out = nullptr;
   const long long fs = (long long)(2.0 * bandwidth_hz);
   if (fs <= 0 || spacing_hz <= 0 || offset_hz < 0 || sampleoffset < 0 || kind < SWSGPU_PCAL_AUTO ||
       kind > SWSGPU_PCAL_IMPLICIT) {
      sws::record_create_error("swsgpu_pcal_create: bad bandwidth, spacing, offset, sample offset or kind");
      return SWSGPU_EINVAL;
   }
   if (kind == SWSGPU_PCAL_AUTO) {
      if (offset_hz == 0) {
         kind = SWSGPU_PCAL_TRIVIAL;
      } else {
         const long long No = fs / gcdll(offset_hz, fs), Np = fs / gcdll((long long)spacing_hz, fs);
         kind = (No % Np == 0) ? SWSGPU_PCAL_IMPLICIT : SWSGPU_PCAL_SHIFTING;
      }
   }
   swsgpu_pcal *p = new swsgpu_pcal();
   p->device = device;
   p->kind = kind;
   p->fs = (double)fs;
   p->spacing = spacing_hz;
   p->offset = offset_hz;
   if (kind == SWSGPU_PCAL_IMPLICIT) {
      p->nbins = (int)(fs / gcdll(offset_hz, fs));
      p->ntones = (int)std::floor((bandwidth_hz - offset_hz) / spacing_hz) + 1;
   } else {
      p->nbins = (int)(fs / gcdll((long long)spacing_hz, fs));
      p->ntones = kind == SWSGPU_PCAL_TRIVIAL ? (int)std::floor(bandwidth_hz / spacing_hz)
                                              : (int)std::floor((bandwidth_hz - offset_hz) / spacing_hz) + 1;
   }
   p->rotlen = kind == SWSGPU_PCAL_SHIFTING ? (int)(fs / gcdll(offset_hz, fs)) : p->nbins;
   if (p->nbins < 1 || p->ntones < 1 || p->nbins > (1 << 24) || p->rotlen > (1 << 24)) {
      delete p;
      sws::record_create_error("swsgpu_pcal_create: no tones, or more than 2^24 bins");
      return SWSGPU_EINVAL;
   }
   p->pcal_index = sampleoffset % p->nbins;
   p->rotator_index = sampleoffset % p->rotlen;
   cudaError_t e = cudaSetDevice(device);
   if (e == cudaSuccess) e = cudaMalloc(&p->d_acc, sizeof(double2) * 2 * (size_t)p->nbins);
   if (e == cudaSuccess) e = cudaMalloc(&p->d_out, sizeof(double2) * (size_t)p->ntones);
   if (e == cudaSuccess) e = cudaMemset(p->d_acc, 0, sizeof(double2) * 2 * (size_t)p->nbins);
   if (e == cudaSuccess && kind == SWSGPU_PCAL_SHIFTING) {
      // the oscillator table of PCalExtractorShifting (:350-355): FP32 values of
      // exp(i dphi n), n < 2R, the argument in double
      float2 *h = (float2 *)malloc(sizeof(float2) * 2 * (size_t)p->rotlen);
      const double dphi = 2 * M_PI * (-(double)offset_hz / p->fs);
      for (int n = 0; n < 2 * p->rotlen; n++) h[n] = make_float2((float)cos(dphi * n), (float)sin(dphi * n));
      e = cudaMalloc(&p->d_rot, sizeof(float2) * 2 * (size_t)p->rotlen);
      if (e == cudaSuccess) e = cudaMemcpy(p->d_rot, h, sizeof(float2) * 2 * (size_t)p->rotlen, cudaMemcpyHostToDevice);
      free(h);
   }
   if (e != cudaSuccess) {
      sws::record_create_error(std::string("swsgpu_pcal_create: ") + cudaGetErrorString(e));
      cudaFree(p->d_acc);
      cudaFree(p->d_out);
      cudaFree(p->d_rot);
      delete p;
      return e == cudaErrorNoDevice || e == cudaErrorInvalidDevice ? SWSGPU_ENODEV : SWSGPU_ECUDA;
   }
   *out = p;
   return SWSGPU_OK;
}

int swsgpu_pcal_info(const swsgpu_pcal *p, int *kind, int *nbins, int *ntones)
{
   if (!p) return SWSGPU_EINVAL;
   if (kind) *kind = p->kind;
   if (nbins) *nbins = p->nbins;
   if (ntones) *ntones = p->ntones;
   return SWSGPU_OK;
}

int swsgpu_pcal_clear(swsgpu_pcal *p)
{
   if (!p) return SWSGPU_EINVAL;
   if (cudaSetDevice(p->device) != cudaSuccess ||
       cudaMemset(p->d_acc, 0, sizeof(double2) * 2 * (size_t)p->nbins) != cudaSuccess)
      return SWSGPU_ECUDA;
   p->samplecount = 0;
   p->finalized = false;
   return SWSGPU_OK;
}

int swsgpu_pcal_adjust_offset(swsgpu_pcal *p, int64_t sampleoffset)
{
   if (!p || sampleoffset < 0) return SWSGPU_EINVAL;
   p->pcal_index = sampleoffset % p->nbins;
   if (p->kind == SWSGPU_PCAL_SHIFTING) p->rotator_index = sampleoffset % p->rotlen;
   return SWSGPU_OK;
}

int swsgpu_pcal_extract(swsgpu_pcal *p, const float *d_samples, int64_t len, void *cuda_stream)
{
   if (!p || (!d_samples && len > 0) || len < 0) return SWSGPU_EINVAL;
   if (p->finalized) return SWSGPU_ESTATE;  // the reference returns false until clear()
   if (len == 0) return SWSGPU_OK;
   if (cudaSetDevice(p->device) != cudaSuccess) return SWSGPU_ECUDA;
   cudaStream_t st = (cudaStream_t)cuda_stream;
   const int R = p->rotlen, N = p->nbins, P = R / N;
   const long long tail = len % R, nper = len / R;
   if (nper > 0) {
      const int per_chunk = 256;
      dim3 grid((unsigned)((R + 255) / 256), (unsigned)((nper + per_chunk - 1) / per_chunk));
      if (grid.y > 65535u) {
         // longer calls: fold in pieces of whole periods
         long long done = 0;
         while (done < nper) {
            const long long part = std::min(nper - done, (long long)65535 * per_chunk);
            dim3 g2(grid.x, (unsigned)((part + per_chunk - 1) / per_chunk));
            k_pcallib_fold<<<g2, 256, 0, st>>>(d_samples + done * R, part, R, N, P, p->kind, p->pcal_index,
                                               p->rotator_index, p->d_rot, p->d_acc, per_chunk);
            done += part;
         }
      } else {
         k_pcallib_fold<<<grid, 256, 0, st>>>(d_samples, nper, R, N, P, p->kind, p->pcal_index, p->rotator_index,
                                              p->d_rot, p->d_acc, per_chunk);
      }
   }
   if (tail > 0)
      k_pcallib_tail<<<(unsigned)((tail + 255) / 256), 256, 0, st>>>(d_samples + nper * R, (int)tail, N, p->kind,
                                                                    p->pcal_index, p->rotator_index, p->d_rot,
                                                                    p->d_acc);
   cudaError_t e = cudaGetLastError();
   if (e != cudaSuccess) {
      sws::record_create_error(std::string("swsgpu_pcal_extract: ") + cudaGetErrorString(e));
      return SWSGPU_ECUDA;
   }
   if (p->kind == SWSGPU_PCAL_SHIFTING) {
      p->rotator_index = (p->rotator_index + tail) % R;
      p->pcal_index = (p->pcal_index + tail % N) % N;
   } else {
      p->pcal_index = (p->pcal_index + tail) % N;
   }
   p->samplecount += (uint64_t)len;
   return SWSGPU_OK;
}

int swsgpu_pcal_final(swsgpu_pcal *p, double *tones_reim, uint64_t *nsamples, void *cuda_stream)
{
   if (!p || !tones_reim) return SWSGPU_EINVAL;
   if (cudaSetDevice(p->device) != cudaSuccess) return SWSGPU_ECUDA;
   cudaStream_t st = (cudaStream_t)cuda_stream;
   const long long step = (long long)std::floor((double)p->nbins * (p->spacing / p->fs));
   const long long off = p->kind == SWSGPU_PCAL_IMPLICIT ? (long long)std::floor((double)p->nbins * p->offset / p->fs) : 0;
   k_pcallib_final<<<(unsigned)((p->ntones + 63) / 64), 64, 0, st>>>(p->d_acc, p->nbins, p->ntones, p->kind, step,
                                                                     off, p->d_out);
   cudaError_t e = cudaGetLastError();
   if (e == cudaSuccess)
      e = cudaMemcpyAsync(tones_reim, p->d_out, sizeof(double2) * (size_t)p->ntones, cudaMemcpyDeviceToHost, st);
   if (e == cudaSuccess) e = cudaStreamSynchronize(st);
   if (e != cudaSuccess) {
      sws::record_create_error(std::string("swsgpu_pcal_final: ") + cudaGetErrorString(e));
      return SWSGPU_ECUDA;
   }
   p->finalized = true;
   if (nsamples) *nsamples = p->samplecount;
   return SWSGPU_OK;
}

void swsgpu_pcal_destroy(swsgpu_pcal *p)
{
   if (!p) return;
   cudaSetDevice(p->device);
   cudaFree(p->d_acc);
   cudaFree(p->d_out);
   cudaFree(p->d_rot);
   delete p;
}

// calcDelay of mark5access's pulse-cal tool (mark5access/examples/m5pcal.c:
// 96-155): the mean phase slope between neighbouring tones inside the valid
// band, each phase difference unwrapped against the one at the middle of the
// list, in ns, folded into +- the ambiguity window 500 / (tone spacing, MHz).
double swsgpu_pcal_delay(int ntones, const int *tone_mhz, const double *phase, double band_center_mhz,
                         double band_valid_mhz)
{
   if (ntones < 2 || !tone_mhz || !phase) return 0.0;
   const double ref = phase[ntones / 2 + 1] - phase[ntones / 2];
   double sum = 0.0;
   int n = 0;
   for (int i = 1; i < ntones; i++) {
      const double f0 = tone_mhz[i - 1], f1 = tone_mhz[i];
      if (std::fabs(f0 - band_center_mhz) > band_valid_mhz || std::fabs(f1 - band_center_mhz) > band_valid_mhz)
         continue;
      double d = phase[i] - phase[i - 1];
      if (d - ref > M_PI) d -= 2.0 * M_PI;
      if (ref - d > M_PI) d += 2.0 * M_PI;
      sum += d / (f1 - f0);
      n++;
   }
   if (n < 1) return 0.0;
   const double window = std::fabs(500.0 / (tone_mhz[ntones / 2 + 1] - tone_mhz[ntones / 2]));
   double delay = 1000.0 * (sum / n) / (2.0 * M_PI);
   while (delay > window) delay -= 2.0 * window;
   while (delay < -window) delay += 2.0 * window;
   return delay;
}

}  // extern "C"
