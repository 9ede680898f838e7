// probe_fp32.cu -- FP32 FMA throughput probe (benchmark support only).
//
// The driver's measured peaks cover HBM copy bandwidth and bf16 tensor GEMM;
// the plain-FP32 spectrometer form is bounded by FP32 FMA issue instead, so
// the benchmark measures that peak here: every thread runs 8 independent FMA
// chains, 2 flops per FMA.
#include <cuda_runtime.h>

__global__ void k_fma_chains(float *out, int iters, float a, float b)
{
   float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
   float x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
   for (int i = 0; i < iters; i++) {
#pragma unroll
      for (int k = 0; k < 16; k++) {
         x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
         x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
      }
   }
   out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

extern "C" int sws_probe_fp32_tflops(int device, double *tflops)
{
   if (cudaSetDevice(device) != cudaSuccess) return -1;
   cudaDeviceProp p;
   cudaGetDeviceProperties(&p, device);
   const int blocks = p.multiProcessorCount * 8, threads = 256, iters = 4096;
   float *out = nullptr;
   if (cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) return -2;
   cudaEvent_t e0, e1;
   cudaEventCreate(&e0);
   cudaEventCreate(&e1);
   k_fma_chains<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
   cudaEventRecord(e0);
   const int reps = 5;
   for (int r = 0; r < reps; r++) k_fma_chains<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
   cudaEventRecord(e1);
   cudaEventSynchronize(e1);
   float ms = 0;
   cudaEventElapsedTime(&ms, e0, e1);
   double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads * reps;
   *tflops = flops / (ms * 1e-3) / 1e12;
   cudaEventDestroy(e0);
   cudaEventDestroy(e1);
   cudaFree(out);
   return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
