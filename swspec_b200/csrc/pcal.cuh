// pcal.cuh -- K4: phase-cal tone folding (TaskCoreIPP::extract_PCal).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sws {

// One folded FFT's worth of samples: N samples of code array `src` from
// chunk sample `start`, accumulated into output slot `out`.
struct PcalJob {
   long long start;
   int src;
   int out;
};

struct PcalArgs {
   const uint32_t *codes;        // phase-decimated code arrays (see SpecArgs)
   long long code_words;
   long long wpp;
   int D;
   const uint32_t *blank;
   long long blank_words;
   const int *blank_any;
   const int *code_stream;
   const PcalJob *jobs;
   int njobs;
   int N;
   int tonebins, rotatorlen, used;
   double dphi;        // 2 pi (-offset / fs)
   float4 levels;
   float *out;         // [nout][tonebins][2]
   double *acc;        // [nout][tonebins][2] FP64 running sums, then [nout] samples folded
   double *tones;      // [nout][ntones][2] tone phasors (null: none)
   int ntones;
   int nout;
   int zero_acc;       // clear acc first (start of an output group)
   int write_out;      // round acc into out (end of an output group)
   int word_fold;      // rotatorlen and every job start are multiples of (32/nbit) * D
};

// Queues zeroing, folding and conversion on `st`; returns 0 or a CUDA error.
int launch_pcal(PcalArgs a, int nbit, cudaStream_t st);

}  // namespace sws
