// plans.cu -- instantiations of the cluster FFT kernel for the supported N.
//
// N = P * Q, cluster of P CTAs, each a Q-point Stockham FFT in shared memory
// with radices R1, R2, R3 (R1 fused with decode + window) and T threads.
#include "plans.cuh"
#include "spectra.cuh"

namespace sws {

#define SWS_PLAN(N_, P_, Q_, T_, R1_, R2_, R3_)                                                     \
   {N_, P_, Q_, T_, R1_, R2_, R3_,                                                                \
    {k_spectra<P_, Q_, T_, R1_, R2_, R3_, 1>, k_spectra<P_, Q_, T_, R1_, R2_, R3_, 2>,            \
     k_spectra<P_, Q_, T_, R1_, R2_, R3_, 8>},                                                    \
    (size_t)((Q_) + (Q_) / 16) * sizeof(float2) + (size_t)(Q_) * sizeof(float)}

static const Plan kPlans[] = {
    SWS_PLAN(65536, 8, 8192, 512, 16, 16, 32),
    SWS_PLAN(32768, 4, 8192, 512, 16, 16, 32),
    SWS_PLAN(16384, 2, 8192, 512, 16, 16, 32),
    SWS_PLAN(8192, 2, 4096, 256, 16, 16, 16),
    SWS_PLAN(4096, 2, 2048, 128, 16, 16, 8),
    SWS_PLAN(20000, 4, 5000, 320, 8, 25, 25),
    SWS_PLAN(131072, 16, 8192, 512, 16, 16, 32),
};

bool find_plan(int N, Plan *out)
{
   for (const Plan &p : kPlans)
      if (p.N == N) {
         *out = p;
         return true;
      }
   return false;
}

}  // namespace sws
