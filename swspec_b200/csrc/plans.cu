// plans.cu -- instantiations of the cluster FFT kernel for the supported N.
//
// N = P * Q, cluster of P CTAs, each a Q-point Stockham FFT in shared memory
// with radices R1, R2, R3 (R1 fused with decode + window) and T threads;
// MINB resident CTAs per SM bound the register budget.
#include "plans.cuh"
#include "spectra.cuh"

namespace sws {

#define SWS_KERN(P_, Q_, T_, R1_, R2_, R3_, MINB_, PREC_)                                        \
   {k_spectra<P_, Q_, T_, R1_, R2_, R3_, 1, MINB_, PREC_>,                                        \
    k_spectra<P_, Q_, T_, R1_, R2_, R3_, 2, MINB_, PREC_>,                                        \
    k_spectra<P_, Q_, T_, R1_, R2_, R3_, 8, MINB_, PREC_>}
#define SWS_SMEM(P_, Q_, R1_, R2_, R3_, PREC_)                                                    \
   {spectra_smem<P_, Q_, R1_, R2_, R3_, 1, PREC_>(), spectra_smem<P_, Q_, R1_, R2_, R3_, 2, PREC_>(), \
    spectra_smem<P_, Q_, R1_, R2_, R3_, 8, PREC_>()}
// plans with tensor-core split forms (Q = 4096 = 16 x 16 x 16, T = 256):
// levels 2-3 on tcgen05 (level 1 in FP32 with the decode), or all three
#define SWS_PLAN_TC(N_, P_, MINB_)                                                                \
   {N_, P_, 4096, 256, 16, 16, 16, SWS_KERN(P_, 4096, 256, 16, 16, 16, MINB_, 0),                 \
    SWS_SMEM(P_, 4096, 16, 16, 16, 0), SWS_KERN(P_, 4096, 256, 16, 16, 16, MINB_, 1),            \
    SWS_SMEM(P_, 4096, 16, 16, 16, 1), SWS_KERN(P_, 4096, 256, 16, 16, 16, MINB_, 2),            \
    SWS_SMEM(P_, 4096, 16, 16, 16, 2)}
#define SWS_PLAN(N_, P_, Q_, T_, R1_, R2_, R3_, MINB_)                                            \
   {N_, P_, Q_, T_, R1_, R2_, R3_, SWS_KERN(P_, Q_, T_, R1_, R2_, R3_, MINB_, 0),                 \
    SWS_SMEM(P_, Q_, R1_, R2_, R3_, 0), {nullptr, nullptr, nullptr}, {0, 0, 0},                  \
    {nullptr, nullptr, nullptr}, {0, 0, 0}}

// The first plan of a length is its default; the others are candidates
// the autotuner times against it (cluster size, CTA size, radix order).
static const Plan kPlans[] = {
    SWS_PLAN_TC(65536, 16, 2),
    SWS_PLAN_TC(32768, 8, 2),
    SWS_PLAN_TC(16384, 4, 2),
    SWS_PLAN_TC(8192, 2, 2),
    SWS_PLAN(4096, 2, 2048, 128, 16, 16, 8, 4),
    SWS_PLAN(4096, 4, 1024, 64, 16, 8, 8, 8),     // 8 CTAs of 2 warps per SM
    SWS_PLAN(4096, 8, 512, 64, 8, 8, 8, 8),       // one radix-8 butterfly per thread and pass
    SWS_PLAN(20000, 4, 5000, 320, 8, 25, 25, 1),
    SWS_PLAN(20000, 4, 5000, 640, 8, 25, 25, 1),  // one butterfly per thread in every pass
    SWS_PLAN(131072, 16, 8192, 256, 16, 16, 32, 1),
    SWS_PLAN(131072, 16, 8192, 512, 16, 32, 16, 1),  // 16 warps per SM, register-capped
};

bool find_plan(int N, Plan *out)
{
   return plan_candidates(N, out, 1) > 0;
}

int plan_candidates(int N, Plan *out, int max)
{
   int n = 0;
   for (const Plan &p : kPlans)
      if (p.N == N && n < max) out[n++] = p;
   return n;
}

}  // namespace sws
