// plans.cuh -- FFT size plans of the cluster kernel.
#pragma once

#include "kernels.cuh"

namespace sws {

typedef void (*SpecKernel)(SpecArgs);

struct Plan {
   int N, P, Q, T;
   int R1, R2, R3;
   SpecKernel kern[3];   // nbit 1, 2, 8 (FP32 form)
   size_t smem[3];       // dynamic shared memory of each variant
   SpecKernel kern_tc[3];  // tensor-core split form (levels 2-3), or null where the plan has none
   size_t smem_tc[3];
   SpecKernel kern_tc2[3]; // tensor-core split form with all three local levels on tensor cores
   size_t smem_tc2[3];
};

// Returns false when N has no single-launch plan; *out = the default plan.
bool find_plan(int N, Plan *out);

// Every plan of length N, the default first; returns how many (<= max).
int plan_candidates(int N, Plan *out, int max);

}  // namespace sws
