// bigfft.cuh -- four-step FFT path for lengths beyond one cluster
// (N = N1 * N2 up to 2^22 and 3,200,000 = 2^10 5^5).
#pragma once

#include "kernels.cuh"

namespace sws {

// One pair FFT: two real frames packed as z = w (a + i b).
struct BigJob {
   long long sa, sb;    // run-relative first sample of frame a / frame b
   int code_a, code_b;  // code arrays (code_b unused in MODE_SINGLE)
   int mode;            // MODE_XPOL / MODE_AUTOSUM / MODE_SINGLE
   int pad;
};

// The jobs [job0, job0 + nfr) of one work item accumulate into partial row
// `item` (layout [item][4][S], as the cluster kernel writes it).
struct BigItem {
   int job0, nfr, mode, item;
};

struct BigArgs {
   // col_layout 0: codes[code * code_words + s / SPW] (no decimation);
   // col_layout 1: decimated by N2, codes[code * code_words + (s % N2) * wpp +
   // (s / N2) / SPW], so that every column of the column pass is one
   // contiguous run of one phase array
   const uint32_t *codes;
   long long code_words;
   long long wpp;
   int col_layout;
   const uint32_t *blank;      // per stream blank bitmap (1 bit per sample-time)
   long long blank_words;
   const int *blank_any;
   const int *code_stream;
   const BigJob *jobs;         // jobs of this batch (scratch slot = index)
   const BigItem *bitems;      // items of this batch
   const float *window;        // N
   const float2 *tw1;          // W_N1^m, m < N1
   const float2 *tw2;          // W_N2^m, m < N2
   const double2 *twA;         // W_N^(2048 h), h < ceil(N / 2048), FP64
   const double2 *twB;         // W_N^l, l < 2048, FP64
   float2 *scratch;            // [job][N1][N2] column FFTs, twiddled
   float *partial;
   int nbjobs;                 // jobs of this batch (column pass)
   int nbitems;                // items of this batch (row pass)
   int N, S;
   float4 levels;
   int *status;                // set to 1 when a bounded wait gave up (null: not reported)
};

typedef void (*BigColsKernel)(BigArgs);
typedef void (*BigRowsKernel)(BigArgs);

struct BigPlan {
   int N, N1, N2, C;            // columns per CTA in the column pass
   int TA, TB;                  // threads of the column / row kernels
   BigColsKernel cols[3];       // nbit 1, 2, 8
   BigRowsKernel rows;
   size_t smem_cols[3], smem_rows;  // column pass per bit depth (1, 2, 8)
   BigRowsKernel rows_tc;       // tensor-core split row pass (N2 = 4096), or null
   size_t smem_rows_tc;
   int TBtc;                    // its threads
};

bool find_big_plan(int N, BigPlan *out);
// Every candidate split of N (default first); returns how many were written.
int big_plan_candidates(int N, BigPlan *out, int max);

}  // namespace sws
