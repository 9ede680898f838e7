// engine.cu -- C ABI of the spectrometer core (include/swsgpu.h).
//
// Host side of one GPU TaskCore: validates the configuration, plans the
// per-run FFT schedule exactly as TaskCoreIPP::doMaths walks a raw buffer
// (src/IA-32/TaskCoreIPP.cpp:394-524), groups FFT jobs into work items, and
// launches K1 (frame validity + corner turn), K2 (cluster FFT + accumulate)
// and K3 (compensated reduction + scaling) on the handle's CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/swsgpu.h"
#include "kernels.cuh"
#include "plans.cuh"
#include "bigfft.cuh"
#include "pcal.cuh"

namespace sws {
__global__ void k_frame_valid(StreamIn s, int2 *valid, int *blank_any);
cudaError_t launch_unpack_codes(cudaStream_t st, StreamIn s, long long nsamp, const int *chans, int nch,
                                uint32_t *codes, int D, long long wpp, const int2 *valid,
                                const int *blank_any, uint32_t *blank, int &launches);
bool unpack_decimation_ok(int D, int nchan, int nbit);
void track_turn_table(int ntrack, int nbit, int nchan, uint32_t *table);
cudaError_t launch_track_turn(cudaStream_t st, const uint8_t *in, long long nbytes, long long grid_offset,
                              int ntrack, int format, const uint32_t *table, uint32_t *out);
__global__ void k_unpack_float(StreamIn s, long long nsamp, int chan, float4 levels, float *out,
                               const int2 *valid, unsigned long long *nvalid);
__global__ void k_reduce(const float *partial, int S, const RedEntry *ent, const OutVec *ov);
}  // namespace sws

using namespace sws;

static thread_local std::string g_create_error;

namespace sws {
// The message swsgpu_last_error(NULL) returns on this thread.
void record_create_error(const std::string &msg) { g_create_error = msg; }
}  // namespace sws

// The kernel and shared-memory size of a cluster plan's form.
static SpecKernel plan_kernel(const Plan &pl, int precision, int nbi)
{
   return precision == SWSGPU_PREC_TCSPLIT ? pl.kern_tc[nbi]
          : precision == SWSGPU_PREC_TCSPLIT_ALL ? pl.kern_tc2[nbi] : pl.kern[nbi];
}
static size_t plan_smem(const Plan &pl, int precision, int nbi)
{
   return precision == SWSGPU_PREC_TCSPLIT ? pl.smem_tc[nbi]
          : precision == SWSGPU_PREC_TCSPLIT_ALL ? pl.smem_tc2[nbi] : pl.smem[nbi];
}

// Launch attributes of the cluster kernel: P CTAs per cluster.  The FP32
// form is placed with the load-balancing policy, which fits one more 16-CTA
// cluster of two CTAs per SM on a B200 than the default spread policy (15
// against 14: 120 SMs busy instead of 112; the FP32 kernel of the
// dual-pol workload went from 4.84 to 4.53 ms).  The tensor-core forms keep
// the spread policy: their grid of 15 load-balanced clusters ran as 14 plus
// a straggler (10.5 ms against 6.9 ms for 14 spread clusters).  Returns the
// number of attributes written.
static unsigned cluster_attrs(cudaLaunchAttribute (&attr)[2], int P, int precision)
{
   attr[0].id = cudaLaunchAttributeClusterDimension;
   attr[0].val.clusterDim.x = P;
   attr[0].val.clusterDim.y = 1;
   attr[0].val.clusterDim.z = 1;
   attr[1].id = cudaLaunchAttributeClusterSchedulingPolicyPreference;
   attr[1].val.clusterSchedulingPolicyPreference = precision == SWSGPU_PREC_FP32
                                                       ? cudaClusterSchedulingPolicyLoadBalancing
                                                       : cudaClusterSchedulingPolicySpread;
   return 2;
}


struct DevBuf {
   void *p = nullptr;
   size_t n = 0;
   cudaError_t ensure(size_t bytes)
   {
      if (bytes <= n) return cudaSuccess;
      if (p) cudaFree(p);
      p = nullptr;
      n = 0;
      cudaError_t e = cudaMalloc(&p, bytes);
      if (e == cudaSuccess) n = bytes;
      return e;
   }
   void release()
   {
      if (p) cudaFree(p);
      p = nullptr;
      n = 0;
   }
};

struct HostBuf {
   void *p = nullptr;
   size_t n = 0;
   cudaError_t ensure(size_t bytes)
   {
      if (bytes <= n) return cudaSuccess;
      if (p) cudaFreeHost(p);
      p = nullptr;
      n = 0;
      cudaError_t e = cudaMallocHost(&p, bytes);
      if (e == cudaSuccess) n = bytes;
      return e;
   }
   void release()
   {
      if (p) cudaFreeHost(p);
      p = nullptr;
      n = 0;
   }
};

// Work schedule of one call (host side).
struct Schedule {
   std::vector<Item> items;
   std::vector<RedEntry> entries;
   std::vector<OutVec> outs;
   std::vector<PcalJob> pcal_jobs;
   std::vector<RedEntry> pcal_entries;
   std::vector<OutVec> pcal_outs;
   int nspec_total = 0;
   long long nsamp = 0;    // chunk sample-times
   int nffts = 0;
   // cluster path: cluster c runs items [cl_first[c], cl_first[c + 1]), ncl clusters
   std::vector<int> cl_first;
   int ncl = 0;
};

// A schedule built once and kept on the device: runs of the same size and
// outputs reuse it, so a submit uploads nothing but its raw bytes.
struct SchedEntry {
   // key
   size_t run_bytes = 0;
   int nruns = 0, rpo = 0, acc_mode = 0;
   float *d_auto = nullptr, *d_xpol = nullptr, *d_pcal = nullptr;
   void *acc_base = nullptr;
   // value
   Schedule sc;
   DevBuf d_items, d_entries, d_outs, d_pcal_jobs, d_bjobs, d_bitems, d_cl_first;
   std::vector<int4> batches;  // four-step: {job0, njobs, item0, nitems}
   int pcal_word_fold = 0;     // phase-cal jobs allow the word-wise fold
   void release()
   {
      d_items.release();
      d_cl_first.release();
      d_entries.release();
      d_outs.release();
      d_pcal_jobs.release();
      d_bjobs.release();
      d_bitems.release();
   }
};

// Device buffers of one pipeline launch: frame validity, decoded codes,
// blank bitmap and per-item partial spectra.  The submit path keeps two
// sets, so that consecutive chunks run on two streams and one chunk's
// unpack and FFT fill the SMs that the previous chunk's last wave leaves.
struct Scratch {
   DevBuf d_valid[SWSGPU_MAX_STREAMS];
   DevBuf d_codes, d_codes1, d_blank, d_blank_any, d_partial;
   DevBuf d_trk[SWSGPU_MAX_STREAMS];  // track formats: the chunk in Mark5B's sample layout
   void release()
   {
      for (int s = 0; s < SWSGPU_MAX_STREAMS; s++) d_valid[s].release();
      for (int s = 0; s < SWSGPU_MAX_STREAMS; s++) d_trk[s].release();
      d_codes.release();
      d_codes1.release();
      d_blank.release();
      d_blank_any.release();
      d_partial.release();
   }
};

struct swsgpu_handle {
   swsgpu_config cfg;
   int device = 0;
   Plan plan;
   bool big = false;   // four-step path (bplan) instead of the cluster kernel
   BigPlan bplan;
   int big_cands = 0;  // candidate splits of N
   int tuned = -1;     // candidate chosen by the autotuner (-1: default)
   int cand = 0;       // candidate in use (index into tw_off)
   std::vector<int2> tw_off;  // per candidate: offsets of its W_N1 and W_N2 tables in d_tw1
   int S = 0;
   int max_clusters = 1;
   const void *rows_fn = nullptr;   // four-step kernels the persistent grids were sized for
   const void *cols_fn = nullptr;
   int rows_grid = 0, cols_grid = 0;
   std::string err;
   cudaStream_t stream = nullptr;     // kernels and result copies
   cudaStream_t cstream = nullptr;    // input copies of submit()
   cudaStream_t stream2 = nullptr;    // chunks of input region 1 (cluster path)
   cudaEvent_t acc_done = nullptr;    // the last chunk's sums and phase-cal folds added
   bool acc_pending = false;          // acc_done recorded since `stream` last waited on it
   cudaEvent_t done = nullptr;        // results of the last submitted run copied back
   // two device input slots per stream: run r+1's copy overlaps run r's kernels
   DevBuf d_slot[2][SWSGPU_MAX_STREAMS];
   cudaEvent_t slot_h2d[2] = {nullptr, nullptr};   // input copy into the slot finished
   cudaEvent_t slot_free[2] = {nullptr, nullptr};  // kernels finished reading the slot
   int next_slot = 0;
   cudaEvent_t last_h2d = nullptr;    // input copy of the last submitted run
   // runs of one output group collected into device chunks of up to chunk_max
   // runs (header-free streams, equal sizes, consecutive payload offsets) and
   // processed by one launch per chunk: one run per launch leaves most of the
   // cluster kernel's CTAs idle at the end of each launch
   DevBuf d_region[2][SWSGPU_MAX_STREAMS];
   cudaEvent_t region_free[2] = {nullptr, nullptr};
   // chunk_target: size of the open chunk, chosen when its first run
   // arrives; the last chunks of a group shrink so that little compute is
   // left once the group's last copy lands
   int chunk_max = 1, chunk_n = 0, chunk_region = 0, chunk_target = 1;
   bool chunk_group_first = false;
   size_t chunk_run_bytes = 0;
   long long chunk_off0[SWSGPU_MAX_STREAMS] = {0, 0};
   bool pending_out = false;          // the pending run completes spectra
   bool pending = false;
   int pending_nspec = 0;
   int last_launches = 0;
   int inject = SWSGPU_INJECT_NONE;  // one-shot fault injection for the next cluster launch
   // code arrays: one per distinct (stream, channel)
   std::vector<int> code_stream, code_chan;
   std::vector<int> src_code;     // source -> code index
   std::vector<int> auto_owner;   // source -> xpol index that owns its auto (-1: none)
   // constant tables
   DevBuf d_window, d_twQ, d_twN, d_code_stream;
   DevBuf d_trk_table;  // track formats: the track turn's unit-byte tables
   DevBuf d_tw1, d_tw2, d_twA, d_twB;               // four-step tables
   DevBuf d_scratch, d_bjobs, d_bitems;             // four-step intermediate and job lists
   DevBuf d_status;                                 // kernel status word (1: a bounded wait gave up)
   // per-call buffers
   DevBuf d_raw[SWSGPU_MAX_STREAMS], d_chans[SWSGPU_MAX_STREAMS];
   DevBuf d_items, d_entries, d_outs;
   // launch buffers: set 0 on `stream`, set 1 on `stream2` (d_codes1 is the
   // undecimated copy for phase-cal when the four-step path uses the column layout)
   Scratch scr[2];
   DevBuf d_pcal_jobs, d_pcal_part, d_pcal_entries, d_pcal_outs;
   DevBuf d_out_auto, d_out_xpol, d_out_pcal, d_out_tones;
   HostBuf h_out;   // pinned staging of one run's outputs
   size_t h_auto_bytes = 0, h_xpol_bytes = 0, h_pcal_bytes = 0, h_tones_bytes = 0;
   // combining of consecutive runs on the device (runs_per_output > 1)
   DevBuf d_acc64;
   int group_pos = 0;
   bool fetch_ready = false;
   // spectra delivered by the submit that completed them (swsgpu_submit_out):
   // straight into pinned caller memory, or through h_out and a copy at wait
   bool delivered = false;
   void *deliver_copy[4] = {nullptr, nullptr, nullptr, nullptr};  // pageable destinations (auto, xpol, pcal, tones)
   // device-resident schedules (a few distinct run shapes per handle)
   std::vector<SchedEntry *> sched;
   // per-stream channel lists of the code arrays (K1), uploaded at create
   std::vector<int> chans_of[SWSGPU_MAX_STREAMS];
   int first_code[SWSGPU_MAX_STREAMS] = {-1, -1};
   // kernel timing
   bool profiling = false;
   std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
};

#define CK(h, call)                                                                                \
   do {                                                                                           \
      cudaError_t e_ = (call);                                                                    \
      if (e_ != cudaSuccess) {                                                                    \
         (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);                           \
         return SWSGPU_ECUDA;                                                                     \
      }                                                                                           \
   } while (0)

static int fail(swsgpu_handle *h, int code, const std::string &msg)
{
   if (h) h->err = msg;
   else g_create_error = msg;
   return code;
}

// ---------------------------------------------------------------------------
// windows (the reference's formulas, TaskCoreIPP.cpp:569-605)
// ---------------------------------------------------------------------------
static void make_window(int type, int n, std::vector<float> &w)
{
   w.resize(n);
   for (int i = 0; i < n; i++) {
      double fi = (double)(float)i, fn = (double)(float)n, v = 1.0;
      double a = 2.0 * M_PI * (double)i / (double)(n - 1);
      switch (type) {
      case SWSGPU_WIN_NONE: v = 1.0; break;
      case SWSGPU_WIN_COSINE: v = std::cos(M_PI * (fi - 0.5 * fn + 0.5) / fn); break;
      case SWSGPU_WIN_COSINE2: {
         double c = std::cos(M_PI * (fi - 0.5 * fn + 0.5) / fn);
         v = c * c;
      } break;
      case SWSGPU_WIN_HAMMING: v = 0.54 - 0.46 * std::cos(a); break;
      case SWSGPU_WIN_HANN: {
         double s = std::sin(M_PI * (double)i / (double)(n - 1));
         v = s * s;
      } break;
      case SWSGPU_WIN_BLACKMAN: v = 0.75 - 0.5 * std::cos(a) - 0.25 * std::cos(2.0 * a); break;
      case SWSGPU_WIN_BLACKMANHARRIS:
         v = 0.35875 - 0.48829 * std::cos(a) + 0.14128 * std::cos(2.0 * a) - 0.01168 * std::cos(3.0 * a);
         break;
      default: v = 1.0;
      }
      w[i] = (float)v;
   }
}

static void make_twiddles(int n, int count, std::vector<float2> &t)
{
   t.resize(count);
   for (int m = 0; m < count; m++) {
      double a = -2.0 * M_PI * (double)m / (double)n;
      t[m] = make_float2((float)std::cos(a), (float)std::sin(a));
   }
}


static int payload_bytes(const swsgpu_layout &l) { return l.frame_bytes - l.header_bytes; }

// Raw single-channel 2-bit data stores the oldest sample in the byte's MSBs.
static int is_msb2(const swsgpu_layout &l)
{
   return ((l.format == SWSGPU_FMT_RAW_SIGNED || l.format == SWSGPU_FMT_RAW_UNSIGNED) && l.nbit == 2 &&
           l.nchan == 1) ? 1 : 0;
}

// Checks a track-format layout (VLBA / Mark4): frame_bytes = 2500 ntrack
// (20000 track-words), tracks 8..64, fanout 1, 2 or 4, at most 32 bits per
// sample-time, payload only.  Returns the number of tracks, or 0.
static int track_layout_ok(const swsgpu_layout &l, std::string &why)
{
   const int ntrack = l.frame_bytes / 2500;
   if (l.header_bytes != 0 || l.frame_bytes % 2500 || (ntrack != 8 && ntrack != 16 && ntrack != 32 && ntrack != 64)) {
      why = "track formats: frame_bytes must be 2500 x tracks (8, 16, 32 or 64) with header_bytes 0";
      return 0;
   }
   if ((l.nbit != 1 && l.nbit != 2) || l.nchan * l.nbit > 64 || ntrack % (l.nchan * l.nbit)) {
      why = "track formats: nbit 1 or 2, nchan * nbit <= 64 and dividing the tracks";
      return 0;
   }
   const int fanout = ntrack / (l.nchan * l.nbit);
   if (fanout != 1 && fanout != 2 && fanout != 4) { why = "track formats: fanout must be 1, 2 or 4"; return 0; }
   return ntrack;
}

// ---------------------------------------------------------------------------
// doMaths frame schedule of one run (TaskCoreIPP.cpp:394-524)
// ---------------------------------------------------------------------------
struct RunShape {
   std::vector<long long> starts;  // run-relative first sample of each FFT
   std::vector<int> spec;          // run-local spectrum of each FFT
   int nspec = 0;
   bool partial = false;
};

static RunShape run_shape(const swsgpu_config &c, long long nsamp)
{
   RunShape r;
   long long pos = 0, hop = c.fft_points / c.overlap;
   int acc = 0, ns = 0;
   while (nsamp - pos >= c.fft_points) {
      r.starts.push_back(pos);
      r.spec.push_back(ns);
      pos += hop;
      if (++acc >= c.core_overlapped_ffts) {
         ns++;
         acc = 0;
         pos += c.fft_points - hop;
      }
   }
   r.partial = acc > 0;
   r.nspec = ns + (acc > 0);
   return r;
}

static long long samples_of(const swsgpu_layout &l, size_t payload_bytes_n)
{
   return (long long)((payload_bytes_n * 8ull) / (unsigned long long)(l.nchan * l.nbit));
}

// Cluster path: cluster c gets the jobs [c J / ncl, (c + 1) J / ncl) of the
// item sequence (J jobs in all), so that every cluster runs the same number
// of jobs however few items there are (a run's spectrum is at most one item,
// so a chunk of a few runs has few).  An item that straddles a boundary is
// split into segments, each with copies of the item's reduction entries.
static void balance_clusters(int max_clusters, Schedule &sc)
{
   long long J = 0;
   for (const Item &it : sc.items) J += it.nfr;
   if (J == 0) return;
   const int ncl = (int)std::max<long long>(1, std::min<long long>(max_clusters, J));
   std::vector<long long> bnd(ncl + 1);
   for (int k = 0; k <= ncl; k++) bnd[k] = J * k / ncl;
   std::vector<Item> items;
   std::vector<std::vector<int>> parts(sc.items.size());
   sc.cl_first.assign(ncl + 1, 0);
   long long pos = 0;  // sequence index of the current item's first job
   int cl = 0;         // cluster of the next segment
   for (size_t i = 0; i < sc.items.size(); i++) {
      const Item &it = sc.items[i];
      int j = 0;
      while (j < it.nfr) {
         while (cl < ncl - 1 && pos + j >= bnd[cl + 1]) {
            cl++;
            sc.cl_first[cl] = (int)items.size();
         }
         const long long end = std::min<long long>(pos + it.nfr, bnd[cl + 1]);
         const int n = (int)(end - (pos + j));
         Item s = it;
         s.start = it.start + (long long)j * it.step;
         s.nfr = n;
         parts[i].push_back((int)items.size());
         items.push_back(s);
         j += n;
      }
      pos += it.nfr;
   }
   for (int k = cl + 1; k <= ncl; k++) sc.cl_first[k] = (int)items.size();
   std::vector<RedEntry> ents;
   for (OutVec &o : sc.outs) {
      const int first = (int)ents.size();
      for (int k = o.first; k < o.first + o.count; k++)
         for (int id : parts[sc.entries[k].item]) {
            RedEntry e = sc.entries[k];
            e.item = id;
            ents.push_back(e);
         }
      o.first = first;
      o.count = (int)ents.size() - first;
   }
   sc.entries.swap(ents);
   sc.items.swap(items);
   sc.ncl = ncl;
}

// Build items, reduction entries and output vectors for `nruns` runs.
static void build_schedule(const swsgpu_handle *h, size_t run_bytes, int nruns, int runs_per_output,
                           float *d_auto, float *d_xpol, float *d_pcal, Schedule &sc)
{
   const swsgpu_config &c = h->cfg;
   const int S = h->S;
   const long long run_samp = samples_of(c.layout[0], run_bytes);
   RunShape rs = run_shape(c, run_samp);
   sc.nsamp = run_samp * nruns;
   const int groups = (nruns + runs_per_output - 1) / runs_per_output;
   sc.nspec_total = groups * rs.nspec;
   sc.nffts = (int)rs.starts.size() * nruns;
   const long long hop = c.fft_points / c.overlap;

   // jobs per spectrum and item size: aim for ~4 items per resident cluster
   long long total_jobs = 0;
   {
      int nxp = c.num_xpols, nauto = 0;
      for (int s = 0; s < c.num_sources; s++)
         if (h->auto_owner[s] < 0) nauto++;
      total_jobs = (long long)sc.nffts * nxp + (long long)(sc.nffts + 1) / 2 * nauto;
   }
   long long target_items = std::max<long long>(1, 4ll * h->max_clusters);
   int fper = (int)std::max<long long>(1, (total_jobs + target_items - 1) / target_items);
   // the four-step row kernel accumulates an item's jobs in FP32 registers
   // per CTA: at most 16 jobs per item, so those sums stay short and the
   // compensated reduction adds the items
   if (h->big) fper = 16;

   // key -> output vector index
   std::map<long long, std::vector<RedEntry>> vec_entries;
   std::map<long long, OutVec> vec_desc;
   auto add_entry = [&](long long key, float *dst, int stride, int item, int prod, float scale) {
      if (!vec_desc.count(key)) {
         OutVec o;
         o.first = 0;
         o.count = 0;
         o.dst = dst;
         o.stride = stride;
         vec_desc[key] = o;
      }
      RedEntry e;
      e.item = item;
      e.prod = prod;
      e.scale = scale;
      vec_entries[key].push_back(e);
   };

   const int nfr_run = (int)rs.starts.size();
   for (int r = 0; r < nruns; r++) {
      const long long base = (long long)r * run_samp;
      const int g0 = (r / runs_per_output) * rs.nspec;
      for (int sp = 0; sp < rs.nspec; sp++) {
         // frames of this spectrum (consecutive, uniform hop)
         int f0 = -1, nf = 0;
         for (int f = 0; f < nfr_run; f++)
            if (rs.spec[f] == sp) {
               if (f0 < 0) f0 = f;
               nf++;
            }
         if (nf == 0) continue;
         const bool full = !(rs.partial && sp == rs.nspec - 1);
         const float scale = 0.25f * (full ? (float)(1.0 / c.core_overlapped_ffts) : 1.0f);
         const int g = g0 + sp;
         const long long first = base + rs.starts[f0];
         // cross pairs
         for (int xp = 0; xp < c.num_xpols; xp++) {
            const int si = c.xpol_pair[xp][0], sj = c.xpol_pair[xp][1];
            for (int j0 = 0; j0 < nf; j0 += fper) {
               Item it;
               it.start = first + (long long)j0 * hop;
               it.src_a = h->src_code[si];
               it.src_b = h->src_code[sj];
               it.step = (int)hop;
               it.offset_b = 0;
               it.nfr = std::min(fper, nf - j0);
               it.mode = MODE_XPOL;
               const int id = (int)sc.items.size();
               sc.items.push_back(it);
               if (h->auto_owner[si] == xp && d_auto)
                  add_entry(((long long)g * 4 + 0) << 32 | (unsigned)si,
                            d_auto + ((size_t)g * c.num_sources + si) * S, 1, id, 0, scale);
               if (h->auto_owner[sj] == xp && d_auto)
                  add_entry(((long long)g * 4 + 0) << 32 | (unsigned)sj,
                            d_auto + ((size_t)g * c.num_sources + sj) * S, 1, id, 1, scale);
               if (d_xpol) {
                  float *xb = d_xpol + ((size_t)g * c.num_xpols + xp) * S * 2;
                  add_entry(((long long)g * 4 + 1) << 32 | (unsigned)xp, xb, 2, id, 2, scale);
                  add_entry(((long long)g * 4 + 2) << 32 | (unsigned)xp, xb + 1, 2, id, 3, scale);
               }
            }
         }
         // auto-only sources: consecutive frame pairs
         for (int s = 0; s < c.num_sources; s++) {
            if (h->auto_owner[s] >= 0 || !d_auto) continue;
            float *dst = d_auto + ((size_t)g * c.num_sources + s) * S;
            const long long key = ((long long)g * 4 + 0) << 32 | (unsigned)s;
            const int npairs = nf / 2;
            const int pper = std::max(1, fper);
            for (int j0 = 0; j0 < npairs; j0 += pper) {
               Item it;
               it.start = first + (long long)(2 * j0) * hop;
               it.src_a = h->src_code[s];
               it.src_b = h->src_code[s];
               it.step = (int)(2 * hop);
               it.offset_b = (int)hop;
               it.nfr = std::min(pper, npairs - j0);
               it.mode = MODE_AUTOSUM;
               const int id = (int)sc.items.size();
               sc.items.push_back(it);
               add_entry(key, dst, 1, id, 0, scale);
            }
            if (nf % 2) {
               Item it;
               it.start = first + (long long)(nf - 1) * hop;
               it.src_a = h->src_code[s];
               it.src_b = -1;
               it.step = 0;
               it.offset_b = 0;
               it.nfr = 1;
               it.mode = MODE_SINGLE;
               const int id = (int)sc.items.size();
               sc.items.push_back(it);
               add_entry(key, dst, 1, id, 0, scale);
            }
         }
         // phase-cal folding: every overlap-th source FFT, counted per source
         // FFT within the run (TaskCoreIPP.cpp:414-418, curr_ffts)
         if (c.extract_pcal && d_pcal) {
            for (int f = f0; f < f0 + nf; f++)
               for (int s = 0; s < c.num_sources; s++) {
                  const int curr = f * c.num_sources + s;
                  if (curr % c.overlap != 0) continue;
                  PcalJob pj;
                  pj.start = base + rs.starts[f];
                  pj.src = h->src_code[s];
                  pj.out = (g * c.num_sources + s);
                  sc.pcal_jobs.push_back(pj);
               }
         }
      }
   }
   for (auto &kv : vec_desc) {
      OutVec o = kv.second;
      auto &ents = vec_entries[kv.first];
      o.first = (int)sc.entries.size();
      o.count = (int)ents.size();
      sc.entries.insert(sc.entries.end(), ents.begin(), ents.end());
      sc.outs.push_back(o);
   }
   if (!h->big) balance_clusters(h->max_clusters, sc);
}

// ---------------------------------------------------------------------------
// four-step path: column and row passes over batches of whole work items
// ---------------------------------------------------------------------------
static const size_t kBigScratchBudget = (size_t)1 << 30;  // bytes of column-pass output per batch

// Whole work items per batch; a single item above the budget runs alone.
static void big_batches(const swsgpu_handle *h, const Schedule &sc, std::vector<BigJob> &jobs,
                        std::vector<BigItem> &bitems, std::vector<int4> &batches)
{
   const size_t job_bytes = sizeof(float2) * (size_t)h->cfg.fft_points;
   size_t i0 = 0;
   while (i0 < sc.items.size()) {
      const int job_base = (int)jobs.size(), item_base = (int)bitems.size();
      size_t i = i0;
      while (i < sc.items.size()) {
         const Item &it = sc.items[i];
         const size_t in_batch = jobs.size() - job_base;
         if (i > i0 && (in_batch + it.nfr) * job_bytes > kBigScratchBudget) break;
         BigItem bi;
         bi.job0 = (int)in_batch;
         bi.nfr = it.nfr;
         bi.mode = it.mode;
         bi.item = (int)i;
         for (int j = 0; j < it.nfr; j++) {
            BigJob jb;
            jb.sa = it.start + (long long)j * it.step;
            jb.sb = (it.mode == MODE_AUTOSUM) ? jb.sa + it.offset_b : jb.sa;
            jb.code_a = it.src_a;
            jb.code_b = (it.mode == MODE_XPOL) ? it.src_b : it.src_a;
            jb.mode = it.mode;
            jb.pad = 0;
            jobs.push_back(jb);
         }
         bitems.push_back(bi);
         i++;
      }
      batches.push_back(make_int4(job_base, (int)jobs.size() - job_base, item_base,
                                  (int)bitems.size() - item_base));
      i0 = i;
   }
}

static int launch_big(swsgpu_handle *h, const SchedEntry &se, long long code_words, long long wpp, bool col,
                      long long blank_words, Scratch &x,
                      cudaStream_t st, int &launches)
{
   const swsgpu_config &c = h->cfg;
   const BigPlan &bp = h->bplan;
   const int nbit = c.layout[0].nbit;
   const int nbi = nbit == 1 ? 0 : nbit == 2 ? 1 : 2;
   const size_t job_bytes = sizeof(float2) * (size_t)c.fft_points;
   int max_jobs = 0;
   for (const int4 &b : se.batches) max_jobs = std::max(max_jobs, b.y);
   CK(h, h->d_scratch.ensure(job_bytes * (size_t)max_jobs));
   BigArgs a;
   a.codes = (const uint32_t *)x.d_codes.p;
   a.code_words = code_words;
   a.wpp = wpp;
   a.col_layout = col ? 1 : 0;
   a.blank = (const uint32_t *)x.d_blank.p;
   a.blank_words = blank_words;
   a.blank_any = (const int *)x.d_blank_any.p;
   a.code_stream = (const int *)h->d_code_stream.p;
   a.window = (const float *)h->d_window.p;
   a.tw1 = (const float2 *)h->d_tw1.p + h->tw_off[h->cand].x;
   a.tw2 = (const float2 *)h->d_tw1.p + h->tw_off[h->cand].y;
   a.twA = (const double2 *)h->d_twA.p;
   a.twB = (const double2 *)h->d_twB.p;
   a.scratch = (float2 *)h->d_scratch.p;
   a.partial = (float *)x.d_partial.p;
   a.N = c.fft_points;
   a.S = h->S;
   a.levels = level_table(c.layout[0].format, nbit);
   a.status = (int *)h->d_status.p;
   const bool tc = c.precision != SWSGPU_PREC_FP32;
   BigRowsKernel rows = tc ? bp.rows_tc : bp.rows;
   const int TB = tc ? bp.TBtc : bp.TB;
   const size_t smem_rows = tc ? bp.smem_rows_tc : bp.smem_rows;
   if (!rows) return fail(h, SWSGPU_EINVAL, "split has no tensor-core row pass");
   if (h->rows_fn != (const void *)rows || h->cols_fn != (const void *)bp.cols[nbi]) {
      // persistent passes: as many CTAs as fit on the device at once (the
      // tensor-core row pass holds 144 KB of shared memory: one per SM)
      int occ_r = 0, occ_c = 0, nsm = 0;
      CK(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_r, rows, TB, smem_rows));
      CK(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, bp.cols[nbi], bp.TA, bp.smem_cols[nbi]));
      CK(h, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
      h->rows_grid = std::max(1, occ_r) * nsm;
      h->cols_grid = std::max(1, occ_c) * nsm;
      h->rows_fn = (const void *)rows;
      h->cols_fn = (const void *)bp.cols[nbi];
   }
   cudaEvent_t ev0 = nullptr, ev1 = nullptr;
   if (h->profiling) {
      CK(h, cudaEventCreate(&ev0));
      CK(h, cudaEventCreate(&ev1));
      CK(h, cudaEventRecord(ev0, st));
   }
   for (const int4 &b : se.batches) {
      a.jobs = (const BigJob *)se.d_bjobs.p + b.x;
      a.bitems = (const BigItem *)se.d_bitems.p + b.z;
      a.nbjobs = b.y;
      bp.cols[nbi]<<<(unsigned)std::min((bp.N2 / bp.C) * b.y, h->cols_grid), bp.TA, bp.smem_cols[nbi], st>>>(a);
      a.nbitems = b.w;
      const int units = (bp.N1 / 2 + 1) * b.w;
      rows<<<(unsigned)std::min(units, h->rows_grid), TB, smem_rows, st>>>(a);
      CK(h, cudaGetLastError());
      launches += 2;
   }
   if (h->profiling) {
      CK(h, cudaEventRecord(ev1, st));
      h->prof_events.push_back(std::make_pair(ev0, ev1));
   }
   return SWSGPU_OK;
}

static void drop_schedules(swsgpu_handle *h)
{
   for (SchedEntry *e : h->sched) {
      e->release();
      delete e;
   }
   h->sched.clear();
}

// The device-resident schedule of a run shape (built and uploaded once).
static int get_schedule(swsgpu_handle *h, size_t run_bytes, int nruns, int rpo, float *d_auto, float *d_xpol,
                        float *d_pcal, int acc_mode, SchedEntry **out)
{
   for (SchedEntry *e : h->sched)
      if (e->run_bytes == run_bytes && e->nruns == nruns && e->rpo == rpo && e->d_auto == d_auto &&
          e->d_xpol == d_xpol && e->d_pcal == d_pcal && e->acc_mode == acc_mode &&
          (acc_mode == 0 || e->acc_base == h->d_acc64.p)) {
         *out = e;
         return SWSGPU_OK;
      }
   if (h->sched.size() >= 8) drop_schedules(h);  // cudaFree waits for work that may still use them
   SchedEntry *e = new SchedEntry();
   e->run_bytes = run_bytes;
   e->nruns = nruns;
   e->rpo = rpo;
   e->d_auto = d_auto;
   e->d_xpol = d_xpol;
   e->d_pcal = d_pcal;
   e->acc_mode = acc_mode;
   Schedule &sc = e->sc;
   build_schedule(h, run_bytes, nruns, rpo, d_auto, d_xpol, d_pcal, sc);
   auto bail = [&](cudaError_t err, const char *what) {
      e->release();
      delete e;
      return fail(h, SWSGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(err));
   };
   if (acc_mode != 0) {
      const size_t need = sizeof(double) * (size_t)h->S * (sc.outs.size() + 1);
      if (need > h->d_acc64.n) {
         // the running sums move: schedules pointing at the old ones go
         std::vector<SchedEntry *> keep;
         for (SchedEntry *o : h->sched) {
            if (o->acc_mode != 0) {
               o->release();
               delete o;
            } else {
               keep.push_back(o);
            }
         }
         h->sched = keep;
         cudaError_t err = h->d_acc64.ensure(need);
         if (err != cudaSuccess) return bail(err, "accumulator allocation");
      }
      e->acc_base = h->d_acc64.p;
      for (size_t i = 0; i < sc.outs.size(); i++) {
         sc.outs[i].acc = (double *)h->d_acc64.p + i * (size_t)h->S;
         sc.outs[i].acc_mode = acc_mode;
      }
   } else {
      for (auto &o : sc.outs) {
         o.acc = nullptr;
         o.acc_mode = 0;
      }
   }
   auto upload = [&](DevBuf &d, const void *src, size_t bytes) {
      if (bytes == 0) return cudaSuccess;
      cudaError_t err = d.ensure(bytes);
      if (err != cudaSuccess) return err;
      return cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice);
   };
   cudaError_t err;
   {
      // word-wise phase-cal fold: periods and job starts on code-word boundaries
      const long long unit = (long long)(32 / h->cfg.layout[0].nbit) * (h->big ? 1 : h->plan.P);
      bool ok = h->cfg.extract_pcal && h->cfg.pcal_rotatorlen % unit == 0;
      for (const PcalJob &pj : sc.pcal_jobs) ok = ok && (pj.start % unit == 0);
      e->pcal_word_fold = ok ? 1 : 0;
   }
   if ((err = upload(e->d_items, sc.items.data(), sizeof(Item) * sc.items.size())) != cudaSuccess ||
       (err = upload(e->d_entries, sc.entries.data(), sizeof(RedEntry) * sc.entries.size())) != cudaSuccess ||
       (err = upload(e->d_outs, sc.outs.data(), sizeof(OutVec) * sc.outs.size())) != cudaSuccess ||
       (err = upload(e->d_pcal_jobs, sc.pcal_jobs.data(), sizeof(PcalJob) * sc.pcal_jobs.size())) != cudaSuccess ||
       (err = upload(e->d_cl_first, sc.cl_first.data(), sizeof(int) * sc.cl_first.size())) != cudaSuccess)
      return bail(err, "schedule upload");
   if (h->big) {
      std::vector<BigJob> jobs;
      std::vector<BigItem> bitems;
      big_batches(h, sc, jobs, bitems, e->batches);
      if ((err = upload(e->d_bjobs, jobs.data(), sizeof(BigJob) * jobs.size())) != cudaSuccess ||
          (err = upload(e->d_bitems, bitems.data(), sizeof(BigItem) * bitems.size())) != cudaSuccess)
         return bail(err, "four-step job upload");
   }
   h->sched.push_back(e);
   *out = e;
   return SWSGPU_OK;
}

// Phase decimation of the code arrays: the cluster size, or N2 on the
// four-step path (the column layout) when every stream's corner turn
// supports it (*col), else 1.
static int code_decimation(const swsgpu_handle *h, bool *col)
{
   const swsgpu_config &c = h->cfg;
   bool cl = h->big;
   for (int s = 0; s < c.num_streams && cl; s++)
      if (!h->chans_of[s].empty()) cl = unpack_decimation_ok(h->bplan.N2, c.layout[s].nchan, c.layout[s].nbit);
   *col = cl;
   return h->big ? (cl ? h->bplan.N2 : 1) : h->plan.P;
}

// ---------------------------------------------------------------------------
// pipeline launch for a chunk already in device memory
// ---------------------------------------------------------------------------
static int launch_chunk(swsgpu_handle *h, const void *const *d_raw, const size_t *raw_bytes,
                        const long long *grid_off, size_t run_bytes, int nruns,
                        int runs_per_output, float *d_auto, float *d_xpol, float *d_pcal,
                        cudaStream_t st, int *nspec_out, int acc_mode = 0, int pcal_zero = 1,
                        int pcal_write = 1, double *d_tones = nullptr, int set = 0,
                        cudaEvent_t after_k1 = nullptr, cudaEvent_t acc_wait = nullptr,
                        cudaEvent_t acc_rec = nullptr)
{
   // set: the scratch set (and so the stream) of this launch; after_k1:
   // recorded once K1 has read the raw bytes; acc_wait / acc_rec: ordering
   // of the reduction and phase-cal folds, which add into sums shared with
   // the chunks of the other stream
   const swsgpu_config &c = h->cfg;
   Scratch &x = h->scr[set];
   SchedEntry *se = nullptr;
   {
      int rc = get_schedule(h, run_bytes, nruns, runs_per_output, d_auto, d_xpol, d_pcal, acc_mode, &se);
      if (rc != SWSGPU_OK) return rc;
   }
   const Schedule &sc = se->sc;
   if (nspec_out) *nspec_out = sc.nspec_total;
   int launches = 0;
   const int S = h->S;
   const int ncode = (int)h->code_stream.size();
   const int nbit = c.layout[0].nbit;
   const int spw = 32 / nbit;
   const long long nsamp = sc.nsamp;
   bool col = false;
   const int D = code_decimation(h, &col);
   const long long per_phase = (nsamp + D - 1) / D;
   // +2: prefetch may touch one word past; a multiple of 4 words, so every
   // phase array starts on a 16-byte boundary (bulk copies of its runs)
   const long long wpp = ((per_phase + spw - 1) / spw + 2 + 3) / 4 * 4;
   const long long code_words = (long long)D * wpp;
   const long long blank_words = (nsamp + 31) / 32;
   // phase-cal folds read undecimated codes (word-wise when the rotator
   // period allows); with the column layout they get their own copy
   const bool pcal_copy = col && c.extract_pcal && d_pcal && !sc.pcal_jobs.empty();
   const long long wpp1 = (nsamp + spw - 1) / spw + 2;

   CK(h, x.d_codes.ensure(sizeof(uint32_t) * (size_t)code_words * ncode + 64));
   if (pcal_copy) CK(h, x.d_codes1.ensure(sizeof(uint32_t) * (size_t)wpp1 * ncode + 64));
   CK(h, x.d_blank.ensure(sizeof(uint32_t) * (size_t)blank_words * c.num_streams + 16));
   CK(h, x.d_blank_any.ensure(sizeof(int) * SWSGPU_MAX_STREAMS));
   // the blank bitmap is written by K1 and read by K2/PCal only for streams
   // with a blanked frame (blank_any), so it needs no clearing
   CK(h, cudaMemsetAsync(x.d_blank_any.p, 0, sizeof(int) * SWSGPU_MAX_STREAMS, st));

   // K1 per stream
   for (int s = 0; s < c.num_streams; s++) {
      const swsgpu_layout &L = c.layout[s];
      StreamIn si;
      si.data = (const uint8_t *)d_raw[s];
      si.nbytes = (long long)raw_bytes[s];
      si.grid_offset = grid_off[s];
      si.frame_bytes = L.frame_bytes;
      si.header_bytes = L.header_bytes;
      si.payload_bytes = payload_bytes(L);
      si.nchan = L.nchan;
      si.nbit = L.nbit;
      si.format = L.format;
      si.msb2 = is_msb2(L);
      set_zones(si);
      const long long last_v = si.grid_offset + ((nsamp * (long long)L.nchan * L.nbit - 1) >> 3);
      si.nframes = last_v / si.payload_bytes + 1;
      CK(h, x.d_valid[s].ensure(sizeof(int2) * (size_t)si.nframes * si.zpf));
      k_frame_valid<<<(unsigned)((si.nframes + 127) / 128), 128, 0, st>>>(
          si, (int2 *)x.d_valid[s].p, (int *)x.d_blank_any.p + s);
      launches++;
      if (track_format(L.format)) {
         // VLBA / Mark4 track-words into Mark5B's sample layout (same size
         // and grid; validity above was read from the track-words)
         CK(h, x.d_trk[s].ensure((raw_bytes[s] + 3) / 4 * 4 + 16));
         CK(h, launch_track_turn(st, (const uint8_t *)d_raw[s], (long long)raw_bytes[s], grid_off[s],
                                 payload_bytes(L) / 2500, L.format, (const uint32_t *)h->d_trk_table.p,
                                 (uint32_t *)x.d_trk[s].p));
         si.data = (const uint8_t *)x.d_trk[s].p;
         launches++;
      }
      const std::vector<int> &chans = h->chans_of[s];
      if (chans.empty()) continue;
      uint32_t *codes = (uint32_t *)x.d_codes.p + (size_t)h->first_code[s] * code_words;
      uint32_t *blank = (uint32_t *)x.d_blank.p + (size_t)s * blank_words;
      CK(h, launch_unpack_codes(st, si, nsamp, (const int *)h->d_chans[s].p, (int)chans.size(), codes, D, wpp,
                                (const int2 *)x.d_valid[s].p, (const int *)x.d_blank_any.p + s, blank, launches));
      if (pcal_copy)
         CK(h, launch_unpack_codes(st, si, nsamp, (const int *)h->d_chans[s].p, (int)chans.size(),
                                   (uint32_t *)x.d_codes1.p + (size_t)h->first_code[s] * wpp1, 1, wpp1,
                                   (const int2 *)x.d_valid[s].p, (const int *)x.d_blank_any.p + s, blank,
                                   launches));
   }
   CK(h, cudaGetLastError());
   if (after_k1) CK(h, cudaEventRecord(after_k1, st));

   // K2
   const int nitems = (int)sc.items.size();
   if (nitems > 0) {
      CK(h, x.d_partial.ensure(sizeof(float) * 4 * (size_t)S * nitems));
      if (h->big) {
         int rc = launch_big(h, *se, code_words, wpp, col, blank_words, x, st, launches);
         if (rc != SWSGPU_OK) return rc;
      } else {
         SpecArgs a;
         a.codes = (const uint32_t *)x.d_codes.p;
         a.code_words = code_words;
         a.wpp = wpp;
         a.D = D;
         a.blank = (const uint32_t *)x.d_blank.p;
         a.blank_words = blank_words;
         a.blank_any = (const int *)x.d_blank_any.p;
         a.code_stream = (const int *)h->d_code_stream.p;
         a.items = (const Item *)se->d_items.p;
         a.nitems = nitems;
         a.cl_first = sc.cl_first.empty() ? nullptr : (const int *)se->d_cl_first.p;
         a.window = (const float *)h->d_window.p;
         a.twQ = (const float2 *)h->d_twQ.p;
         a.twN = (const float2 *)h->d_twN.p;
         a.partial = (float *)x.d_partial.p;
         a.N = c.fft_points;
         a.S = S;
         a.levels = level_table(c.layout[0].format, nbit);
         a.status = (int *)h->d_status.p;
         a.drop_last_exchange = h->inject == SWSGPU_INJECT_DROP_EXCHANGE;
         h->inject = SWSGPU_INJECT_NONE;
         const Plan &pl = h->plan;
         const int nbi = nbit == 1 ? 0 : nbit == 2 ? 1 : 2;
         SpecKernel kern = plan_kernel(pl, c.precision, nbi);
         const int ncl = sc.cl_first.empty() ? std::max(1, std::min(nitems, h->max_clusters)) : sc.ncl;
         cudaLaunchConfig_t cfgl = {};
         cfgl.gridDim = dim3(ncl * pl.P);
         cfgl.blockDim = dim3(pl.T);
         cfgl.dynamicSmemBytes = plan_smem(pl, c.precision, nbi);
         cfgl.stream = st;
         cudaLaunchAttribute attr[2];
         cfgl.numAttrs = cluster_attrs(attr, pl.P, c.precision);
         cfgl.attrs = attr;
         cudaEvent_t ev0 = nullptr, ev1 = nullptr;
         if (h->profiling) {
            CK(h, cudaEventCreate(&ev0));
            CK(h, cudaEventCreate(&ev1));
            CK(h, cudaEventRecord(ev0, st));
         }
         CK(h, cudaLaunchKernelEx(&cfgl, kern, a));
         if (h->profiling) {
            CK(h, cudaEventRecord(ev1, st));
            h->prof_events.push_back(std::make_pair(ev0, ev1));
         }
         launches++;
      }
   }
   if (acc_wait) CK(h, cudaStreamWaitEvent(st, acc_wait, 0));
   if (nitems > 0) {
      // K3
      const int nouts = (int)sc.outs.size();
      if (nouts > 0) {
         dim3 grid((S + 255) / 256, nouts);
         k_reduce<<<grid, 256, 0, st>>>((const float *)x.d_partial.p, S,
                                         (const RedEntry *)se->d_entries.p, (const OutVec *)se->d_outs.p);
         launches++;
      }
   }
   // phase cal
   if (c.extract_pcal && d_pcal) {
      const int nout = sc.nspec_total * c.num_sources;
      if (pcal_write && sc.pcal_jobs.empty()) {
         CK(h, cudaMemsetAsync(d_pcal, 0, sizeof(float) * 2 * c.pcal_tonebins * (size_t)nout, st));
         if (d_tones && c.pcal_ntones > 0)
            CK(h, cudaMemsetAsync(d_tones, 0, sizeof(double) * 2 * c.pcal_ntones * (size_t)nout, st));
         launches++;
      }
      if (!sc.pcal_jobs.empty()) {
         // FP64 sums [nout][tonebins][2] followed by the samples folded per output
         CK(h, h->d_pcal_part.ensure(sizeof(double) * (2 * c.pcal_tonebins + 1) * (size_t)nout));
         int njobs = (int)sc.pcal_jobs.size();
         PcalArgs pa;
         pa.codes = (const uint32_t *)(pcal_copy ? x.d_codes1.p : x.d_codes.p);
         pa.code_words = pcal_copy ? wpp1 : code_words;
         pa.wpp = pcal_copy ? wpp1 : wpp;
         pa.D = pcal_copy ? 1 : D;
         pa.blank = (const uint32_t *)x.d_blank.p;
         pa.blank_words = blank_words;
         pa.blank_any = (const int *)x.d_blank_any.p;
         pa.code_stream = (const int *)h->d_code_stream.p;
         pa.jobs = (const PcalJob *)se->d_pcal_jobs.p;
         pa.njobs = njobs;
         pa.N = c.fft_points;
         pa.tonebins = c.pcal_tonebins;
         pa.rotatorlen = c.pcal_rotatorlen;
         pa.used = (c.pcal_rotatorlen / c.pcal_tonebins) * c.pcal_tonebins;
         pa.dphi = 2.0 * M_PI * (-c.pcal_offset_hz / c.samplingfreq);
         pa.levels = level_table(c.layout[0].format, nbit);
         pa.out = d_pcal;
         pa.acc = (double *)h->d_pcal_part.p;
         pa.tones = d_tones;
         pa.ntones = d_tones ? c.pcal_ntones : 0;
         pa.nout = nout;
         pa.zero_acc = pcal_zero;
         pa.write_out = pcal_write;
         pa.word_fold = se->pcal_word_fold;
         int rc = launch_pcal(pa, nbit, st);
         if (rc) return fail(h, SWSGPU_ECUDA, std::string("pcal launch: ") + cudaGetErrorString(cudaGetLastError()));
         launches += 2;
      }
   }
   if (acc_rec) CK(h, cudaEventRecord(acc_rec, st));
   CK(h, cudaGetLastError());
   h->last_launches = launches;
   return SWSGPU_OK;
}

static void drop_prof_events(swsgpu_handle *h)
{
   for (auto &pr : h->prof_events) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
   }
   h->prof_events.clear();
}

// Makes `stream` wait for every chunk launched so far (the last chunk's
// sums were added after all earlier chunks' sums).
static int join_chunks(swsgpu_handle *h)
{
   if (h->acc_pending) {
      CK(h, cudaStreamWaitEvent(h->stream, h->acc_done, 0));
      h->acc_pending = false;
   }
   return SWSGPU_OK;
}

// Launches the open chunk of collected runs as one multi-run chunk whose
// spectra are summed into the group's FP64 running sums (group_end: and
// written out).
static int flush_chunk(swsgpu_handle *h, bool group_end, int *nspec)
{
   const swsgpu_config &c = h->cfg;
   if (h->chunk_n == 0) return SWSGPU_OK;
   const int region = h->chunk_region;
   const void *d_raw[SWSGPU_MAX_STREAMS];
   size_t raw_bytes[SWSGPU_MAX_STREAMS];
   long long grid_off[SWSGPU_MAX_STREAMS];
   for (int s = 0; s < c.num_streams; s++) {
      d_raw[s] = h->d_region[region][s].p;
      raw_bytes[s] = h->chunk_run_bytes * (size_t)h->chunk_n;
      grid_off[s] = h->chunk_off0[s] % payload_bytes(c.layout[s]);
   }
   const bool first = h->chunk_group_first;
   const int acc_mode = group_end ? (first ? 0 : 3) : (first ? 1 : 2);
   // cluster path: region 1's chunks run on the second stream with the
   // second scratch set; the four-step path shares its intermediate buffer
   // between launches and keeps one stream
   const int set = (!h->big && h->stream2 && region == 1) ? 1 : 0;
   cudaStream_t st = set ? h->stream2 : h->stream;
   CK(h, cudaStreamWaitEvent(st, h->last_h2d, 0));
   // the region is free for the next copies once K1 has decoded it
   const int rc = launch_chunk(h, d_raw, raw_bytes, grid_off, h->chunk_run_bytes, h->chunk_n, h->chunk_n,
                               (float *)h->d_out_auto.p, c.num_xpols ? (float *)h->d_out_xpol.p : nullptr,
                               c.extract_pcal ? (float *)h->d_out_pcal.p : nullptr, st, nspec, acc_mode,
                               first ? 1 : 0, group_end ? 1 : 0,
                               h->h_tones_bytes ? (double *)h->d_out_tones.p : nullptr, set,
                               h->region_free[region], h->acc_done, h->acc_done);
   if (rc) return rc;
   h->acc_pending = true;
   h->chunk_region ^= 1;
   h->chunk_n = 0;
   h->chunk_group_first = false;
   return SWSGPU_OK;
}

static int autotune_big(swsgpu_handle *h, int iters);
static int autotune_cluster(swsgpu_handle *h, int iters);

// Makes `pl` the handle's cluster plan: its per-CTA twiddle table W_Q, the
// launch attributes of its kernel and the number of co-resident clusters
// (the grid of every launch).  Kept schedules depend on the plan's cluster
// size and grid, so they are dropped.
static int set_cluster_plan(swsgpu_handle *h, const Plan &pl)
{
   const swsgpu_config &c = h->cfg;
   const int nbit = c.layout[0].nbit;
   const int nbi = nbit == 1 ? 0 : nbit == 2 ? 1 : 2;
   const SpecKernel kern = plan_kernel(pl, c.precision, nbi);
   if (!kern) return fail(h, SWSGPU_EINVAL, "the plan has no kernel of this form");
   const size_t smem = plan_smem(pl, c.precision, nbi);
   std::vector<float2> twQ;
   make_twiddles(pl.Q, pl.Q, twQ);
   CK(h, cudaStreamSynchronize(h->stream));
   CK(h, h->d_twQ.ensure(sizeof(float2) * twQ.size()));
   CK(h, cudaMemcpy(h->d_twQ.p, twQ.data(), sizeof(float2) * twQ.size(), cudaMemcpyHostToDevice));
   CK(h, cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
   if (pl.P > 8) CK(h, cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
   cudaLaunchConfig_t cfgl = {};
   cfgl.gridDim = dim3(pl.P);
   cfgl.blockDim = dim3(pl.T);
   cfgl.dynamicSmemBytes = smem;
   cudaLaunchAttribute attr[2];
   cfgl.numAttrs = cluster_attrs(attr, pl.P, c.precision);
   cfgl.attrs = attr;
   // The occupancy query reports one resident CTA per SM for any kernel
   // that allocates tensor memory, whatever its footprint; two 113 KB
   // tensor-core CTAs (128 TMEM columns each, 512 per SM) do co-reside,
   // and a grid sized for one CTA per SM runs at 0.69x the speed of one
   // sized for two.  So the grid of a tensor-core form is sized by the
   // FP32 form's kernel of the same plan (same threads and register cap)
   // at the tensor-core form's shared-memory footprint.
   const void *occ_kern = (const void *)kern;
   if (c.precision != SWSGPU_PREC_FP32) {
      occ_kern = (const void *)pl.kern[nbi];
      CK(h, cudaFuncSetAttribute(occ_kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      if (pl.P > 8) CK(h, cudaFuncSetAttribute(occ_kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
   }
   int ncl = 0;
   CK(h, cudaOccupancyMaxActiveClusters(&ncl, occ_kern, &cfgl));
   if (ncl < 1) return fail(h, SWSGPU_ECUDA, "cluster configuration does not fit on this device");
   h->max_clusters = ncl;
   h->plan = pl;
   drop_schedules(h);
   return SWSGPU_OK;
}
static cudaError_t set_big_attrs(const swsgpu_handle *h, const BigPlan &bp);
static std::mutex &tune_mutex();
static int tuned_choice(int N, int nbit, bool tc, bool big);

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int swsgpu_version(void) { return 10000; }

int swsgpu_device_ok(int device)
{
   cudaDeviceProp p;
   if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return 0;
   return p.major >= 10 ? 1 : 0;
}

const char *swsgpu_last_error(const swsgpu_handle *h)
{
   return h ? h->err.c_str() : g_create_error.c_str();
}

static int validate_config(const swsgpu_config *c, std::string &why)
{
   if (c->num_streams < 1 || c->num_streams > SWSGPU_MAX_STREAMS) { why = "num_streams must be 1 or 2"; return 0; }
   for (int s = 0; s < c->num_streams; s++) {
      const swsgpu_layout &l = c->layout[s];
      if (l.nbit != 1 && l.nbit != 2 && l.nbit != 8) { why = "nbit must be 1, 2 or 8"; return 0; }
      if (l.nchan < 1 || l.nchan * l.nbit > 64) { why = "nchan*nbit must be 1..64"; return 0; }
      if (l.format < SWSGPU_FMT_MARK5B || l.format > SWSGPU_FMT_MARK4) { why = "unknown format"; return 0; }
      if (track_format(l.format) && !track_layout_ok(l, why)) return 0;
      if (l.format == SWSGPU_FMT_RAW_SIGNED || l.format == SWSGPU_FMT_RAW_UNSIGNED) {
         // the reference's raw unpackers (DataUnpackerFactory.h:44-67)
         if (l.nbit == 1) { why = "raw formats have no 1-bit unpacker"; return 0; }
         if (l.nbit == 2 && !(l.nchan == 1 || l.nchan % 4 == 0)) {
            why = "raw 2-bit data needs one channel or a multiple of 4";
            return 0;
         }
      }
      if (l.header_bytes < 0 || l.frame_bytes <= l.header_bytes) { why = "bad frame layout"; return 0; }
      if ((l.frame_bytes % 8) || (l.header_bytes % 4) || ((l.frame_bytes - l.header_bytes) % 8)) {
         why = "frame, header and payload sizes must be multiples of 8, 4 and 8 bytes";
         return 0;
      }
      if (l.nbit != c->layout[0].nbit || l.nchan != c->layout[0].nchan || l.format != c->layout[0].format) {
         why = "all streams must share format, channels and bits (as in the reference's settings)";
         return 0;
      }
   }
   if (c->overlap < 1 || c->fft_points % c->overlap) { why = "overlap must divide fft_points"; return 0; }
   if (c->core_overlapped_ffts < 1) { why = "core_overlapped_ffts must be >= 1"; return 0; }
   if (c->num_sources < 1 || c->num_sources > SWSGPU_MAX_SOURCES) { why = "num_sources out of range"; return 0; }
   for (int s = 0; s < c->num_sources; s++) {
      if (c->source_stream[s] < 0 || c->source_stream[s] >= c->num_streams) { why = "source_stream out of range"; return 0; }
      if (c->source_channel[s] < 0 || c->source_channel[s] >= c->layout[c->source_stream[s]].nchan) {
         why = "source_channel out of range";
         return 0;
      }
   }
   if (c->num_xpols < 0 || c->num_xpols > SWSGPU_MAX_SOURCES) { why = "num_xpols out of range"; return 0; }
   for (int x = 0; x < c->num_xpols; x++)
      for (int k = 0; k < 2; k++)
         if (c->xpol_pair[x][k] < 0 || c->xpol_pair[x][k] >= c->num_sources) { why = "xpol_pair out of range"; return 0; }
   if (c->window < 0 || c->window > SWSGPU_WIN_BLACKMANHARRIS) { why = "unknown window"; return 0; }
   if (c->precision != SWSGPU_PREC_FP32 && c->precision != SWSGPU_PREC_TCSPLIT &&
       c->precision != SWSGPU_PREC_TCSPLIT_ALL) {
      why = "unknown precision";
      return 0;
   }
   if (c->runs_per_output < 0) { why = "runs_per_output must be >= 0"; return 0; }
   if (c->plan_family < SWSGPU_PLAN_DEFAULT || c->plan_family > SWSGPU_PLAN_FOURSTEP) { why = "unknown plan_family"; return 0; }
   if (c->plan_candidate < 0) { why = "plan_candidate must be >= 0"; return 0; }
   if (c->extract_pcal) {
      if (c->pcal_tonebins < 1 || c->pcal_rotatorlen < c->pcal_tonebins || c->fft_points % c->pcal_rotatorlen) {
         why = "pcal: need tonebins >= 1, rotatorlen >= tonebins and N % rotatorlen == 0";
         return 0;
      }
      if (c->pcal_tonebins > 4096) { why = "pcal_tonebins > 4096"; return 0; }
      if (c->pcal_ntones < 0 || c->pcal_ntones > c->pcal_tonebins / 2) {
         why = "pcal_ntones must be 0..pcal_tonebins/2";
         return 0;
      }
   } else if (c->pcal_ntones != 0) {
      why = "pcal_ntones needs extract_pcal";
      return 0;
   }
   return 1;
}

int swsgpu_create(const swsgpu_config *cfg, int device, swsgpu_handle **out)
{
   if (!cfg || !out) return fail(nullptr, SWSGPU_EINVAL, "null argument");
   *out = nullptr;
   std::string why;
   if (!validate_config(cfg, why)) return fail(nullptr, SWSGPU_EINVAL, why);
   Plan plan = {};
   BigPlan bplan = {};
   bool cluster_plan = find_plan(cfg->fft_points, &plan);
   const bool four_step = find_big_plan(cfg->fft_points, &bplan);
   if (cfg->plan_family == SWSGPU_PLAN_FOURSTEP) {
      if (!four_step)
         return fail(nullptr, SWSGPU_EINVAL, "fft_points " + std::to_string(cfg->fft_points) + " has no four-step plan");
      cluster_plan = false;
   } else if (cfg->plan_family == SWSGPU_PLAN_CLUSTER && !cluster_plan) {
      return fail(nullptr, SWSGPU_EINVAL, "fft_points " + std::to_string(cfg->fft_points) + " has no cluster plan");
   }
   if (!cluster_plan && !four_step)
      return fail(nullptr, SWSGPU_EINVAL, "fft_points " + std::to_string(cfg->fft_points) + " has no GPU plan");
   if (cfg->precision != SWSGPU_PREC_FP32) {
      // cluster lengths: the plan's tensor-core kernels; four-step lengths:
      // a split with 4096-point rows (the tensor-core row pass)
      bool tc_ok = cluster_plan && plan.kern_tc[1];
      if (!cluster_plan && four_step) {
         BigPlan cand[16];
         const int nc = big_plan_candidates(cfg->fft_points, cand, 16);
         for (int k = 0; k < nc; k++) tc_ok = tc_ok || cand[k].rows_tc;
      }
      if (!tc_ok)
         return fail(nullptr, SWSGPU_EINVAL,
                     "tensor-core split form not available for fft_points " + std::to_string(cfg->fft_points));
   }
   int ndev = 0;
   if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
      return fail(nullptr, SWSGPU_ENODEV, "no CUDA device " + std::to_string(device));
   if (!swsgpu_device_ok(device)) return fail(nullptr, SWSGPU_ENODEV, "device is not sm_100 class");
   if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, SWSGPU_ENODEV, "cudaSetDevice failed");

   swsgpu_handle *h = new swsgpu_handle();
   h->cfg = *cfg;
   h->device = device;
   h->plan = plan;
   h->big = !cluster_plan;
   h->bplan = bplan;
   h->S = cfg->fft_points / 2 + 1;
   auto bail = [&](int rc) {
      std::string e = h->err;
      swsgpu_destroy(h);
      g_create_error = e;
      return rc;
   };
   // code arrays
   std::map<std::pair<int, int>, int> code_of;
   for (int s = 0; s < cfg->num_sources; s++) {
      auto key = std::make_pair(cfg->source_stream[s], cfg->source_channel[s]);
      if (!code_of.count(key)) {
         code_of[key] = (int)h->code_stream.size();
         h->code_stream.push_back(key.first);
         h->code_chan.push_back(key.second);
      }
      h->src_code.push_back(code_of[key]);
   }
   // reorder code arrays so each stream's are contiguous (K1 writes per stream)
   {
      std::vector<int> order;
      for (int st = 0; st < cfg->num_streams; st++)
         for (int k = 0; k < (int)h->code_stream.size(); k++)
            if (h->code_stream[k] == st) order.push_back(k);
      std::vector<int> inv(order.size()), cs, cc;
      for (int i = 0; i < (int)order.size(); i++) {
         inv[order[i]] = i;
         cs.push_back(h->code_stream[order[i]]);
         cc.push_back(h->code_chan[order[i]]);
      }
      h->code_stream = cs;
      h->code_chan = cc;
      for (auto &x : h->src_code) x = inv[x];
   }
   for (int s = 0; s < cfg->num_streams; s++) {
      for (int k = 0; k < (int)h->code_stream.size(); k++)
         if (h->code_stream[k] == s) {
            if (h->first_code[s] < 0) h->first_code[s] = k;
            h->chans_of[s].push_back(h->code_chan[k]);
         }
   }
   h->auto_owner.assign(cfg->num_sources, -1);
   for (int x = 0; x < cfg->num_xpols; x++)
      for (int k = 0; k < 2; k++)
         if (h->auto_owner[cfg->xpol_pair[x][k]] < 0) h->auto_owner[cfg->xpol_pair[x][k]] = x;
   // a pair (i, i) cannot own both autos twice; treat it as owning source i once
   bool ev_ok = cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking) == cudaSuccess;
   for (int k = 0; k < 2 && ev_ok; k++)
      ev_ok = cudaEventCreateWithFlags(&h->slot_h2d[k], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&h->slot_free[k], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&h->region_free[k], cudaEventDisableTiming) == cudaSuccess;
   h->chunk_max = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(1, cfg->runs_per_output),
                                                            ((size_t)32 << 20) / std::max<size_t>(1, cfg->max_run_bytes)));
   if (!ev_ok || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
       cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->acc_done, cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&h->done, cudaEventDisableTiming) != cudaSuccess) {
      h->err = "stream/event creation failed";
      return bail(SWSGPU_ECUDA);
   }
   std::vector<float> win;
   make_window(cfg->window, cfg->fft_points, win);
   std::vector<float2> twN;
   if (!h->big) make_twiddles(cfg->fft_points, cfg->fft_points / 2 + 1, twN);
#define CKB(call)                                                                                  \
   do {                                                                                           \
      cudaError_t e_ = (call);                                                                    \
      if (e_ != cudaSuccess) {                                                                    \
         h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                             \
         return bail(SWSGPU_ECUDA);                                                               \
      }                                                                                           \
   } while (0)
   CKB(h->d_window.ensure(sizeof(float) * win.size()));
   CKB(cudaMemcpy(h->d_window.p, win.data(), sizeof(float) * win.size(), cudaMemcpyHostToDevice));
   if (track_format(cfg->layout[0].format)) {
      // the track turn's unit-byte tables (every stream shares the mode)
      const swsgpu_layout &L = cfg->layout[0];
      std::vector<uint32_t> tab(TRACK_TABLE_WORDS);
      track_turn_table(L.frame_bytes / 2500, L.nbit, L.nchan, tab.data());
      CKB(h->d_trk_table.ensure(sizeof(uint32_t) * tab.size()));
      CKB(cudaMemcpy(h->d_trk_table.p, tab.data(), sizeof(uint32_t) * tab.size(), cudaMemcpyHostToDevice));
   }
   if (!h->big) {
      CKB(h->d_twN.ensure(sizeof(float2) * twN.size()));
      CKB(cudaMemcpy(h->d_twN.p, twN.data(), sizeof(float2) * twN.size(), cudaMemcpyHostToDevice));
   } else {
      // four-step tables, each entry rounded once from double: W_N1 and
      // W_N2 of every candidate split (one buffer), W_N^(2048 h), W_N^l
      std::vector<float2> t1;
      {
         BigPlan cand[16];
         const int nc = big_plan_candidates(cfg->fft_points, cand, 16);
         for (int k = 0; k < nc; k++) {
            std::vector<float2> a1, a2;
            make_twiddles(cand[k].N1, cand[k].N1, a1);
            make_twiddles(cand[k].N2, cand[k].N2, a2);
            h->tw_off.push_back(make_int2((int)t1.size(), (int)(t1.size() + a1.size())));
            t1.insert(t1.end(), a1.begin(), a1.end());
            t1.insert(t1.end(), a2.begin(), a2.end());
         }
      }
      // the four-step twiddle W_N^m = W_N^(2048 h) W_N^l from two FP64 tables
      std::vector<double2> dA, dB(2048);
      for (int l = 0; l < 2048; l++) {
         const double ang = -2.0 * M_PI * (double)l / (double)cfg->fft_points;
         dB[l] = make_double2(std::cos(ang), std::sin(ang));
      }
      const int nA = (cfg->fft_points + 2047) / 2048;
      dA.resize(nA);
      for (int k = 0; k < nA; k++) {
         const double ang = -2.0 * M_PI * (double)((long long)k * 2048) / (double)cfg->fft_points;
         dA[k] = make_double2(std::cos(ang), std::sin(ang));
      }
      CKB(h->d_tw1.ensure(sizeof(float2) * t1.size()));
      CKB(cudaMemcpy(h->d_tw1.p, t1.data(), sizeof(float2) * t1.size(), cudaMemcpyHostToDevice));
      const std::pair<DevBuf *, std::vector<double2> *> tabs[2] = {{&h->d_twA, &dA}, {&h->d_twB, &dB}};
      for (const auto &t : tabs) {
         CKB(t.first->ensure(sizeof(double2) * t.second->size()));
         CKB(cudaMemcpy(t.first->p, t.second->data(), sizeof(double2) * t.second->size(), cudaMemcpyHostToDevice));
      }
   }
   for (int s = 0; s < cfg->num_streams; s++) {
      if (h->chans_of[s].empty()) continue;
      CKB(h->d_chans[s].ensure(sizeof(int) * h->chans_of[s].size()));
      CKB(cudaMemcpy(h->d_chans[s].p, h->chans_of[s].data(), sizeof(int) * h->chans_of[s].size(),
                     cudaMemcpyHostToDevice));
   }
   CKB(h->d_status.ensure(sizeof(int)));
   CKB(cudaMemset(h->d_status.p, 0, sizeof(int)));
   CKB(h->d_code_stream.ensure(sizeof(int) * h->code_stream.size()));
   CKB(cudaMemcpy(h->d_code_stream.p, h->code_stream.data(), sizeof(int) * h->code_stream.size(),
                  cudaMemcpyHostToDevice));
   // kernel attributes and cluster occupancy
   const int nbit = cfg->layout[0].nbit;
   const int nbi = nbit == 1 ? 0 : nbit == 2 ? 1 : 2;
   if (h->big) {
      {
         BigPlan cand[16];
         h->big_cands = big_plan_candidates(cfg->fft_points, cand, 16);
         // a split tuned earlier in this process for the same length, bits and form
         const bool tc = cfg->precision != SWSGPU_PREC_FP32;
         const int t = tuned_choice(cfg->fft_points, nbit, tc, true);
         if (tc) {
            // the tensor-core form runs only splits with 4096-point rows
            for (int k = 0; k < h->big_cands; k++)
               if (cand[k].rows_tc) {
                  h->bplan = cand[k];
                  h->cand = k;
                  break;
               }
         }
         if (cfg->plan_candidate > 0 && !cfg->autotune) {
            if (cfg->plan_candidate >= h->big_cands) {
               h->err = "plan_candidate beyond the candidates of this length";
               return bail(SWSGPU_EINVAL);
            }
            if (tc && !cand[cfg->plan_candidate].rows_tc) {
               h->err = "plan_candidate has no tensor-core row pass (rows of 4096 points)";
               return bail(SWSGPU_EINVAL);
            }
            h->bplan = cand[cfg->plan_candidate];
            h->cand = cfg->plan_candidate;
         } else if (t >= 0 && t < h->big_cands) {
            h->bplan = cand[t];
            h->tuned = t;
            h->cand = t;
         }
      }
      CKB(set_big_attrs(h, h->bplan));
      for (int k = 0; k < 2; k++)
         for (int s = 0; s < cfg->num_streams; s++)
            CKB(h->d_slot[k][s].ensure(cfg->max_run_bytes + (cfg->max_run_bytes / 8) + 1024 + 128));
      if (cfg->autotune && h->tuned < 0) {
         const int rc = autotune_big(h, 3);
         if (rc != SWSGPU_OK) return bail(rc);
      }
      *out = h;
      return SWSGPU_OK;
   }
   {
      // the default plan, a candidate asked for, or the one the autotuner
      // chose earlier in this process for this length, bit depth and form
      Plan cand[8];
      const int nc = plan_candidates(cfg->fft_points, cand, 8);
      const bool tc = cfg->precision != SWSGPU_PREC_FP32;
      int pick = 0;
      if (cfg->plan_candidate > 0 && !cfg->autotune) {
         if (cfg->plan_candidate >= nc) {
            h->err = "plan_candidate beyond the candidates of this length";
            return bail(SWSGPU_EINVAL);
         }
         if (!plan_kernel(cand[cfg->plan_candidate], cfg->precision, nbi)) {
            h->err = "plan_candidate has no kernel of this form";
            return bail(SWSGPU_EINVAL);
         }
         pick = cfg->plan_candidate;
      } else {
         const int t = tuned_choice(cfg->fft_points, nbit, tc, false);
         if (t >= 0 && t < nc && plan_kernel(cand[t], cfg->precision, nbi)) {
            pick = t;
            h->tuned = t;
         }
      }
      h->cand = pick;
      const int rc = set_cluster_plan(h, cand[pick]);
      if (rc != SWSGPU_OK) return bail(rc);
   }
   // device buffers for submit()
   for (int k = 0; k < 2; k++)
      for (int s = 0; s < cfg->num_streams; s++) CKB(h->d_slot[k][s].ensure(cfg->max_run_bytes + (cfg->max_run_bytes / 8) + 1024 + 128));
#undef CKB
   if (cfg->autotune && h->tuned < 0) {
      const int rc = autotune_cluster(h, 3);
      if (rc != SWSGPU_OK) return bail(rc);
   }
   *out = h;
   return SWSGPU_OK;
}

void swsgpu_destroy(swsgpu_handle *h)
{
   if (!h) return;
   cudaSetDevice(h->device);
   if (h->stream) cudaStreamSynchronize(h->stream);
   if (h->stream2) cudaStreamSynchronize(h->stream2);
   DevBuf *bufs[] = {&h->d_window, &h->d_twQ, &h->d_twN, &h->d_code_stream, &h->d_items, &h->d_entries,
                     &h->d_outs, &h->d_pcal_jobs, &h->d_pcal_part, &h->d_pcal_entries,
                     &h->d_pcal_outs, &h->d_out_auto, &h->d_out_xpol, &h->d_out_pcal, &h->d_out_tones,
                     &h->d_tw1, &h->d_tw2, &h->d_twA, &h->d_twB, &h->d_scratch, &h->d_bjobs, &h->d_status,
                     &h->d_bitems, &h->d_trk_table};
   for (DevBuf *b : bufs) b->release();
   for (Scratch &x : h->scr) x.release();
   drop_schedules(h);
   if (h->cstream) cudaStreamSynchronize(h->cstream);
   for (int k = 0; k < 2; k++) {
      for (int s = 0; s < SWSGPU_MAX_STREAMS; s++) h->d_slot[k][s].release();
      if (h->slot_h2d[k]) cudaEventDestroy(h->slot_h2d[k]);
      if (h->slot_free[k]) cudaEventDestroy(h->slot_free[k]);
      if (h->region_free[k]) cudaEventDestroy(h->region_free[k]);
      for (int s = 0; s < SWSGPU_MAX_STREAMS; s++) h->d_region[k][s].release();
   }
   for (int s = 0; s < SWSGPU_MAX_STREAMS; s++) {
      h->d_raw[s].release();
      h->d_chans[s].release();
   }
   h->h_out.release();
   h->d_acc64.release();
   drop_prof_events(h);
   if (h->done) cudaEventDestroy(h->done);
   if (h->acc_done) cudaEventDestroy(h->acc_done);
   if (h->stream) cudaStreamDestroy(h->stream);
   if (h->stream2) cudaStreamDestroy(h->stream2);
   if (h->cstream) cudaStreamDestroy(h->cstream);
   delete h;
}

int swsgpu_run_shape(const swsgpu_handle *h, size_t nbytes, int *nspectra, int *nffts, int *partial)
{
   if (!h) return SWSGPU_EINVAL;
   RunShape rs = run_shape(h->cfg, samples_of(h->cfg.layout[0], nbytes));
   if (nspectra) *nspectra = rs.nspec;
   if (nffts) *nffts = (int)rs.starts.size();
   if (partial) *partial = rs.partial ? 1 : 0;
   return SWSGPU_OK;
}

// True when host pointer p is page-locked memory the GPU can copy into
// asynchronously.
static bool host_pinned(const void *p)
{
   cudaPointerAttributes at;
   if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
      cudaGetLastError();
      return false;
   }
   return at.type == cudaMemoryTypeHost;
}

static int submit_impl(swsgpu_handle *h, const void *const *raw, const size_t *nbytes,
                       const int64_t *stream_payload_offset, const swsgpu_outputs *dest)
{
   if (!h || !raw || !nbytes) return SWSGPU_EINVAL;
   if (h->pending && h->pending_out)
      return fail(h, SWSGPU_ESTATE, "submit while a run's spectra are pending (wait and fetch first)");
   const swsgpu_config &c = h->cfg;
   CK(h, cudaSetDevice(h->device));
   // payload bytes per stream: the reference walks min over sources
   size_t payload_min = (size_t)-1;
   long long grid_off[SWSGPU_MAX_STREAMS];
   long long offs[SWSGPU_MAX_STREAMS];
   bool framed = false, equal = true;
   for (int s = 0; s < c.num_streams; s++) {
      const swsgpu_layout &L = c.layout[s];
      const int pb = payload_bytes(L);
      offs[s] = stream_payload_offset ? (long long)stream_payload_offset[s] : 0;
      long long off = offs[s] % pb;
      if (off % 4) return fail(h, SWSGPU_EINVAL, "payload offset must be a multiple of 4 bytes");
      size_t pay;
      if (L.header_bytes == 0) {
         pay = nbytes[s];
         grid_off[s] = off;
      } else {
         if (off != 0) return fail(h, SWSGPU_EINVAL, "framed input must start on a frame");
         size_t nfr = nbytes[s] / L.frame_bytes;
         size_t rem = nbytes[s] - nfr * L.frame_bytes;
         pay = nfr * pb + (rem > (size_t)L.header_bytes ? rem - L.header_bytes : 0);
         grid_off[s] = 0;
         framed = true;
      }
      if (nbytes[s] > c.max_run_bytes + (size_t)c.max_run_bytes / 8 + 1024 + 64)
         return fail(h, SWSGPU_EINVAL, "buffer larger than max_run_bytes");
      if (nbytes[s] != nbytes[0]) equal = false;
      payload_min = std::min(payload_min, pay);
   }
   RunShape rs = run_shape(c, samples_of(c.layout[0], payload_min));
   const int S = h->S;
   const int nsp = std::max(rs.nspec, 0);
   h->h_auto_bytes = sizeof(float) * (size_t)nsp * c.num_sources * S;
   h->h_xpol_bytes = sizeof(float) * 2 * (size_t)nsp * c.num_xpols * S;
   h->h_pcal_bytes = c.extract_pcal ? sizeof(float) * 2 * (size_t)nsp * c.num_sources * c.pcal_tonebins : 0;
   h->h_tones_bytes = (c.extract_pcal && c.pcal_ntones > 0)
                          ? sizeof(double) * 2 * (size_t)nsp * c.num_sources * c.pcal_ntones : 0;
   CK(h, h->d_out_auto.ensure(h->h_auto_bytes + 16));
   CK(h, h->d_out_xpol.ensure(h->h_xpol_bytes + 16));
   CK(h, h->d_out_pcal.ensure(h->h_pcal_bytes + 16));
   CK(h, h->d_out_tones.ensure(h->h_tones_bytes + 16));
   CK(h, h->h_out.ensure(h->h_auto_bytes + h->h_xpol_bytes + h->h_pcal_bytes + h->h_tones_bytes + 64));
   int nspec = 0;
   const int rpo = std::max(1, c.runs_per_output);
   bool group_end = true;
   int acc_mode = 0, pcal_zero = 1, pcal_write = 1;
   if (rpo > 1) {
      if (rs.nspec != 1 || rs.partial)
         return fail(h, SWSGPU_EINVAL, "runs_per_output > 1 needs runs of exactly one full spectrum");
      const bool first = h->group_pos == 0;
      group_end = h->group_pos == rpo - 1;
      acc_mode = group_end ? 3 : (first ? 1 : 2);
      if (first && group_end) acc_mode = 0;
      pcal_zero = first ? 1 : 0;
      pcal_write = group_end ? 1 : 0;
   }
   // collect the runs of a group into device chunks when they continue the
   // recording (equal header-free buffers at consecutive payload offsets)
   const bool chunkable = rpo > 1 && h->chunk_max > 1 && !framed && equal && nsp == 1;
   bool continues = chunkable && h->chunk_n > 0 && nbytes[0] == h->chunk_run_bytes;
   for (int s = 0; continues && s < c.num_streams; s++)
      if (offs[s] != h->chunk_off0[s] + (long long)h->chunk_n * (long long)h->chunk_run_bytes) continues = false;
   if (h->chunk_n > 0 && !continues) {
      int ns = 0;
      const int rc = flush_chunk(h, false, &ns);
      if (rc) return rc;
   }
   if (chunkable) {
      const int region = h->chunk_region;
      if (h->chunk_n == 0) {
         for (int k = 0; k < 2; k++)
            for (int s = 0; s < c.num_streams; s++)
               CK(h, h->d_region[k][s].ensure((size_t)h->chunk_max * c.max_run_bytes + 64));
         CK(h, cudaStreamWaitEvent(h->cstream, h->region_free[region], 0));
         for (int s = 0; s < c.num_streams; s++) h->chunk_off0[s] = offs[s];
         h->chunk_run_bytes = nbytes[0];
         h->chunk_group_first = h->group_pos == 0;
         // R runs left in the group: full chunks while R > 2 chunk_max,
         // then about half of what is left (8, 8, ..., 6, 3, 2, 1, 1)
         const int left = rpo - h->group_pos;
         h->chunk_target = left > 2 * h->chunk_max ? h->chunk_max
                                                   : std::max(1, std::min(h->chunk_max, left / 2));
      }
      for (int s = 0; s < c.num_streams; s++)
         CK(h, cudaMemcpyAsync((char *)h->d_region[region][s].p + (size_t)h->chunk_n * h->chunk_run_bytes, raw[s],
                               nbytes[s], cudaMemcpyHostToDevice, h->cstream));
      const int ev = h->next_slot;
      CK(h, cudaEventRecord(h->slot_h2d[ev], h->cstream));
      h->last_h2d = h->slot_h2d[ev];
      h->next_slot ^= 1;
      h->chunk_n++;
      h->group_pos = group_end ? 0 : h->group_pos + 1;
      if (h->chunk_n >= h->chunk_target || group_end) {
         const int rc = flush_chunk(h, group_end, &nspec);
         if (rc) return rc;
      } else {
         h->last_launches = 0;
      }
   } else {
      // one run per launch through the two input slots
      if (int rc = join_chunks(h)) return rc;
      const int slot = h->next_slot;
      CK(h, cudaStreamWaitEvent(h->cstream, h->slot_free[slot], 0));
      const void *d_raw[SWSGPU_MAX_STREAMS];
      size_t raw_bytes[SWSGPU_MAX_STREAMS];
      for (int s = 0; s < c.num_streams; s++) {
         CK(h, cudaMemcpyAsync(h->d_slot[slot][s].p, raw[s], nbytes[s], cudaMemcpyHostToDevice, h->cstream));
         raw_bytes[s] = nbytes[s];
         d_raw[s] = h->d_slot[slot][s].p;
      }
      CK(h, cudaEventRecord(h->slot_h2d[slot], h->cstream));
      CK(h, cudaStreamWaitEvent(h->stream, h->slot_h2d[slot], 0));
      h->last_h2d = h->slot_h2d[slot];
      h->next_slot ^= 1;
      if (nsp > 0) {
         int rc = launch_chunk(h, d_raw, raw_bytes, grid_off, payload_min, 1, 1, (float *)h->d_out_auto.p,
                               c.num_xpols ? (float *)h->d_out_xpol.p : nullptr,
                               c.extract_pcal ? (float *)h->d_out_pcal.p : nullptr, h->stream, &nspec,
                               acc_mode, pcal_zero, pcal_write,
                               h->h_tones_bytes ? (double *)h->d_out_tones.p : nullptr, 0, nullptr,
                               nullptr, h->acc_done);
         if (rc) return rc;
         if (rpo > 1) h->group_pos = group_end ? 0 : h->group_pos + 1;
      } else {
         h->last_launches = 0;
      }
      CK(h, cudaEventRecord(h->slot_free[slot], h->stream));
   }
   h->fetch_ready = group_end && !dest;
   h->delivered = false;
   for (void *&p : h->deliver_copy) p = nullptr;
   if (nsp > 0 && group_end) {
      if (int rc = join_chunks(h)) return rc;
      char *hp = (char *)h->h_out.p;
      // each output goes to pinned caller memory directly, else to the
      // staging buffer (copied to a pageable destination at wait, or kept
      // for swsgpu_fetch)
      void *const stage[4] = {hp, hp + h->h_auto_bytes, hp + h->h_auto_bytes + h->h_xpol_bytes,
                              hp + h->h_auto_bytes + h->h_xpol_bytes + h->h_pcal_bytes};
      const void *const src[4] = {h->d_out_auto.p, h->d_out_xpol.p, h->d_out_pcal.p, h->d_out_tones.p};
      const size_t bytes[4] = {h->h_auto_bytes, h->h_xpol_bytes, h->h_pcal_bytes, h->h_tones_bytes};
      void *const want[4] = {dest ? (void *)dest->auto_out : nullptr, dest ? (void *)dest->xpol_out : nullptr,
                             dest ? (void *)dest->pcal_out : nullptr, dest ? (void *)dest->tones_out : nullptr};
      for (int k = 0; k < 4; k++) {
         if (bytes[k] == 0 || (dest && !want[k])) continue;
         const bool direct = want[k] && host_pinned(want[k]);
         CK(h, cudaMemcpyAsync(direct ? want[k] : stage[k], src[k], bytes[k], cudaMemcpyDeviceToHost, h->stream));
         if (want[k] && !direct) h->deliver_copy[k] = want[k];
      }
      h->delivered = dest != nullptr;
   }
   CK(h, cudaEventRecord(h->done, h->stream));
   h->pending = true;
   h->pending_out = nsp > 0 && group_end;
   h->pending_nspec = group_end ? nspec : 0;
   return SWSGPU_OK;
}

int swsgpu_submit(swsgpu_handle *h, const void *const *raw, const size_t *nbytes,
                  const int64_t *stream_payload_offset)
{
   return submit_impl(h, raw, nbytes, stream_payload_offset, nullptr);
}

int swsgpu_submit_out(swsgpu_handle *h, const void *const *raw, const size_t *nbytes,
                      const int64_t *stream_payload_offset, const swsgpu_outputs *dest)
{
   if (!dest) return SWSGPU_EINVAL;
   return submit_impl(h, raw, nbytes, stream_payload_offset, dest);
}

int swsgpu_wait(swsgpu_handle *h, int timeout_ms, int *nspectra)
{
   if (!h) return SWSGPU_EINVAL;
   if (!h->pending) return fail(h, SWSGPU_ESTATE, "wait without a submitted run");
   CK(h, cudaSetDevice(h->device));
   // a run that completes no spectrum only has to release its input buffers
   cudaEvent_t ev = (h->pending_out || !h->last_h2d) ? h->done : h->last_h2d;
   auto t0 = std::chrono::steady_clock::now();
   while (true) {
      cudaError_t e = cudaEventQuery(ev);
      if (e == cudaSuccess) break;
      if (e != cudaErrorNotReady) {
         h->pending = false;
         return fail(h, SWSGPU_ECUDA, std::string("run failed: ") + cudaGetErrorString(e));
      }
      const auto us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
      if (timeout_ms >= 0 && us >= 1000ll * timeout_ms)
         return fail(h, SWSGPU_ETIMEOUT, "run not complete within timeout");
      // a run's copy or kernels finish within a few hundred microseconds:
      // poll tightly at first (a sleep costs a scheduler quantum per run),
      // then back off
      if (us < 2000) std::this_thread::yield();
      else std::this_thread::sleep_for(std::chrono::microseconds(50));
   }
   h->pending = false;
   const bool had_out = h->pending_out;
   h->pending_out = false;
   if (had_out && h->d_status.p) {
      int st = 0;
      CK(h, cudaMemcpy(&st, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
      if (st) {
         cudaMemset(h->d_status.p, 0, sizeof(int));
         return fail(h, SWSGPU_ECUDA, "a device-side wait for cluster data gave up; the spectra are invalid");
      }
   }
   if (had_out) {
      // pageable destinations of swsgpu_submit_out: from the staging buffer,
      // whose four regions follow one another
      const char *hp = (const char *)h->h_out.p;
      const size_t bytes[4] = {h->h_auto_bytes, h->h_xpol_bytes, h->h_pcal_bytes, h->h_tones_bytes};
      size_t at = 0;
      for (int k = 0; k < 4; k++) {
         if (h->deliver_copy[k]) memcpy(h->deliver_copy[k], hp + at, bytes[k]);
         h->deliver_copy[k] = nullptr;
         at += bytes[k];
      }
   }
   if (nspectra) *nspectra = h->pending_nspec;
   return SWSGPU_OK;
}

int swsgpu_sync(swsgpu_handle *h, void *cuda_stream)
{
   if (!h) return SWSGPU_EINVAL;
   CK(h, cudaSetDevice(h->device));
   CK(h, cudaStreamSynchronize(cuda_stream ? (cudaStream_t)cuda_stream : h->stream));
   if (!cuda_stream && h->stream2) CK(h, cudaStreamSynchronize(h->stream2));
   if (h->d_status.p) {
      int st = 0;
      CK(h, cudaMemcpy(&st, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
      if (st) {
         CK(h, cudaMemset(h->d_status.p, 0, sizeof(int)));
         return fail(h, SWSGPU_ECUDA, "a device-side wait for cluster data gave up; the spectra are invalid");
      }
   }
   return SWSGPU_OK;
}

int swsgpu_inject(swsgpu_handle *h, int kind)
{
   if (!h) return SWSGPU_EINVAL;
   if (kind != SWSGPU_INJECT_NONE && kind != SWSGPU_INJECT_DROP_EXCHANGE)
      return fail(h, SWSGPU_EINVAL, "unknown fault-injection kind");
   if (kind == SWSGPU_INJECT_DROP_EXCHANGE && h->big)
      return fail(h, SWSGPU_EINVAL, "the four-step path has no cluster exchange to drop");
   h->inject = kind;
   return SWSGPU_OK;
}

int swsgpu_host_register(void *p, size_t bytes)
{
   if (!p || bytes == 0) return SWSGPU_EINVAL;
   cudaPointerAttributes at;
   if (cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeHost) return SWSGPU_OK;
   cudaGetLastError();
   cudaError_t e = cudaHostRegister(p, bytes, cudaHostRegisterDefault);
   if (e == cudaErrorHostMemoryAlreadyRegistered) {
      cudaGetLastError();
      return SWSGPU_OK;
   }
   if (e != cudaSuccess) {
      cudaGetLastError();
      g_create_error = std::string("cudaHostRegister: ") + cudaGetErrorString(e);
      return SWSGPU_ECUDA;
   }
   return SWSGPU_OK;
}

int swsgpu_host_unregister(void *p)
{
   if (!p) return SWSGPU_EINVAL;
   cudaError_t e = cudaHostUnregister(p);
   if (e != cudaSuccess) {
      cudaGetLastError();
      return e == cudaErrorHostMemoryNotRegistered ? SWSGPU_EINVAL : SWSGPU_ECUDA;
   }
   return SWSGPU_OK;
}

int swsgpu_fetch(swsgpu_handle *h, const swsgpu_outputs *out)
{
   if (!h || !out) return SWSGPU_EINVAL;
   if (h->pending) return fail(h, SWSGPU_ESTATE, "fetch before wait");
   const char *hp = (const char *)h->h_out.p;
   if (h->delivered)
      return fail(h, SWSGPU_ESTATE, "the spectra went to the destination given to swsgpu_submit_out");
   if (!hp || !h->fetch_ready) return fail(h, SWSGPU_ESTATE, "no completed spectra to fetch");
   if (out->auto_out) memcpy(out->auto_out, hp, h->h_auto_bytes);
   if (out->xpol_out && h->h_xpol_bytes) memcpy(out->xpol_out, hp + h->h_auto_bytes, h->h_xpol_bytes);
   if (out->pcal_out && h->h_pcal_bytes)
      memcpy(out->pcal_out, hp + h->h_auto_bytes + h->h_xpol_bytes, h->h_pcal_bytes);
   if (out->tones_out && h->h_tones_bytes)
      memcpy(out->tones_out, hp + h->h_auto_bytes + h->h_xpol_bytes + h->h_pcal_bytes, h->h_tones_bytes);
   return SWSGPU_OK;
}

static int process_device_on(swsgpu_handle *h, const void *const *d_raw, size_t run_bytes, int nruns,
                             int runs_per_output, const swsgpu_outputs *d_out, cudaStream_t st);

int swsgpu_process_device(swsgpu_handle *h, const void *const *d_raw, size_t run_bytes, int nruns,
                          int runs_per_output, const swsgpu_outputs *d_out, void *cuda_stream)
{
   if (!h || !d_raw || !d_out || nruns < 1 || runs_per_output < 1) return SWSGPU_EINVAL;
   CK(h, cudaSetDevice(h->device));
   return process_device_on(h, d_raw, run_bytes, nruns, runs_per_output, d_out,
                            cuda_stream ? (cudaStream_t)cuda_stream : h->stream);
}

}  // extern "C"

static int process_device_on(swsgpu_handle *h, const void *const *d_raw, size_t run_bytes, int nruns,
                             int runs_per_output, const swsgpu_outputs *d_out, cudaStream_t st)
{
   const swsgpu_config &c = h->cfg;
   long long grid_off[SWSGPU_MAX_STREAMS];
   size_t raw_bytes[SWSGPU_MAX_STREAMS];
   for (int s = 0; s < c.num_streams; s++)
      if (!d_raw[s] || ((uintptr_t)d_raw[s] % 4))
         return fail(h, SWSGPU_EINVAL, "device input must be 4-byte aligned (the decoders read 32-bit words)");
   for (int s = 0; s < c.num_streams; s++) {
      const swsgpu_layout &L = c.layout[s];
      const int pb = payload_bytes(L);
      size_t pay = run_bytes * (size_t)nruns;
      grid_off[s] = 0;
      if (L.header_bytes == 0) raw_bytes[s] = pay;
      else raw_bytes[s] = ((pay + pb - 1) / pb) * (size_t)L.frame_bytes;
   }
   int nspec = 0;
   return launch_chunk(h, d_raw, raw_bytes, grid_off, run_bytes, nruns, runs_per_output,
                       d_out->auto_out, c.num_xpols ? d_out->xpol_out : nullptr,
                       c.extract_pcal ? d_out->pcal_out : nullptr, st, &nspec, 0, 1, 1,
                       (c.extract_pcal && c.pcal_ntones > 0) ? d_out->tones_out : nullptr);
}

// ---------------------------------------------------------------------------
// autotuning of the four-step split
// ---------------------------------------------------------------------------
__global__ void k_fill_hash(uint32_t *p, size_t n, uint32_t seed)
{
   const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   uint32_t x = (uint32_t)i * 2654435761u ^ seed;
   x ^= x >> 16;
   x *= 0x7feb352du;
   x ^= x >> 15;
   x *= 0x846ca68bu;
   x ^= x >> 16;
   p[i] = x;
}

static std::mutex g_tune_mu;
static std::map<std::pair<int, int>, int> g_tuned;  // (N, tune_key) -> candidate
// bit depth, + 100 for a tensor-core form, + 1000 for the four-step family
static int tune_key(int nbit, bool tc, bool big) { return nbit + (tc ? 100 : 0) + (big ? 1000 : 0); }

static cudaError_t set_big_attrs(const swsgpu_handle *h, const BigPlan &bp)
{
   const int nbit = h->cfg.layout[0].nbit;
   const int nbi = nbit == 1 ? 0 : nbit == 2 ? 1 : 2;
   cudaError_t e = cudaFuncSetAttribute((const void *)bp.cols[nbi], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)bp.smem_cols[nbi]);
   if (e != cudaSuccess) return e;
   if (h->cfg.precision != SWSGPU_PREC_FP32)
      return bp.rows_tc ? cudaFuncSetAttribute((const void *)bp.rows_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)bp.smem_rows_tc)
                        : cudaErrorInvalidValue;
   return cudaFuncSetAttribute((const void *)bp.rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)bp.smem_rows);
}

// Times every candidate split on a hash-filled run (the handle's own
// sources, pairs and window) of enough frames for about 16 pair FFTs, so
// that both passes fill the device as a full run does, and keeps the one
// with the shortest single iteration.
static int autotune_big(swsgpu_handle *h, int iters)
{
   const swsgpu_config &c = h->cfg;
   BigPlan cand[16];
   const int nc = big_plan_candidates(c.fft_points, cand, 16);
   h->big_cands = nc;
   if (nc <= 1) return SWSGPU_OK;
   const int nbit = c.layout[0].nbit;
   const int frames = 2 * std::max(1, (16 + c.num_sources - 1) / std::max(1, c.num_sources));
   const long long nsamp = (long long)frames * c.fft_points;
   const int pb = payload_bytes(c.layout[0]);
   size_t pay = (size_t)((nsamp * c.layout[0].nchan * nbit + 7) / 8);
   pay = ((pay + pb - 1) / pb) * pb;
   DevBuf raw[SWSGPU_MAX_STREAMS], oa, ox;
   const void *d_raw[SWSGPU_MAX_STREAMS];
   size_t raw_bytes[SWSGPU_MAX_STREAMS];
   long long grid_off[SWSGPU_MAX_STREAMS];
   auto cleanup = [&]() {
      cudaStreamSynchronize(h->stream);
      for (auto &r : raw) r.release();
      oa.release();
      ox.release();
      drop_schedules(h);
   };
   for (int s = 0; s < c.num_streams; s++) {
      const swsgpu_layout &L = c.layout[s];
      raw_bytes[s] = L.header_bytes ? (pay / pb) * (size_t)L.frame_bytes : pay;
      grid_off[s] = 0;
      if (raw[s].ensure(raw_bytes[s] + 64) != cudaSuccess) {
         cleanup();
         return fail(h, SWSGPU_ECUDA, "autotune: allocation failed");
      }
      const size_t nw = raw_bytes[s] / 4;
      k_fill_hash<<<(unsigned)((nw + 255) / 256), 256, 0, h->stream>>>((uint32_t *)raw[s].p, nw, 1234u + s);
      d_raw[s] = raw[s].p;
   }
   if (oa.ensure(sizeof(float) * (size_t)h->S * c.num_sources * (frames + 1) + 64) != cudaSuccess ||
       ox.ensure(sizeof(float) * 2 * (size_t)h->S * std::max(c.num_xpols, 1) * (frames + 1) + 64) != cudaSuccess) {
      cleanup();
      return fail(h, SWSGPU_ECUDA, "autotune: allocation failed");
   }
   int best = -1;
   float best_ms = 0.0f;
   const int nit = std::max(1, std::min(iters, 16));
   cudaEvent_t ev[17];
   for (int i = 0; i <= nit; i++) cudaEventCreate(&ev[i]);
   for (int k = 0; k < nc; k++) {
      if (c.precision != SWSGPU_PREC_FP32 && !cand[k].rows_tc) continue;  // no tensor-core row pass
      if (set_big_attrs(h, cand[k]) != cudaSuccess) {
         cudaGetLastError();
         continue;
      }
      h->bplan = cand[k];
      h->cand = k;
      int nspec = 0, rc = SWSGPU_OK;
      // one untimed iteration, then nit timed ones
      for (int it = 0; it <= nit && rc == SWSGPU_OK; it++) {
         if (it >= 1) cudaEventRecord(ev[it - 1], h->stream);
         rc = launch_chunk(h, d_raw, raw_bytes, grid_off, pay, 1, 1, (float *)oa.p,
                           c.num_xpols ? (float *)ox.p : nullptr, nullptr, h->stream, &nspec);
      }
      cudaEventRecord(ev[nit], h->stream);
      if (rc != SWSGPU_OK || cudaEventSynchronize(ev[nit]) != cudaSuccess) {
         cudaGetLastError();
         continue;
      }
      float ms = 0.0f;
      for (int i = 0; i < nit; i++) {
         float t = 0.0f;
         cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
         if (i == 0 || t < ms) ms = t;
      }
      if (best < 0 || ms < best_ms) {
         best = k;
         best_ms = ms;
      }
   }
   for (int i = 0; i <= nit; i++) cudaEventDestroy(ev[i]);
   cleanup();
   if (best < 0) return fail(h, SWSGPU_ECUDA, "autotune: no candidate ran");
   h->bplan = cand[best];
   h->tuned = best;
   h->cand = best;
   CK(h, set_big_attrs(h, h->bplan));
   std::lock_guard<std::mutex> lk(g_tune_mu);
   g_tuned[std::make_pair(c.fft_points, tune_key(nbit, c.precision != SWSGPU_PREC_FP32, true))] = best;
   return SWSGPU_OK;
}

// Times every cluster plan of the length that has a kernel of the handle's
// form (cluster size, threads per CTA, radix order) on one run of
// max_run_bytes of synthetic codes -- the job count the core's runs give --
// and keeps the fastest single iteration.  The choice is remembered per
// length, bit depth and form for the rest of the process.
static int autotune_cluster(swsgpu_handle *h, int iters)
{
   const swsgpu_config &c = h->cfg;
   Plan cand[8];
   const int nc = plan_candidates(c.fft_points, cand, 8);
   const int nbit = c.layout[0].nbit;
   const int nbi = nbit == 1 ? 0 : nbit == 2 ? 1 : 2;
   int nrun_ok = 0;
   for (int k = 0; k < nc; k++) nrun_ok += plan_kernel(cand[k], c.precision, nbi) ? 1 : 0;
   if (nrun_ok <= 1) return SWSGPU_OK;
   const Plan keep = h->plan;
   const int keep_cand = h->cand;
   const int pb = payload_bytes(c.layout[0]);
   // one run's samples (at least two FFTs per source), capped at 64 MiB of payload
   size_t pay = std::min<size_t>(c.max_run_bytes, (size_t)64 << 20);
   if (c.layout[0].header_bytes) pay = pay / c.layout[0].frame_bytes * (size_t)pb;
   long long nsamp = samples_of(c.layout[0], pay);
   nsamp = std::max<long long>(nsamp, 2LL * c.fft_points);
   pay = (size_t)((nsamp * c.layout[0].nchan * nbit + 7) / 8);
   pay = ((pay + pb - 1) / pb) * pb;
   const RunShape rs = run_shape(c, samples_of(c.layout[0], pay));
   const int nspec = std::max(rs.nspec, 1) + 1;
   DevBuf raw[SWSGPU_MAX_STREAMS], oa, ox;
   const void *d_raw[SWSGPU_MAX_STREAMS];
   size_t raw_bytes[SWSGPU_MAX_STREAMS];
   long long grid_off[SWSGPU_MAX_STREAMS];
   auto cleanup = [&]() {
      cudaStreamSynchronize(h->stream);
      for (auto &r : raw) r.release();
      oa.release();
      ox.release();
      drop_schedules(h);
   };
   for (int s = 0; s < c.num_streams; s++) {
      const swsgpu_layout &L = c.layout[s];
      raw_bytes[s] = L.header_bytes ? (pay / pb) * (size_t)L.frame_bytes : pay;
      grid_off[s] = 0;
      if (raw[s].ensure(raw_bytes[s] + 64) != cudaSuccess) {
         cleanup();
         return fail(h, SWSGPU_ECUDA, "autotune: allocation failed");
      }
      const size_t nw = raw_bytes[s] / 4;
      k_fill_hash<<<(unsigned)((nw + 255) / 256), 256, 0, h->stream>>>((uint32_t *)raw[s].p, nw, 1234u + s);
      d_raw[s] = raw[s].p;
   }
   if (oa.ensure(sizeof(float) * (size_t)h->S * c.num_sources * nspec + 64) != cudaSuccess ||
       ox.ensure(sizeof(float) * 2 * (size_t)h->S * std::max(c.num_xpols, 1) * nspec + 64) != cudaSuccess) {
      cleanup();
      return fail(h, SWSGPU_ECUDA, "autotune: allocation failed");
   }
   int best = -1;
   float best_ms = 0.0f;
   const int nit = std::max(1, std::min(iters, 16));
   cudaEvent_t ev[17];
   for (int i = 0; i <= nit; i++) cudaEventCreate(&ev[i]);
   for (int k = 0; k < nc; k++) {
      if (!plan_kernel(cand[k], c.precision, nbi)) continue;
      if (set_cluster_plan(h, cand[k]) != SWSGPU_OK) {
         cudaGetLastError();
         continue;
      }
      h->cand = k;
      int ns = 0, rc = SWSGPU_OK;
      // one untimed iteration, then nit timed ones
      for (int it = 0; it <= nit && rc == SWSGPU_OK; it++) {
         if (it >= 1) cudaEventRecord(ev[it - 1], h->stream);
         rc = launch_chunk(h, d_raw, raw_bytes, grid_off, pay, 1, 1, (float *)oa.p,
                           c.num_xpols ? (float *)ox.p : nullptr, nullptr, h->stream, &ns);
      }
      cudaEventRecord(ev[nit], h->stream);
      if (rc != SWSGPU_OK || cudaEventSynchronize(ev[nit]) != cudaSuccess) {
         cudaGetLastError();
         continue;
      }
      float ms = 0.0f;
      for (int i = 0; i < nit; i++) {
         float t = 0.0f;
         cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
         if (i == 0 || t < ms) ms = t;
      }
      if (best < 0 || ms < best_ms) {
         best = k;
         best_ms = ms;
      }
   }
   for (int i = 0; i <= nit; i++) cudaEventDestroy(ev[i]);
   cleanup();
   if (best < 0) {
      set_cluster_plan(h, keep);
      h->cand = keep_cand;
      return fail(h, SWSGPU_ECUDA, "autotune: no candidate ran");
   }
   {
      const int rc = set_cluster_plan(h, cand[best]);
      if (rc != SWSGPU_OK) return rc;
   }
   h->tuned = best;
   h->cand = best;
   std::lock_guard<std::mutex> lk(g_tune_mu);
   g_tuned[std::make_pair(c.fft_points, tune_key(nbit, c.precision != SWSGPU_PREC_FP32, false))] = best;
   return SWSGPU_OK;
}

// ---------------------------------------------------------------------------
// batches: many cores' runs captured as one CUDA graph
// ---------------------------------------------------------------------------
struct swsgpu_batch {
   int device = 0;
   std::vector<swsgpu_handle *> cores;
   struct Work {
      bool set = false;
      const void *d_raw[SWSGPU_MAX_STREAMS] = {nullptr, nullptr};
      size_t run_bytes = 0;
      int nruns = 0, rpo = 0;
      swsgpu_outputs out = {};
   };
   std::vector<Work> work;
   cudaStream_t cap = nullptr;
   cudaEvent_t fork = nullptr;
   std::vector<cudaEvent_t> join;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   bool dirty = true;
   int kernels = 0;
};

static void batch_drop_graph(swsgpu_batch *b)
{
   if (b->exec) cudaGraphExecDestroy(b->exec);
   if (b->graph) cudaGraphDestroy(b->graph);
   b->exec = nullptr;
   b->graph = nullptr;
   b->dirty = true;
}

extern "C" {

int swsgpu_workspace_size(const swsgpu_handle *h, size_t run_bytes, int nruns, size_t *bytes)
{
   if (!h || !bytes || nruns < 1) return SWSGPU_EINVAL;
   const swsgpu_config &c = h->cfg;
   const long long nsamp = samples_of(c.layout[0], run_bytes) * nruns;
   const int spw = 32 / c.layout[0].nbit;
   const size_t ncode = h->code_stream.size();
   bool col = false;
   const int D = code_decimation(h, &col);
   const long long wpp = (((nsamp + D - 1) / D + spw - 1) / spw + 2 + 3) / 4 * 4;
   size_t total = sizeof(uint32_t) * (size_t)D * (size_t)wpp * ncode + 64;       // codes
   if (col && c.extract_pcal)                                                      // undecimated copy
      total += sizeof(uint32_t) * (size_t)((nsamp + spw - 1) / spw + 2) * ncode + 64;
   total += sizeof(uint32_t) * (size_t)((nsamp + 31) / 32) * c.num_streams + 16;  // blank bitmaps
   for (int s = 0; s < c.num_streams; s++)                                         // frame validity
      total += sizeof(int2) * (size_t)(run_bytes * (size_t)nruns / payload_bytes(c.layout[s]) + 2);
   // the schedule's partial rows and, on the four-step path, its scratch;
   // the output addresses are only recorded in the entries, never used here
   Schedule sc;
   float *unused = reinterpret_cast<float *>(alignof(float2));
   build_schedule(h, run_bytes, nruns, nruns, unused, c.num_xpols ? unused : nullptr, nullptr, sc);
   total += sizeof(float) * 4 * (size_t)h->S * sc.items.size();
   // FP64 running sums, used when an output group spans launches
   if (nruns > 1) total += sizeof(double) * (size_t)h->S * (sc.outs.size() + 1);
   if (h->big) {
      std::vector<BigJob> jobs;
      std::vector<BigItem> bitems;
      std::vector<int4> batches;
      big_batches(h, sc, jobs, bitems, batches);
      int max_jobs = 0;
      for (const int4 &b : batches) max_jobs = std::max(max_jobs, b.y);
      total += sizeof(float2) * (size_t)c.fft_points * (size_t)max_jobs;
   }
   *bytes = total;
   return SWSGPU_OK;
}

int swsgpu_unpack_device(const swsgpu_layout *lay, const void *d_raw, size_t nbytes,
                         int64_t payload_offset, int chan, int64_t nsamp, float *d_out,
                         int64_t *nvalid, void *cuda_stream)
{
   if (!lay || !d_raw || !d_out || chan < 0 || chan >= lay->nchan || nsamp < 0) return SWSGPU_EINVAL;
   if (lay->nbit != 1 && lay->nbit != 2 && lay->nbit != 8) return SWSGPU_EINVAL;
   if ((uintptr_t)d_raw % 4 || (uintptr_t)d_out % 4) return SWSGPU_EINVAL;  // 32-bit loads and stores
   const int pb = lay->frame_bytes - lay->header_bytes;
   if (pb <= 0 || (pb % 8) || (lay->header_bytes % 4) || (payload_offset % 4)) return SWSGPU_EINVAL;
   if (lay->header_bytes > 0 && payload_offset != 0) return SWSGPU_EINVAL;
   std::string why;
   const int ntrack = track_format(lay->format) ? track_layout_ok(*lay, why) : 0;
   if (track_format(lay->format) && (!ntrack || payload_offset % (ntrack / 8))) return SWSGPU_EINVAL;
   cudaStream_t st = (cudaStream_t)cuda_stream;
   StreamIn si;
   si.data = (const uint8_t *)d_raw;
   si.nbytes = (long long)nbytes;
   si.grid_offset = payload_offset % pb;
   si.frame_bytes = lay->frame_bytes;
   si.header_bytes = lay->header_bytes;
   si.payload_bytes = pb;
   si.nchan = lay->nchan;
   si.nbit = lay->nbit;
   si.format = lay->format;
   si.msb2 = is_msb2(*lay);
   set_zones(si);
   if (nsamp == 0) {
      if (nvalid) *nvalid = 0;
      return SWSGPU_OK;
   }
   const long long last_v = si.grid_offset + ((nsamp * (long long)lay->nchan * lay->nbit - 1) >> 3);
   si.nframes = last_v / pb + 1;
   // bytes needed
   long long need = lay->header_bytes ? si.nframes * lay->frame_bytes - (lay->frame_bytes - lay->header_bytes - (last_v % pb) - 1)
                                      : (last_v - si.grid_offset + 1);
   if (need > (long long)nbytes) return SWSGPU_EINVAL;
   int2 *d_valid = nullptr;
   int *d_any = nullptr;
   unsigned long long *d_cnt = nullptr;
   uint32_t *d_trk = nullptr;
   if (cudaMalloc(&d_valid, sizeof(int2) * si.nframes * si.zpf) != cudaSuccess) return SWSGPU_ECUDA;
   if (cudaMalloc(&d_any, sizeof(int)) != cudaSuccess || cudaMalloc(&d_cnt, sizeof(unsigned long long)) != cudaSuccess) {
      cudaFree(d_valid);
      if (d_any) cudaFree(d_any);
      return SWSGPU_ECUDA;
   }
   cudaMemsetAsync(d_any, 0, sizeof(int), st);
   cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st);
   // validity from the stream's own bytes (the track-words, for VLBA / Mark4)
   k_frame_valid<<<(unsigned)((si.nframes + 127) / 128), 128, 0, st>>>(si, d_valid, d_any);
   uint32_t *d_tab = nullptr;
   if (ntrack) {
      // VLBA / Mark4 track-words into Mark5B's sample layout
      std::vector<uint32_t> tab(TRACK_TABLE_WORDS);
      track_turn_table(ntrack, lay->nbit, lay->nchan, tab.data());
      cudaError_t e = cudaMalloc(&d_trk, (nbytes + 3) / 4 * 4 + 16);
      if (e == cudaSuccess) e = cudaMalloc(&d_tab, sizeof(uint32_t) * tab.size());
      if (e == cudaSuccess)
         e = cudaMemcpyAsync(d_tab, tab.data(), sizeof(uint32_t) * tab.size(), cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
         e = launch_track_turn(st, (const uint8_t *)d_raw, (long long)nbytes, si.grid_offset, ntrack, lay->format,
                               d_tab, d_trk);
      if (e != cudaSuccess) {
         cudaStreamSynchronize(st);
         cudaFree(d_valid);
         cudaFree(d_any);
         cudaFree(d_cnt);
         if (d_trk) cudaFree(d_trk);
         if (d_tab) cudaFree(d_tab);
         return SWSGPU_ECUDA;
      }
      si.data = (const uint8_t *)d_trk;
   }
   k_unpack_float<<<(unsigned)((nsamp + 255) / 256), 256, 0, st>>>(si, nsamp, chan,
                                                                    level_table(lay->format, lay->nbit),
                                                                    d_out, d_valid, d_cnt);
   unsigned long long cnt = 0;
   cudaMemcpyAsync(&cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st);
   cudaError_t e = cudaStreamSynchronize(st);
   cudaFree(d_valid);
   cudaFree(d_any);
   cudaFree(d_cnt);
   if (d_trk) cudaFree(d_trk);
   if (d_tab) cudaFree(d_tab);
   if (e != cudaSuccess) {
      g_create_error = cudaGetErrorString(e);
      return SWSGPU_ECUDA;
   }
   if (nvalid) *nvalid = (int64_t)cnt;
   return SWSGPU_OK;
}

int swsgpu_last_launch_count(const swsgpu_handle *h) { return h ? h->last_launches : 0; }

int swsgpu_profile(swsgpu_handle *h, int enable)
{
   if (!h) return SWSGPU_EINVAL;
   CK(h, cudaSetDevice(h->device));
   if (enable) {
      CK(h, cudaStreamSynchronize(h->stream));
      drop_prof_events(h);
   }
   h->profiling = enable != 0;
   return SWSGPU_OK;
}

int swsgpu_profile_read(swsgpu_handle *h, int *launches, double *total_ms)
{
   if (!h) return SWSGPU_EINVAL;
   CK(h, cudaSetDevice(h->device));
   double tot = 0.0;
   for (auto &pr : h->prof_events) {
      CK(h, cudaEventSynchronize(pr.second));
      float ms = 0.0f;
      CK(h, cudaEventElapsedTime(&ms, pr.first, pr.second));
      tot += ms;
   }
   if (launches) *launches = (int)h->prof_events.size();
   if (total_ms) *total_ms = tot;
   drop_prof_events(h);
   return SWSGPU_OK;
}

int swsgpu_autotune(swsgpu_handle *h, int iterations)
{
   if (!h || iterations < 1) return SWSGPU_EINVAL;
   CK(h, cudaSetDevice(h->device));
   if (h->pending) return fail(h, SWSGPU_ESTATE, "autotune while a run is pending");
   return h->big ? autotune_big(h, iterations) : autotune_cluster(h, iterations);
}

int swsgpu_plan_info(const swsgpu_handle *h, char *buf, size_t len)
{
   if (!h || !buf || len == 0) return SWSGPU_EINVAL;
   if (h->big) {
      snprintf(buf, len, "four-step %d x %d, %d columns per CTA, candidate %d of %d%s", h->bplan.N1, h->bplan.N2,
               h->bplan.C, h->cand, h->big_cands,
               h->tuned >= 0 ? " (tuned)" : (h->cand > 0 ? " (pinned)" : " (default)"));
   } else {
      Plan cand[8];
      const int nc = plan_candidates(h->cfg.fft_points, cand, 8);
      snprintf(buf, len, "cluster %d x %d (CTAs x points), %d threads, radices %d/%d/%d, candidate %d of %d%s, %s form",
               h->plan.P, h->plan.Q, h->plan.T, h->plan.R1, h->plan.R2, h->plan.R3, h->cand, nc,
               h->tuned >= 0 ? " (tuned)" : (h->cand > 0 ? " (pinned)" : " (default)"),
               h->cfg.precision == SWSGPU_PREC_TCSPLIT       ? "tensor-core split (tcgen05 levels 2-3)"
               : h->cfg.precision == SWSGPU_PREC_TCSPLIT_ALL ? "tensor-core split (tcgen05 levels 1-3)"
                                                             : "FP32");
   }
   return SWSGPU_OK;
}

int swsgpu_batch_create(swsgpu_handle *const *cores, int ncores, swsgpu_batch **out)
{
   if (!cores || ncores < 1 || !out) return fail(nullptr, SWSGPU_EINVAL, "batch: no cores");
   *out = nullptr;
   for (int i = 0; i < ncores; i++) {
      if (!cores[i]) return fail(nullptr, SWSGPU_EINVAL, "batch: null core");
      if (cores[i]->device != cores[0]->device) return fail(nullptr, SWSGPU_EINVAL, "batch: cores on different devices");
      for (int j = 0; j < i; j++)
         if (cores[j] == cores[i]) return fail(nullptr, SWSGPU_EINVAL, "batch: a core appears twice");
   }
   if (cudaSetDevice(cores[0]->device) != cudaSuccess) return fail(nullptr, SWSGPU_ENODEV, "batch: cudaSetDevice");
   swsgpu_batch *b = new swsgpu_batch();
   b->device = cores[0]->device;
   b->cores.assign(cores, cores + ncores);
   b->work.resize(ncores);
   b->join.assign(ncores, nullptr);
   bool ok = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
   for (int i = 0; i < ncores && ok; i++) ok = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
   if (!ok) {
      swsgpu_batch_destroy(b);
      return fail(nullptr, SWSGPU_ECUDA, "batch: stream/event creation failed");
   }
   *out = b;
   return SWSGPU_OK;
}

int swsgpu_batch_set(swsgpu_batch *b, int i, const void *const *d_raw, size_t run_bytes, int nruns,
                     int runs_per_output, const swsgpu_outputs *d_out)
{
   if (!b || i < 0 || i >= (int)b->cores.size() || !d_raw || !d_out || nruns < 1 || runs_per_output < 1)
      return fail(nullptr, SWSGPU_EINVAL, "batch_set: bad argument");
   for (int s = 0; s < b->cores[i]->cfg.num_streams; s++)
      if (!d_raw[s] || ((uintptr_t)d_raw[s] % 4))
         return fail(nullptr, SWSGPU_EINVAL, "batch_set: device input must be 4-byte aligned");
   swsgpu_batch::Work &w = b->work[i];
   for (int s = 0; s < b->cores[i]->cfg.num_streams; s++) w.d_raw[s] = d_raw[s];
   w.run_bytes = run_bytes;
   w.nruns = nruns;
   w.rpo = runs_per_output;
   w.out = *d_out;
   w.set = true;
   batch_drop_graph(b);
   return SWSGPU_OK;
}

int swsgpu_batch_launch(swsgpu_batch *b, void *cuda_stream, int *kernels)
{
   if (!b) return SWSGPU_EINVAL;
   for (const auto &w : b->work)
      if (!w.set) return fail(nullptr, SWSGPU_EINVAL, "batch_launch: a core has no work (swsgpu_batch_set)");
   if (cudaSetDevice(b->device) != cudaSuccess) return fail(nullptr, SWSGPU_ENODEV, "batch: cudaSetDevice");
   const int n = (int)b->cores.size();
   auto cuda_fail = [&](cudaError_t e, const char *what) {
      cudaGetLastError();
      return fail(nullptr, SWSGPU_ECUDA, std::string("batch ") + what + ": " + cudaGetErrorString(e));
   };
   if (b->dirty) {
      // eager pass: every allocation and device schedule is made here, so the
      // captured launches allocate and upload nothing
      int total = 0;
      for (int i = 0; i < n; i++) {
         swsgpu_handle *h = b->cores[i];
         if (h->pending) return fail(nullptr, SWSGPU_ESTATE, "batch: a core has a run pending");
         const auto &w = b->work[i];
         const int rc = process_device_on(h, w.d_raw, w.run_bytes, w.nruns, w.rpo, &w.out, h->stream);
         if (rc != SWSGPU_OK) return fail(nullptr, rc, "batch eager run of core " + std::to_string(i) + ": " + h->err);
         total += h->last_launches;
      }
      for (int i = 0; i < n; i++) {
         cudaError_t e = cudaStreamSynchronize(b->cores[i]->stream);
         if (e != cudaSuccess) return cuda_fail(e, "eager run");
      }
      // capture: each core's pipeline on its own stream, forked from and
      // joined back into the capture stream, so the cores run concurrently
      cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return cuda_fail(e, "begin capture");
      int rc = SWSGPU_OK;
      e = cudaEventRecord(b->fork, b->cap);
      for (int i = 0; i < n && e == cudaSuccess && rc == SWSGPU_OK; i++) {
         swsgpu_handle *h = b->cores[i];
         const auto &w = b->work[i];
         e = cudaStreamWaitEvent(h->stream, b->fork, 0);
         if (e != cudaSuccess) break;
         rc = process_device_on(h, w.d_raw, w.run_bytes, w.nruns, w.rpo, &w.out, h->stream);
         if (rc != SWSGPU_OK) break;
         e = cudaEventRecord(b->join[i], h->stream);
         if (e == cudaSuccess) e = cudaStreamWaitEvent(b->cap, b->join[i], 0);
      }
      cudaGraph_t g = nullptr;
      cudaError_t e2 = cudaStreamEndCapture(b->cap, &g);
      if (e != cudaSuccess || rc != SWSGPU_OK || e2 != cudaSuccess) {
         if (g) cudaGraphDestroy(g);
         if (rc != SWSGPU_OK) return fail(nullptr, rc, "batch capture");
         return cuda_fail(e != cudaSuccess ? e : e2, "capture");
      }
      b->graph = g;
      e = cudaGraphInstantiate(&b->exec, b->graph, 0);
      if (e != cudaSuccess) {
         batch_drop_graph(b);
         return cuda_fail(e, "instantiate");
      }
      b->dirty = false;
      b->kernels = total;
      if (kernels) *kernels = total;
      return SWSGPU_OK;  // the eager pass produced this launch's results
   }
   cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)cuda_stream);
   if (e != cudaSuccess) return cuda_fail(e, "graph launch");
   if (kernels) *kernels = b->kernels;
   return SWSGPU_OK;
}

void swsgpu_batch_destroy(swsgpu_batch *b)
{
   if (!b) return;
   cudaSetDevice(b->device);
   if (b->cap) cudaStreamSynchronize(b->cap);
   batch_drop_graph(b);
   for (cudaEvent_t e : b->join)
      if (e) cudaEventDestroy(e);
   if (b->fork) cudaEventDestroy(b->fork);
   if (b->cap) cudaStreamDestroy(b->cap);
   delete b;
}

}  // extern "C"

static std::mutex &tune_mutex() { return g_tune_mu; }

static int tuned_choice(int N, int nbit, bool tc, bool big)
{
   std::lock_guard<std::mutex> lk(tune_mutex());
   auto it = g_tuned.find(std::make_pair(N, tune_key(nbit, tc, big)));
   return it == g_tuned.end() ? -1 : it->second;
}
