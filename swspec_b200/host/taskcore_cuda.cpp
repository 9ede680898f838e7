// taskcore_cuda.cpp -- TaskCore implementation over the GPU C ABI.
//
// Replaces TaskCoreIPP (src/IA-32/TaskCoreIPP.cpp): prepare() creates the
// device core from the settings, run() queues the buffers (H2D + kernels)
// and returns, join() waits and copies the run's spectra into the output
// buffers with the lengths doMaths sets (:526-541), combineResults() adds
// them into the dispatcher's buffers (:311-349).  With GpuCombineOnDevice the
// runs of one spectrum are summed on the device (FP64 between runs) and only
// the completed spectrum is copied back.
#include <algorithm>
#include <chrono>
#include <cstring>

#include "sws_host.h"

namespace swshost {

TaskCoreCUDA::~TaskCoreCUDA()
{
   if (h_) swsgpu_destroy(h_);
   for (void *p : pinned_) swsgpu_host_unregister(p);
}

static int window_code(WindowFunctionType w)
{
   switch (w) {
   case None: return SWSGPU_WIN_NONE;
   case Cosine: return SWSGPU_WIN_COSINE;
   case Cosine2: return SWSGPU_WIN_COSINE2;
   case Hamming: return SWSGPU_WIN_HAMMING;
   case Hann: return SWSGPU_WIN_HANN;
   case Blackman: return SWSGPU_WIN_BLACKMAN;
   case BlackmanHarris: return SWSGPU_WIN_BLACKMANHARRIS;
   }
   return SWSGPU_WIN_COSINE2;
}

void TaskCoreCUDA::prepare(Settings *s)
{
   cfg_ = s;
   swsgpu_config c;
   memset(&c, 0, sizeof(c));
   c.layout[0] = c.layout[1] = s->layout;
   c.num_streams = s->num_sources;
   c.fft_points = (int)s->fft_points;
   c.overlap = s->fft_overlap_factor;
   c.window = window_code(s->wf_type);
   c.precision = s->gpu_precision;
   c.core_overlapped_ffts = s->core_overlapped_ffts;
   c.num_sources = s->num_sources;
   for (int i = 0; i < s->num_sources; i++) {
      c.source_stream[i] = i;
      c.source_channel[i] = (i == 0) ? s->use_channel_file1 : s->use_channel_file2;
      // raw 2-bit multi-channel data with ChannelOrderIncreasing = no keeps
      // channel 0 in the highest bits (TwoBitUnpacker, DataUnpackers.cpp:201-211)
      if (s->layout.format >= SWSGPU_FMT_RAW_SIGNED && s->layout.nbit == 2 && s->layout.nchan % 4 == 0 &&
          !s->channelorder_increasing)
         c.source_channel[i] = s->layout.nchan - 1 - c.source_channel[i];
   }
   c.num_xpols = s->num_xpols;
   if (s->num_xpols) {
      c.xpol_pair[0][0] = 0;
      c.xpol_pair[0][1] = 1;
   }
   c.extract_pcal = s->extract_PCal ? 1 : 0;
   c.pcal_tonebins = s->pcal_tonebins;
   c.pcal_rotatorlen = s->pcal_rotatorlen;
   c.samplingfreq = s->samplingfreq;
   c.pcal_offset_hz = s->pcaloffsethz;
   c.max_run_bytes = s->rawbuf_size;
   c.runs_per_output = (s->gpu_combine_on_device && s->max_buffers_per_spectrum > 1) ? s->max_buffers_per_spectrum : 1;
   c.autotune = s->gpu_autotune ? 1 : 0;
   int rc = swsgpu_create(&c, s->gpu_device, &h_);
   if (rc != SWSGPU_OK) {
      *s->tlog << "CUDA core " << rank_ << ": " << swsgpu_last_error(nullptr) << std::endl;
      h_ = nullptr;
   }
}

int TaskCoreCUDA::run(Buffer **inbuf, Buffer **outbuf, Buffer **xpolbuf, Buffer **pcalbuf)
{
   out_ = outbuf;
   xpol_ = xpolbuf;
   pcal_ = pcalbuf;
   if (!h_) return -1;
   const void *raw[SWSGPU_MAX_STREAMS];
   size_t nbytes[SWSGPU_MAX_STREAMS];
   int64_t offs[SWSGPU_MAX_STREAMS];
   size_t minlen = (size_t)-1;
   for (int s = 0; s < cfg_->num_sources; s++) minlen = std::min(minlen, inbuf[s]->getLength());
   for (int s = 0; s < cfg_->num_sources; s++) {
      raw[s] = inbuf[s]->getData();
      nbytes[s] = minlen;  // doMaths walks the shortest source buffer
      // main allocates the raw buffers once (swspectrometer.cpp:373-413):
      // page-lock each on first sight so its copy is an asynchronous DMA
      void *p = inbuf[s]->getData();
      if (std::find(pinned_.begin(), pinned_.end(), p) == pinned_.end() &&
          swsgpu_host_register(p, inbuf[s]->getAllocated()) == SWSGPU_OK)
         pinned_.push_back(p);
   }
   int nspec = 0, nffts = 0, partial = 0;
   swsgpu_run_shape(h_, minlen, &nspec, &nffts, &partial);
   run_nspec_ = nspec;
   total_ffts_ += (int64_t)nffts * cfg_->num_sources;
   // buffers of one core are every num_cores-th raw buffer of the stream;
   // their payload offsets place mark5access's per-frame blanking zones
   const int64_t run_index = total_runs_++;
   for (int s = 0; s < cfg_->num_sources; s++)
      offs[s] = (run_index * cfg_->num_cores + rank_) * (int64_t)cfg_->rawbuf_size;
   t_submit_ = std::chrono::steady_clock::now().time_since_epoch().count();
   if (swsgpu_submit(h_, raw, nbytes, offs) != SWSGPU_OK) {
      *cfg_->tlog << "CUDA core " << rank_ << " submit: " << swsgpu_last_error(h_) << std::endl;
      return -1;
   }
   return 0;
}

int TaskCoreCUDA::join()
{
   if (!h_) return -1;
   int nready = 0;
   if (swsgpu_wait(h_, -1, &nready) != SWSGPU_OK) {
      *cfg_->tlog << "CUDA core " << rank_ << " join: " << swsgpu_last_error(h_) << std::endl;
      return -1;
   }
   total_runtime_ += 1e-9 * (double)(std::chrono::steady_clock::now().time_since_epoch().count() - t_submit_);
   if (nready > 0) {
      swsgpu_outputs o = {};
      // the C ABI writes [spec][source][bins]; the reference keeps one buffer
      // per source, so fetch into a staging copy and scatter
      staged_.resize((size_t)nready * cfg_->num_sources * cfg_->fft_ssb_points);
      stagedx_.resize((size_t)nready * cfg_->num_xpols * cfg_->fft_ssb_points * 2);
      stagedp_.resize((size_t)nready * cfg_->num_sources * cfg_->pcal_tonebins * 2 + 1);
      o.auto_out = staged_.data();
      o.xpol_out = cfg_->num_xpols ? stagedx_.data() : nullptr;
      o.pcal_out = cfg_->extract_PCal ? stagedp_.data() : nullptr;
      if (swsgpu_fetch(h_, &o) != SWSGPU_OK) return -1;
      const size_t S = cfg_->fft_ssb_points;
      for (int s = 0; s < cfg_->num_sources; s++) {
         float *dst = reinterpret_cast<float *>(out_[s]->getData());
         for (int k = 0; k < nready; k++)
            memcpy(dst + k * S, staged_.data() + ((size_t)k * cfg_->num_sources + s) * S, S * sizeof(float));
         out_[s]->setLength(cfg_->fft_bytes_ssb * nready);
         if (cfg_->extract_PCal) {
            float *pd = reinterpret_cast<float *>(pcal_[s]->getData());
            const size_t tb = (size_t)cfg_->pcal_tonebins * 2;
            for (int k = 0; k < nready; k++)
               memcpy(pd + k * tb, stagedp_.data() + ((size_t)k * cfg_->num_sources + s) * tb, tb * sizeof(float));
            pcal_[s]->setLength(cfg_->pcal_result_bytes * nready);
         }
      }
      for (int x = 0; x < cfg_->num_xpols; x++) {
         float *dst = reinterpret_cast<float *>(xpol_[x]->getData());
         for (int k = 0; k < nready; k++)
            memcpy(dst + k * 2 * S, stagedx_.data() + ((size_t)k * cfg_->num_xpols + x) * 2 * S, 2 * S * sizeof(float));
         xpol_[x]->setLength(cfg_->fft_bytes_xpol * nready);
      }
      fetched_ = true;
   } else {
      fetched_ = false;
   }
   return run_nspec_;
}

int TaskCoreCUDA::combineResults(Buffer **outbuf, Buffer **pcalbuf)
{
   if (!out_ || !outbuf || !pcalbuf) {
      std::cerr << "TaskCoreCUDA combine : null buffer(s)!" << std::endl;
      return 0;
   }
   if (fetched_) {
      const size_t S = cfg_->fft_ssb_points;
      for (int s = 0; s < cfg_->num_sources; s++) {
         float *d = reinterpret_cast<float *>(outbuf[s]->getData());
         const float *m = reinterpret_cast<const float *>(out_[s]->getData());
         for (size_t k = 0; k < S; k++) d[k] += m[k];
         outbuf[s]->setLength(sizeof(float) * S);
      }
      for (int x = 0; x < cfg_->num_xpols; x++) {
         const int xo = x + cfg_->num_sources;
         float *d = reinterpret_cast<float *>(outbuf[xo]->getData());
         const float *m = reinterpret_cast<const float *>(xpol_[x]->getData());
         for (size_t k = 0; k < 2 * S; k++) d[k] += m[k];
         // the reference sets 4*(N/2+1) bytes here, half of the complex data
         // (TaskCoreIPP.cpp:333); FixXpolLength writes all of it
         outbuf[xo]->setLength(sizeof(float) * S * (cfg_->fix_xpol_length ? 2 : 1));
      }
      if (cfg_->extract_PCal) {
         for (int s = 0; s < cfg_->num_sources; s++) {
            float *d = reinterpret_cast<float *>(pcalbuf[s]->getData());
            const float *m = reinterpret_cast<const float *>(pcal_[s]->getData());
            for (int k = 0; k < 2 * cfg_->pcal_tonebins; k++) d[k] += m[k];
            pcalbuf[s]->setLength(sizeof(float) * 2 * cfg_->pcal_tonebins);
         }
      }
      fetched_ = false;
   }
   for (int s = 0; s < cfg_->num_sources; s++) resetBuffer(out_[s]);
   for (int x = 0; x < cfg_->num_xpols; x++) resetBuffer(xpol_[x]);
   if (cfg_->extract_PCal)
      for (int s = 0; s < cfg_->num_sources; s++) resetBuffer(pcal_[s]);
   return 0;
}

void TaskCoreCUDA::resetBuffer(Buffer *buf)
{
   if (buf) memset(buf->getData(), 0, buf->getAllocated());
}

int TaskCoreCUDA::finalize()
{
   *cfg_->tlog << "CUDA core " << rank_ << " completed: " << total_runtime_ << "s total run-to-join time, "
               << total_ffts_ << " FFTs" << std::endl;
   if (h_) swsgpu_destroy(h_);
   h_ = nullptr;
   for (void *p : pinned_) swsgpu_host_unregister(p);
   pinned_.clear();
   return 0;
}

}  // namespace swshost
