// TaskCoreCUDA.cpp -- the reference-interface GPU core (see TaskCoreCUDA.h).
//
// Replaces TaskCoreIPP (src/IA-32/TaskCoreIPP.cpp): the settings the
// reference's main derives (src/swspectrometer.cpp:166-231) become one
// swsgpu_config; every run() queues one raw buffer per source and returns;
// join() waits and scatters the run's spectra into the per-source output
// buffers with the lengths doMaths sets (TaskCoreIPP.cpp:526-541).
#include "TaskCoreCUDA.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <strings.h>

#include "Buffer.h"
#include "LogFile.h"

namespace {

int window_code(WindowFunctionType w)
{
   switch (w) {
   case None: return SWSGPU_WIN_NONE;
   case Cosine: return SWSGPU_WIN_COSINE;
   case Cosine2: return SWSGPU_WIN_COSINE2;
   case Hamming: return SWSGPU_WIN_HAMMING;
   case Hann: return SWSGPU_WIN_HANN;
   case Blackman: return SWSGPU_WIN_BLACKMAN;
   }
   return SWSGPU_WIN_COSINE2;
}

// Byte layout of the buffers FileSource::read delivers (src/FileSource.cpp:
// 36-110, 167-215): the framed formats arrive with their headers removed.
bool layout_of(const swspect_settings_t *s, swsgpu_layout &l, std::string &why)
{
   l.nchan = s->source_channels;
   l.nbit = s->bits_per_sample;
   l.header_bytes = 0;
   if (s->sourceformat == Mk5B) {
      l.format = SWSGPU_FMT_MARK5B;
      l.frame_bytes = 10000;
      return true;
   }
   if (s->sourceformat == VDIF) {
      l.format = SWSGPU_FMT_VDIF;
      l.frame_bytes = 8000;
      return true;
   }
   if (s->sourceformat == RawSigned || s->sourceformat == RawUnsigned) {
      // header-free sampler data; the frame size only delimits blanking zones
      l.format = s->sourceformat == RawSigned ? SWSGPU_FMT_RAW_SIGNED : SWSGPU_FMT_RAW_UNSIGNED;
      l.frame_bytes = 8192;
      return true;
   }
   if (s->sourceformat == iBOB) {
      l.format = SWSGPU_FMT_RAW_SIGNED;  // 4-byte headers stripped by FileSource, signed samples
      l.frame_bytes = 4096;
      return true;
   }
   why = "source format '" + s->sourceformat_str + "' is not decoded by the GPU core (Mk5B, VDIF, RawSigned, "
         "RawUnsigned, iBob)";
   return false;
}

int precision_from_env()
{
   const char *p = std::getenv("SWSGPU_PRECISION");
   if (!p) return SWSGPU_PREC_FP32;
   if (!strcasecmp(p, "tcsplit")) return SWSGPU_PREC_TCSPLIT;
   if (!strcasecmp(p, "tcsplit_all")) return SWSGPU_PREC_TCSPLIT_ALL;
   return SWSGPU_PREC_FP32;
}

}  // namespace

TaskCoreCUDA::~TaskCoreCUDA()
{
   if (h_) swsgpu_destroy(h_);
   for (void *p : pinned_) swsgpu_host_unregister(p);
}

void TaskCoreCUDA::prepare(swspect_settings_t *s)
{
   cfg_ = s;
   swsgpu_config c;
   std::memset(&c, 0, sizeof(c));
   std::string why;
   if (!layout_of(s, c.layout[0], why)) {
      *s->tlog << "TaskCoreCUDA " << rank_ << ": " << why << std::endl;
      return;
   }
   c.layout[1] = c.layout[0];
   c.num_streams = s->num_sources;
   c.fft_points = (int)s->fft_points;
   c.overlap = s->fft_overlap_factor;
   c.window = window_code(s->wf_type);
   c.precision = precision_from_env();
   c.core_overlapped_ffts = s->core_overlapped_ffts;
   c.num_sources = s->num_sources;
   for (int i = 0; i < s->num_sources; i++) {
      c.source_stream[i] = i;
      c.source_channel[i] = (i == 0) ? s->use_channel_file1 : s->use_channel_file2;  // 0-based after main
      // raw 2-bit multi-channel data with ChannelOrderIncreasing = no keeps
      // channel 0 in the highest bits (TwoBitUnpacker, DataUnpackers.cpp:201-211)
      if (c.layout[0].format >= SWSGPU_FMT_RAW_SIGNED && c.layout[0].nbit == 2 && c.layout[0].nchan % 4 == 0 &&
          !s->channelorder_increasing)
         c.source_channel[i] = c.layout[0].nchan - 1 - c.source_channel[i];
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
   // The dispatcher adds max_buffers_per_spectrum joins into one spectrum,
   // each loop taking one run from every core: with an even split every
   // core's share is summed on the device and copied back once.
   runs_per_output_ = 1;
   if (s->max_buffers_per_spectrum > 1 && s->max_buffers_per_spectrum % s->num_cores == 0)
      runs_per_output_ = s->max_buffers_per_spectrum / s->num_cores;
   c.runs_per_output = runs_per_output_;
   if (swsgpu_create(&c, 0, &h_) != SWSGPU_OK) {
      *s->tlog << "TaskCoreCUDA " << rank_ << ": " << swsgpu_last_error(nullptr) << std::endl;
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
   size_t shortest = (size_t)-1;
   for (int s = 0; s < cfg_->num_sources; s++) shortest = std::min(shortest, inbuf[s]->getLength());
   const int64_t run = runs_++;
   for (int s = 0; s < cfg_->num_sources; s++) {
      raw[s] = inbuf[s]->getData();
      nbytes[s] = shortest;  // doMaths walks the shortest source buffer
      // the raw buffers live for the whole run (src/swspectrometer.cpp:
      // 373-413): page-lock each on first sight so its copy is a DMA
      void *p = inbuf[s]->getData();
      if (std::find(pinned_.begin(), pinned_.end(), p) == pinned_.end() &&
          swsgpu_host_register(p, inbuf[s]->getAllocated()) == SWSGPU_OK)
         pinned_.push_back(p);
      // core `rank_` gets every num_cores-th buffer of each source: the
      // payload offset places mark5access's per-frame blanking zones
      offs[s] = (run * cfg_->num_cores + rank_) * (int64_t)cfg_->rawbuf_size;
   }
   int nspec = 0, nffts = 0, partial = 0;
   swsgpu_run_shape(h_, shortest, &nspec, &nffts, &partial);
   run_nspec_ = nspec;
   ffts_ += (int64_t)nffts * cfg_->num_sources;
   if (swsgpu_submit(h_, raw, nbytes, offs) != SWSGPU_OK) {
      *cfg_->tlog << "TaskCoreCUDA " << rank_ << " run: " << swsgpu_last_error(h_) << std::endl;
      return -1;
   }
   return 0;
}

int TaskCoreCUDA::join()
{
   if (!h_) return -1;
   int ready = 0;
   if (swsgpu_wait(h_, -1, &ready) != SWSGPU_OK) {
      *cfg_->tlog << "TaskCoreCUDA " << rank_ << " join: " << swsgpu_last_error(h_) << std::endl;
      return -1;
   }
   fetched_ = false;
   if (ready > 0) {
      const size_t S = cfg_->fft_ssb_points;
      staged_.resize((size_t)ready * cfg_->num_sources * S);
      stagedx_.resize((size_t)ready * cfg_->num_xpols * S * 2 + 1);
      stagedp_.resize((size_t)ready * cfg_->num_sources * cfg_->pcal_tonebins * 2 + 1);
      swsgpu_outputs o = {};
      o.auto_out = staged_.data();
      o.xpol_out = cfg_->num_xpols ? stagedx_.data() : nullptr;
      o.pcal_out = cfg_->extract_PCal ? stagedp_.data() : nullptr;
      if (swsgpu_fetch(h_, &o) != SWSGPU_OK) return -1;
      // the C ABI writes [spectrum][source][bin]; the reference keeps one
      // buffer per source with its spectra back to back
      for (int s = 0; s < cfg_->num_sources; s++) {
         float *dst = reinterpret_cast<float *>(out_[s]->getData());
         for (int k = 0; k < ready; k++)
            std::memcpy(dst + k * S, staged_.data() + ((size_t)k * cfg_->num_sources + s) * S, S * sizeof(float));
         out_[s]->setLength(cfg_->fft_bytes_ssb * ready);
         if (cfg_->extract_PCal) {
            float *pd = reinterpret_cast<float *>(pcal_[s]->getData());
            const size_t tb = (size_t)cfg_->pcal_tonebins * 2;
            for (int k = 0; k < ready; k++)
               std::memcpy(pd + k * tb, stagedp_.data() + ((size_t)k * cfg_->num_sources + s) * tb, tb * sizeof(float));
            pcal_[s]->setLength(cfg_->pcal_result_bytes * ready);
         }
      }
      for (int x = 0; x < cfg_->num_xpols; x++) {
         float *dst = reinterpret_cast<float *>(xpol_[x]->getData());
         for (int k = 0; k < ready; k++)
            std::memcpy(dst + k * 2 * S, stagedx_.data() + ((size_t)k * cfg_->num_xpols + x) * 2 * S,
                        2 * S * sizeof(float));
         xpol_[x]->setLength(cfg_->fft_bytes_xpol * ready);
      }
      fetched_ = true;
   }
   // TaskCore::join returns the number of complete spectra of the run
   // (TaskCoreIPP::join, src/IA-32/TaskCoreIPP.cpp:173-183)
   return run_nspec_;
}

int TaskCoreCUDA::combineResults(Buffer **outbuf, Buffer **pcalbuf)
{
   if (!out_ || !outbuf || !pcalbuf) {
      std::cerr << "TaskCoreCUDA combineResults: null buffer(s)" << std::endl;
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
         // the length TaskCoreIPP::combineResults sets (TaskCoreIPP.cpp:333)
         outbuf[xo]->setLength(sizeof(float) * S);
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
   if (buf) std::memset(buf->getData(), 0, buf->getAllocated());
}

int TaskCoreCUDA::finalize()
{
   if (cfg_ && cfg_->tlog)
      *cfg_->tlog << "TaskCoreCUDA " << rank_ << ": " << runs_ << " runs, " << ffts_ << " FFTs" << std::endl;
   if (h_) swsgpu_destroy(h_);
   h_ = nullptr;
   for (void *p : pinned_) swsgpu_host_unregister(p);
   pinned_.clear();
   return 0;
}
