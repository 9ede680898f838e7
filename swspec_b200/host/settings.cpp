// settings.cpp -- INI keys and derived parameters of the spectrometer run,
// as main() computes them (src/swspectrometer.cpp:67-231).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <sstream>
#include <strings.h>

#include "sws_host.h"

namespace swshost {

int load_ini(Settings &s, const std::string &inifile, std::string &err)
{
   IniParser ini(inifile);
   if (!ini.ok() || !ini.selectSection("Spectrometer")) {
      err = "INI could not be read or it is missing the [Spectrometer] section";
      return -1;
   }
   std::string keyval;
   ini.getKeyValue("NumCPUCores", s.num_cores);
   if (ini.getKeyValue("MaxSourceBufferMB", s.max_rawbuf_size)) s.max_rawbuf_size *= 1024 * 1024 / 2;
   ini.getKeyValue("FFTpoints", s.fft_points);
   ini.getKeyValue("FFTIntegrationTimeSec", s.fft_integ_seconds);
   ini.getKeyValue("FFToverlapFactor", s.fft_overlap_factor);
   if (ini.getKeyValue("WindowType", keyval)) s.wf_type = parse_Windowing(keyval.c_str());
   if (ini.getKeyValue("BandwidthHz", s.samplingfreq)) s.samplingfreq *= 2.0f;
   ini.getKeyValue("PCalOffsetHz", s.pcaloffsethz);
   ini.getKeyValue("SourceFormat", s.sourceformat_str);
   ini.getKeyValue("SourceSkipSeconds", s.seconds_to_skip);
   ini.getKeyValue("BitsPerSample", s.bits_per_sample);
   ini.getKeyValue("ChannelOrderIncreasing", s.channelorder_increasing);
   ini.getKeyValue("SourceChannels", s.source_channels);
   ini.getKeyValue("UseFile1Channel", s.use_channel_file1);
   ini.getKeyValue("UseFile2Channel", s.use_channel_file2);
   ini.getKeyValue("ExtractPCal", s.extract_PCal);
   ini.getKeyValue("PlotProgress", s.use_live_plot);
   ini.getKeyValue("DoCrossPolarization", s.calc_Xpol);
   ini.getKeyValue("DoCostasLoop", s.costas_loop);
   keyval.clear();
   ini.getKeyValue("SinkFormat", keyval);
   if (strcasecmp(keyval.c_str(), "ASCII") == 0) s.sinkformat = Ascii;
   if (!ini.getKeyValue("BaseFilename1", s.basefilename1_pattern)) {
      err = "BaseFilename1 setting is missing from the INI file!";
      return -1;
   }
   if (!ini.getKeyValue("BaseFilename2", s.basefilename2_pattern)) {
      std::cerr << "Note: the INI has no BaseFilename2; the second input's files are named after "
                   "BaseFilename1 with '_file2' appended" << std::endl;
      s.basefilename2_pattern = s.basefilename1_pattern + "_file2";
   }
   // keys of the GPU core
   if (ini.getKeyValue("GpuPrecision", keyval))
      s.gpu_precision = (strcasecmp(keyval.c_str(), "TCSPLIT") == 0)       ? SWSGPU_PREC_TCSPLIT
                        : (strcasecmp(keyval.c_str(), "TCSPLIT_ALL") == 0) ? SWSGPU_PREC_TCSPLIT_ALL
                                                                            : SWSGPU_PREC_FP32;
   ini.getKeyValue("GpuDevice", s.gpu_device);
   ini.getKeyValue("VdifThread", s.vdif_thread);
   ini.getKeyValue("GpuCombineOnDevice", s.gpu_combine_on_device);
   ini.getKeyValue("GpuAutotune", s.gpu_autotune);
   ini.getKeyValue("FixXpolLength", s.fix_xpol_length);
   return 0;
}

std::string cfg_to_filename(std::string pattern, const Settings &s, int filenr)
{
   const int ch = (filenr == 1) ? s.use_channel_file1 : s.use_channel_file2;
   const std::pair<std::string, std::string> keys[3] = {
       {"%fftpoints%", std::to_string((int)s.fft_points)},
       {"%integrtime%", std::to_string((int)s.fft_integ_seconds)},
       {"%channel%", std::to_string(ch + 1)}};
   std::replace(pattern.begin(), pattern.end(), ' ', '_');
   std::string fn = pattern;
   for (const auto &k : keys) {
      while (true) {
         size_t idx = fn.find(k.first, 0);
         if (idx == std::string::npos) break;
         fn.replace(idx, k.first.length(), k.second);
      }
   }
   return fn;
}

int parse_format(Settings &s, std::string &err)
{
   const std::string &f = s.sourceformat_str;
   int mbps = 0, nch = 0, nbit = 0, payload = 0;
   if (strncasecmp(f.c_str(), "Mark5B-", 7) == 0 && sscanf(f.c_str() + 7, "%d-%d-%d", &mbps, &nch, &nbit) == 3) {
      s.sourceformat = Mark5B;
      s.layout = {SWSGPU_FMT_MARK5B, nch, nbit, 10000, 0};
      s.source_channels = nch;
      s.bits_per_sample = nbit;
   } else if (strncasecmp(f.c_str(), "VDIF_", 5) == 0 &&
              sscanf(f.c_str() + 5, "%d-%d-%d-%d", &payload, &mbps, &nch, &nbit) == 4) {
      s.sourceformat = VDIF;
      s.layout = {SWSGPU_FMT_VDIF, nch, nbit, payload, 0};
      s.source_channels = nch;
      s.bits_per_sample = nbit;
   } else if ((strncasecmp(f.c_str(), "VLBA1_", 6) == 0 || strncasecmp(f.c_str(), "MKIV1_", 6) == 0) &&
              sscanf(f.c_str() + 6, "%d-%d-%d-%d", &payload, &mbps, &nch, &nbit) == 4) {
      // mark5access's VLBA1_<fanout>-<Mbps>-<nchan>-<nbit> and MKIV1_ modes:
      // frames of 20000 track-words of nchan * nbit * fanout tracks; the GPU
      // core takes VLBA payloads with the headers removed, Mark4 frames whole
      const bool vlba = strncasecmp(f.c_str(), "VLBA1_", 6) == 0;
      const int fanout = payload, ntrack = nch * nbit * fanout;
      if ((fanout != 1 && fanout != 2 && fanout != 4) || (ntrack != 8 && ntrack != 16 && ntrack != 32 && ntrack != 64)) {
         err = "source format '" + f + "': fanout 1, 2 or 4 and 8, 16, 32 or 64 tracks";
         return -1;
      }
      s.sourceformat = vlba ? VLBA : MKIV;
      s.layout = {vlba ? SWSGPU_FMT_VLBA : SWSGPU_FMT_MARK4, nch, nbit, 2500 * ntrack, 0};
      s.source_channels = nch;
      s.bits_per_sample = nbit;
   } else if (strcasecmp(f.c_str(), "Mk5B") == 0) {
      // the reference's framed Mark5B: 16-byte headers, 10000-byte payloads
      s.sourceformat = Mk5B;
      s.layout = {SWSGPU_FMT_MARK5B, s.source_channels, s.bits_per_sample, 10000, 0};
   } else if (strcasecmp(f.c_str(), "VDIF") == 0) {
      // the reference's framed VDIF: 16-byte legacy headers, 8000-byte payloads
      s.sourceformat = VDIF;
      s.layout = {SWSGPU_FMT_VDIF, s.source_channels, s.bits_per_sample, 8000, 0};
   } else if (strcasecmp(f.c_str(), "RawSigned") == 0 || strcasecmp(f.c_str(), "RawUnsigned") == 0) {
      // header-free sampler data (the reference's default format); the frame
      // size only delimits blanking zones, and raw data has none
      const bool sgn = strcasecmp(f.c_str(), "RawSigned") == 0;
      s.sourceformat = sgn ? RawSigned : RawUnsigned;
      s.layout = {sgn ? SWSGPU_FMT_RAW_SIGNED : SWSGPU_FMT_RAW_UNSIGNED, s.source_channels, s.bits_per_sample, 8192, 0};
   } else if (strcasecmp(f.c_str(), "iBob") == 0) {
      // iBOB UDP captures: 4-byte sequence headers, 4096-byte payloads of
      // signed samples (src/FileSource.cpp:53-57, DataUnpackerFactory.h:91-95)
      s.sourceformat = iBOB;
      s.layout = {SWSGPU_FMT_RAW_SIGNED, s.source_channels, s.bits_per_sample, 4096, 0};
   } else {
      err = "source format '" + f + "' is not decoded by the GPU core (Mark5B-*, VDIF_*, VLBA1_*, MKIV1_*, Mk5B, "
            "VDIF, RawSigned, RawUnsigned, iBob)";
      return -1;
   }
   if (nbit != 0 && nbit != 1 && nbit != 2 && nbit != 8) {
      err = "GPU core decodes 1, 2 or 8 bits per sample";
      return -1;
   }
   return 0;
}

int derive(Settings &s, int ninputs, std::string &err)
{
   if (s.use_channel_file1 < 1 || s.use_channel_file1 > s.source_channels) {
      err = "UseFile1Channel setting " + std::to_string(s.use_channel_file1) + " is an invalid channel number";
      return -1;
   }
   if (s.use_channel_file2 < 1 || s.use_channel_file2 > s.source_channels) {
      err = "UseFile2Channel setting " + std::to_string(s.use_channel_file2) + " is an invalid channel number";
      return -1;
   }
   if (s.calc_Xpol && ninputs != 2) {
      std::cerr << "Note: cross-polarisation needs two input files; one was given, so no cross spectrum "
                   "is computed" << std::endl;
      s.calc_Xpol = false;
   }
   s.use_channel_file1--;
   s.use_channel_file2--;
   // swsfloat_t arithmetic as in the reference
   s.dt = 1.0f / s.samplingfreq;
   s.df = s.samplingfreq / (swsfloat_t)s.fft_points;
   s.averaged_ffts = (int)((s.samplingfreq * s.fft_integ_seconds) / (swsfloat_t)s.fft_points);
   s.fft_overlap_points = (int)(s.fft_points / s.fft_overlap_factor);
   s.fft_ssb_points = (int)(s.fft_points / 2) + 1;
   s.rawbytes_per_channelsample = (s.bits_per_sample * s.source_channels) / 8.0;
   s.raw_fullfft_bytes = (size_t)(int)(s.fft_points * s.rawbytes_per_channelsample);
   s.raw_overlap_bytes = (size_t)(int)(s.fft_overlap_points * s.rawbytes_per_channelsample);
   s.fft_bytes = s.fft_points * sizeof(swsfloat_t);
   s.fft_bytes_ssb = s.fft_ssb_points * sizeof(swsfloat_t);
   s.fft_bytes_xpol = 2 * s.fft_bytes_ssb;
   if (s.extract_PCal) {
      if (s.pcaloffsethz == 0) {
         err = "PCalOffsetHz must be nonzero";
         return -1;
      }
      s.pcal_tonebins = (int)(s.samplingfreq / s.pcalharmonicshz);
      s.pcal_rotatorlen = (int)(s.samplingfreq / (swsfloat_t)gcd((long long)s.samplingfreq, (long long)s.pcaloffsethz));
      s.pcal_pulses = s.pcal_rotatorlen / s.pcal_tonebins;
      s.pcal_result_bytes = s.pcal_tonebins * 2 * sizeof(float);
      s.pcal_pulses_per_fft = (int)(s.fft_points / s.pcal_rotatorlen);
      if ((s.fft_points % s.pcal_rotatorlen) != 0) {
         std::cerr << "Note: phase-cal extraction is off: the rotator period of " << s.pcal_rotatorlen
                   << " samples does not divide the " << s.fft_points << "-point FFT" << std::endl;
         s.extract_PCal = false;
      }
   }
   if (!s.extract_PCal) {
      s.pcal_tonebins = s.pcal_rotatorlen = s.pcal_pulses = s.pcal_pulses_per_fft = 0;
      s.pcal_result_bytes = 0;
   }
   s.max_rawbuf_size = s.max_rawbuf_size / s.num_cores;
   size_t tent = s.raw_fullfft_bytes * s.averaged_ffts;
   if (tent > s.max_rawbuf_size) {
      s.max_spectra_per_buffer = 0;
      s.max_specffts_per_buffer = 1;
      s.max_buffers_per_spectrum = s.averaged_ffts;
      tent = s.raw_fullfft_bytes;
      while (tent <= s.max_rawbuf_size && (s.max_buffers_per_spectrum % 2) == 0) {
         tent *= 2;
         s.max_buffers_per_spectrum /= 2;
         s.max_specffts_per_buffer *= 2;
      }
   } else {
      s.max_spectra_per_buffer = 1;
      s.max_specffts_per_buffer = s.averaged_ffts;
      s.max_buffers_per_spectrum = 0;
      while (2 * tent <= s.max_rawbuf_size) {
         tent *= 2;
         s.max_spectra_per_buffer *= 2;
      }
   }
   s.rawbuf_size = tent;
   s.core_averaged_ffts = s.max_specffts_per_buffer;
   s.core_overlapped_ffts = s.fft_overlap_factor * s.max_specffts_per_buffer - (s.fft_overlap_factor - 1);
   s.basefilename1 = cfg_to_filename(s.basefilename1_pattern, s, 1);
   // the reference derives both names from BaseFilename1 (swspectrometer.cpp:234-235)
   s.basefilename2 = cfg_to_filename(s.basefilename1_pattern, s, 2);
   return 0;
}

std::string settings_json(const Settings &s)
{
   std::ostringstream o;
   o << "{\"fft_points\": " << s.fft_points << ", \"samplingfreq\": " << s.samplingfreq
     << ", \"averaged_ffts\": " << s.averaged_ffts << ", \"fft_ssb_points\": " << s.fft_ssb_points
     << ", \"raw_fullfft_bytes\": " << s.raw_fullfft_bytes << ", \"raw_overlap_bytes\": " << s.raw_overlap_bytes
     << ", \"rawbuf_size\": " << s.rawbuf_size << ", \"max_spectra_per_buffer\": " << s.max_spectra_per_buffer
     << ", \"max_specffts_per_buffer\": " << s.max_specffts_per_buffer
     << ", \"max_buffers_per_spectrum\": " << s.max_buffers_per_spectrum
     << ", \"core_overlapped_ffts\": " << s.core_overlapped_ffts << ", \"extract_PCal\": " << (s.extract_PCal ? 1 : 0)
     << ", \"pcal_tonebins\": " << s.pcal_tonebins << ", \"pcal_rotatorlen\": " << s.pcal_rotatorlen
     << ", \"pcal_pulses_per_fft\": " << s.pcal_pulses_per_fft << ", \"wf_type\": " << (int)s.wf_type
     << ", \"use_channel_file1\": " << s.use_channel_file1 << ", \"use_channel_file2\": " << s.use_channel_file2
     << ", \"source_channels\": " << s.source_channels << ", \"bits_per_sample\": " << s.bits_per_sample
     << ", \"calc_Xpol\": " << (s.calc_Xpol ? 1 : 0) << ", \"sinkformat\": \"" << (s.sinkformat == Ascii ? "ascii" : "binary")
     << "\", \"basefilename1\": \"" << s.basefilename1 << "\", \"basefilename2\": \"" << s.basefilename2
     << "\", \"gpu_precision\": " << s.gpu_precision << ", \"gpu_autotune\": " << (s.gpu_autotune ? 1 : 0) << "}";
   return o.str();
}

}  // namespace swshost
