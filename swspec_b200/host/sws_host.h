// sws_host.h -- C++ host side of the GPU spectrometer core.
//
// Mirrors the reference's host classes so that the GPU core drops in behind
// the same dispatcher, INI settings and output files:
//   Settings       <- swspect_settings_t (src/Settings.h:59-159) and the
//                     derivation in main() (src/swspectrometer.cpp:67-231)
//   IniParser      <- src/IniParser.cpp:48-265
//   Buffer         <- src/Buffer.cpp:32-100
//   FileSource     <- src/FileSource.cpp:36-250 (framed formats, headers stripped)
//   FileSink       <- src/FileSink.cpp:31-110
//   TaskCore       <- src/TaskCore.h:36-89 (abstract core)
//   TaskCoreCUDA   -- the GPU core over include/swsgpu.h
//   TaskDispatcher <- src/TaskDispatcher.cpp:38-247
#pragma once

#include <cstddef>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "swsgpu.h"

namespace swshost {

enum WindowFunctionType { None, Cosine, Cosine2, Hamming, Hann, Blackman, BlackmanHarris };
enum OutputFormat { Ascii, Binary };
enum InputFormat { Unknown = -1, RawSigned, RawUnsigned, Mk5B, iBOB, VDIF, VLBA, MKIV, Mark5B, Maxim };

typedef float swsfloat_t;

class Buffer {
public:
   explicit Buffer(size_t bytes);
   ~Buffer();
   Buffer(const Buffer &) = delete;
   Buffer &operator=(const Buffer &) = delete;
   char *getData() { return data_; }
   size_t getLength() const { return length_; }
   size_t getAllocated() const { return allocated_; }
   void setLength(size_t len) { length_ = len; }

private:
   char *data_ = nullptr;
   size_t length_ = 0, allocated_ = 0;
};

class IniParser {
public:
   explicit IniParser(const std::string &filename);
   bool selectSection(const std::string &name);
   bool hasKey(const std::string &key) const;
   bool getKeyValue(const char *key, std::string &value) const;
   bool getKeyValue(const char *key, int &value) const;
   bool getKeyValue(const char *key, size_t &value) const;
   bool getKeyValue(const char *key, float &value) const;
   bool getKeyValue(const char *key, bool &value) const;
   bool ok() const { return opened_; }

private:
   struct KV {
      std::string key, value;
   };
   struct Section {
      std::string name;
      std::vector<KV> entries;
   };
   std::vector<Section> sections_;
   int section_index_ = -1;
   bool opened_ = false;
};

WindowFunctionType parse_Windowing(const char *str);
bool parse_YesNo(const char *str);
long long gcd(long long a, long long b);

class DataSource;
class DataSink;

struct Settings {
   // INI / command line
   int num_cores = 1;
   size_t max_rawbuf_size = 32u * 1024u * 1024u;  // PLATFORM_MAX_RAW_BUF_SIZE_MB of the IPP build
   size_t fft_points = 320000;
   swsfloat_t fft_integ_seconds = 20;
   int fft_overlap_factor = 2;
   WindowFunctionType wf_type = Cosine2;
   int bits_per_sample = 8;
   bool channelorder_increasing = true;
   int seconds_to_skip = 0;
   int source_channels = 1;
   int use_channel_file1 = 1;  // 1-based in the INI, 0-based after derive()
   int use_channel_file2 = 1;
   swsfloat_t samplingfreq = 16e6;
   swsfloat_t pcaloffsethz = 10e3;
   swsfloat_t pcalharmonicshz = 1e6;
   bool extract_PCal = false;
   bool calc_Xpol = false;
   bool costas_loop = false;
   bool use_live_plot = false;
   std::string basefilename1_pattern = "ProjDate_StationID_Instrument_ScanNo_%fftpoints%_%integrtime%_%channel%";
   std::string basefilename2_pattern;
   std::string sourceformat_str = "RawSigned";
   OutputFormat sinkformat = Binary;
   // GPU core keys (new; the reference's parser ignores unknown keys)
   int gpu_precision = SWSGPU_PREC_FP32;  // GpuPrecision = FP32 | TCSPLIT
   int gpu_device = 0;                    // GpuDevice
   int vdif_thread = -1;                  // VdifThread: keep only the frames of this VDIF thread (-1: all)
   bool gpu_combine_on_device = true;     // GpuCombineOnDevice
   bool gpu_autotune = false;             // GpuAutotune: time the four-step splits of the length at prepare
   bool fix_xpol_length = false;          // FixXpolLength (reference quirk: half of XY* written)
   // counts
   int num_sources = 0, num_sinks = 0, num_xpols = 0;
   InputFormat sourceformat = Unknown;
   // derived
   std::string basefilename1, basefilename2;
   swsfloat_t dt = 0, df = 0;
   int averaged_ffts = 0, averaged_overlapped_ffts = 0;
   int fft_overlap_points = 0, fft_ssb_points = 0;
   double rawbytes_per_channelsample = 0;
   size_t raw_fullfft_bytes = 0, raw_overlap_bytes = 0;
   size_t fft_bytes = 0, fft_bytes_ssb = 0, fft_bytes_xpol = 0;
   size_t rawbuf_size = 0;
   int max_spectra_per_buffer = 0, max_specffts_per_buffer = 0, max_buffers_per_spectrum = 0;
   int core_overlapped_ffts = 0, core_averaged_ffts = 0;
   int pcal_tonebins = 0, pcal_rotatorlen = 0, pcal_pulses = 0, pcal_pulses_per_fft = 0;
   size_t pcal_result_bytes = 0;
   // stream layout (from the source format string)
   swsgpu_layout layout = {SWSGPU_FMT_MARK5B, 1, 2, 10000, 0};
   // runtime objects
   std::vector<DataSource *> sources;
   std::vector<DataSink *> sinks;
   std::vector<DataSink *> pcalsinks;
   std::vector<std::vector<std::vector<Buffer *>>> rawbuffers;  // [core][2][source]
   std::vector<std::vector<Buffer *>> outbuffers;               // [core][source]
   std::vector<std::vector<Buffer *>> outbuffersXpol;           // [core][xpol]
   std::vector<std::vector<Buffer *>> outbuffersPCal;           // [core][source]
   std::ostream *tlog = &std::cerr;
   std::ofstream *startlog = nullptr;
};

// INI keys of src/swspectrometer.cpp:103-145 (+ the GPU keys above).
int load_ini(Settings &s, const std::string &inifile, std::string &err);
// Checks and derived parameters of src/swspectrometer.cpp:147-231.
int derive(Settings &s, int ninputs, std::string &err);
std::string cfg_to_filename(std::string pattern, const Settings &s, int filenr);
// Stream layout of a source format string (Mark5B-<Mbps>-<nch>-<nbit>,
// VDIF_<payload>-<Mbps>-<nch>-<nbit>, Mk5B, VDIF with the INI's bits/channels).
int parse_format(Settings &s, std::string &err);
std::string settings_json(const Settings &s);

class DataSource {
public:
   virtual ~DataSource() {}
   virtual int open(const std::string &uri) = 0;
   virtual int read(Buffer *buf) = 0;
   virtual int close() = 0;
   virtual bool eof() = 0;
   // payload byte offset (within the recording) of the buffer filled last
   virtual int64_t last_payload_offset() const = 0;
};

// Framed recordings: locates the first frame, then fills buffers with
// payload bytes only (headers stripped), like the reference's framed path
// (FileSource.cpp:184-215).  Writes the first frame's time to the
// start-timing log.
class FileSource : public DataSource {
public:
   explicit FileSource(Settings *s) : cfg_(s) {}
   int open(const std::string &uri) override;
   int read(Buffer *buf) override;
   int close() override;
   bool eof() override { return got_eof_; }
   int64_t last_payload_offset() const override { return last_offset_; }

private:
   Settings *cfg_;
   std::ifstream ifile_;
   bool got_eof_ = false;
   int frame_bytes_ = 0, header_bytes_ = 0;
   int64_t first_frame_ = 0;
   int64_t in_frame_ = 0;       // payload bytes of the current frame already consumed
   int64_t payload_total_ = 0;  // payload bytes delivered so far
   int64_t last_offset_ = 0;
   int64_t frames_ = 0;         // frame headers consumed so far
   int64_t bad_sync_ = 0;       // of them, Mark5B headers without the sync word
   bool pending_header_ = true;

public:
   int64_t frames_read() const { return frames_; }
   int64_t bad_sync_frames() const { return bad_sync_; }
};

class DataSink {
public:
   virtual ~DataSink() {}
   virtual int open(const std::string &uri) = 0;
   virtual size_t write(Buffer *buf) = 0;
   virtual int close() = 0;
};

class FileSink : public DataSink {
public:
   explicit FileSink(const Settings *s) : cfg_(s) {}
   int open(const std::string &uri) override;
   size_t write(Buffer *buf) override;
   int close() override;

private:
   const Settings *cfg_;
   std::ofstream ofile_;
};

class TaskCore {
public:
   virtual ~TaskCore() {}
   virtual void prepare(Settings *settings) = 0;
   virtual int run(Buffer **inbuf, Buffer **outbuf, Buffer **xpolbuf, Buffer **pcalbuf) = 0;
   virtual int join() { return 1; }
   virtual int finalize() { return 0; }
   virtual int combineResults(Buffer **outbuf, Buffer **pcalbuf) { return 0; }
   virtual void resetBuffer(Buffer *buf) {}
};

class TaskCoreCUDA : public TaskCore {
public:
   explicit TaskCoreCUDA(int rank) : rank_(rank) {}
   ~TaskCoreCUDA() override;
   void prepare(Settings *settings) override;
   int run(Buffer **inbuf, Buffer **outbuf, Buffer **xpolbuf, Buffer **pcalbuf) override;
   int join() override;
   int finalize() override;
   int combineResults(Buffer **outbuf, Buffer **pcalbuf) override;
   void resetBuffer(Buffer *buf) override;
   bool ok() const { return h_ != nullptr; }

private:
   int rank_;
   Settings *cfg_ = nullptr;
   swsgpu_handle *h_ = nullptr;
   Buffer **out_ = nullptr, **xpol_ = nullptr, **pcal_ = nullptr;
   bool fetched_ = false;  // out_/xpol_/pcal_ hold spectra not yet combined
   int run_nspec_ = 0;
   int64_t total_ffts_ = 0, total_runs_ = 0;
   int64_t t_submit_ = 0;
   double total_runtime_ = 0;
   std::vector<float> staged_, stagedx_, stagedp_;
   std::vector<void *> pinned_;  // raw buffers page-locked for asynchronous input copies
};

class TaskDispatcher {
public:
   explicit TaskDispatcher(Settings *s);
   ~TaskDispatcher();
   void run();

private:
   Settings *set_;
   std::vector<TaskCore *> cores_;
   std::vector<Buffer *> corecombined_spectra_;
   std::vector<Buffer *> corecombined_pcals_;
};

}  // namespace swshost
