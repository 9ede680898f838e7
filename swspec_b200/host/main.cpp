// main.cpp -- command-line front end (src/swspectrometer.cpp:46-427) with the
// GPU core in place of the IPP core:
//   swspectrometer_gpu <inifile> <infile1> [<infile2>]
//   swspectrometer_gpu --print-settings <inifile> [ninputs]   (no GPU needed)
//   swspectrometer_gpu --read-source <inifile> <infile> <outfile>  (no GPU needed)
#include <cstring>
#include <fstream>
#include <streambuf>

#include "sws_host.h"

using namespace swshost;

// stream that writes to two streambufs (the reference's TeeStream)
class TeeBuf : public std::streambuf {
public:
   TeeBuf(std::streambuf *a, std::streambuf *b) : a_(a), b_(b) {}

protected:
   int overflow(int c) override
   {
      if (c == EOF) return !EOF;
      const int r1 = a_->sputc((char)c), r2 = b_->sputc((char)c);
      return (r1 == EOF || r2 == EOF) ? EOF : c;
   }
   int sync() override { return (a_->pubsync() == 0 && b_->pubsync() == 0) ? 0 : -1; }

private:
   std::streambuf *a_, *b_;
};

int main(int argc, char *argv[])
{
   std::string err;
   if (argc >= 3 && strcmp(argv[1], "--print-settings") == 0) {
      Settings s;
      if (load_ini(s, argv[2], err) || parse_format(s, err) || derive(s, argc >= 4 ? atoi(argv[3]) : 1, err)) {
         std::cerr << "Error: " << err << std::endl;
         return 1;
      }
      std::cout << settings_json(s) << std::endl;
      return 0;
   }
   if (argc == 5 && strcmp(argv[1], "--read-source") == 0) {
      // the front end alone: read <infile> into buffers of the INI's raw
      // buffer size, append the payload bytes to <outfile>, print one JSON
      // line with the buffer lengths; messages go to stderr and the start
      // timing to <outfile>.starttiming.txt (no GPU needed)
      Settings s;
      if (load_ini(s, argv[2], err) || parse_format(s, err) || derive(s, 1, err)) {
         std::cerr << "Error: " << err << std::endl;
         return 1;
      }
      std::ofstream st(std::string(argv[4]) + ".starttiming.txt");
      s.tlog = &std::cerr;
      s.startlog = &st;
      FileSource f(&s);
      if (f.open(argv[3])) return 2;
      std::ofstream o(argv[4], std::ios::binary);
      Buffer b(s.rawbuf_size);
      std::cout << "{\"buffers\": [";
      for (int k = 0; !f.eof(); k++) {
         const int n = f.read(&b);
         o.write(b.getData(), n);
         std::cout << (k ? ", " : "") << n;
      }
      std::cout << "], \"frames\": " << f.frames_read() << ", \"bad_sync_frames\": " << f.bad_sync_frames() << "}"
                << std::endl;
      f.close();
      return 0;
   }
   std::cout << std::endl << "SWSpec GPU core (sm_100a)" << std::endl << std::endl;
   if (!(argc == 3 || argc == 4)) {
      std::cout << " Usage: swspectrometer_gpu <inifile> <infile1> [<infile2>]" << std::endl;
      return 0;
   }
   Settings set;
   if (load_ini(set, argv[1], err) || parse_format(set, err) || derive(set, argc - 2, err)) {
      std::cerr << "Error: " << err << std::endl;
      return -1;
   }
   std::ofstream runlog(set.basefilename1 + "_runlog.txt");
   std::ofstream startlog(set.basefilename1 + "_starttiming.txt");
   TeeBuf tee(std::cerr.rdbuf(), runlog.rdbuf());
   std::ostream tlog(&tee);
   set.tlog = &tlog;
   set.startlog = &startlog;
   std::ostream &out = tlog;
   out << "Config file  : " << argv[1] << std::endl;
   out << "Input file 1 : " << argv[2] << std::endl;
   out << "Input file 2 : " << (argc == 4 ? argv[3] : "") << std::endl;
   out << "File format  : " << set.bits_per_sample << " bits/sample, " << set.source_channels << " channels, selected "
       << "channel " << (set.use_channel_file1 + 1) << " of input 1, channel " << (set.use_channel_file2 + 1)
       << " of input 2" << std::endl;
   out << "DFT info     : " << set.fft_points << " points, " << set.df << " Hz resolution, " << set.averaged_ffts
       << "-fold averaging, " << 100.0 * (1.0 - 1.0 / set.fft_overlap_factor) << "% overlap" << std::endl;
   out << "Raw buffers  : " << set.rawbuf_size / 1024.0 << " kB per source" << std::endl;

   const std::string out1 = set.basefilename1 + "_swspec.bin", out2 = set.basefilename2 + "_swspec.bin";
   const std::string pcal1 = set.basefilename1 + "_pcal.bin", pcal2 = set.basefilename2 + "_pcal.bin";
   const std::string outx = set.basefilename1 + "_xpol_swspec.bin";
   auto add_source = [&](const char *uri) {
      FileSource *f = new FileSource(&set);
      if (f->open(uri)) return false;
      set.sources.push_back(f);
      return true;
   };
   auto add_sink = [&](const std::string &uri, std::vector<DataSink *> &v) {
      FileSink *k = new FileSink(&set);
      if (k->open(uri)) return false;
      v.push_back(k);
      return true;
   };
   if (!add_source(argv[2]) || !add_sink(out1, set.sinks) || (set.extract_PCal && !add_sink(pcal1, set.pcalsinks))) {
      out << "Error: could not open input 1 or its outputs" << std::endl;
      return -1;
   }
   if (argc == 4) {
      if (!add_source(argv[3]) || !add_sink(out2, set.sinks) || (set.extract_PCal && !add_sink(pcal2, set.pcalsinks))) {
         out << "Error: could not open input 2 or its outputs" << std::endl;
         return -1;
      }
   }
   if (set.calc_Xpol) {
      if (!add_sink(outx, set.sinks)) return -1;
      set.num_xpols = 1;
   }
   set.num_sources = (int)set.sources.size();
   set.num_sinks = (int)set.sinks.size();
   // double-buffered raw buffers [core][2][source] and output buffers (swspectrometer.cpp:373-413)
   set.rawbuffers.resize(set.num_cores);
   set.outbuffers.resize(set.num_cores);
   set.outbuffersXpol.resize(set.num_cores);
   set.outbuffersPCal.resize(set.num_cores);
   const size_t nsp = std::max(set.max_spectra_per_buffer, 1);
   for (int c = 0; c < set.num_cores; c++) {
      set.rawbuffers[c].resize(2);
      for (int b = 0; b < 2; b++)
         for (int s = 0; s < set.num_sources; s++) set.rawbuffers[c][b].push_back(new Buffer(set.rawbuf_size));
      for (int s = 0; s < set.num_sources; s++) {
         set.outbuffers[c].push_back(new Buffer(nsp * set.fft_bytes_ssb));
         set.outbuffersPCal[c].push_back(new Buffer(std::max<size_t>(nsp * set.pcal_result_bytes, 8)));
      }
      for (int x = 0; x < set.num_xpols; x++) set.outbuffersXpol[c].push_back(new Buffer(nsp * set.fft_bytes_xpol));
   }
   {
      TaskDispatcher td(&set);
      td.run();
   }
   for (auto &cb : set.rawbuffers)
      for (auto &bb : cb)
         for (Buffer *b : bb) delete b;
   for (auto *v : {&set.outbuffers, &set.outbuffersXpol, &set.outbuffersPCal})
      for (auto &cb : *v)
         for (Buffer *b : cb) delete b;
   for (DataSource *s : set.sources) delete s;
   for (DataSink *k : set.sinks) delete k;
   for (DataSink *k : set.pcalsinks) delete k;
   return 0;
}
