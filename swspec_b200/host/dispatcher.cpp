// dispatcher.cpp -- TaskDispatcher (src/TaskDispatcher.cpp:38-247): prefill,
// run every core on its buffers, read the next buffers meanwhile, join,
// combine sub-spectra (max_buffers_per_spectrum > 1) or write whole spectra,
// flip the double buffer, stop at the first end of file.  The buffer read
// when the end of file is met is not processed (as in the reference).
#include <algorithm>

#include "sws_host.h"

namespace swshost {

TaskDispatcher::TaskDispatcher(Settings *s) : set_(s)
{
   std::ostream &log = *s->tlog;
   log << "TaskDispatcher buffer prefill..." << std::endl;
   for (int c = 0; c < s->num_cores; c++)
      for (int src = 0; src < s->num_sources; src++) s->sources[src]->read(s->rawbuffers[c][0][src]);
   log << "TaskDispatcher core init... ";
   for (int c = 0; c < s->num_cores; c++) {
      log << c << " ";
      TaskCoreCUDA *core = new TaskCoreCUDA(c);
      core->prepare(s);
      cores_.push_back(core);
   }
   log << std::endl;
   const size_t peak = std::max(s->fft_bytes_xpol, s->fft_bytes_ssb);
   for (int cc = 0; cc < s->num_sinks; cc++) {
      Buffer *b = new Buffer(peak);
      b->setLength(peak);
      cores_[0]->resetBuffer(b);
      corecombined_spectra_.push_back(b);
   }
   for (int cp = 0; cp < s->num_sources; cp++) {
      Buffer *b = new Buffer(std::max<size_t>(s->pcal_result_bytes, 8));
      b->setLength(s->pcal_result_bytes);
      cores_[0]->resetBuffer(b);
      corecombined_pcals_.push_back(b);
   }
}

TaskDispatcher::~TaskDispatcher()
{
   for (TaskCore *c : cores_) delete c;
   for (Buffer *b : corecombined_spectra_) delete b;
   for (Buffer *b : corecombined_pcals_) delete b;
}

void TaskDispatcher::run()
{
   Settings *set = set_;
   const int ncores = set->num_cores;
   int dblbuf = 0;
   bool gotEOF = false;
   int num_combined = 0, total_spectra = 0;
   std::ostream &log = *set->tlog;
   log << "TaskDispatcher processing all input chunks... " << std::endl;
   bool failed = false;
   do {
      for (int c = 0; c < ncores; c++) {
         std::vector<Buffer *> &in = set->rawbuffers[c][dblbuf];
         if (cores_[c]->run(in.data(), set->outbuffers[c].data(), set->outbuffersXpol[c].data(),
                            set->outbuffersPCal[c].data()) != 0)
            failed = true;
      }
      for (int c = 0; c < ncores; c++)
         for (int s = 0; s < set->num_sources; s++) set->sources[s]->read(set->rawbuffers[c][(dblbuf + 1) % 2][s]);
      for (int c = 0; c < ncores && !failed; c++) {
         const int numcompleted = cores_[c]->join();
         if (numcompleted < 0) {
            failed = true;
            break;
         }
         if (set->max_buffers_per_spectrum > 1) {
            cores_[c]->combineResults(corecombined_spectra_.data(), corecombined_pcals_.data());
            if (++num_combined == set->max_buffers_per_spectrum) {
               for (int sk = 0; sk < set->num_sinks; sk++) {
                  set->sinks[sk]->write(corecombined_spectra_[sk]);
                  cores_[0]->resetBuffer(corecombined_spectra_[sk]);
               }
               if (set->extract_PCal)
                  for (int pc = 0; pc < set->num_sources; pc++) {
                     set->pcalsinks[pc]->write(corecombined_pcals_[pc]);
                     cores_[0]->resetBuffer(corecombined_pcals_[pc]);
                  }
               total_spectra++;
               num_combined = 0;
            }
         } else {
            for (int sk = 0; sk < set->num_sinks && sk < set->num_sources; sk++)
               set->sinks[sk]->write(set->outbuffers[c][sk]);
            for (int xp = 0; xp < set->num_xpols; xp++)
               set->sinks[set->num_sources + xp]->write(set->outbuffersXpol[c][xp]);
            if (set->extract_PCal)
               for (int pc = 0; pc < set->num_sources; pc++) {
                  set->pcalsinks[pc]->write(set->outbuffersPCal[c][pc]);
                  cores_[0]->resetBuffer(set->outbuffersPCal[c][pc]);
               }
            total_spectra += set->max_spectra_per_buffer;
         }
      }
      if (failed) {
         log << "TaskDispatcher: a core failed, stopping" << std::endl;
         break;
      }
      dblbuf = (dblbuf + 1) % 2;
      for (int s = 0; s < set->num_sources; s++) {
         if (set->sources[s]->eof()) gotEOF = true;
         if (set->rawbuffers[0][dblbuf][s]->getLength() > 0) break;
      }
   } while (!gotEOF);
   for (TaskCore *c : cores_) c->finalize();
   for (DataSink *k : set->sinks) k->close();
   if (set->extract_PCal)
      for (DataSink *k : set->pcalsinks) k->close();
   log << "TaskDispatcher completed, " << total_spectra << " spectra." << std::endl;
}

}  // namespace swshost
