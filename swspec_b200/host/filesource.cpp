// filesource.cpp -- framed recordings to payload-only buffers.
//
// Follows the reference's framed reading (src/FileSource.cpp:36-250):
// locate the first frame header, optionally skip whole seconds, then fill
// each buffer with payload bytes, consuming every frame header on the way.
// Mark5B frames are found by two consecutive sync words 10016 bytes apart
// (as mark5access's findfirstframe, mark5_format_mark5b.c:98-131); the first
// frame's BCD time is written to the start-timing log.
#include <cmath>
#include <cstring>

#include "sws_host.h"

namespace swshost {

static const uint32_t kMark5BSync = 0xABADDEEDu;

int FileSource::open(const std::string &uri)
{
   const Settings &s = *cfg_;
   const bool mark5b = (s.sourceformat == Mark5B || s.sourceformat == Mk5B);
   const bool raw = (s.sourceformat == RawSigned || s.sourceformat == RawUnsigned);
   const bool tracks = (s.sourceformat == VLBA || s.sourceformat == MKIV);
   const int tb = s.layout.frame_bytes / 20000;  // track formats: bytes per track-word
   if (raw) header_bytes_ = 0;
   else if (s.sourceformat == iBOB) header_bytes_ = 4;  // packet sequence header (src/FileSource.cpp:53-57)
   // VLBA frames are 20160 track-words with the payload at 96 .. 20095
   // (mark5access's framebytes and payloadoffset): 160 track-words lie
   // between two payloads; Mark4 frames (data replacement) are read whole
   else if (tracks) header_bytes_ = s.sourceformat == VLBA ? 160 * tb : 0;
   else header_bytes_ = mark5b ? 16 : (s.sourceformat_str.size() > 4 && s.sourceformat_str[4] == '_' ? 32 : 16);
   frame_bytes_ = header_bytes_ + s.layout.frame_bytes;
   ifile_.open(uri.c_str(), std::ios::binary | std::ios::in);
   if (!ifile_.is_open()) {
      *cfg_->tlog << "Could not open input file " << uri << std::endl;
      got_eof_ = true;
      return -1;
   }
   // locate the first frame
   first_frame_ = 0;
   if (mark5b) {
      std::vector<unsigned char> win(1 << 20);
      ifile_.read(reinterpret_cast<char *>(win.data()), win.size());
      const int64_t got = ifile_.gcount();
      int64_t found = -1;
      for (int64_t i = 0; i + 10020 <= got; i++) {
         uint32_t a, b;
         memcpy(&a, &win[i], 4);
         memcpy(&b, &win[i + 10016], 4);
         if (a == kMark5BSync && b == kMark5BSync) {
            found = i;
            break;
         }
      }
      if (found < 0) {
         *cfg_->tlog << "FileSource: no Mark5B frame found in " << uri << std::endl;
         return -1;
      }
      first_frame_ = found;
      if (found > 0)
         *cfg_->tlog << "FileSource: first Mark5B frame at byte " << found << " (" << found
                     << " leading bytes skipped)" << std::endl;
      if (cfg_->startlog) {
         // header word 2 holds the time as 8 BCD digits JJJSSSSS (MJD mod
         // 1000, second of day); the reference reads it without checks
         // (src/FileSource.cpp:338-339), here a digit above 9 is reported
         const unsigned char *h = &win[found + 8];
         int nib[8];
         bool bcd_ok = true;
         for (int i = 0; i < 4; i++) {
            nib[2 * i] = h[3 - i] >> 4;
            nib[2 * i + 1] = h[3 - i] & 15;
         }
         for (int i = 0; i < 8; i++) bcd_ok = bcd_ok && nib[i] <= 9;
         const int mjd3 = nib[0] * 100 + nib[1] * 10 + nib[2];
         const int sec = nib[3] * 10000 + nib[4] * 1000 + nib[5] * 100 + nib[6] * 10 + nib[7];
         *cfg_->startlog << "First frame at byte " << found << ": MJD(mod 1000) " << mjd3 << " second " << sec
                         << std::endl;
         if (!bcd_ok || sec >= 86400) {
            *cfg_->tlog << "FileSource: Mark5B time code of the first frame is not a valid BCD time (digits";
            for (int i = 0; i < 8; i++) *cfg_->tlog << " " << nib[i];
            *cfg_->tlog << ")" << std::endl;
         }
      }
   }
   if (tracks) {
      // the frame sync word: 32 track-words of all ones, two frames apart
      // (as mark5access's findfirstframe); VLBA frames start with it, Mark4
      // frames carry it after 64 track-words of auxiliary data
      const int64_t sync_len = 32 * tb, sync_at = s.sourceformat == VLBA ? 0 : 64 * tb;
      std::vector<unsigned char> win((size_t)(3 * frame_bytes_ + sync_len));
      ifile_.read(reinterpret_cast<char *>(win.data()), win.size());
      const int64_t got = ifile_.gcount();
      auto ones = [&](int64_t at) {
         for (int64_t k = 0; k < sync_len; k++)
            if (win[at + k] != 0xFF) return false;
         return true;
      };
      int64_t found = -1;
      for (int64_t i = 0; i + frame_bytes_ + sync_len <= got && found < 0; i++)
         if (ones(i) && ones(i + frame_bytes_)) found = i;
      if (found < 0) {
         *cfg_->tlog << "FileSource: no " << (s.sourceformat == VLBA ? "VLBA" : "Mark4") << " frame found in " << uri
                     << std::endl;
         return -1;
      }
      // the first whole frame
      first_frame_ = found >= sync_at ? found - sync_at : found - sync_at + frame_bytes_;
      if (first_frame_ > 0)
         *cfg_->tlog << "FileSource: first frame at byte " << first_frame_ << " (" << first_frame_
                     << " leading bytes skipped)" << std::endl;
      if (cfg_->startlog) {
         // the time code follows the sync word: BCD nibbles of four
         // track-words each, most significant bit first, every bit the
         // majority of the track-word's tracks as mark5access reads it (set
         // when more than ntrack / 16 tracks are set;
         // mark5_format_vlba.c:314-334).  VLBA: JJJ SSSSS ssss (MJD mod
         // 1000, second of day, 0.1 ms); Mark4: Y DDD HH MM SS ss s (last
         // digit of the year, day of year, time of day)
         const int nnib = s.sourceformat == VLBA ? 12 : 13;
         const int64_t t0 = found + sync_len;
         int nib[13] = {0};
         bool bcd_ok = t0 + (int64_t)4 * nnib * tb <= got;
         for (int i = 0; bcd_ok && i < nnib; i++) {
            for (int b = 0; b < 4; b++) {
               int c = 0;
               for (int j = 0; j < tb; j++) c += __builtin_popcount(win[t0 + (int64_t)tb * (4 * i + 3 - b) + j]);
               if (c > tb / 2) nib[i] |= 1 << b;
            }
            bcd_ok = bcd_ok && nib[i] <= 9;
         }
         *cfg_->startlog << "First frame at byte " << first_frame_ << ": ";
         if (s.sourceformat == VLBA) {
            const int mjd3 = nib[0] * 100 + nib[1] * 10 + nib[2];
            const int sec = nib[3] * 10000 + nib[4] * 1000 + nib[5] * 100 + nib[6] * 10 + nib[7];
            const int frac = nib[8] * 1000 + nib[9] * 100 + nib[10] * 10 + nib[11];
            *cfg_->startlog << "MJD(mod 1000) " << mjd3 << " second " << sec << " + " << frac << " x 0.1 ms"
                            << std::endl;
            bcd_ok = bcd_ok && sec < 86400;
         } else {
            const int doy = nib[1] * 100 + nib[2] * 10 + nib[3];
            const int sec = (nib[4] * 10 + nib[5]) * 3600 + (nib[6] * 10 + nib[7]) * 60 + nib[8] * 10 + nib[9];
            *cfg_->startlog << "year digit " << nib[0] << " day " << doy << " second " << sec << std::endl;
            bcd_ok = bcd_ok && doy >= 1 && doy <= 366 && sec < 86400;
         }
         if (!bcd_ok) {
            *cfg_->tlog << "FileSource: time code of the first frame is not a valid BCD time (digits";
            for (int i = 0; i < nnib; i++) *cfg_->tlog << " " << nib[i];
            *cfg_->tlog << ")" << std::endl;
         }
      }
   }
   // skip whole seconds (FileSource.cpp:132-153)
   int64_t seek = first_frame_;
   if (s.seconds_to_skip > 0) {
      const double smp_bytes = (double)s.bits_per_sample * s.source_channels * s.samplingfreq / 8.0 * s.seconds_to_skip;
      if (header_bytes_ == 0) {
         seek += (int64_t)smp_bytes;  // unframed data: a plain byte offset
         *cfg_->tlog << "Skipping " << s.seconds_to_skip << " sample-seconds: " << (int64_t)smp_bytes << " bytes"
                     << std::endl;
      } else {
         const int64_t frames = (int64_t)std::ceil(smp_bytes / (double)s.layout.frame_bytes);
         seek += frames * frame_bytes_;
         *cfg_->tlog << "Skipping " << s.seconds_to_skip << " sample-seconds: " << frames << " frames" << std::endl;
      }
   }
   ifile_.clear();
   ifile_.seekg(seek, std::ios::beg);
   *cfg_->tlog << "FileSource   : processing framed data with " << header_bytes_ << "-byte headers and "
               << s.layout.frame_bytes << "-byte payloads" << std::endl;
   got_eof_ = false;
   pending_header_ = true;
   in_frame_ = 0;
   if (s.sourceformat == VLBA) {
      // the first payload follows the frame's 96-track-word header
      ifile_.seekg(seek + 96 * tb, std::ios::beg);
      pending_header_ = false;
   }
   return 0;
}

int FileSource::read(Buffer *buf)
{
   last_offset_ = payload_total_;
   if (!ifile_.is_open() || !buf) {
      if (buf) buf->setLength(0);
      return 0;
   }
   const int64_t payload = cfg_->layout.frame_bytes;
   char *dst = buf->getData();
   int64_t want = (int64_t)buf->getAllocated(), got = 0;
   std::vector<char> hdr(header_bytes_);
   while (want > 0 && !got_eof_) {
      if (pending_header_) {
         ifile_.read(hdr.data(), header_bytes_);
         if (ifile_.gcount() != header_bytes_) {
            got_eof_ = true;
            break;
         }
         frames_++;
         if (cfg_->sourceformat == Mark5B || cfg_->sourceformat == Mk5B) {
            // the reference logs a header without the sync word and keeps
            // reading (src/FileSource.cpp:401-427); so does this reader
            uint32_t sync;
            memcpy(&sync, hdr.data(), 4);
            if (sync != kMark5BSync) {
               bad_sync_++;
               *cfg_->tlog << "FileSource: Mark5B sync word mismatch in frame " << frames_ - 1 << " at byte "
                           << (int64_t)ifile_.tellg() - header_bytes_ << std::endl;
            }
         }
         if (cfg_->sourceformat == VDIF && cfg_->vdif_thread >= 0) {
            // multi-thread VDIF: the thread id is bits 16-25 of header word 3;
            // frames of other threads are skipped whole, so the kept frames
            // form one contiguous stream
            uint32_t w3;
            memcpy(&w3, hdr.data() + 12, 4);
            if ((int)((w3 >> 16) & 0x3FFu) != cfg_->vdif_thread) {
               ifile_.seekg(payload, std::ios::cur);
               if (!ifile_.good()) {
                  got_eof_ = true;
                  break;
               }
               continue;
            }
         }
         pending_header_ = false;
         in_frame_ = 0;
      }
      const int64_t n = std::min(want, payload - in_frame_);
      ifile_.read(dst + got, n);
      const int64_t r = ifile_.gcount();
      got += r;
      want -= r;
      in_frame_ += r;
      if (r < n) {
         got_eof_ = true;
         if (r > 0 || in_frame_ > 0)
            *cfg_->tlog << "FileSource: file ends inside frame " << frames_ - 1 << " after " << in_frame_ << " of "
                        << payload << " payload bytes" << std::endl;
         break;
      }
      if (in_frame_ == payload) pending_header_ = true;
   }
   payload_total_ += got;
   buf->setLength((size_t)got);
   return (int)got;
}

int FileSource::close()
{
   ifile_.close();
   return 0;
}

}  // namespace swshost
