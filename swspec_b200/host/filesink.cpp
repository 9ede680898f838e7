// filesink.cpp -- spectrum output files (src/FileSink.cpp:31-110).
// Binary: the buffer's bytes appended as they are.  ASCII: the reference's
// text layout -- a marker line, a bin-count line, the first float of every
// float pair, then the second float of the buffer as "Nyquist".
#include "sws_host.h"

namespace swshost {

int FileSink::open(const std::string &uri)
{
   if (ofile_.is_open()) ofile_.close();
   ofile_.open(uri.c_str(), std::ofstream::trunc | std::ios::out | std::ios::binary);
   if (!ofile_.is_open()) {
      std::cerr << "Could not open output file " << uri << std::endl;
      return -1;
   }
   ofile_.precision(12);
   return 0;
}

size_t FileSink::write(Buffer *buf)
{
   if (!buf || buf->getLength() == 0 || !cfg_) return 0;
   if (!ofile_.is_open() || !ofile_.good()) {
      std::cerr << "FileSink write: file not open or in bad state" << std::endl;
      return 0;
   }
   const float *src = reinterpret_cast<const float *>(buf->getData());
   const size_t len = buf->getLength() / (2 * sizeof(float));
   if (cfg_->sinkformat == Binary) {
      ofile_.write(buf->getData(), (std::streamsize)buf->getLength());
   } else {
      ofile_ << "// --------------------- DATA SET TIMESTAMP xxxx ---------------------" << std::endl;
      ofile_ << "// FFT bins 0.." << (len - 1) << " + Nyquist" << std::endl;
      const float nyq = src[1];
      for (size_t i = 0; i < len; i++) ofile_ << src[2 * i] << std::endl;
      ofile_ << nyq << std::endl;
   }
   ofile_.flush();
   if (!ofile_.good()) std::cerr << "Write I/O error!" << std::endl;
   return buf->getLength();
}

int FileSink::close()
{
   ofile_.close();
   return 0;
}

}  // namespace swshost
