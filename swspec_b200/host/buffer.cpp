// buffer.cpp -- 128-byte aligned host buffer (src/Buffer.cpp:32-100).
#include <cstdlib>

#include "sws_host.h"

namespace swshost {

Buffer::Buffer(size_t bytes)
{
   void *p = nullptr;
   if (posix_memalign(&p, 128, bytes ? bytes : 128) != 0) {
      std::cerr << "Failed to allocate " << bytes << " bytes." << std::endl;
      return;
   }
   data_ = static_cast<char *>(p);
   allocated_ = bytes;
}

Buffer::~Buffer() { free(data_); }

}  // namespace swshost
