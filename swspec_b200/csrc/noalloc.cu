// noalloc.cu -- channel decode that allocates no device memory.
//
// swsgpu_unpack_device obtains its small scratch area (one valid-byte range
// per frame, a sample counter and a flag) from cudaMalloc on every call.
// Some callers cannot allocate device memory where they decode: a recorder's
// acquisition thread that must not stall on the implicit device-wide
// synchronisation cudaMalloc/cudaFree can cause, an application whose memory
// manager owns every device allocation and forbids others, or a process that
// reserves all of its device memory once at start-up.
// swsgpu_unpack_device_noalloc does the same decode with its scratch in one
// fixed array compiled into this library (SWSGPU_NOALLOC_SCRATCH_BYTES per
// device that loads the library, held until the process exits).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/swsgpu.h"
#include "kernels.cuh"

namespace sws {
void record_create_error(const std::string &msg);
__global__ void k_frame_valid(StreamIn s, int2 *valid, int *blank_any);
__global__ void k_unpack_float(StreamIn s, long long nsamp, int chan, float4 levels, float *out,
                               const int2 *valid, unsigned long long *nvalid);
}  // namespace sws

using namespace sws;

// Scratch layout: int2 valid[SWSGPU_NOALLOC_MAX_FRAMES], then the 64-bit
// sample counter, then the int blank flag.
static constexpr size_t kValidBytes = sizeof(int2) * (size_t)SWSGPU_NOALLOC_MAX_FRAMES;
static constexpr size_t kCounterOff = kValidBytes;
static constexpr size_t kFlagOff = kValidBytes + 8;
static_assert(kFlagOff + sizeof(int) <= (size_t)SWSGPU_NOALLOC_SCRATCH_BYTES, "scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[SWSGPU_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// names a host-side stand-in, not device memory, so the address must come
// from cudaGetSymbolAddress, resolved once per device with that device
// current.
static constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mu;
static void *g_scratch_ptr[kMaxDevices] = {};

static int scratch_for_current_device(unsigned char **out)
{
   int dev = -1;
   if (cudaGetDevice(&dev) != cudaSuccess) return SWSGPU_ENODEV;
   if (dev < 0 || dev >= kMaxDevices) return SWSGPU_ENODEV;
   std::lock_guard<std::mutex> lock(g_scratch_mu);
   if (!g_scratch_ptr[dev]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) return SWSGPU_ECUDA;
      g_scratch_ptr[dev] = p;
   }
   *out = static_cast<unsigned char *>(g_scratch_ptr[dev]);
   return SWSGPU_OK;
}


extern "C" int swsgpu_unpack_device_noalloc(const swsgpu_layout *lay, const void *d_raw,
                                            size_t nbytes, int64_t payload_offset, int chan,
                                            int64_t nsamp, float *d_out, int64_t *nvalid,
                                            void *cuda_stream)
{
   if (!lay || !d_raw || !d_out || chan < 0 || chan >= lay->nchan || nsamp < 0) return SWSGPU_EINVAL;
   if (lay->nbit != 1 && lay->nbit != 2 && lay->nbit != 8) return SWSGPU_EINVAL;
   if ((uintptr_t)d_raw % 4 || (uintptr_t)d_out % 4) return SWSGPU_EINVAL;  // 32-bit loads and stores
   const int pb = lay->frame_bytes - lay->header_bytes;
   if (pb <= 0 || (pb % 8) || (lay->header_bytes % 4) || (payload_offset % 4)) return SWSGPU_EINVAL;
   if (lay->header_bytes > 0 && payload_offset != 0) return SWSGPU_EINVAL;
   // track formats (VLBA, Mark4) are decoded through a conversion buffer of
   // the data's size, which this entry has no room for
   if (lay->format == SWSGPU_FMT_VLBA || lay->format == SWSGPU_FMT_MARK4) return SWSGPU_EINVAL;
   if (nsamp == 0) {
      if (nvalid) *nvalid = 0;
      return SWSGPU_OK;
   }
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
   si.msb2 = (lay->format >= SWSGPU_FMT_RAW_SIGNED && lay->nbit == 2 && lay->nchan == 1) ? 1 : 0;
   set_zones(si);  // one range per frame for every format taken here
   const long long last_v = si.grid_offset + ((nsamp * (long long)lay->nchan * lay->nbit - 1) >> 3);
   si.nframes = last_v / pb + 1;
   // the fixed scratch holds one valid range per frame
   if (si.nframes > SWSGPU_NOALLOC_MAX_FRAMES) return SWSGPU_ETOOBIG;
   long long need = lay->header_bytes
                        ? si.nframes * lay->frame_bytes - (lay->frame_bytes - lay->header_bytes - (last_v % pb) - 1)
                        : (last_v - si.grid_offset + 1);
   if (need > (long long)nbytes) return SWSGPU_EINVAL;

   unsigned char *scr = nullptr;
   int rc = scratch_for_current_device(&scr);
   if (rc != SWSGPU_OK) return rc;
   int2 *valid = reinterpret_cast<int2 *>(scr);
   unsigned long long *counter = reinterpret_cast<unsigned long long *>(scr + kCounterOff);
   int *flag = reinterpret_cast<int *>(scr + kFlagOff);

   cudaStream_t st = (cudaStream_t)cuda_stream;
   // the scratch keeps the previous call's contents: the counter and flag
   // must start at zero; valid[0, nframes) is rewritten by k_frame_valid
   if (cudaMemsetAsync(scr + kCounterOff, 0, kFlagOff + sizeof(int) - kCounterOff, st) != cudaSuccess)
      return SWSGPU_ECUDA;
   k_frame_valid<<<(unsigned)((si.nframes + 127) / 128), 128, 0, st>>>(si, valid, flag);
   k_unpack_float<<<(unsigned)((nsamp + 255) / 256), 256, 0, st>>>(
       si, nsamp, chan, level_table(lay->format, lay->nbit), d_out, valid, counter);
   cudaError_t e = cudaGetLastError();
   unsigned long long cnt = 0;
   if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, counter, sizeof(cnt), cudaMemcpyDeviceToHost, st);
   if (e == cudaSuccess) e = cudaStreamSynchronize(st);
   if (e != cudaSuccess) {
      record_create_error(std::string("swsgpu_unpack_device_noalloc: ") + cudaGetErrorString(e));
      return SWSGPU_ECUDA;
   }
   if (nvalid) *nvalid = (int64_t)cnt;
   return SWSGPU_OK;
}
