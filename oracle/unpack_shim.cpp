// unpack_shim.cpp -- C entry into the reference's own raw-data unpackers
// (test infrastructure: compiled with src/IA-32/DataUnpackers.cpp from the
// reference tree into oracle/_ref/libunpackref.so by oracle/Makefile; never
// linked into the GPU product).
//
// The unpackers are the ones DataUnpackerFactory picks for RawSigned and
// RawUnsigned data (src/IA-32/DataUnpackerFactory.h:44-67):
//   kind 0  SignedUnpacker              8-bit  (DataUnpackers.cpp:68-114)
//   kind 1  UnsignedUnpacker            8-bit  (:125-171)
//   kind 2  TwoBitUnpacker              2-bit, channels % 4 == 0 (:191-249)
//   kind 3  TwoBitSinglechannelUnpacker 2-bit, 1 channel (:261-310)
// IPP is absent: the stub ippcore.h / ipps.h that the recipe generates give
// Ipp32f its meaning (float) and an element copy, nothing else.
#include <cstring>

#include "DataUnpackers.h"
#include "Settings.h"

extern "C" long refunpack_raw(int kind, int nbit, int nchan, int increasing, const char *src, float *dst,
                              long count, int channel)
{
   swspect_settings_t s;
   s.bits_per_sample = nbit;
   s.source_channels = nchan;
   s.channelorder_increasing = increasing != 0;
   switch (kind) {
   case 0: return (long)SignedUnpacker(&s).extract_samples(src, dst, (size_t)count, channel);
   case 1: return (long)UnsignedUnpacker(&s).extract_samples(src, dst, (size_t)count, channel);
   case 2: return (long)TwoBitUnpacker(&s).extract_samples(src, dst, (size_t)count, channel);
   case 3: return (long)TwoBitSinglechannelUnpacker(&s).extract_samples(src, dst, (size_t)count, channel);
   }
   return -1;
}
