// kernels.cuh -- device data structures shared by the spectrometer kernels.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/swsgpu.h"

namespace sws {

constexpr uint32_t FILL32 = 0x11223344u;              // mark5 fill pattern (blanker_mark5.c:42-48)
constexpr unsigned long long FILL64 = 0x1122334411223344ull;

// One input stream of a chunk.  data[0] is the first byte of frame 0 (framed
// layouts) or the first payload byte of the chunk (header-free layouts).
// grid_offset: payload bytes of frame 0 that precede the chunk's first
// payload byte.  Virtual payload byte v = grid_offset + x for chunk payload
// byte x; frame f = v / payload_bytes.
struct StreamIn {
   const uint8_t *data;
   long long nbytes;
   long long grid_offset;
   int frame_bytes;
   int header_bytes;
   int payload_bytes;
   int nchan;
   int nbit;
   int format;   // SWSGPU_FMT_*
   long long nframes;  // frames touched by the chunk
   int msb2;     // 2-bit samples stored oldest-first from the byte's MSB (raw single channel)
   // blanking zones: a frame's valid byte ranges are valid[f * zpf + (o >> zshift)]
   // for payload byte o of frame f (set by set_zones)
   int zpf;
   int zshift;
};

// Level table of a format, as decode_level reads it: 1-bit {x, y}; 2-bit
// {x, y, z, w} for codes 0..3; 8-bit v = x * (code ^ bits(z)) + y (exact
// for every 8-bit table: VDIF (2b - 255)/256, raw b - 128 and (int8)b).
__host__ __device__ inline float4 level_table(int format, int nbit)
{
   const float H = 3.3359f;  // OPTIMAL_2BIT_HIGH (mark5access) = the reference's 2-bit high level
   if (format == SWSGPU_FMT_MARK5B || format == SWSGPU_FMT_VLBA || format == SWSGPU_FMT_MARK4) {
      // the track formats are turned into Mark5B's sample layout first
      if (nbit == 2) return make_float4(-H, 1.0f, -1.0f, H);
      return make_float4(1.0f, -1.0f, 0.0f, 0.0f);
   }
   if (format == SWSGPU_FMT_RAW_SIGNED || format == SWSGPU_FMT_RAW_UNSIGNED) {
      if (nbit == 2) return make_float4(1.0f, -1.0f, H, -H);
      float x;
      const uint32_t xm = format == SWSGPU_FMT_RAW_SIGNED ? 0x80u : 0u;
      memcpy(&x, &xm, 4);
      return make_float4(1.0f, -128.0f, x, 0.0f);
   }
   if (nbit == 2) return make_float4(-H, -1.0f, 1.0f, H);
   if (nbit == 8) return make_float4(1.0f / 128.0f, -255.0f / 256.0f, 0.0f, 0.0f);
   return make_float4(-1.0f, 1.0f, 0.0f, 0.0f);
}

__host__ __device__ inline bool track_format(int format)
{
   return format == SWSGPU_FMT_VLBA || format == SWSGPU_FMT_MARK4;
}

// Unit-byte tables of a VLBA / Mark4 mode's track turn: [8 bytes][256 values]
// x two 32-bit output words (unpack.cu, track_turn_table).
constexpr int TRACK_TABLE_WORDS = 8 * 256 * 2;

// mark5access blanks VLBA and Mark4 payloads by 32 KiB zones, each with its
// own valid byte range (blanker_mark5.c:126-280, log2blankzonesize = 15);
// the other formats have one range per frame.
inline void set_zones(StreamIn &s)
{
   if (track_format(s.format)) {
      s.zshift = 15;
      s.zpf = (s.payload_bytes + 32767) >> 15;
   } else {
      s.zshift = 31;
      s.zpf = 1;
   }
}
__device__ __forceinline__ int2 valid_range(const StreamIn &s, const int2 *valid, long long f, int o)
{
   return valid[f * s.zpf + (o >> s.zshift)];
}

// Tracks of sample j (< fanout) of channel c in a track-word of a VLBA /
// Mark4 mode: the sign bit's track, and for 2-bit samples the magnitude
// bit's (-1 for 1-bit).  Up to 16 tracks a channel's tracks are contiguous
// (sign tracks then magnitude tracks, f of each); with 32 and 64 tracks the
// channels interleave within groups of 32 tracks (4 bytes): a group holds
// 32 / (nbit f) channels, and the rules below give, per group, the
// assignment mark5access's decoders read (mark5_format_vlba.c and
// mark5_format_mark4.c: the 32/64-track decoders, their byte reordering of
// fanout-4 2-bit modes included).
__host__ __device__ inline int2 track_of(int ntrack, int fanout, int nbit, int c, int j)
{
   const int f = fanout;
   if (ntrack <= 16) {
      if (nbit == 1) return make_int2(f * c + j, -1);
      const int s = 2 * f * c + j;
      return make_int2(s, s + f);
   }
   if (nbit == 1) {
      if (f == 1) {
         const int g = c / 32, q = c % 32;
         return make_int2(32 * g + 2 * (q % 16) + q / 16, -1);
      }
      if (f == 2) {
         const int g = c / 16, q = c % 16;
         return make_int2(32 * g + 4 * (q % 8) + q / 8 + 2 * j, -1);
      }
      const int g = c / 8, q = c % 8;
      return make_int2(32 * g + 8 * (q % 4) + q / 4 + 2 * j, -1);
   }
   if (f == 1) {
      const int g = c / 16, q = c % 16, s = 32 * g + 4 * (q % 8) + q / 8;
      return make_int2(s, s + 2);
   }
   if (f == 2) {
      const int g = c / 8, q = c % 8, s = 32 * g + 8 * (q % 4) + q / 4 + 2 * j;
      return make_int2(s, s + 4);
   }
   const int g = c / 4, q = c % 4, s = 32 * g + 16 * (q % 2) + q / 2 + 2 * j;
   return make_int2(s, s + 8);
}

// Reverses the order of the four 2-bit fields of every byte of w.
__host__ __device__ inline uint32_t swap2_in_bytes(uint32_t w)
{
   return ((w & 0x03030303u) << 6) | ((w & 0x0C0C0C0Cu) << 2) | ((w & 0x30303030u) >> 2) |
          ((w & 0xC0C0C0C0u) >> 6);
}

// A run of consecutive FFT jobs that share their accumulators.
// mode 0 (XPOL):    job j packs A = source a, B = source b, both starting at
//                   start + j*step; products |A|^2, |B|^2, A conj(B).
// mode 1 (AUTOSUM): A = source a at start + j*step, B = source a at
//                   start + j*step + offset_b; product |A|^2 + |B|^2.
// mode 2 (SINGLE):  A = source a at start (one job), B = 0; product |A|^2.
struct Item {
   long long start;
   int src_a, src_b;
   int step, offset_b;
   int nfr, mode;
};

constexpr int MODE_XPOL = 0, MODE_AUTOSUM = 1, MODE_SINGLE = 2;

// Code arrays are phase-decimated (see k_unpack_codes): array c holds
// D phase arrays of wpp words; sample s at phase s % D, index s / D.
struct SpecArgs {
   const uint32_t *codes;        // [ncode][D][wpp]
   long long code_words;         // words per code array (D * wpp)
   long long wpp;                // words per phase array
   int D;                        // decimation (the plan's cluster size)
   const uint32_t *blank;        // [nstream][blank_words] bitmaps (1 = blanked sample-time)
   long long blank_words;
   const int *blank_any;         // [nstream]
   const int *code_stream;       // stream of each code array
   const Item *items;
   int nitems;
   const int *cl_first;          // [clusters + 1]: cluster c runs items [cl_first[c], cl_first[c + 1]) (null: every ncl-th item)
   const float *window;          // [N]
   const float2 *twQ;            // W_Q^m, m < Q
   const float2 *twN;            // W_N^m, m < N/2 (+1)
   float *partial;               // [nitems][4][S]
   int N, S;
   float4 levels;                // level table for 1/2-bit codes
   int *status;                  // set to 1 when a bounded wait gave up (null: not reported)
   int drop_last_exchange;       // fault injection: the last job of each cluster pushes nothing
};

// Reduction of item partial sums into output spectra.
struct RedEntry {
   int item, prod;
   float scale;
};
// acc_mode: 0 dst = sum; 1 acc = sum; 2 acc += sum; 3 acc += sum, dst = acc
// (acc is an FP64 running sum across runs, element k at acc[k])
struct OutVec {
   int first, count;             // entries [first, first+count)
   float *dst;                   // base of the output vector
   int stride;                   // element stride (1 real, 2 complex)
   double *acc;
   int acc_mode;
};

}  // namespace sws
