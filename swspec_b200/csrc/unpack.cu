// unpack.cu -- K1: raw Mark5B / VDIF bytes -> per-channel sample codes.
//
// Restates mark5access's decoders (mark5access/mark5access/
// mark5_format_mark5b.c:1043-1909, format_vdif.c:564-610, :1097-1137) as a
// corner turn: sample-time t occupies nchan*nbit bits of the payload stream
// from bit t*nchan*nbit, channel c at bit offset c*nbit, LSB-first.  Each
// thread owns one 32-bit output word (32/nbit consecutive samples) of every
// requested channel, reads the payload words once and writes one code word
// per channel, so only the channels a run uses are touched.  Headers are
// skipped by index arithmetic.
//
// Blanking follows mark5access exactly: per frame, a valid byte range
// [start, end) (blanker_mark5.c:126-200 with its binary search for the fill
// pattern, blanker_vdif :282-310, and whole-frame blanking when a VDIF frame
// fails validation on its invalid bit, format_vdif.c:2873-2914 and
// mark5_stream.c:136-145); a sample-time whose first byte lies outside the
// range decodes to 0.  Blanked sample-times are marked in a bitmap the FFT
// kernel consults only when a chunk has any.
#include "kernels.cuh"

namespace sws {

__device__ __forceinline__ long long payload_addr(const StreamIn &s, long long v)
{
   // byte offset into s.data of virtual payload byte v
   if (s.header_bytes == 0) return v - s.grid_offset;
   long long f = v / s.payload_bytes;
   long long o = v - f * s.payload_bytes;
   return f * s.frame_bytes + s.header_bytes + o;
}

// 64-bit word `w` of frame f's payload; words outside the chunk read as
// "not fill" (only possible for partial frames of header-free chunks).
__device__ __forceinline__ unsigned long long frame_word64(const StreamIn &s, long long f, int w)
{
   long long v = f * s.payload_bytes + 8ll * w;
   if (v < s.grid_offset) return 0ull;
   long long a = payload_addr(s, v);
   if (a < 0 || a + 8 > s.nbytes) return 0ull;
   const uint32_t *p = reinterpret_cast<const uint32_t *>(s.data + a);
   return (unsigned long long)p[0] | ((unsigned long long)p[1] << 32);
}
__device__ __forceinline__ uint32_t frame_word32(const StreamIn &s, long long f, int w)
{
   long long v = f * s.payload_bytes + 4ll * w;
   if (v < s.grid_offset) return 0u;
   long long a = payload_addr(s, v);
   if (a < 0 || a + 4 > s.nbytes) return 0u;
   return *reinterpret_cast<const uint32_t *>(s.data + a);
}

// blanker_mark5's findfirstinvalid / findfirstvalid over words [0, n)
__device__ int m5_first_invalid(const StreamIn &s, long long f, int n)
{
   int i = n / 2, r = n - 1;
   for (int st = n / 4; st > 0; st >>= 1) {
      if (frame_word64(s, f, i) == FILL64) { r = i; i -= st; }
      else i += st;
   }
   r = 8 * r;
   if (frame_word32(s, f, r / 4 - 1) == FILL32) r -= 4;
   return r;
}
__device__ int m5_first_valid(const StreamIn &s, long long f, int n)
{
   int i = n / 2, r = n - 1;
   for (int st = n / 4; st > 0; st >>= 1) {
      if (frame_word64(s, f, i) != FILL64) { r = i; i -= st; }
      else i += st;
   }
   r = 8 * r;
   if (frame_word32(s, f, r / 4 - 2) == FILL32) r += 4;
   return r;
}

// Valid payload byte range of every frame the chunk touches.
__global__ void k_frame_valid(StreamIn s, int2 *valid, int *blank_any)
{
   long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (f >= s.nframes) return;
   const int big = 1 << 30;
   int vs = 0, ve = big;
   const int nword = s.payload_bytes / 8;
   if (s.format == 1) {
      // VDIF: invalid bit in header word 0 (framed layouts only), then fill check
      bool bad = false;
      if (s.header_bytes > 0) {
         long long a = f * s.frame_bytes;
         if (a + 4 <= s.nbytes) bad = (*reinterpret_cast<const uint32_t *>(s.data + a) >> 31) & 1u;
      }
      if (bad) { vs = big; ve = 0; }
      else if (frame_word64(s, f, 0) == FILL64 || frame_word64(s, f, nword - 1) == FILL64) { vs = 0; ve = 0; }
   } else {
      // Mark5B: one 32 KiB zone per 10000-byte payload
      bool startOK = frame_word64(s, f, 0) != FILL64;
      bool endOK = frame_word64(s, f, nword - 1) != FILL64;
      if (startOK && endOK) { vs = 0; ve = big; }
      else if (!startOK && !endOK) { vs = big; ve = 0; }
      else if (startOK) { vs = 0; ve = m5_first_invalid(s, f, nword); }
      else { vs = m5_first_valid(s, f, nword); ve = big; }
   }
   valid[f] = make_int2(vs, ve);
   if (!(vs <= 0 && ve >= s.payload_bytes)) atomicOr(blank_any, 1);
}

// Corner turn into a phase-decimated code layout.  For decimation D (the
// FFT plan's cluster size), sample s of a channel is stored in phase array
// s % D at index s / D, SPW = 32/NBIT codes per 32-bit word:
//   codes[c * D * wpp + (s % D) * wpp + (s / D) / SPW], bits NBIT * ((s / D) % SPW).
// A CTA of the FFT cluster that owns residue p then reads its samples as one
// contiguous run.  Thread t writes word t / D of phase t % D for every
// requested channel; each payload word is read by exactly one thread.
// Blank bits (1 per sample-time, standard order) go to `blank` (pre-zeroed).
template <int NBIT>
__global__ void k_unpack_codes(StreamIn s, long long nsamp, const int *chans, int nch,
                               uint32_t *codes, int D, long long wpp, const int2 *valid,
                               uint32_t *blank)
{
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT == 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= (long long)D * wpp) return;
   const int ph = (int)(t % D);
   const long long iw = t / D;
   const long long stride = (long long)s.nchan * NBIT;
   const int nb = s.payload_bytes;
   uint32_t acc[16];
   int c0 = blockIdx.y * 16;
   int cn = min(16, nch - c0);
#pragma unroll
   for (int c = 0; c < 16; c++) acc[c] = 0u;
   long long cached_idx = -1;
   uint32_t cached = 0u;
   for (int k = 0; k < SPW; k++) {
      const long long smp = (iw * SPW + k) * D + ph;
      if (smp >= nsamp) break;
      long long bit0 = smp * stride;
      long long v0 = s.grid_offset + (bit0 >> 3);
      long long f = v0 / nb;
      int o = (int)(v0 - f * nb);
      int2 vr = valid[f];
      if (!((o >= vr.x) && (o < vr.y))) {
         if (blockIdx.y == 0) atomicOr(&blank[smp >> 5], 1u << (smp & 31));
         continue;
      }
#pragma unroll
      for (int c = 0; c < 16; c++) {
         if (c < cn) {
            long long bit = bit0 + (long long)chans[c0 + c] * NBIT;
            long long widx = bit >> 5;   // 32-bit payload word (frames are multiples of 4 bytes)
            if (widx != cached_idx) {
               // grid_offset and payload sizes are multiples of 4 bytes, so a
               // payload word never straddles a frame boundary
               cached = *reinterpret_cast<const uint32_t *>(s.data + payload_addr(s, s.grid_offset + 4 * widx));
               cached_idx = widx;
            }
            acc[c] |= ((cached >> (bit & 31)) & MASK) << (NBIT * k);
         }
      }
   }
   const long long code_words = (long long)D * wpp;
#pragma unroll
   for (int c = 0; c < 16; c++)
      if (c < cn) codes[(long long)(c0 + c) * code_words + (long long)ph * wpp + iw] = acc[c];
}

// Decoded float samples of one channel (test path; same rules as above).
__global__ void k_unpack_float(StreamIn s, long long nsamp, int chan, float4 levels, float *out,
                               const int2 *valid, unsigned long long *nvalid)
{
   long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= nsamp) return;
   const int nbit = s.nbit;
   long long bit = t * (long long)s.nchan * nbit + (long long)chan * nbit;
   long long v0 = s.grid_offset + ((t * (long long)s.nchan * nbit) >> 3);
   long long f = v0 / s.payload_bytes;
   int o = (int)(v0 - f * s.payload_bytes);
   int2 vr = valid[f];
   float val = 0.0f;
   if (o >= vr.x && o < vr.y) {
      long long widx = bit >> 5;
      uint32_t word = *reinterpret_cast<const uint32_t *>(s.data + payload_addr(s, s.grid_offset + 4 * widx));
      uint32_t code = (word >> (bit & 31)) & ((nbit == 8) ? 0xffu : ((1u << nbit) - 1u));
      if (nbit == 8) val = (float)((int)code * 2 - 255) * (1.0f / 256.0f);
      else if (nbit == 2) val = (code == 0) ? levels.x : (code == 1) ? levels.y : (code == 2) ? levels.z : levels.w;
      else val = code ? levels.y : levels.x;
      atomicAdd(nvalid, 1ull);
   }
   out[t] = val;
}

void launch_unpack_codes(int nbit, dim3 grid, int block, cudaStream_t st, StreamIn s,
                         long long nsamp, const int *chans, int nch, uint32_t *codes, int D,
                         long long wpp, const int2 *valid, uint32_t *blank)
{
   if (nbit == 1)
      k_unpack_codes<1><<<grid, block, 0, st>>>(s, nsamp, chans, nch, codes, D, wpp, valid, blank);
   else if (nbit == 2)
      k_unpack_codes<2><<<grid, block, 0, st>>>(s, nsamp, chans, nch, codes, D, wpp, valid, blank);
   else
      k_unpack_codes<8><<<grid, block, 0, st>>>(s, nsamp, chans, nch, codes, D, wpp, valid, blank);
}

}  // namespace sws
