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
#include <algorithm>

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

// blanker_mark5's findfirstinvalid / findfirstvalid: binary search of words
// [b, e) of a frame for the start / end of its fill pattern, in bytes, with
// the 32-bit straggler check just before the found word.
__device__ int m5_first_invalid(const StreamIn &s, long long f, int b, int e)
{
   const int n = e - b;
   int i = n / 2, r = n - 1;
   for (int st = n / 4; st > 0; st >>= 1) {
      if (frame_word64(s, f, b + i) == FILL64) { r = i; i -= st; }
      else i += st;
   }
   r = 8 * (b + r);
   if (frame_word32(s, f, r / 4 - 1) == FILL32) r -= 4;
   return r;
}
__device__ int m5_first_valid(const StreamIn &s, long long f, int b, int e)
{
   const int n = e - b;
   int i = n / 2, r = n - 1;
   for (int st = n / 4; st > 0; st >>= 1) {
      if (frame_word64(s, f, b + i) != FILL64) { r = i; i -= st; }
      else i += st;
   }
   r = 8 * (b + r);
   if (frame_word32(s, f, r / 4 - 2) == FILL32) r += 4;
   return r;
}

// Valid byte range of words [b, e) of frame f from the fill pattern at their
// two ends (blanker_mark5.c:159-196).
__device__ int2 fill_zone(const StreamIn &s, long long f, int b, int e)
{
   const int big = 1 << 30;
   const bool startOK = frame_word64(s, f, b) != FILL64;
   const bool endOK = frame_word64(s, f, e - 1) != FILL64;
   if (startOK && endOK) return make_int2(0, big);
   if (!startOK && !endOK) return make_int2(big, 0);
   if (startOK) return make_int2(0, m5_first_invalid(s, f, b, e));
   return make_int2(m5_first_valid(s, f, b, e), big);
}

// Valid payload byte ranges of every frame the chunk touches (zpf per frame).
// Reads the stream's own bytes: for the track formats, the track-words
// before they are turned.
__global__ void k_frame_valid(StreamIn s, int2 *valid, int *blank_any)
{
   long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (f >= s.nframes) return;
   const int big = 1 << 30;
   int vs = 0, ve = big;
   const int nword = s.payload_bytes / 8;
   if (s.format == SWSGPU_FMT_RAW_SIGNED || s.format == SWSGPU_FMT_RAW_UNSIGNED) {
      // raw sampler data: the reference's raw unpackers blank nothing
   } else if (track_format(s.format)) {
      // VLBA (blanker_mark5 on the header-free payload) and Mark4
      // (blanker_mark5.c:199-280, blanker_mark4, on the whole frame): 4096-word zones.
      // Mark4 starts its first zone after the frame's 160 header
      // track-words (20 n words, n = ntrack / 8 bytes per track-word) by
      // moving the loop's start, so each later zone is examined 20 n words
      // past its place on the 32 KiB grid the decoders look it up by; its
      // first zone starts no earlier than byte 160 n.  The decoders test a
      // track-word's first byte, so ranges are rounded up to whole
      // track-words.
      const int n = s.payload_bytes / 20000;
      const bool mk4 = s.format == SWSGPU_FMT_MARK4;
      int z = 0;
      for (int b = 0; b < nword && z < s.zpf; b += 4096, z++) {
         const int e = min(b + 4096, nword);
         if (mk4 && b == 0) b = 20 * n;
         int2 r = fill_zone(s, f, b, e);
         if (mk4 && z == 0) r.x = max(r.x, 160 * n);
         r.x = (r.x + n - 1) / n * n;
         r.y = (r.y + n - 1) / n * n;
         valid[f * s.zpf + z] = r;
         if (!(r.x <= 32768 * z && r.y >= min(32768 * (z + 1), s.payload_bytes))) atomicOr(blank_any, 1);
      }
      for (; z < s.zpf; z++) valid[f * s.zpf + z] = make_int2(0, big);
      return;
   } else if (s.format == SWSGPU_FMT_VDIF) {
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
      const int2 r = fill_zone(s, f, 0, nword);
      vs = r.x;
      ve = r.y;
   }
   valid[f] = make_int2(vs, ve);
   if (!(vs <= 0 && ve >= s.payload_bytes)) atomicOr(blank_any, 1);
}

// The VLBA modulation sequence: the 16-stage feedback shift register of the
// VLBA recording format (feedback from stages 10, 12, 13 and 15, all ones at
// the start of a frame, one extra step after every eighth output, which
// skips the parity bit), one bit per track-word of a frame; every sample of
// track-word i is negated where bit i is set.  Generated at compile time.
struct VlbaModulation {
   uint32_t w[625];
};
constexpr VlbaModulation make_vlba_modulation()
{
   VlbaModulation m{};
   uint32_t reg = 0xFFFFu;  // bit n = stage n
   for (int i = 0; i < 20000; i++) {
      uint32_t k = ((reg >> 10) ^ (reg >> 12) ^ (reg >> 13) ^ (reg >> 15)) & 1u;
      reg = ((reg << 1) | k) & 0xFFFFu;
      if (k) m.w[i >> 5] |= 1u << (i & 31);
      if (i % 8 == 7) {
         k = ((reg >> 10) ^ (reg >> 12) ^ (reg >> 13) ^ (reg >> 15)) & 1u;
         reg = ((reg << 1) | k) & 0xFFFFu;
      }
   }
   return m;
}
__constant__ VlbaModulation c_vlba_mod = make_vlba_modulation();

// Track-word stream (VLBA payload or Mark4 frames) -> Mark5B's sample layout:
// sample-time t of the chunk takes bits [t B, t B + B) of the output, B =
// nchan * nbit, channel c at bit offset c * nbit, 2-bit codes sign + 2 mag.
// A track-word of ntrack bits is `fanout` sample-times of B bits, so the
// output has the input's size and frame grid (frame validity, blanking and
// the corner turn treat it as Mark5B payload), and the turn is a fixed
// permutation of the bits of every unit of max(32, ntrack) bits: output bit
// o of a unit comes from one input bit of the same unit.  The permutation
// is tabulated per mode as unit-byte tables (track_turn_table): the output
// unit is the OR of one table entry per input byte.  VLBA modulation
// negates every sample of a modulated track-word, i.e. flips all of its
// bits before the permutation.
void track_turn_table(int ntrack, int nbit, int nchan, uint32_t *table)
{
   std::fill(table, table + TRACK_TABLE_WORDS, 0u);
   const int B = nchan * nbit, fanout = ntrack / B;
   const int U = ntrack > 32 ? 64 : 32;  // unit bits
   for (int o = 0; o < U; o++) {
      const int wi = o / ntrack, r = o % ntrack;  // track-word of the unit, bit of its sample-times
      const int j = r / B, c = (r % B) / nbit, b = r % nbit;
      const int2 tr = track_of(ntrack, fanout, nbit, c, j);
      const int src = wi * ntrack + (b == 0 ? tr.x : tr.y);
      for (int v = 0; v < 256; v++)
         if ((v >> (src & 7)) & 1) table[((src >> 3) * 256 + v) * 2 + (o >> 5)] |= 1u << (o & 31);
   }
}

// One thread per unit (4 bytes, or 8 at 64 tracks), the tables in shared
// memory.  The chunk starts on a track-word (grid_offset a multiple of
// ntrack / 8); the bytes of a track-word cut off by the chunk's end read as
// zero (modulation still applied).
__global__ void __launch_bounds__(256) k_track_turn(const uint8_t *__restrict__ in, long long nbytes,
                                                    long long grid_offset, int ntrack, int vlba, int aligned,
                                                    const uint2 *__restrict__ table, uint32_t *__restrict__ out)
{
   __shared__ uint2 s_tab[8 * 256];
   const int UB = ntrack > 32 ? 8 : 4;  // bytes per unit
   for (int i = threadIdx.x; i < UB * 256; i += blockDim.x) s_tab[i] = table[i];
   __syncthreads();
   const int tb = ntrack / 8;           // bytes per track-word
   const int tpu = UB / tb;             // track-words per unit
   const long long W0 = 8 * grid_offset / ntrack;  // grid track-word of the chunk's first byte
   const long long nunit = (nbytes + UB - 1) / UB;
   const long long nw = (nbytes + 3) / 4;
   for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < nunit;
        u += (long long)gridDim.x * blockDim.x) {
      const long long a = u * UB;
      uint32_t lo = 0u, hi = 0u;
      if (aligned && a + UB <= nbytes) {
         if (UB == 8) {
            const uint2 v = __ldg(reinterpret_cast<const uint2 *>(in + a));
            lo = v.x;
            hi = v.y;
         } else {
            lo = __ldg(reinterpret_cast<const uint32_t *>(in + a));
         }
      } else {
         // bytes of whole track-words (an unaligned source reads bytewise)
         const int whole = (int)std::min<long long>((nbytes - a) / tb * tb, UB);
         for (int k = 0; k < whole; k++) {
            if (k < 4) lo |= (uint32_t)in[a + k] << (8 * k);
            else hi |= (uint32_t)in[a + k] << (8 * (k - 4));
         }
      }
      if (vlba) {
         for (int t = 0; t < tpu; t++) {
            const int i = (int)((W0 + u * tpu + t) % 20000);
            if ((c_vlba_mod.w[i >> 5] >> (i & 31)) & 1u) {
               if (tb >= 4) {
                  lo = ~lo;
                  if (tb == 8) hi = ~hi;
               } else {
                  lo ^= ((1u << (8 * tb)) - 1u) << (8 * tb * t);
               }
            }
         }
      }
      uint32_t r0 = 0u, r1 = 0u;
#pragma unroll
      for (int p = 0; p < 4; p++) {
         const uint2 e = s_tab[p * 256 + ((lo >> (8 * p)) & 0xFFu)];
         r0 |= e.x;
         r1 |= e.y;
      }
      if (UB == 8) {
#pragma unroll
         for (int p = 0; p < 4; p++) {
            const uint2 e = s_tab[(4 + p) * 256 + ((hi >> (8 * p)) & 0xFFu)];
            r0 |= e.x;
            r1 |= e.y;
         }
         out[2 * u] = r0;
         if (2 * u + 1 < nw) out[2 * u + 1] = r1;
      } else {
         out[u] = r0;
      }
   }
}

cudaError_t launch_track_turn(cudaStream_t st, const uint8_t *in, long long nbytes, long long grid_offset,
                              int ntrack, int format, const uint32_t *table, uint32_t *out)
{
   const int UB = ntrack > 32 ? 8 : 4;
   const long long nunit = (nbytes + UB - 1) / UB;
   if (nunit == 0) return cudaSuccess;
   // a resident grid (8 CTAs of 256 threads per SM) striding over the
   // units, so each CTA loads the tables once for many units
   const long long nblk = std::min<long long>((nunit + 255) / 256, 148LL * 8);
   const int aligned = ((uintptr_t)in % UB) == 0 ? 1 : 0;
   k_track_turn<<<(unsigned)nblk, 256, 0, st>>>(in, nbytes, grid_offset, ntrack,
                                                 format == SWSGPU_FMT_VLBA ? 1 : 0, aligned,
                                                 reinterpret_cast<const uint2 *>(table), out);
   return cudaGetLastError();
}

// Corner turn into a phase-decimated code layout.  For decimation D (the
// FFT plan's cluster size), sample s of a channel is stored in phase array
// s % D at index s / D, SPW = 32/NBIT codes per 32-bit word:
//   codes[c * D * wpp + (s % D) * wpp + (s / D) / SPW], bits NBIT * ((s / D) % SPW).
// A CTA of the FFT cluster that owns residue p then reads its samples as one
// contiguous run.
//
// One CTA owns G consecutive code words (a multiple of 32) of every phase of
// every requested channel, i.e. the sample-times of G*SW payload words
// (SW = D * nchan words hold the SPW*D sample-times behind one code word).
//   1. The chunk's payload words are read once, coalesced (16-byte loads
//      when frames allow), into shared memory with one pad word per SW so
//      that lanes reading the same offset of consecutive blocks hit
//      distinct banks.  Words outside their frame's valid range read as 0
//      and are flagged in a shared bitmap.
//   2. A warp builds 32 consecutive code words of one phase: each lane
//      gathers its SPW sample-times.  When one payload word is exactly one
//      sample-time of 32/NBIT channels (16 ch x 2 bit, 32 x 1, 4 x 8) the
//      lane loads SPW words and transposes the SPW x SPW matrix of NBIT-bit
//      codes in registers, giving every channel's code word at once; other
//      layouts extract channel by channel.  Stores are 128-byte rows.
//   3. With any blanked frame in the run, the CTA writes the blank bitmap
//      words of its sample-times (1 bit per sample-time, standard order);
//      otherwise the bitmap is left unwritten and unread.
__host__ __device__ constexpr uint32_t transpose_mask(int sh)
{
   // low sh bits of every 2*sh-bit group
   uint32_t m = 0u;
   for (int i = 0; i < 32; i += 2 * sh) m |= ((1u << sh) - 1u) << i;
   return m;
}

// In-register transpose of the E x E matrix of NBIT-bit codes held in
// x[0..E), E = 32/NBIT: code (r, c) at bits NBIT*c of x[r] moves to bits
// NBIT*r of x[c].  Block swaps of halving size (E/2, ..., 1 codes).
template <int NBIT>
__device__ __forceinline__ void transpose_codes(uint32_t (&x)[32 / NBIT])
{
   constexpr int E = 32 / NBIT;
#pragma unroll
   for (int j = E / 2; j >= 1; j >>= 1) {
      const int sh = NBIT * j;
      const uint32_t mask = transpose_mask(sh);
#pragma unroll
      for (int r = 0; r < E; r++)
         if (!(r & j)) {
            const uint32_t t = ((x[r] >> sh) ^ x[r + j]) & mask;
            x[r + j] ^= t;
            x[r] ^= t << sh;
         }
   }
}

struct UnpackGeom {
   int D, G, SW, nw;   // decimation, code words per CTA, payload words per block, per chunk
   int vec16;          // 16-byte payload loads allowed
   long long wpp, words_total, blank_words;
   // Phase blocks (decimations whose D * nchan payload words per code word
   // exceed shared memory): CTA (x, y) owns phases [y Dt, (y + 1) Dt) and
   // reads, per code word, SPW pieces of PW = Dt nchan nbit / 32 payload
   // words RS = D nchan nbit / 32 words apart; SW = Dt nchan.  Without
   // phase blocks Dt = D and the pieces are contiguous.
   int pblock, Dt, PW;
   long long RS;
};

template <int NBIT>
__global__ void __launch_bounds__(256) k_unpack_codes(StreamIn s, long long nsamp, const int *chans, int nch,
                                                      uint32_t *codes, UnpackGeom g, const int2 *valid,
                                                      const int *blank_any, uint32_t *blank)
{
   constexpr int SPW = 32 / NBIT;
   constexpr uint32_t MASK = (NBIT == 32) ? 0xffffffffu : ((1u << NBIT) - 1u);
   extern __shared__ uint32_t sm[];
   const int SW = g.SW, SWp = g.SW + 1, nw = g.nw, D = g.D, Dt = g.Dt;
   const int ph0 = blockIdx.y * Dt;
   uint32_t *vbits = sm + (size_t)g.G * SWp;          // invalid-word flags, nw / 32 words
   int *pos = reinterpret_cast<int *>(vbits + nw / 32);  // channel -> output slot (transpose path)
   int *sch = pos + SPW;                                 // requested channels
   const bool any = *blank_any != 0;
   const long long w0 = (long long)blockIdx.x * nw;
   const bool tpath = (s.nchan * NBIT == 32);
   // sample-times of a 1/R payload word (R = 2: 8 x 2 bit, 16 x 1, 2 x 8;
   // R = 4: 4 x 2 bit, 8 x 1; R = 8, 16: 2 x 2 bit, 4 x 1, 2 x 1) at a phase
   // count that R divides: a payload word holds R consecutive phases of
   // the same row
   const int BW = s.nchan * NBIT;
   const int RPW = (s.nchan > 1 && BW < 32 && 32 % BW == 0) ? 32 / BW : 0;
   const bool tpath2 = RPW > 0 && Dt % RPW == 0;
   for (int j = threadIdx.x; j < nch; j += blockDim.x) sch[j] = chans[j];
   if (tpath || tpath2)
      for (int c = threadIdx.x; c < SPW; c += blockDim.x) {
         int p = -1;
         for (int k = 0; k < nch; k++)
            if (chans[k] == c) p = k;
         pos[c] = p;
      }
   if (any)
      for (int j = threadIdx.x; j < nw / 32; j += blockDim.x) vbits[j] = 0u;
   __syncthreads();

   // 1. payload words -> shared memory
   const int pb = s.payload_bytes;
   if (g.pblock) {
      // piece q / nq (code word iw = piece / SPW, sample offset k = piece % SPW)
      // covers sample-times ((x G + iw) SPW + k) D + y Dt + [0, Dt)
      constexpr int UNR = 4;
      const int wpl = g.vec16 ? 4 : 1;
      const int nq = g.PW / wpl, nload = g.G * SPW * nq;
      const bool need_f = s.header_bytes != 0 || any;  // frame position for headers / validity
      const long long row0 = (long long)blockIdx.x * g.G * SPW, col0 = (long long)blockIdx.y * g.PW;
      for (int qb = threadIdx.x; qb < nload; qb += UNR * blockDim.x) {
         uint32_t val[UNR][4];
         long long fu[UNR];
         int ou[UNR];
#pragma unroll
         for (int u = 0; u < UNR; u++) {
            const int q = qb + u * blockDim.x;
            const int piece = q / nq;
            const long long gw = (row0 + piece) * g.RS + col0 + (long long)(q - piece * nq) * wpl;
            const long long v = s.grid_offset + 4 * gw;
            fu[u] = need_f ? v / pb : 0;
            ou[u] = (int)(v - fu[u] * pb);
#pragma unroll
            for (int i = 0; i < 4; i++) val[u][i] = 0u;
            if (q < nload && gw < g.words_total) {
               const long long a = s.header_bytes ? fu[u] * s.frame_bytes + s.header_bytes + ou[u] : 4 * gw;
               if (wpl == 4 && a + 16 <= s.nbytes) {
                  const uint4 t = __ldg(reinterpret_cast<const uint4 *>(s.data + a));
                  val[u][0] = t.x;
                  val[u][1] = t.y;
                  val[u][2] = t.z;
                  val[u][3] = t.w;
               } else {
                  for (int i = 0; i < wpl; i++)
                     if (a + 4 * i + 4 <= s.nbytes) val[u][i] = __ldg(reinterpret_cast<const uint32_t *>(s.data + a + 4 * i));
               }
            }
         }
#pragma unroll
         for (int u = 0; u < UNR; u++) {
            const int q = qb + u * blockDim.x;
            if (q >= nload) break;
            const int piece = q / nq;
            const long long gw = (row0 + piece) * g.RS + col0 + (long long)(q - piece * nq) * wpl;
            const int jl = piece * g.PW + (q - piece * nq) * wpl;
            for (int i = 0; i < wpl; i++) {
               uint32_t x = val[u][i];
               if (s.msb2) x = swap2_in_bytes(x);
               if (gw + i >= g.words_total) x = 0u;
               else if (any) {
                  const int oi = ou[u] + 4 * i;
                  const int2 vr = valid_range(s, valid, fu[u], oi);
                  if (!(oi >= vr.x && oi < vr.y)) x = 0u;
               }
               sm[jl + i + piece / SPW] = x;  // one pad word per code word's block
            }
         }
      }
   } else if (g.vec16) {
      // UNR 16-byte loads in flight per thread before any shared store
      constexpr int UNR = 4;
      const int step = 16 * blockDim.x;
      long long v = s.grid_offset + 4 * (w0 + 4 * threadIdx.x);
      long long f = v / pb;
      int o = (int)(v - f * pb);
      for (int jb = 4 * threadIdx.x; jb < nw; jb += UNR * 4 * blockDim.x) {
         uint4 q[UNR];
         long long fu[UNR];
         int ou[UNR];
#pragma unroll
         for (int u = 0; u < UNR; u++) {
            const int j = jb + u * 4 * blockDim.x;
            const long long w = w0 + j;
            fu[u] = f;
            ou[u] = o;
            q[u] = make_uint4(0u, 0u, 0u, 0u);
            if (j < nw && w < g.words_total) {
               const long long a = s.header_bytes ? f * s.frame_bytes + s.header_bytes + o : v - s.grid_offset;
               if (a + 16 <= s.nbytes) {
                  q[u] = __ldg(reinterpret_cast<const uint4 *>(s.data + a));
               } else {
                  // ragged end of the buffer: word by word
                  uint32_t t4[4] = {0u, 0u, 0u, 0u};
                  for (int i = 0; i < 4; i++)
                     if (a + 4 * i + 4 <= s.nbytes) t4[i] = __ldg(reinterpret_cast<const uint32_t *>(s.data + a + 4 * i));
                  q[u] = make_uint4(t4[0], t4[1], t4[2], t4[3]);
               }
            }
            v += step;
            o += step;
            while (o >= pb) {
               o -= pb;
               f++;
            }
         }
#pragma unroll
         for (int u = 0; u < UNR; u++) {
            const int j = jb + u * 4 * blockDim.x;
            if (j >= nw) break;
            const long long w = w0 + j;
            uint32_t val[4] = {q[u].x, q[u].y, q[u].z, q[u].w};
            if (s.msb2)
               for (int i = 0; i < 4; i++) val[i] = swap2_in_bytes(val[i]);
            const int pj = j / SW, rj = j - pj * SW;  // block and offset of word j
#pragma unroll
            for (int i = 0; i < 4; i++) {
               if (w + i >= g.words_total) val[i] = 0u;
               else if (any) {
                  const int oi = ou[u] + 4 * i;
                  const int2 vr = valid_range(s, valid, fu[u], oi);
                  if (!(oi >= vr.x && oi < vr.y)) {
                     val[i] = 0u;
                     atomicOr(&vbits[(j + i) >> 5], 1u << ((j + i) & 31));
                  }
               }
               sm[j + i + pj + (SW >= 4 ? (int)(rj + i >= SW) : (rj + i) / SW)] = val[i];
            }
         }
      }
   } else {
      const int step = 4 * blockDim.x;
      long long v = s.grid_offset + 4 * (w0 + threadIdx.x);
      long long f = v / pb;
      int o = (int)(v - f * pb);
      for (int j = threadIdx.x; j < nw; j += blockDim.x) {
         uint32_t val = 0u;
         const long long w = w0 + j;
         if (w < g.words_total) {
            const long long a = s.header_bytes ? f * s.frame_bytes + s.header_bytes + o : v - s.grid_offset;
            if (a + 4 <= s.nbytes) val = __ldg(reinterpret_cast<const uint32_t *>(s.data + a));
            if (s.msb2) val = swap2_in_bytes(val);
            if (any) {
               const int2 vr = valid_range(s, valid, f, o);
               if (!(o >= vr.x && o < vr.y)) {
                  val = 0u;
                  atomicOr(&vbits[j >> 5], 1u << (j & 31));
               }
            }
         }
         sm[j + j / SW] = val;
         v += step;
         o += step;
         while (o >= pb) {
            o -= pb;
            f++;
         }
      }
   }
   __syncthreads();

   // 2. code words, one warp task = 32 consecutive words of one phase
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
   const long long code_words = (long long)D * g.wpp;
   if (s.nchan == 1 && Dt % SPW == 0) {
      // One channel: payload word wc of sample index iw SPW + k (row k of
      // the block) holds phases wc SPW + m at bits NBIT m, so the SPW x SPW
      // transpose gives SPW phases' code words at once.
      const int PWs = Dt / SPW;
      const int nt1 = PWs * (g.G / 32);
      for (int t = warp; t < nt1; t += nwarp) {
         const int wc = t % PWs;
         const int iw = (t / PWs) * 32 + lane;
         const long long iwg = (long long)blockIdx.x * g.G + iw;
         const uint32_t *blk = sm + (size_t)iw * SWp;
         uint32_t x[SPW];
#pragma unroll
         for (int k = 0; k < SPW; k++) x[k] = blk[k * PWs + wc];
         transpose_codes<NBIT>(x);
         if (iwg < g.wpp) {
#pragma unroll
            for (int m = 0; m < SPW; m++) codes[(long long)(ph0 + wc * SPW + m) * g.wpp + iwg] = x[m];
         }
      }
   } else if (s.nchan == 1 && Dt == 1) {
      // one channel, no decimation: the code words are the payload words
      for (int iw = threadIdx.x; iw < g.G; iw += blockDim.x) {
         const long long iwg = (long long)blockIdx.x * g.G + iw;
         if (iwg < g.wpp) codes[iwg] = sm[(size_t)iw * SWp];
      }
   } else if (tpath2) {
      // Row k of a code word's block holds phases R pp ... R pp + R - 1 in
      // one payload word, so the SPW x SPW transpose gives those phases'
      // code words of every channel: code word c' is channel c' % nchan of
      // phase R pp + c' / nchan.
      const int nc = s.nchan, WR = Dt / RPW;  // payload words per row
      const int ntask = WR * (g.G / 32);
      for (int t = warp; t < ntask; t += nwarp) {
         const int pp = t % WR;
         const int iw = (t / WR) * 32 + lane;
         const long long iwg = (long long)blockIdx.x * g.G + iw;
         const uint32_t *blk = sm + (size_t)iw * SWp;
         uint32_t x[SPW];
#pragma unroll
         for (int k = 0; k < SPW; k++) x[k] = blk[k * WR + pp];
         transpose_codes<NBIT>(x);
         if (iwg < g.wpp) {
#pragma unroll
            for (int c = 0; c < SPW; c++) {
               const int p = pos[c % nc];
               if (p >= 0)
                  codes[(long long)p * code_words + (long long)(ph0 + RPW * pp + c / nc) * g.wpp + iwg] = x[c];
            }
         }
      }
   } else {
   const int ntask = Dt * (g.G / 32);
   for (int t = warp; t < ntask; t += nwarp) {
      const int ph = t % Dt;
      const int iw = (t / Dt) * 32 + lane;
      const long long iwg = (long long)blockIdx.x * g.G + iw;
      const uint32_t *blk = sm + (size_t)iw * SWp;
      if (tpath) {
         uint32_t x[SPW];
#pragma unroll
         for (int k = 0; k < SPW; k++) x[k] = blk[k * Dt + ph];
         transpose_codes<NBIT>(x);
         if (iwg < g.wpp) {
#pragma unroll
            for (int c = 0; c < SPW; c++) {
               const int p = pos[c];
               if (p >= 0) codes[(long long)p * code_words + (long long)(ph0 + ph) * g.wpp + iwg] = x[c];
            }
         }
      } else {
         const int stride = s.nchan * NBIT;
         for (int c0 = 0; c0 < nch; c0 += 16) {
            const int cn = min(16, nch - c0);
            uint32_t acc[16];
#pragma unroll
            for (int c = 0; c < 16; c++) acc[c] = 0u;
            int cached_idx = -1;
            uint32_t cached = 0u;
            for (int k = 0; k < SPW; k++) {
               const int bit0 = (k * Dt + ph) * stride;
#pragma unroll
               for (int c = 0; c < 16; c++) {
                  if (c < cn) {
                     const int bit = bit0 + sch[c0 + c] * NBIT;
                     const int widx = bit >> 5;
                     if (widx != cached_idx) {
                        cached = blk[widx];
                        cached_idx = widx;
                     }
                     acc[c] |= ((cached >> (bit & 31)) & MASK) << (NBIT * k);
                  }
               }
            }
            if (iwg < g.wpp) {
#pragma unroll
               for (int c = 0; c < 16; c++)
                  if (c < cn) codes[(long long)(c0 + c) * code_words + (long long)(ph0 + ph) * g.wpp + iwg] = acc[c];
            }
         }
      }
   }

   }

   // 3. blank bitmap words of the chunk's sample-times (k_blank_bits with
   // phase blocks, whose sample-times are not contiguous)
   if (any && !g.pblock) {
      const int stride = s.nchan * NBIT;
      const int nbw = g.G * SPW * D / 32;
      const long long b0 = (long long)blockIdx.x * nbw;
      for (int j = threadIdx.x; j < nbw; j += blockDim.x) {
         if (b0 + j >= g.blank_words) break;
         uint32_t m = 0u;
         for (int i = 0; i < 32; i++) {
            const long long st = 32ll * j + i;   // sample-time within the chunk
            const int widx = (int)((st * stride) >> 5);
            if ((b0 + j) * 32 + i < nsamp && ((vbits[widx >> 5] >> (widx & 31)) & 1u)) m |= 1u << i;
         }
         blank[b0 + j] = m;
      }
   }
}

// Blank bitmap for phase-blocked corner turns, with the rule of step 3
// above: sample-time t is blanked when the payload word holding its first
// bit lies outside its frame's valid byte range.
__global__ void k_blank_bits(StreamIn s, long long nsamp, long long words_total, long long blank_words,
                             const int2 *valid, const int *blank_any, uint32_t *blank)
{
   if (*blank_any == 0) return;
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= blank_words) return;
   const int stride = s.nchan * s.nbit;
   uint32_t m = 0u;
   for (int i = 0; i < 32; i++) {
      const long long t = 32 * j + i;
      if (t >= nsamp) break;
      const long long w = (t * stride) >> 5;
      if (w >= words_total) continue;
      const long long v = s.grid_offset + 4 * w;
      const long long f = v / s.payload_bytes;
      const int o = (int)(v - f * s.payload_bytes);
      const int2 vr = valid_range(s, valid, f, o);
      if (!(o >= vr.x && o < vr.y)) m |= 1u << i;
   }
   blank[j] = m;
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
   const int2 vr = valid_range(s, valid, f, o);
   float val = 0.0f;
   if (o >= vr.x && o < vr.y) {
      long long widx = bit >> 5;
      uint32_t word = *reinterpret_cast<const uint32_t *>(s.data + payload_addr(s, s.grid_offset + 4 * widx));
      if (s.msb2) word = swap2_in_bytes(word);
      uint32_t code = (word >> (bit & 31)) & ((nbit == 8) ? 0xffu : ((1u << nbit) - 1u));
      if (nbit == 8) val = fmaf(levels.x, (float)(code ^ __float_as_uint(levels.z)), levels.y);
      else if (nbit == 2) val = (code == 0) ? levels.x : (code == 1) ? levels.y : (code == 2) ? levels.z : levels.w;
      else val = code ? levels.y : levels.x;
      atomicAdd(nvalid, 1ull);
   }
   out[t] = val;
}

// Largest phase block Dt | D whose pieces are whole 16-byte loads (else
// whole words) with at most kMaxBlockWords payload words per code word;
// 0 when there is none.
static constexpr int kMaxBlockWords = 512;
static int phase_block(int D, int nchan, int nbit, bool *whole16)
{
   for (int unit : {128, 32}) {
      int best = 0;
      for (int dt = 1; dt <= D && dt * nchan <= kMaxBlockWords; dt++)
         if (D % dt == 0 && ((long long)dt * nchan * nbit) % unit == 0) best = dt;
      if (best) {
         if (whole16) *whole16 = unit == 128;
         return best;
      }
   }
   return 0;
}

bool unpack_decimation_ok(int D, int nchan, int nbit)
{
   return D * nchan <= kMaxBlockWords || phase_block(D, nchan, nbit, nullptr) > 0;
}

UnpackGeom unpack_geometry(const StreamIn &s, long long nsamp, int D, long long wpp)
{
   UnpackGeom g;
   g.D = D;
   g.wpp = wpp;
   g.words_total = (nsamp * s.nchan * s.nbit + 31) / 32;
   g.blank_words = (nsamp + 31) / 32;
   const bool frames16 = (s.payload_bytes % 16 == 0) &&
                         (s.header_bytes == 0 || (s.header_bytes % 16 == 0 && s.frame_bytes % 16 == 0));
   g.vec16 = frames16 && (s.grid_offset % 16 == 0) && ((uintptr_t)s.data % 16 == 0);
   bool whole16 = false;
   g.pblock = D * s.nchan > kMaxBlockWords;
   g.Dt = g.pblock ? phase_block(D, s.nchan, s.nbit, &whole16) : D;
   g.SW = g.Dt * s.nchan;
   g.G = g.pblock ? 32 : 32 * std::max(1, (8192 / std::max(g.SW, 1)) / 32);
   g.nw = g.G * g.SW;
   g.PW = (int)(((long long)g.Dt * s.nchan * s.nbit) / 32);
   g.RS = ((long long)D * s.nchan * s.nbit) / 32;
   if (g.pblock) g.vec16 = g.vec16 && whole16 && g.RS % 4 == 0;
   return g;
}

size_t unpack_smem_bytes(const UnpackGeom &g, int nch)
{
   return sizeof(uint32_t) * ((size_t)g.G * (g.SW + 1) + g.nw / 32 + 32 + nch);
}

template <int NBIT>
static cudaError_t launch_codes_t(const UnpackGeom &g, cudaStream_t st, StreamIn s, long long nsamp,
                                  const int *chans, int nch, uint32_t *codes, const int2 *valid,
                                  const int *blank_any, uint32_t *blank)
{
   const size_t smem = unpack_smem_bytes(g, nch);
   if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_unpack_codes<NBIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
   }
   const unsigned nblk = (unsigned)((g.wpp + g.G - 1) / g.G);
   k_unpack_codes<NBIT><<<dim3(nblk, (unsigned)(g.D / g.Dt)), 256, smem, st>>>(s, nsamp, chans, nch, codes, g, valid,
                                                                                blank_any, blank);
   return cudaGetLastError();
}

cudaError_t launch_unpack_codes(cudaStream_t st, StreamIn s, long long nsamp, const int *chans, int nch,
                                uint32_t *codes, int D, long long wpp, const int2 *valid,
                                const int *blank_any, uint32_t *blank, int &launches)
{
   const UnpackGeom g = unpack_geometry(s, nsamp, D, wpp);
   if (g.Dt <= 0 || unpack_smem_bytes(g, nch) > 227 * 1024) return cudaErrorInvalidValue;
   cudaError_t e;
   if (s.nbit == 1) e = launch_codes_t<1>(g, st, s, nsamp, chans, nch, codes, valid, blank_any, blank);
   else if (s.nbit == 2) e = launch_codes_t<2>(g, st, s, nsamp, chans, nch, codes, valid, blank_any, blank);
   else e = launch_codes_t<8>(g, st, s, nsamp, chans, nch, codes, valid, blank_any, blank);
   if (e != cudaSuccess) return e;
   launches++;
   if (g.pblock) {
      k_blank_bits<<<(unsigned)((g.blank_words + 255) / 256), 256, 0, st>>>(s, nsamp, g.words_total, g.blank_words,
                                                                            valid, blank_any, blank);
      launches++;
      e = cudaGetLastError();
   }
   return e;
}

}  // namespace sws
