/*
 * swspec_oracle.c -- CPU restatement of the SWSpec IPP spectrometer core.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline.  Only the test suite, the smoke check and the CPU-baseline leg of
 * the benchmark load it; the GPU product never links or calls it.
 *
 * It restates, without Intel IPP:
 *   - the mark5access level tables and bit layouts used to decode Mark5B and
 *     VDIF payloads (mark5access/mark5access/mark5_format_mark5b.c:59-96,
 *     :1690-1909 and mark5access/mark5access/format_vdif.c:69-143,
 *     :564-610, :1097-1137);
 *   - the window functions of TaskCoreIPP::generate_windowfunction
 *     (src/IA-32/TaskCoreIPP.cpp:569-605).  Hann = sin^2(pi n/(N-1)) as in
 *     src/IA-32/TaskCoreMKL.cpp:53 and src/Cell/TaskCoreFFTW.cpp:65; Hamming
 *     and Blackman(alpha) follow the published IPP definitions (IPP itself is
 *     closed and absent, so those two are unpinned); BlackmanHarris is the
 *     4-term Harris (1978) window, which the reference does not have;
 *   - the per-buffer loop of TaskCoreIPP::doMaths
 *     (src/IA-32/TaskCoreIPP.cpp:355-560): hop by N/overlap, DC/Nyquist
 *     handling, cross product X_i conj(X_j), scaling by 1/core_overlapped_ffts,
 *     the spectrum hop, the unscaled partial spectrum at the end of a buffer,
 *     and the PCal cadence curr_ffts % overlap (counted per source FFT);
 *   - TaskCoreIPP::extract_PCal (src/IA-32/TaskCoreIPP.cpp:633-693) with the
 *     rotator built in TaskCoreIPP::prepare (:129-136).
 *
 * Two arithmetic variants of the same loop are provided:
 *   orc_domaths64 : FP64 window products, FP64 FFT, FP64 accumulation -- the
 *                   accuracy reference ("FP64 oracle");
 *   orc_domaths32 : FP32 throughout with plain sums, one worker thread per
 *                   core, as the IPP core does -- the timed CPU baseline.
 * Both use this file's own mixed-radix (2,3,4,5,generic) Stockham FFT.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* Decoding (mark5access level tables)                                      */
/* ------------------------------------------------------------------------ */

#define ORC_FMT_MARK5B 0
#define ORC_FMT_VDIF 1
#define ORC_FMT_RAW_SIGNED 2
#define ORC_FMT_RAW_UNSIGNED 3

static const float ORC_HIMAG = 3.3359f; /* OPTIMAL_2BIT_HIGH, mark5_stream.h:72 */

/* Value of one sample given its nbit-wide code (bit 0 = first bit in stream).
 * Mark5B 2-bit: level[sign + 2*mag] = {-H, +1, -1, +H}
 *   (mark5_format_mark5b.c:63, sign bit first); 1-bit: {+1, -1}[bit] (:62).
 * VDIF 2-bit: {-H, -1, +1, +H}[code] (format_vdif.c:73); 1-bit {-1,+1}
 *   (:72); 8-bit (2b-255)/256 (:117). */
static float orc_level(int fmt, int nbit, unsigned code)
{
   if (fmt == ORC_FMT_MARK5B) {
      if (nbit == 1) return code ? -1.0f : 1.0f;
      if (nbit == 2) {
         static const float l4[4] = {-3.3359f, 1.0f, -1.0f, 3.3359f};
         return l4[code & 3];
      }
   } else {
      if (nbit == 1) return code ? 1.0f : -1.0f;
      if (nbit == 2) {
         static const float l4[4] = {-3.3359f, -1.0f, 1.0f, 3.3359f};
         return l4[code & 3];
      }
      if (nbit == 8) return (float)(((double)code * 2.0 - 255.0) / 256.0);
   }
   return 0.0f;
}

/* The reference's raw unpackers (src/IA-32/DataUnpackers.cpp):
 * SignedUnpacker 8-bit: (signed char) byte (:68-90); UnsignedUnpacker
 * 8-bit: byte - 128 (:125-147); TwoBitUnpacker and the single-channel one:
 * map_rev[code] = {1, -1, 3.3359, -3.3359} (:214, :280). */
static float orc_raw_level(int fmt, int nbit, unsigned code)
{
   if (nbit == 8) return fmt == ORC_FMT_RAW_SIGNED ? (float)(signed char)code : (float)code - 128.0f;
   static const float map_rev[4] = {1.0f, -1.0f, 3.3359f, -3.3359f};
   return map_rev[code & 3];
}

/* Raw sampler data, channel `chan` (0-based, as the unpacker sees it):
 *  8-bit: byte t*nchan + chan (SignedUnpacker / UnsignedUnpacker :74-78);
 *  2-bit, nchan % 4 == 0: byte t*nchan/4 + chan/4, bits 2*(chan%4) .. +1
 *    (TwoBitUnpacker :207-243 with ChannelOrderIncreasing; the decreasing
 *    order is channel nchan-1-chan);
 *  2-bit, one channel: byte t/4, bits 6-2*(t%4) .. +1, the oldest sample
 *    in the most significant bits (TwoBitSinglechannelUnpacker :261-265;
 *    its table lookup at :280-284 masks with the top two bits for every
 *    sample position, so only the first sample of each byte reads a
 *    defined table entry there: this restates the layout the function
 *    documents). */
static int orc_decode_raw(int fmt, int nchan, int nbit, const uint8_t *payload, int64_t nsamp, int chan,
                          float *out)
{
   if (nbit == 8) {
      for (int64_t t = 0; t < nsamp; t++) out[t] = orc_raw_level(fmt, 8, payload[t * nchan + chan]);
      return 0;
   }
   if (nbit != 2) return -1;
   if (nchan == 1) {
      for (int64_t t = 0; t < nsamp; t++) out[t] = orc_raw_level(fmt, 2, (payload[t >> 2] >> (6 - 2 * (t & 3))) & 3u);
      return 0;
   }
   if (nchan % 4) return -1;
   const int64_t step = nchan / 4;
   for (int64_t t = 0; t < nsamp; t++)
      out[t] = orc_raw_level(fmt, 2, (payload[t * step + chan / 4] >> (2 * (chan % 4))) & 3u);
   return 0;
}

/* Decode channel `chan` of a header-free payload byte stream: sample-time t
 * occupies nchan*nbit consecutive bits starting at bit t*nchan*nbit, channel c
 * at bit offset c*nbit inside it, bits numbered LSB-first within each byte.
 * This is the layout every mark5access Mark5B decoder and the single-thread
 * VDIF decoders read. */
int orc_decode(int fmt, int nchan, int nbit, const uint8_t *payload, int64_t nsamp, int chan,
               float *out)
{
   if (chan < 0 || chan >= nchan) return -1;
   if (fmt == ORC_FMT_RAW_SIGNED || fmt == ORC_FMT_RAW_UNSIGNED)
      return orc_decode_raw(fmt, nchan, nbit, payload, nsamp, chan, out);
   const int64_t stride = (int64_t)nchan * nbit;
   for (int64_t t = 0; t < nsamp; t++) {
      int64_t bit = t * stride + (int64_t)chan * nbit;
      unsigned code = 0;
      for (int b = 0; b < nbit; b++) {
         int64_t p = bit + b;
         code |= ((payload[p >> 3] >> (p & 7)) & 1u) << b;
      }
      out[t] = orc_level(fmt, nbit, code);
   }
   (void)ORC_HIMAG;
   return 0;
}

/* ------------------------------------------------------------------------ */
/* Blanking (mark5access blankers)                                          */
/* ------------------------------------------------------------------------ */

#define ORC_FILL32 0x11223344u
#define ORC_FILL64 0x1122334411223344ull
#define ORC_ZONE_LOG2 15 /* blanker_mark5.c:138, 32768-byte zones */
#define ORC_BIG (1 << 30)

static uint64_t orc_w64(const uint8_t *p, int64_t w)
{
   uint64_t v;
   memcpy(&v, p + 8 * w, 8);
   return v;
}
static uint32_t orc_w32(const uint8_t *p, int64_t w)
{
   uint32_t v;
   memcpy(&v, p + 4 * w, 4);
   return v;
}

/* Binary search for the edge of a fill zone between 64-bit words [b, e) of
 * a payload, then the 32-bit straggler check (blanker_mark5.c:53-123).
 * want_fill = 1 finds the first fill word (start of a trailing zone),
 * 0 the first data word (end of a leading zone); byte offsets. */
static int orc_zone_edge(const uint8_t *pay, int b, int e, int want_fill)
{
   int n = e - b, i = n / 2, r = n - 1;
   for (int s = n / 4; s > 0; s >>= 1) {
      const int hit = (orc_w64(pay, b + i) == ORC_FILL64) == want_fill;
      if (hit) {
         r = i;
         i -= s;
      } else {
         i += s;
      }
   }
   r = 8 * (b + r);
   if (want_fill) {
      if (orc_w32(pay, r / 4 - 1) == ORC_FILL32) r -= 4;
   } else {
      if (orc_w32(pay, r / 4 - 2) == ORC_FILL32) r += 4;
   }
   return r;
}

/* Valid byte range [zs[z], ze[z]) of each zone of one frame payload:
 * Mark5B checks the first and last 64-bit word of every 32 KiB zone
 * (blanker_mark5.c:126-200), VDIF blanks a whole frame whose first or last
 * word is fill (:282-310) or whose header has the invalid bit set
 * (format_vdif.c:2873-2914).  Returns the number of zones. */
static int orc_frame_zones(int fmt, const uint8_t *pay, int payload_bytes, int invalid, int *zs, int *ze)
{
   const int nword = payload_bytes / 8;
   if (fmt == ORC_FMT_VDIF) {
      zs[0] = 0;
      ze[0] = (invalid || orc_w64(pay, 0) == ORC_FILL64 || orc_w64(pay, nword - 1) == ORC_FILL64) ? 0 : ORC_BIG;
      if (invalid) zs[0] = ORC_BIG;
      return 1;
   }
   const int zw = 1 << (ORC_ZONE_LOG2 - 3);
   int z = 0;
   for (int b = 0; b < nword; b += zw, z++) {
      const int e = (b + zw > nword) ? nword : b + zw;
      const int startOK = orc_w64(pay, b) != ORC_FILL64;
      const int endOK = orc_w64(pay, e - 1) != ORC_FILL64;
      if (startOK && endOK) {
         zs[z] = 0;
         ze[z] = ORC_BIG;
      } else if (!startOK && !endOK) {
         zs[z] = ORC_BIG;
         ze[z] = 0;
      } else if (startOK) {
         zs[z] = 0;
         ze[z] = orc_zone_edge(pay, b, e, 1);
      } else {
         zs[z] = orc_zone_edge(pay, b, e, 0);
         ze[z] = ORC_BIG;
      }
   }
   return z;
}

/* orc_decode with mark5access's blanking: the payload stream starts at a
 * frame boundary, frames are payload_bytes long, frame_invalid[f] (or NULL)
 * carries VDIF header invalid bits.  A sample-time whose first byte lies
 * outside its zone's valid range decodes to 0 (the per-byte test of every
 * mark5access decoder, e.g. mark5_format_mark5b.c:1216-1223).  Returns the
 * number of blanked sample-times, or -1. */
int64_t orc_decode_blanked(int fmt, int nchan, int nbit, const uint8_t *payload, int64_t payload_len,
                           int payload_bytes, const uint8_t *frame_invalid, int64_t nsamp, int chan,
                           float *out)
{
   if (chan < 0 || chan >= nchan || payload_bytes <= 0 || (payload_bytes % 8)) return -1;
   const int64_t stride = (int64_t)nchan * nbit;
   if (nsamp > 0 && ((nsamp * stride + 7) >> 3) > payload_len) return -1;
   if (orc_decode(fmt, nchan, nbit, payload, nsamp, chan, out)) return -1;
   const int maxz = (payload_bytes >> ORC_ZONE_LOG2) + 2;
   int *zs = (int *)malloc(sizeof(int) * maxz), *ze = (int *)malloc(sizeof(int) * maxz);
   int64_t nblank = 0, cur = -1;
   for (int64_t t = 0; t < nsamp; t++) {
      const int64_t byte = (t * stride) >> 3;
      const int64_t f = byte / payload_bytes;
      const int o = (int)(byte - f * payload_bytes);
      if (f != cur) {
         /* a frame cut short by the end of the stream is checked as far as it goes */
         if ((f + 1) * payload_bytes <= payload_len) {
            orc_frame_zones(fmt, payload + f * payload_bytes, payload_bytes, frame_invalid ? frame_invalid[f] : 0,
                            zs, ze);
         } else {
            zs[0] = 0;
            ze[0] = ORC_BIG;
            for (int z = 1; z < maxz; z++) zs[z] = 0, ze[z] = ORC_BIG;
         }
         cur = f;
      }
      const int z = (fmt == ORC_FMT_VDIF) ? 0 : (o >> ORC_ZONE_LOG2);
      if (o < zs[z] || o >= ze[z]) {
         out[t] = 0.0f;
         nblank++;
      }
   }
   free(zs);
   free(ze);
   return nblank;
}

/* ------------------------------------------------------------------------ */
/* Windows                                                                  */
/* ------------------------------------------------------------------------ */

enum { W_NONE = 0, W_COSINE, W_COSINE2, W_HAMMING, W_HANN, W_BLACKMAN, W_BLACKMANHARRIS };

/* FP32 window exactly as the reference builds it (double arithmetic on
 * float-valued arguments, rounded to float once). */
void orc_window(int type, int n, float *out)
{
   for (int i = 0; i < n; i++) {
      double w;
      double fi = (double)(float)i, fn = (double)(float)n;
      double a = 2.0 * M_PI * (double)i / (double)(n - 1);
      switch (type) {
      case W_NONE: w = 1.0; break;
      case W_COSINE: w = cos(M_PI * (fi - 0.5 * fn + 0.5) / fn); break;
      case W_COSINE2: {
         double c = cos(M_PI * (fi - 0.5 * fn + 0.5) / fn);
         w = c * c;
      } break;
      case W_HAMMING: w = 0.54 - 0.46 * cos(a); break;
      case W_HANN: {
         double s = sin(M_PI * (double)i / (double)(n - 1));
         w = s * s;
      } break;
      case W_BLACKMAN: /* IPP ippsWinBlackman, alpha = 0.5 hard-coded by the reference */
         w = (0.5 + 1.0) / 2.0 - 0.5 * cos(a) - (0.5 / 2.0) * cos(2.0 * a);
         break;
      case W_BLACKMANHARRIS:
         w = 0.35875 - 0.48829 * cos(a) + 0.14128 * cos(2.0 * a) - 0.01168 * cos(3.0 * a);
         break;
      default: w = 1.0; break;
      }
      out[i] = (float)w;
   }
}

/* ------------------------------------------------------------------------ */
/* Mixed-radix Stockham FFT (forward, unscaled), FP64 and FP32              */
/* ------------------------------------------------------------------------ */

typedef struct { double re, im; } c64;
typedef struct { float re, im; } c32;

static int orc_factor(int n, int *rad)
{
   int nr = 0;
   while (n % 4 == 0 && n > 4) { rad[nr++] = 4; n /= 4; }
   while (n % 2 == 0) { rad[nr++] = 2; n /= 2; }
   for (int p = 3; n > 1; p += 2)
      while (n % p == 0) { rad[nr++] = p; n /= p; }
   return nr;
}

/* W_n^k table in FP64: angle reduced exactly via integer k < n.  The last
 * table is cached per thread (callers free only tables they own). */
static __thread c64 *tw_cache = NULL;
static __thread int tw_cache_n = 0;
static c64 *orc_twiddles64(int n)
{
   if (tw_cache_n == n) return tw_cache;
   c64 *w = (c64 *)malloc(sizeof(c64) * (size_t)n);
   for (int k = 0; k < n; k++) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      w[k].re = cos(a);
      w[k].im = sin(a);
   }
   free(tw_cache);
   tw_cache = w;
   tw_cache_n = n;
   return w;
}

/* One radix-R DFT on v[0..R) in FP64 (generic, O(R^2) for odd primes). */
static void dft_small64(int R, c64 *v, const c64 *w, int n)
{
   c64 t[64];
   if (R == 2) {
      c64 a = v[0], b = v[1];
      v[0].re = a.re + b.re; v[0].im = a.im + b.im;
      v[1].re = a.re - b.re; v[1].im = a.im - b.im;
      return;
   }
   if (R == 4) {
      c64 a = v[0], b = v[1], c = v[2], d = v[3];
      c64 s0 = {a.re + c.re, a.im + c.im}, s1 = {a.re - c.re, a.im - c.im};
      c64 s2 = {b.re + d.re, b.im + d.im}, s3 = {b.re - d.re, b.im - d.im};
      v[0].re = s0.re + s2.re; v[0].im = s0.im + s2.im;
      v[2].re = s0.re - s2.re; v[2].im = s0.im - s2.im;
      v[1].re = s1.re + s3.im; v[1].im = s1.im - s3.re; /* s1 - i s3 */
      v[3].re = s1.re - s3.im; v[3].im = s1.im + s3.re; /* s1 + i s3 */
      return;
   }
   for (int k = 0; k < R; k++) {
      double sr = 0, si = 0;
      for (int r = 0; r < R; r++) {
         int idx = (int)(((long long)r * k % R) * (n / R));
         double wr = w[idx].re, wi = w[idx].im;
         sr += v[r].re * wr - v[r].im * wi;
         si += v[r].re * wi + v[r].im * wr;
      }
      t[k].re = sr; t[k].im = si;
   }
   memcpy(v, t, sizeof(c64) * (size_t)R);
}

/* Forward FFT, x (length n) -> out.  Stockham autosort, DIT:
 * for each pass with current span Ns and radix R, butterfly j reads
 * d0[j + r n/R], twiddles by W_{Ns R}^{(j mod Ns) r}, and writes
 * d1[(j/Ns) Ns R + (j mod Ns) + r Ns]. */
int orc_fft64(int n, const double *in_reim, double *out_reim)
{
   int rad[64];
   int nr = orc_factor(n, rad);
   c64 *w = orc_twiddles64(n);
   c64 *d0 = (c64 *)malloc(sizeof(c64) * (size_t)n);
   c64 *d1 = (c64 *)malloc(sizeof(c64) * (size_t)n);
   memcpy(d0, in_reim, sizeof(c64) * (size_t)n);
   int Ns = 1;
   for (int p = 0; p < nr; p++) {
      int R = rad[p];
      int nb = n / R;
      for (int j = 0; j < nb; j++) {
         c64 v[64];
         int k = j % Ns;
         for (int r = 0; r < R; r++) {
            c64 a = d0[j + r * nb];
            long long ti = (long long)k * r * (n / (Ns * R));
            c64 t = w[ti % n];
            v[r].re = a.re * t.re - a.im * t.im;
            v[r].im = a.re * t.im + a.im * t.re;
         }
         dft_small64(R, v, w, n);
         int dst = (j / Ns) * Ns * R + k;
         for (int r = 0; r < R; r++) d1[dst + r * Ns] = v[r];
      }
      c64 *tmp = d0; d0 = d1; d1 = tmp;
      Ns *= R;
   }
   memcpy(out_reim, d0, sizeof(c64) * (size_t)n);
   free(d0); free(d1);
   return 0;
}

/* FP32 plan: radices + FP32 twiddle table (values rounded from FP64). */
typedef struct {
   int n, nr, rad[64];
   c32 *w;
} plan32;

static plan32 *plan32_new(int n)
{
   plan32 *p = (plan32 *)calloc(1, sizeof(plan32));
   p->n = n;
   p->nr = orc_factor(n, p->rad);
   p->w = (c32 *)malloc(sizeof(c32) * (size_t)n);
   for (int k = 0; k < n; k++) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      p->w[k].re = (float)cos(a);
      p->w[k].im = (float)sin(a);
   }
   return p;
}

static void plan32_free(plan32 *p)
{
   if (!p) return;
   free(p->w);
   free(p);
}

static void dft_small32(int R, c32 *v, const c32 *w, int n)
{
   c32 t[64];
   if (R == 2) {
      c32 a = v[0], b = v[1];
      v[0].re = a.re + b.re; v[0].im = a.im + b.im;
      v[1].re = a.re - b.re; v[1].im = a.im - b.im;
      return;
   }
   if (R == 4) {
      c32 a = v[0], b = v[1], c = v[2], d = v[3];
      c32 s0 = {a.re + c.re, a.im + c.im}, s1 = {a.re - c.re, a.im - c.im};
      c32 s2 = {b.re + d.re, b.im + d.im}, s3 = {b.re - d.re, b.im - d.im};
      v[0].re = s0.re + s2.re; v[0].im = s0.im + s2.im;
      v[2].re = s0.re - s2.re; v[2].im = s0.im - s2.im;
      v[1].re = s1.re + s3.im; v[1].im = s1.im - s3.re;
      v[3].re = s1.re - s3.im; v[3].im = s1.im + s3.re;
      return;
   }
   for (int k = 0; k < R; k++) {
      float sr = 0, si = 0;
      for (int r = 0; r < R; r++) {
         int idx = (int)(((long long)r * k % R) * (n / R));
         float wr = w[idx].re, wi = w[idx].im;
         sr += v[r].re * wr - v[r].im * wi;
         si += v[r].re * wi + v[r].im * wr;
      }
      t[k].re = sr; t[k].im = si;
   }
   memcpy(v, t, sizeof(c32) * (size_t)R);
}

/* FP32 complex FFT in d0 (scratch d1); returns pointer to the result buffer. */
static c32 *fft32(const plan32 *pl, c32 *d0, c32 *d1)
{
   int n = pl->n, Ns = 1;
   for (int p = 0; p < pl->nr; p++) {
      int R = pl->rad[p];
      int nb = n / R;
      int tstep = n / (Ns * R);
      for (int j = 0; j < nb; j++) {
         c32 v[64];
         int k = j % Ns;
         for (int r = 0; r < R; r++) {
            c32 a = d0[j + r * nb];
            c32 t = pl->w[(long long)k * r * tstep % n];
            v[r].re = a.re * t.re - a.im * t.im;
            v[r].im = a.re * t.im + a.im * t.re;
         }
         dft_small32(R, v, pl->w, n);
         int dst = (j / Ns) * Ns * R + k;
         for (int r = 0; r < R; r++) d1[dst + r * Ns] = v[r];
      }
      c32 *tmp = d0; d0 = d1; d1 = tmp;
      Ns *= R;
   }
   return d0;
}

/* ------------------------------------------------------------------------ */
/* doMaths restatement                                                      */
/* ------------------------------------------------------------------------ */

/* Configuration of one core run.  Field meanings follow swspect_settings_t
 * (src/Settings.h:59-159); the sample counts are per source. */
typedef struct {
   int fft_points;            /* N */
   int overlap;               /* fft_overlap_factor */
   int core_overlapped_ffts;  /* FFTs per spectrum in one run */
   int num_sources;           /* 1 or more */
   int num_xpols;             /* cross pairs taken in the reference's pair order */
   int window;                /* window type */
   int extract_pcal;          /* 0/1 */
   int pcal_tonebins;
   int pcal_rotatorlen;
   double samplingfreq;
   double pcaloffsethz;
   int nthreads;              /* FP32 baseline only: worker threads */
} orc_cfg;

/* Pair order of doMaths (TaskCoreIPP.cpp:457-464): xp_i starts at 0,
 * xp_j = xp_i+1, and advances xp_i once xp_j exceeds the source count. */
int orc_xpol_pairs(int num_sources, int num_xpols, int *pairs)
{
   int xp_i = 0;
   for (int xp = 0; xp < num_xpols; xp++) {
      int xp_j = xp_i + 1;
      if (xp_j > num_sources) xp_j = (++xp_i) + 1;
      pairs[2 * xp] = xp_i;
      pairs[2 * xp + 1] = xp_j;
   }
   return 0;
}

/* Frame schedule of doMaths for one buffer of nsamp samples per source:
 * writes the first sample of each FFT and the spectrum it belongs to.
 * Returns the FFT count; *nspec gets the number of (possibly partial)
 * spectra and *partial whether the last one is an unscaled partial. */
int orc_schedule(const orc_cfg *c, int64_t nsamp, int64_t *starts, int *spec_of, int maxf,
                 int *nspec, int *partial)
{
   int64_t pos = 0, hop = c->fft_points / c->overlap;
   int nf = 0, acc = 0, ns = 0;
   while (nsamp - pos >= c->fft_points) {
      if (nf < maxf && starts) { starts[nf] = pos; spec_of[nf] = ns; }
      nf++;
      pos += hop;
      if (++acc >= c->core_overlapped_ffts) {
         ns++;
         acc = 0;
         pos += c->fft_points - hop;
      }
   }
   *partial = acc > 0;
   *nspec = ns + (acc > 0);
   return nf;
}

/* FP64 oracle over one buffer.
 * samples[s]   : decoded samples of source s (nsamp each)
 * out_auto     : [nspec][num_sources][N/2+1]
 * out_xpol     : [nspec][num_xpols][N/2+1][2]
 * out_pcal     : [nspec][num_sources][tonebins][2]
 * Returns number of spectra (incl. a trailing partial one). */
typedef struct {
   const orc_cfg *c;
   const float *const *samples;
   const int64_t *starts;
   const int *spec_of;
   int f0, f1;
   const float *win;
   const c64 *rot;
   const int *pairs;
   double *auto_acc, *xpol_acc, *pcal_acc; /* [nspec][...] (thread-private when threaded) */
} orc_job64;

static void *orc_worker64(void *arg)
{
   orc_job64 *j = (orc_job64 *)arg;
   const orc_cfg *c = j->c;
   const int N = c->fft_points, S = N / 2 + 1;
   double *in = (double *)malloc(sizeof(double) * 2 * (size_t)N);
   double **X = (double **)malloc(sizeof(double *) * (size_t)c->num_sources);
   for (int s = 0; s < c->num_sources; s++) X[s] = (double *)malloc(sizeof(double) * 2 * (size_t)N);
   /* curr_ffts counts source FFTs in doMaths order (TaskCoreIPP.cpp:633) */
   int curr_ffts = j->f0 * c->num_sources;
   for (int f = j->f0; f < j->f1; f++) {
      int sp = j->spec_of[f];
      for (int s = 0; s < c->num_sources; s++) {
         const float *x = j->samples[s] + j->starts[f];
         if (c->extract_pcal && (curr_ffts % c->overlap) == 0) {
            double *pc = j->pcal_acc + 2 * ((size_t)sp * c->num_sources + s) * c->pcal_tonebins;
            /* only whole tone periods of each rotator block are folded
             * (the reference's integer division rotatorlen/tonebins) */
            int used = (c->pcal_rotatorlen / c->pcal_tonebins) * c->pcal_tonebins;
            for (int n = 0; n < N; n++) {
               int ph = n % c->pcal_rotatorlen;
               if (ph >= used) continue;
               int b = ph % c->pcal_tonebins;
               pc[2 * b] += (double)x[n] * j->rot[ph].re;
               pc[2 * b + 1] += (double)x[n] * j->rot[ph].im;
            }
         }
         for (int n = 0; n < N; n++) {
            in[2 * n] = (double)x[n] * (double)j->win[n];
            in[2 * n + 1] = 0.0;
         }
         orc_fft64(N, in, X[s]);
         curr_ffts++;
         double *oa = j->auto_acc + ((size_t)sp * c->num_sources + s) * S;
         for (int k = 0; k < S; k++) oa[k] += X[s][2 * k] * X[s][2 * k] + X[s][2 * k + 1] * X[s][2 * k + 1];
      }
      for (int xp = 0; xp < c->num_xpols; xp++) {
         const double *A = X[j->pairs[2 * xp]], *B = X[j->pairs[2 * xp + 1]];
         double *ox = j->xpol_acc + 2 * ((size_t)sp * c->num_xpols + xp) * S;
         for (int k = 0; k < S; k++) {
            ox[2 * k] += A[2 * k] * B[2 * k] + A[2 * k + 1] * B[2 * k + 1];
            ox[2 * k + 1] += A[2 * k + 1] * B[2 * k] - A[2 * k] * B[2 * k + 1];
         }
         ox[1] = 0.0;
         ox[2 * (S - 1) + 1] = 0.0;
      }
   }
   free(in);
   for (int s = 0; s < c->num_sources; s++) free(X[s]);
   free(X);
   return NULL;
}

/* FP64 oracle over one buffer (doMaths, TaskCoreIPP.cpp:355-560).  With
 * c->nthreads > 1 the FFTs are split into contiguous ranges, one per
 * thread, and the thread-private FP64 sums are added in thread order. */
int orc_domaths64(const orc_cfg *c, const float *const *samples, int64_t nsamp, double *out_auto,
                  double *out_xpol, double *out_pcal)
{
   const int N = c->fft_points, S = N / 2 + 1;
   int nspec, partial;
   int nf = orc_schedule(c, nsamp, NULL, NULL, 0, &nspec, &partial);
   int64_t *starts = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nf + 1));
   int *spec_of = (int *)malloc(sizeof(int) * (size_t)(nf + 1));
   orc_schedule(c, nsamp, starts, spec_of, nf, &nspec, &partial);

   float *win = (float *)malloc(sizeof(float) * (size_t)N);
   orc_window(c->window, N, win);
   int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(c->num_xpols + 1));
   orc_xpol_pairs(c->num_sources, c->num_xpols, pairs);
   c64 *rot = NULL;
   if (c->extract_pcal) {
      rot = (c64 *)malloc(sizeof(c64) * (size_t)c->pcal_rotatorlen);
      double dphi = 2 * M_PI * (-c->pcaloffsethz / c->samplingfreq);
      for (int i = 0; i < c->pcal_rotatorlen; i++) {
         rot[i].re = cos(dphi * (double)i);
         rot[i].im = sin(dphi * (double)i);
      }
   }
   size_t na = (size_t)nspec * c->num_sources * S, nx = 2 * (size_t)nspec * c->num_xpols * S,
          np = 2 * (size_t)nspec * c->num_sources * (c->extract_pcal ? c->pcal_tonebins : 0);
   memset(out_auto, 0, sizeof(double) * na);
   if (nx) memset(out_xpol, 0, sizeof(double) * nx);
   if (np) memset(out_pcal, 0, sizeof(double) * np);

   int nt = c->nthreads < 1 ? 1 : c->nthreads;
   if (nt > nf) nt = nf > 0 ? nf : 1;
   orc_job64 *jobs = (orc_job64 *)calloc((size_t)nt, sizeof(orc_job64));
   pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
   for (int t = 0; t < nt; t++) {
      orc_job64 *j = &jobs[t];
      j->c = c; j->samples = samples; j->starts = starts; j->spec_of = spec_of;
      j->f0 = (int)((long long)nf * t / nt);
      j->f1 = (int)((long long)nf * (t + 1) / nt);
      j->win = win; j->rot = rot; j->pairs = pairs;
      if (nt == 1) {
         j->auto_acc = out_auto; j->xpol_acc = out_xpol; j->pcal_acc = out_pcal;
         orc_worker64(j);
      } else {
         j->auto_acc = (double *)calloc(na + 1, sizeof(double));
         j->xpol_acc = (double *)calloc(nx + 1, sizeof(double));
         j->pcal_acc = (double *)calloc(np + 1, sizeof(double));
         pthread_create(&th[t], NULL, orc_worker64, j);
      }
   }
   if (nt > 1) {
      for (int t = 0; t < nt; t++) {
         pthread_join(th[t], NULL);
         for (size_t i = 0; i < na; i++) out_auto[i] += jobs[t].auto_acc[i];
         for (size_t i = 0; i < nx; i++) out_xpol[i] += jobs[t].xpol_acc[i];
         for (size_t i = 0; i < np; i++) out_pcal[i] += jobs[t].pcal_acc[i];
         free(jobs[t].auto_acc); free(jobs[t].xpol_acc); free(jobs[t].pcal_acc);
      }
   }
   /* scale completed spectra; a trailing partial spectrum stays unscaled */
   int nfull = nspec - partial;
   double sc = 1.0 / (double)c->core_overlapped_ffts;
   for (size_t i = 0; i < (size_t)nfull * c->num_sources * S; i++) out_auto[i] *= sc;
   for (size_t i = 0; i < 2 * (size_t)nfull * c->num_xpols * S; i++) out_xpol[i] *= sc;

   free(jobs); free(th); free(starts); free(spec_of); free(win); free(pairs); free(rot);
   return nspec;
}

/* ---------------- FP32 baseline (threaded over contiguous FFT ranges) --- */

typedef struct {
   const orc_cfg *c;
   const float *const *samples;
   const int64_t *starts;
   const int *spec_of;
   int f0, f1;
   const float *win;
   const plan32 *pl;   /* N-point plan (odd N) or the N/2-point plan of the real FFT */
   const c32 *wn;      /* W_N^k, k < N/2: real-FFT post-processing twiddles (even N) */
   const c32 *rot;
   const int *pairs;
   int nspec;
   float *auto_acc, *xpol_acc, *pcal_acc; /* thread-private [nspec][...] */
   int curr0;                             /* curr_ffts value at f0 */
} orc_job32;

static void *orc_worker32(void *arg)
{
   orc_job32 *j = (orc_job32 *)arg;
   const orc_cfg *c = j->c;
   const int N = c->fft_points, S = N / 2 + 1;
   c32 *d0 = (c32 *)malloc(sizeof(c32) * (size_t)N);
   c32 *d1 = (c32 *)malloc(sizeof(c32) * (size_t)N);
   const int H = N / 2;
   c32 **X = (c32 **)malloc(sizeof(c32 *) * (size_t)c->num_sources);
   for (int s = 0; s < c->num_sources; s++) X[s] = (c32 *)malloc(sizeof(c32) * (size_t)S);
   int curr = j->curr0;
   for (int f = j->f0; f < j->f1; f++) {
      int sp = j->spec_of[f];
      for (int s = 0; s < c->num_sources; s++) {
         const float *x = j->samples[s] + j->starts[f];
         if (c->extract_pcal && (curr % c->overlap) == 0) {
            float *pc = j->pcal_acc + 2 * ((size_t)sp * c->num_sources + s) * c->pcal_tonebins;
            int used = (c->pcal_rotatorlen / c->pcal_tonebins) * c->pcal_tonebins;
            for (int n0 = 0; n0 < N; n0 += c->pcal_rotatorlen)
               for (int i = 0; i < used; i++) {
                  int b = i % c->pcal_tonebins;
                  pc[2 * b] += x[n0 + i] * j->rot[i].re;
                  pc[2 * b + 1] += x[n0 + i] * j->rot[i].im;
               }
         }
         if (j->wn) {
            /* real FFT of the windowed samples as one complex FFT of N/2
             * points: z[n] = x[2n] + i x[2n+1], then
             * X[k] = (Z[k] + conj Z[H-k])/2 + W_N^k (Z[k] - conj Z[H-k])/(2i) */
            for (int n = 0; n < H; n++) {
               d0[n].re = x[2 * n] * j->win[2 * n];
               d0[n].im = x[2 * n + 1] * j->win[2 * n + 1];
            }
            const c32 *Z = fft32(j->pl, d0, d1);
            X[s][0].re = Z[0].re + Z[0].im; X[s][0].im = 0.0f;
            X[s][H].re = Z[0].re - Z[0].im; X[s][H].im = 0.0f;
            for (int k = 1; k < H; k++) {
               const c32 a = Z[k], b = Z[H - k];
               const float er = 0.5f * (a.re + b.re), ei = 0.5f * (a.im - b.im);
               const float o_r = 0.5f * (a.im + b.im), o_i = -0.5f * (a.re - b.re);
               const c32 w = j->wn[k];
               X[s][k].re = er + w.re * o_r - w.im * o_i;
               X[s][k].im = ei + w.re * o_i + w.im * o_r;
            }
         } else {
            /* odd N: complex FFT of the windowed samples */
            for (int n = 0; n < N; n++) {
               d0[n].re = x[n] * j->win[n];
               d0[n].im = 0.0f;
            }
            c32 *r = fft32(j->pl, d0, d1);
            memcpy(X[s], r, sizeof(c32) * (size_t)S);
         }
         curr++;
         float *oa = j->auto_acc + ((size_t)sp * c->num_sources + s) * S;
         for (int k = 0; k < S; k++) oa[k] += X[s][k].re * X[s][k].re + X[s][k].im * X[s][k].im;
      }
      for (int xp = 0; xp < c->num_xpols; xp++) {
         const c32 *A = X[j->pairs[2 * xp]], *B = X[j->pairs[2 * xp + 1]];
         float *ox = j->xpol_acc + 2 * ((size_t)sp * c->num_xpols + xp) * S;
         for (int k = 0; k < S; k++) {
            ox[2 * k] += A[k].re * B[k].re + A[k].im * B[k].im;
            ox[2 * k + 1] += A[k].im * B[k].re - A[k].re * B[k].im;
         }
         ox[1] = 0.0f;
         ox[2 * (S - 1) + 1] = 0.0f;
      }
   }
   free(d0); free(d1);
   for (int s = 0; s < c->num_sources; s++) free(X[s]);
   free(X);
   return NULL;
}

/* FP32 CPU baseline over one buffer; same output layout as orc_domaths64 but
 * in float.  FFTs are split into contiguous ranges, one per thread, and the
 * thread-private sums are added at the end (the reference splits work across
 * cores the same way and adds partial spectra in combineResults). */
int orc_domaths32(const orc_cfg *c, const float *const *samples, int64_t nsamp, float *out_auto,
                  float *out_xpol, float *out_pcal)
{
   const int N = c->fft_points, S = N / 2 + 1;
   int nspec, partial;
   int nf = orc_schedule(c, nsamp, NULL, NULL, 0, &nspec, &partial);
   int64_t *starts = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nf + 1));
   int *spec_of = (int *)malloc(sizeof(int) * (size_t)(nf + 1));
   orc_schedule(c, nsamp, starts, spec_of, nf, &nspec, &partial);
   float *win = (float *)malloc(sizeof(float) * (size_t)N);
   orc_window(c->window, N, win);
   /* even N: the real transform runs as an N/2-point complex FFT (the IPP
    * core's ippsDFTFwd_RToPerm_32f is a real-input transform too) */
   plan32 *pl = plan32_new(N % 2 == 0 ? N / 2 : N);
   c32 *wn = NULL;
   if (N % 2 == 0) {
      wn = (c32 *)malloc(sizeof(c32) * (size_t)(N / 2));
      for (int k = 0; k < N / 2; k++) {
         double a = -2.0 * M_PI * (double)k / (double)N;
         wn[k].re = (float)cos(a);
         wn[k].im = (float)sin(a);
      }
   }
   int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(c->num_xpols + 1));
   orc_xpol_pairs(c->num_sources, c->num_xpols, pairs);
   c32 *rot = NULL;
   if (c->extract_pcal) {
      rot = (c32 *)malloc(sizeof(c32) * (size_t)c->pcal_rotatorlen);
      double dphi = 2 * M_PI * (-c->pcaloffsethz / c->samplingfreq);
      for (int i = 0; i < c->pcal_rotatorlen; i++) {
         rot[i].re = (float)cos(dphi * (double)i);
         rot[i].im = (float)sin(dphi * (double)i);
      }
   }
   int nt = c->nthreads < 1 ? 1 : c->nthreads;
   if (nt > nf) nt = nf > 0 ? nf : 1;
   size_t na = (size_t)nspec * c->num_sources * S, nx = 2 * (size_t)nspec * c->num_xpols * S,
          np = 2 * (size_t)nspec * c->num_sources * (c->extract_pcal ? c->pcal_tonebins : 0);
   orc_job32 *jobs = (orc_job32 *)calloc((size_t)nt, sizeof(orc_job32));
   pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
   for (int t = 0; t < nt; t++) {
      orc_job32 *j = &jobs[t];
      j->c = c; j->samples = samples; j->starts = starts; j->spec_of = spec_of;
      j->f0 = (int)((long long)nf * t / nt);
      j->f1 = (int)((long long)nf * (t + 1) / nt);
      j->win = win; j->pl = pl; j->wn = wn; j->rot = rot; j->pairs = pairs; j->nspec = nspec;
      j->auto_acc = (float *)calloc(na + 1, sizeof(float));
      j->xpol_acc = (float *)calloc(nx + 1, sizeof(float));
      j->pcal_acc = (float *)calloc(np + 1, sizeof(float));
      j->curr0 = j->f0 * c->num_sources;
      pthread_create(&th[t], NULL, orc_worker32, j);
   }
   memset(out_auto, 0, sizeof(float) * na);
   if (nx) memset(out_xpol, 0, sizeof(float) * nx);
   if (np) memset(out_pcal, 0, sizeof(float) * np);
   for (int t = 0; t < nt; t++) {
      pthread_join(th[t], NULL);
      for (size_t i = 0; i < na; i++) out_auto[i] += jobs[t].auto_acc[i];
      for (size_t i = 0; i < nx; i++) out_xpol[i] += jobs[t].xpol_acc[i];
      for (size_t i = 0; i < np; i++) out_pcal[i] += jobs[t].pcal_acc[i];
      free(jobs[t].auto_acc); free(jobs[t].xpol_acc); free(jobs[t].pcal_acc);
   }
   int nfull = nspec - partial;
   float sc = (float)(1.0 / c->core_overlapped_ffts);
   for (size_t i = 0; i < (size_t)nfull * c->num_sources * S; i++) out_auto[i] *= sc;
   for (size_t i = 0; i < 2 * (size_t)nfull * c->num_xpols * S; i++) out_xpol[i] *= sc;
   free(jobs); free(th); free(starts); free(spec_of); free(win); free(pairs); free(rot); free(wn);
   plan32_free(pl);
   return nspec;
}

/* ------------------------------------------------------------------------ */
/* Phase-cal tone extraction from folded bins                               */
/* ------------------------------------------------------------------------ */

/* Tone phasors from the folded, de-rotated bins that extract_PCal produces:
 * tone k (frequency k*spacing + offset) is DFT bin k of the tonebins folded
 * samples, normalised by the number of samples folded (nfolded).  FP64.
 * This follows the final step of the PCal library's ImplicitShift extractor
 * (src/IA-32/PhaseCal/PCal.cpp:654-678: DFT of the folded bins, pick bins
 * offset + n*step), applied to the rotate-and-fold output. */
int orc_pcal_tones(int tonebins, const double *bins_reim, double nfolded, int ntones,
                   double *tones_reim)
{
   for (int k = 0; k < ntones; k++) {
      double sr = 0, si = 0;
      for (int b = 0; b < tonebins; b++) {
         double a = -2.0 * M_PI * (double)((long long)k * b % tonebins) / (double)tonebins;
         double c = cos(a), s = sin(a);
         sr += bins_reim[2 * b] * c - bins_reim[2 * b + 1] * s;
         si += bins_reim[2 * b] * s + bins_reim[2 * b + 1] * c;
      }
      tones_reim[2 * k] = sr / nfolded;
      tones_reim[2 * k + 1] = si / nfolded;
   }
   return 0;
}

/* ------------------------------------------------------------------------ */
/* The PCal extractor library (src/IA-32/PhaseCal/PCal.cpp)                 */
/* ------------------------------------------------------------------------ */

/* State of one extractor.  kind: 1 Trivial (:183-318), 2 Shifting
 * (:321-517), 3 ImplicitShift (:521-678).  Sums are kept in FP64 here (the
 * reference adds in FP32); the index bookkeeping and the tone selection are
 * the reference's, quirks included: Shifting adds, per full rotator period,
 * only the first floor(R/N)*N rotated samples (:451-462), and both indices
 * start from the sample offset given at creation (the reference's
 * constructors leave them unset until adjustSampleOffset). */
typedef struct {
   int kind;
   double fs, spacing, offset;
   int nbins, ntones, rotlen;
   int64_t pcal_index, rotator_index;
   uint64_t samplecount;
   float *rot_re, *rot_im; /* FP32 oscillator table, 2 * rotlen entries (:350-355) */
   double *acc;            /* [2 * nbins][re, im] */
} orc_pcallib;

static long long orc_gcdll(long long a, long long b)
{
   while (b) {
      long long t = a % b;
      a = b;
      b = t;
   }
   return a < 0 ? -a : a;
}

void *orc_pcallib_new(double bandwidth_hz, double spacing_hz, int offset_hz, int64_t sampleoffset, int kind)
{
   orc_pcallib *p = (orc_pcallib *)calloc(1, sizeof(orc_pcallib));
   const long long fs = (long long)(2.0 * bandwidth_hz);
   p->fs = (double)fs;
   p->spacing = spacing_hz;
   p->offset = offset_hz;
   if (kind == 0) { /* PCal::getNew (:92-112) */
      if (offset_hz == 0) kind = 1;
      else {
         long long No = fs / orc_gcdll(offset_hz, fs), Np = fs / orc_gcdll((long long)spacing_hz, fs);
         kind = (No % Np == 0) ? 3 : 2;
      }
   }
   p->kind = kind;
   if (kind == 3) {
      p->nbins = (int)(fs / orc_gcdll(offset_hz, fs));
      p->ntones = (int)floor((bandwidth_hz - offset_hz) / spacing_hz) + 1;
   } else {
      p->nbins = (int)(fs / orc_gcdll((long long)fabs(spacing_hz), fs));
      p->ntones = kind == 1 ? (int)floor(bandwidth_hz / spacing_hz)
                            : (int)floor((bandwidth_hz - offset_hz) / spacing_hz) + 1;
   }
   p->rotlen = kind == 2 ? (int)(fs / orc_gcdll((long long)abs(offset_hz), fs)) : p->nbins;
   p->acc = (double *)calloc(4 * (size_t)p->nbins, sizeof(double));
   if (kind == 2) {
      p->rot_re = (float *)malloc(sizeof(float) * 2 * (size_t)p->rotlen);
      p->rot_im = (float *)malloc(sizeof(float) * 2 * (size_t)p->rotlen);
      double dphi = 2 * M_PI * (-(double)offset_hz / p->fs);
      for (int n = 0; n < 2 * p->rotlen; n++) {
         p->rot_re[n] = (float)cos(dphi * (double)n);
         p->rot_im[n] = (float)sin(dphi * (double)n);
      }
   }
   p->pcal_index = sampleoffset % p->nbins;
   p->rotator_index = sampleoffset % p->rotlen;
   return p;
}

void orc_pcallib_free(void *h)
{
   orc_pcallib *p = (orc_pcallib *)h;
   if (!p) return;
   free(p->acc); free(p->rot_re); free(p->rot_im); free(p);
}

void orc_pcallib_clear(void *h)
{
   orc_pcallib *p = (orc_pcallib *)h;
   memset(p->acc, 0, sizeof(double) * 4 * (size_t)p->nbins);
   p->samplecount = 0;
}

void orc_pcallib_adjust(void *h, int64_t sampleoffset)
{
   orc_pcallib *p = (orc_pcallib *)h;
   p->pcal_index = sampleoffset % p->nbins;
   if (p->kind == 2) p->rotator_index = sampleoffset % p->rotlen;
}

static void orc_pcallib_add(orc_pcallib *p, int64_t slot, double re, double im)
{
   p->acc[2 * slot] += re;
   p->acc[2 * slot + 1] += im;
}

void orc_pcallib_extract(void *h, const float *x, int64_t len)
{
   orc_pcallib *p = (orc_pcallib *)h;
   const int N = p->nbins;
   if (p->kind != 2) {
      /* real fold into nbins (:265-296, :610-652): sample n at slot pcal_index + n mod N */
      int64_t tail = len % N, end = len - tail;
      for (int64_t n = 0; n < len; n++) {
         int64_t slot = n < end ? p->pcal_index + (n % N) : p->pcal_index + (n - end);
         orc_pcallib_add(p, slot, (double)x[n], 0.0);
      }
      p->pcal_index = (p->pcal_index + tail) % N;
   } else {
      const int R = p->rotlen, P = R / N;
      int64_t tail = len % R, end = len - tail;
      for (int64_t n = 0; n < end; n++) {
         int64_t j = n % R;
         if (j >= (int64_t)P * N) continue; /* the samples past the last whole pulse */
         int64_t r = p->rotator_index + j;
         orc_pcallib_add(p, p->pcal_index + (j % N), (double)x[n] * p->rot_re[r], (double)x[n] * p->rot_im[r]);
      }
      for (int64_t m = 0; m < tail; m++) {
         int64_t r = p->rotator_index + m;
         orc_pcallib_add(p, p->pcal_index + (m % N), (double)x[end + m] * p->rot_re[r],
                         (double)x[end + m] * p->rot_im[r]);
      }
      int64_t tail2 = tail % N;
      p->rotator_index = (p->rotator_index + tail) % R;
      p->pcal_index = (p->pcal_index + tail2) % N;
   }
   p->samplecount += (uint64_t)len;
}

int orc_pcallib_info(void *h, int *kind, int *nbins, int *ntones)
{
   orc_pcallib *p = (orc_pcallib *)h;
   *kind = p->kind; *nbins = p->nbins; *ntones = p->ntones;
   return 0;
}

/* getFinalPCal: bins [0, N) += [N, 2N), forward DFT scaled by 1/N
 * (IPP_FFT_DIV_FWD_BY_N), then the tone bins: Trivial the first ntones,
 * Shifting every step-th, ImplicitShift every step-th from the offset bin;
 * tones whose bin falls past N stay zero.  Returns the samples integrated. */
uint64_t orc_pcallib_final(void *h, double *out_reim)
{
   orc_pcallib *p = (orc_pcallib *)h;
   const int N = p->nbins;
   double *b = (double *)malloc(sizeof(double) * 2 * (size_t)N);
   for (int k = 0; k < N; k++) {
      b[2 * k] = p->acc[2 * k] + p->acc[2 * (k + N)];
      b[2 * k + 1] = p->acc[2 * k + 1] + p->acc[2 * (k + N) + 1];
   }
   const long long step = (long long)floor((double)N * (p->spacing / p->fs));
   const long long off = p->kind == 3 ? (long long)floor((double)N * p->offset / p->fs) : 0;
   for (int t = 0; t < p->ntones; t++) {
      long long idx = p->kind == 1 ? t : off + (long long)t * step;
      out_reim[2 * t] = out_reim[2 * t + 1] = 0.0;
      if (idx >= N) continue;
      long double sr = 0, si = 0;
      for (int k = 0; k < N; k++) {
         long long e = (idx * (long long)k) % N;
         long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)N;
         long double c = cosl(a), s = sinl(a);
         sr += b[2 * k] * c - b[2 * k + 1] * s;
         si += b[2 * k] * s + b[2 * k + 1] * c;
      }
      out_reim[2 * t] = (double)(sr / N);
      out_reim[2 * t + 1] = (double)(si / N);
   }
   free(b);
   return p->samplecount;
}
