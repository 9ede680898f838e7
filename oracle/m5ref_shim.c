/*
 * m5ref_shim.c -- thin C entry points over the reference's own mark5access
 * library, compiled from the reference sources into oracle/_ref/ by
 * oracle/Makefile.  TEST INFRASTRUCTURE ONLY: used to pin the decode
 * restatement and the GPU unpacker bit-exactly against mark5access itself.
 *
 * m5ref_decode  : framed decode of an in-memory stream, as FileSource /
 *                 m5spec do it (mark5access/mark5access/mark5_stream.c
 *                 mark5_stream_decode, mark5_stream_memory.c): frame search,
 *                 header skip, fill-pattern blanking.
 * m5ref_unpack  : header-free unpack of a payload buffer through
 *                 new_mark5_stream_unpacker(noheaders=1) + mark5_unpack
 *                 (mark5_stream_unpacker.c:112-129), the route
 *                 src/IA-32/DataUnpackers.cpp:671-674,733 uses.
 */
#include <stdlib.h>
#include <string.h>
#include "mark5access/mark5_stream.h"

/* Stream properties of a format string; returns 0 on success. */
int m5ref_format_info(const char *fmt, int *nchan, int *nbit, int *framebytes, int *payloadoffset,
                      int *framesamples, int *samplegranularity)
{
   struct mark5_stream *ms = new_mark5_stream(new_mark5_stream_unpacker(0),
                                              new_mark5_format_generic_from_string(fmt));
   if (!ms) return -1;
   *nchan = ms->nchan;
   *nbit = ms->nbit;
   *framebytes = ms->framebytes;
   *payloadoffset = ms->payloadoffset;
   *framesamples = ms->framesamples;
   *samplegranularity = ms->samplegranularity;
   delete_mark5_stream(ms);
   return 0;
}

/* Decode nsamp samples of every channel from a framed memory stream.
 * out is [nchan][nsamp]; returns mark5_stream_decode's result (samples not
 * blanked) or a negative value; *frameoffset gets the first frame offset. */
int m5ref_decode(const char *fmt, void *data, unsigned nbytes, int nsamp, int nchan_max, float *out,
                 int *frameoffset)
{
   struct mark5_stream *ms = new_mark5_stream(new_mark5_stream_memory(data, nbytes),
                                              new_mark5_format_generic_from_string(fmt));
   if (!ms) return -100;
   if (ms->nchan > nchan_max) { delete_mark5_stream(ms); return -101; }
   float **ptr = (float **)malloc(sizeof(float *) * (size_t)ms->nchan);
   for (int c = 0; c < ms->nchan; c++) ptr[c] = out + (size_t)c * nsamp;
   if (frameoffset) *frameoffset = ms->frameoffset;
   int r = mark5_stream_decode(ms, nsamp, ptr);
   free(ptr);
   delete_mark5_stream(ms);
   return r;
}

/* Header-free unpack of nsamp samples of every channel from `payload`. */
int m5ref_unpack(const char *fmt, void *payload, int nsamp, int nchan_max, float *out)
{
   struct mark5_stream *ms = new_mark5_stream(new_mark5_stream_unpacker(1),
                                              new_mark5_format_generic_from_string(fmt));
   if (!ms) return -100;
   if (ms->nchan > nchan_max) { delete_mark5_stream(ms); return -101; }
   float **ptr = (float **)malloc(sizeof(float *) * (size_t)ms->nchan);
   for (int c = 0; c < ms->nchan; c++) ptr[c] = out + (size_t)c * nsamp;
   int r = mark5_unpack(ms, payload, ptr, nsamp);
   free(ptr);
   delete_mark5_stream(ms);
   return r;
}

/* Time of the first frame of an in-memory framed stream, as mark5access
 * decodes its header (mark5_stream_get_frame_time); returns 0 on success. */
int m5ref_frame_time(const char *fmt, void *data, unsigned nbytes, int *mjd, int *sec, double *ns,
                     int *frameoffset)
{
   struct mark5_stream *ms = new_mark5_stream(new_mark5_stream_memory(data, nbytes),
                                              new_mark5_format_generic_from_string(fmt));
   if (!ms) return -100;
   *frameoffset = ms->frameoffset;
   int r = mark5_stream_get_frame_time(ms, mjd, sec, ns);
   delete_mark5_stream(ms);
   return r;
}
