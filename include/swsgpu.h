/*
 * swsgpu.h -- C ABI of the B200 spectrometer core (libswsgpu.so, sm_100a).
 *
 * This is the boundary a TaskCore implementation calls.  It replaces the
 * compute half of the reference's abstract core, src/TaskCore.h:36-89, whose
 * only complete implementation is TaskCoreIPP (src/IA-32/TaskCoreIPP.h:49-177):
 *
 *   TaskCore::prepare(settings)     (TaskCore.h:47)  -> swsgpu_create
 *   TaskCore::run(in,out,xpol,pcal) (TaskCore.h:58)  -> swsgpu_submit
 *   TaskCore::join()                (TaskCore.h:65)  -> swsgpu_wait + swsgpu_fetch
 *   TaskCore::finalize()            (TaskCore.h:71)  -> swsgpu_destroy
 *   TaskCore::resetBuffer(buf)      (TaskCore.h:87)  -> host memset (no device work)
 *   TaskCore::combineResults(...)   (TaskCore.h:81)  -> host add of fetched spectra, or
 *                                                       swsgpu_process_device with
 *                                                       runs_per_output > 1
 *
 * One call of swsgpu_submit is one core run over one raw buffer per input
 * stream: the per-buffer loop of TaskCoreIPP::doMaths
 * (src/IA-32/TaskCoreIPP.cpp:355-560) -- FFTs every N/overlap samples,
 * spectra of core_overlapped_ffts FFTs scaled by 1/core_overlapped_ffts, the
 * hop over the overlap remainder between spectra, a trailing partial spectrum
 * left unscaled, and PCal folding (TaskCoreIPP.cpp:633-693) on every
 * overlap-th source FFT.  Sample decoding follows mark5access
 * (mark5_format_mark5b.c, format_vdif.c), bit-exact, including fill-pattern
 * blanking.
 *
 * All entry points return 0 on success and a negative SWSGPU_E* code on
 * failure; swsgpu_last_error() describes the last failure of a handle (or,
 * with a NULL handle, the last failure of swsgpu_create on this thread).
 * Memory passed in is owned by the caller.  A handle is used by one host
 * thread at a time.
 */
#ifndef SWSGPU_H
#define SWSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWSGPU_OK 0
#define SWSGPU_EINVAL (-1)       /* bad argument or unsupported configuration */
#define SWSGPU_ECUDA (-2)        /* CUDA runtime error (message has details) */
#define SWSGPU_ETIMEOUT (-3)     /* swsgpu_wait timed out; the run is still queued */
#define SWSGPU_ENODEV (-4)       /* no usable sm_100 device */
#define SWSGPU_ESTATE (-5)       /* call out of order (e.g. fetch before wait) */
#define SWSGPU_ETOOBIG (-6)      /* request exceeds a fixed capacity (see the _noalloc entry) */

/* Sample tables (level values) of the stream. */
#define SWSGPU_FMT_MARK5B 0      /* Mark5B: 2-bit {-H,+1,-1,+H}[s+2m], 1-bit {+1,-1} */
#define SWSGPU_FMT_VDIF 1        /* VDIF: 2-bit {-H,-1,+1,+H}, 1-bit {-1,+1}, 8-bit (2b-255)/256 */
/* Raw sampler data, the reference's RawSigned / RawUnsigned formats
 * (src/IA-32/DataUnpackerFactory.h:44-67): 8-bit samples byte-interleaved by
 * channel, signed (int8) or unsigned (b - 128) (DataUnpackers.cpp:68-171);
 * 2-bit with nchan % 4 == 0: channel c's code at bit 2c of the sample-time's
 * nchan/4 bytes (:191-249; ChannelOrderIncreasing = no is channel
 * nchan-1-c); 2-bit with one channel: four samples per byte, the oldest in
 * the two most significant bits (:261-310).  2-bit codes map to
 * {+1, -1, +H, -H}.  No fill-pattern blanking. */
#define SWSGPU_FMT_RAW_SIGNED 2
#define SWSGPU_FMT_RAW_UNSIGNED 3
/* Track formats, decoded as mark5access decodes them (VLBA1_f / MKIV1_f
 * modes, mark5_format_vlba.c, mark5_format_mark4.c; the reference's
 * VLBAUnpacker / MarkIVUnpacker, src/IA-32/DataUnpackers.cpp:459-658, go
 * through mark5access): a track-word of ntrack bits (tracks 8, 16, 32 or 64,
 * the low track in bit 0 of the first byte) carries `fanout` consecutive
 * samples of every channel, ntrack = nchan * nbit * fanout, fanout 1, 2 or 4,
 * nbit 1 or 2, nchan * nbit <= 32; levels as Mark5B's.  A frame is 20000
 * track-words: frame_bytes = 2500 * ntrack, header_bytes = 0.  VLBA: the
 * payload stream with the frame headers removed (the 96 track-words before
 * and the 64 after each frame's 20000); every sample of track-word i of a
 * frame is negated where the VLBA modulation sequence has bit i set.  Mark4
 * (data replacement): whole frames, whose first 160 track-words (auxiliary
 * data, sync word, time code) decode as blanked samples.  No fill-pattern
 * blanking. */
#define SWSGPU_FMT_VLBA 4
#define SWSGPU_FMT_MARK4 5

/* Window functions: the reference's WindowFunctionType (src/Settings.h:45)
 * plus BlackmanHarris (4-term Harris 1978), which the reference lacks. */
#define SWSGPU_WIN_NONE 0
#define SWSGPU_WIN_COSINE 1
#define SWSGPU_WIN_COSINE2 2
#define SWSGPU_WIN_HAMMING 3
#define SWSGPU_WIN_HANN 4
#define SWSGPU_WIN_BLACKMAN 5
#define SWSGPU_WIN_BLACKMANHARRIS 6

/* Arithmetic of the FFT stages. */
/* FFT paths: the cluster kernel (one thread-block cluster per pair FFT,
 * N <= 131072) or the four-step column/row kernels (intermediate in HBM). */
#define SWSGPU_PLAN_DEFAULT 0     /* cluster kernel where it exists, else four-step */
#define SWSGPU_PLAN_CLUSTER 1
#define SWSGPU_PLAN_FOURSTEP 2

#define SWSGPU_PREC_FP32 0       /* plain FP32 throughout */
#define SWSGPU_PREC_TCSPLIT 1    /* the CTA's inner radix-16 levels 2-3 as tcgen05 GEMMs (FP16 hi+lo
                                    split operands, FP32 accumulators in tensor memory); level 1
                                    in FP32 registers fused with the decode */
#define SWSGPU_PREC_TCSPLIT_ALL 2 /* as TCSPLIT with level 1 on the tensor cores too */

#define SWSGPU_MAX_SOURCES 64
#define SWSGPU_MAX_STREAMS 2

/* Byte layout of one input stream.  A stream is a sequence of frames of
 * frame_bytes bytes, each starting with header_bytes of header followed by
 * the payload.  header_bytes = 0 describes a header-free payload stream (the
 * reference's FileSource strips Mk5B/VDIF headers, src/FileSource.cpp:184-215);
 * frame_bytes then still gives the payload size of one recorded frame, which
 * delimits mark5access's blanking zones. */
typedef struct swsgpu_layout {
   int format;          /* SWSGPU_FMT_* */
   int nchan;           /* channels per sample-time */
   int nbit;            /* bits per sample: 1, 2 or 8 */
   int frame_bytes;     /* header + payload bytes of one frame */
   int header_bytes;    /* header bytes at the start of each frame (0: payload only) */
} swsgpu_layout;

/* Processing configuration; the fields mirror swspect_settings_t
 * (src/Settings.h:59-159) as derived in src/swspectrometer.cpp:166-231. */
typedef struct swsgpu_config {
   swsgpu_layout layout[SWSGPU_MAX_STREAMS];
   int num_streams;                 /* input buffers per run (reference: input files) */
   int fft_points;                  /* N (even, factors 2,3,5) */
   int overlap;                     /* fft_overlap_factor */
   int window;                      /* SWSGPU_WIN_* */
   int precision;                   /* SWSGPU_PREC_* */
   int core_overlapped_ffts;        /* FFTs per spectrum within one run */
   int num_sources;                 /* processed channels */
   int source_stream[SWSGPU_MAX_SOURCES];   /* stream of each source */
   int source_channel[SWSGPU_MAX_SOURCES];  /* 0-based channel of each source */
   int num_xpols;                   /* cross spectra */
   int xpol_pair[SWSGPU_MAX_SOURCES][2];    /* X_i conj(X_j) source indices */
   int extract_pcal;                /* fold phase-cal tones */
   int pcal_tonebins;               /* fs / comb spacing */
   int pcal_rotatorlen;             /* fs / gcd(fs, offset) */
   double samplingfreq;             /* Hz */
   double pcal_offset_hz;           /* Hz */
   size_t max_run_bytes;            /* largest raw buffer per stream and run */
   int runs_per_output;             /* >1: consecutive submits are summed on the device and
                                       one combined spectrum set is returned every
                                       runs_per_output runs -- the dispatcher's
                                       max_buffers_per_spectrum combining
                                       (src/TaskDispatcher.cpp:143-171,
                                       TaskCoreIPP::combineResults :311-349); sums are
                                       kept in FP64 between runs */
   int pcal_ntones;                 /* >0: also return the phasors of the first pcal_ntones
                                       tones (k * spacing + offset, k < ntones <= tonebins/2),
                                       the PCal library's tone output (src/IA-32/PhaseCal/
                                       PCal.cpp:654-678), computed in FP64 */
   int autotune;                    /* 1: swsgpu_create times the candidate plans of the
                                       length -- four-step splits, or cluster plans (cluster
                                       size, threads per CTA, radix order) -- and keeps the
                                       fastest (once per length, bit depth and form per
                                       process; see swsgpu_autotune) */
   int plan_family;                 /* SWSGPU_PLAN_*: which FFT path a length with both uses */
   int plan_candidate;              /* 0 = the default plan, k > 0 = the k-th candidate
                                       split or cluster plan (as the autotuner numbers them);
                                       ignored when autotune is set */
} swsgpu_config;

typedef struct swsgpu_handle swsgpu_handle;

/* Spectra of one run: layouts of TaskCoreIPP's output buffers.
 *   auto_out : float [nspectra][num_sources][N/2+1]
 *   xpol_out : float [nspectra][num_xpols][N/2+1][2]   (re, im)
 *   pcal_out : float [nspectra][num_sources][pcal_tonebins][2]
 *   tones_out: double [nspectra][num_sources][pcal_ntones][2]  (re, im of each tone
 *              phasor: mean over the folded samples; amplitude = |.|, phase = arg)
 * Pointers for outputs that are not configured may be NULL. */
typedef struct swsgpu_outputs {
   float *auto_out;
   float *xpol_out;
   float *pcal_out;
   double *tones_out;
} swsgpu_outputs;

/* Library / device checks. */
int swsgpu_version(void);
int swsgpu_device_ok(int device);

/* TaskCore::prepare.  Validates the configuration, selects `device`,
 * allocates device buffers for runs of up to max_run_bytes per stream,
 * uploads window and twiddle tables. */
int swsgpu_create(const swsgpu_config *cfg, int device, swsgpu_handle **out);

/* TaskCore::finalize. */
void swsgpu_destroy(swsgpu_handle *h);

/* Describes the last failure. */
const char *swsgpu_last_error(const swsgpu_handle *h);

/* Number of spectra (including a trailing partial one) and FFTs a run of
 * `nbytes` payload bytes per stream yields; *partial is set when the last
 * spectrum is an unscaled partial one (TaskCoreIPP.cpp:519-524). */
int swsgpu_run_shape(const swsgpu_handle *h, size_t nbytes, int *nspectra, int *nffts,
                     int *partial);

/* TaskCore::run: queue one run on the handle's CUDA stream and return.
 * raw[s] points to host memory holding nbytes[s] bytes of stream s, whole
 * frames when the layout has headers.  The host memory must stay valid and
 * unchanged until swsgpu_wait returns (the reference's double-buffer rule).
 * Input copies run on their own stream into one of two device slots, so a
 * run's copy overlaps the previous run's kernels; pinned host memory (see
 * swsgpu_host_register) makes them asynchronous.  A run that completes no
 * spectrum (runs_per_output > 1, not the last of its group) may be followed
 * by the next submit before its wait; a run that completes spectra must be
 * waited for (and fetched) first, else SWSGPU_ESTATE.
 * stream_payload_offset[s] is the payload byte offset of raw[s] within its
 * recording (fixes mark5access's per-frame blanking zones; 0 for a run that
 * starts on a frame). */
int swsgpu_submit(swsgpu_handle *h, const void *const *raw, const size_t *nbytes,
                  const int64_t *stream_payload_offset);

/* TaskCore::join: wait up to timeout_ms (<0: forever) until the submitted
 * input buffers may be reused and any spectra the run completes are in
 * host memory; *nspectra gets the spectrum count (TaskCore::join's return
 * value).  With runs_per_output > 1 it is 0 until the run that completes a
 * group, whose fetch returns the combined spectra; for the other runs the
 * wait ends when their input copy has finished (their kernels keep running
 * and are ordered before the group's last run).  Device errors of earlier
 * runs are reported by the wait that follows them. */
int swsgpu_wait(swsgpu_handle *h, int timeout_ms, int *nspectra);

/* Copy the spectra of the completed run into caller memory. */
int swsgpu_fetch(swsgpu_handle *h, const swsgpu_outputs *out);

/* TaskCore::run(in, out, xpol, pcal) (TaskCore.h:58) with its output
 * buffers: swsgpu_submit, plus where the spectra of this run go if it
 * completes any (layouts as swsgpu_fetch; NULL members are not written).
 * Destinations in page-locked memory (cudaHostAlloc, swsgpu_host_register)
 * are written by the run's own device-to-host copies, with no host copy;
 * others through the library's staging buffer during swsgpu_wait.  Either
 * way they hold the spectra once swsgpu_wait returns, and must stay valid
 * until then; swsgpu_fetch is not used for such a run (SWSGPU_ESTATE). */
int swsgpu_submit_out(swsgpu_handle *h, const void *const *raw, const size_t *nbytes,
                      const int64_t *stream_payload_offset, const swsgpu_outputs *dest);

/* Page-lock caller memory that will be passed to swsgpu_submit, so its
 * input copies are DMA transfers that overlap kernels (the reference's raw
 * buffers are allocated once by main, src/swspectrometer.cpp:373-413, and
 * live for the whole run).  Memory already pinned is accepted as is.  No
 * counterpart in the reference (its cores read host memory directly). */
int swsgpu_host_register(void *p, size_t bytes);
/* Undo swsgpu_host_register before the memory is freed. */
int swsgpu_host_unregister(void *p);

/* Autotuner (no counterpart in the reference, whose IPP core has one FFT
 * plan per length): for a length on the four-step path, times every
 * candidate split N = N1 x N2 and columns-per-CTA width on a hash-filled run
 * with this core's sources, pairs and window (enough frames for about 16
 * pair FFTs); for a cluster length, every cluster plan of the handle's form
 * (cluster size, threads per CTA, radix order: 4096, 20000 and 131072 have
 * several) on one hash-filled run of max_run_bytes (at most 64 MiB of
 * payload).  Keeps the candidate with the shortest of `iterations` (at most
 * 16) timed iterations; later cores of the same length, bit depth and form
 * in this process start with that choice.  Synchronous; call it with no run
 * pending. */
int swsgpu_autotune(swsgpu_handle *h, int iterations);

/* Text description of the plan a core uses (split, tile, candidate). */
int swsgpu_plan_info(const swsgpu_handle *h, char *buf, size_t len);

/* Batches: the runs of many cores -- streams of different FFT lengths, bit
 * depths and integrations -- recorded once as a CUDA graph and then issued
 * with a single launch per step; each core's kernels go on its own forked
 * stream inside the graph, so the cores run concurrently.  No counterpart
 * in the reference (one dispatcher per recording).  swsgpu_batch_set gives
 * core i its device inputs and outputs as for swsgpu_process_device.  The
 * first swsgpu_batch_launch after a set runs every core eagerly (that run
 * makes all allocations and device schedules and produces this launch's
 * results) and records the graph; later launches replay it on cuda_stream
 * (asynchronous, over the same device buffers).  *kernels (optional) gets
 * the kernel count of one batch.  The cores must not be used otherwise
 * while their batch is in flight. */
typedef struct swsgpu_batch swsgpu_batch;
int swsgpu_batch_create(swsgpu_handle *const *cores, int ncores, swsgpu_batch **out);
int swsgpu_batch_set(swsgpu_batch *b, int i, const void *const *d_raw, size_t run_bytes, int nruns,
                     int runs_per_output, const swsgpu_outputs *d_out);
int swsgpu_batch_launch(swsgpu_batch *b, void *cuda_stream, int *kernels);
void swsgpu_batch_destroy(swsgpu_batch *b);

/* Throughput path with data already in device memory: processes `nruns`
 * consecutive runs of run_bytes payload bytes per stream (d_raw[s] holds
 * nruns*run_bytes payload bytes, or the framed bytes that carry them) and
 * writes the sum of every `runs_per_output` consecutive runs' spectra --
 * the dispatcher's combineResults path (src/TaskDispatcher.cpp:143-171) --
 * into the device outputs, using runs * nspectra_per_run / runs_per_output
 * spectrum slots.  `cuda_stream` is a cudaStream_t (NULL: the handle's).
 * Every d_raw[s] must be 4-byte aligned (SWSGPU_EINVAL otherwise; the
 * decoders read 32-bit words), as for swsgpu_batch_set. */
int swsgpu_process_device(swsgpu_handle *h, const void *const *d_raw, size_t run_bytes, int nruns,
                          int runs_per_output, const swsgpu_outputs *d_out, void *cuda_stream);

/* swsgpu_process_device and swsgpu_batch_launch only queue work.  This waits
 * for cuda_stream (NULL: the handle's stream) and then reads and clears the
 * handle's device status word: SWSGPU_ECUDA when a kernel of an earlier call
 * on this handle gave up a bounded device-side wait (its spectra are
 * invalid; the GPU context stays usable) or the stream reports a CUDA
 * error.  swsgpu_wait performs the same check for submitted runs.  No
 * counterpart in the reference (its join() has no failure path). */
int swsgpu_sync(swsgpu_handle *h, void *cuda_stream);

/* Fault injection for tests, on the host side of the launch (no device
 * fault): SWSGPU_INJECT_DROP_EXCHANGE makes the next cluster-kernel launch
 * of this handle skip the distributed-shared-memory pushes of each
 * cluster's last job, so every receiving CTA's bounded wait for that job
 * runs out; the kernel finishes, sets the status word, and the next
 * swsgpu_wait / swsgpu_sync returns SWSGPU_ECUDA.  One-shot;
 * SWSGPU_INJECT_NONE cancels it.  SWSGPU_EINVAL on four-step plans. */
#define SWSGPU_INJECT_NONE 0
#define SWSGPU_INJECT_DROP_EXCHANGE 1
int swsgpu_inject(swsgpu_handle *h, int kind);

/* Device memory (bytes) the core allocates for a process_device call of
 * `nruns` runs of `run_bytes` as one output group, beyond the caller's
 * inputs and outputs: code arrays, blank bitmaps, frame validity, per-item
 * partial spectra, FP64 running sums for groups that span launches and,
 * for four-step lengths, the column-pass scratch (an upper bound). */
int swsgpu_workspace_size(const swsgpu_handle *h, size_t run_bytes, int nruns, size_t *bytes);

/* Unpack test entry: decode channel `chan` of `nsamp` samples from the
 * device stream d_raw (layout `lay`, payload offset `payload_offset`) to
 * float32 d_out on the device, with mark5access blanking.  Returns the
 * number of non-blanked samples through *nvalid (may be NULL).  d_raw and
 * d_out must be 4-byte aligned (SWSGPU_EINVAL otherwise). */
int swsgpu_unpack_device(const swsgpu_layout *lay, const void *d_raw, size_t nbytes,
                         int64_t payload_offset, int chan, int64_t nsamp, float *d_out,
                         int64_t *nvalid, void *cuda_stream);

/* No counterpart in the reference.  The same decode as swsgpu_unpack_device
 * without any device allocation, for callers that cannot allocate device
 * memory at the point where they decode: an acquisition thread that must not
 * stall on the device-wide synchronisation cudaMalloc/cudaFree can cause, an
 * application whose memory manager owns every device allocation, or a
 * process that reserves its device memory once at start-up.  Its scratch is
 * one fixed array of SWSGPU_NOALLOC_SCRATCH_BYTES compiled into the library;
 * every device that loads the library holds it until the process exits.
 * Limit: at most SWSGPU_NOALLOC_MAX_FRAMES frames per call (about 160 MB of
 * Mark5B data); larger requests return SWSGPU_ETOOBIG.  The caller still
 * provides d_raw and d_out.  The first call on each device is the one that
 * is not allocation-free: it looks up the scratch address for that device
 * (cudaGetSymbolAddress), which loads the library's device code and
 * allocates the array there; make one small warm-up call per device at
 * start-up, outside the thread that must not allocate.  Every call
 * synchronises its stream (it reads the sample count back), so it cannot
 * be issued on a stream that is being captured.  All calls share the one
 * scratch array: calls that overlap on the GPU (for example on two streams
 * at once) race and must be serialised by the caller.  Track formats (VLBA,
 * Mark4) need a conversion buffer of the data's size and return
 * SWSGPU_EINVAL here.  Returns like swsgpu_unpack_device; on a CUDA error
 * swsgpu_last_error(NULL) describes it. */
#define SWSGPU_NOALLOC_MAX_FRAMES 16384
#define SWSGPU_NOALLOC_SCRATCH_BYTES (SWSGPU_NOALLOC_MAX_FRAMES * 8 + 256)
int swsgpu_unpack_device_noalloc(const swsgpu_layout *lay, const void *d_raw, size_t nbytes,
                                 int64_t payload_offset, int chan, int64_t nsamp, float *d_out,
                                 int64_t *nvalid, void *cuda_stream);

/* The reference's phase-cal extractor library (src/IA-32/PhaseCal/PCal.h,
 * PCal.cpp) on the GPU: a stateful extractor over a stream of float samples
 * in device memory (e.g. swsgpu_unpack_device output).
 *   swsgpu_pcal_create      -> PCal::getNew (PCal.cpp:92-112); kind
 *                              SWSGPU_PCAL_AUTO takes the factory's choice,
 *                              the others force a class; the indices start
 *                              from sampleoffset (the reference's
 *                              constructors leave them unset)
 *   swsgpu_pcal_info        -> getLength (tone count), plus class and bins
 *   swsgpu_pcal_clear       -> clear (:229-241, :387-400, :575-587)
 *   swsgpu_pcal_adjust_offset -> adjustSampleOffset (:243-247, :402-406, :589-592)
 *   swsgpu_pcal_extract     -> extractAndIntegrate (:265-296, :424-487, :610-652);
 *                              asynchronous on cuda_stream; SWSGPU_ESTATE
 *                              after a final until clear, as the reference
 *                              returns false
 *   swsgpu_pcal_final       -> getFinalPCal (:298-318, :489-517, :654-678):
 *                              ntones complex tones (re, im doubles) into
 *                              host memory, *nsamples = samples integrated;
 *                              waits for cuda_stream
 * Sums and the DFT are FP64 (the reference's are FP32).  Shifting keeps the
 * reference's per-period sample selection (only floor(R/N)*N rotated
 * samples of every whole rotator period R are added). */
#define SWSGPU_PCAL_AUTO 0
#define SWSGPU_PCAL_TRIVIAL 1
#define SWSGPU_PCAL_SHIFTING 2
#define SWSGPU_PCAL_IMPLICIT 3
typedef struct swsgpu_pcal swsgpu_pcal;
int swsgpu_pcal_create(double bandwidth_hz, double spacing_hz, int offset_hz, int64_t sampleoffset, int kind,
                       int device, swsgpu_pcal **out);
int swsgpu_pcal_info(const swsgpu_pcal *p, int *kind, int *nbins, int *ntones);
int swsgpu_pcal_clear(swsgpu_pcal *p);
int swsgpu_pcal_adjust_offset(swsgpu_pcal *p, int64_t sampleoffset);
int swsgpu_pcal_extract(swsgpu_pcal *p, const float *d_samples, int64_t len, void *cuda_stream);
int swsgpu_pcal_final(swsgpu_pcal *p, double *tones_reim, uint64_t *nsamples, void *cuda_stream);
void swsgpu_pcal_destroy(swsgpu_pcal *p);

/* Tone-phase delay in ns from extracted tones: calcDelay of mark5access's
 * pulse-cal tool (mark5access/examples/m5pcal.c:96-155) -- the mean slope
 * of neighbouring tones' phase differences (radians, frequencies in MHz)
 * within band_valid_mhz of band_center_mhz, each unwrapped against the
 * difference at the middle of the list, folded into +- 500 / spacing. */
double swsgpu_pcal_delay(int ntones, const int *tone_mhz, const double *phase, double band_center_mhz,
                         double band_valid_mhz);

/* Number of kernel launches the last submit / process_device call issued. */
int swsgpu_last_launch_count(const swsgpu_handle *h);

/* Kernel timing on the launching stream: enable=1 starts recording CUDA
 * events around every FFT/accumulate kernel launch (resetting the totals),
 * enable=0 stops.  swsgpu_profile_read waits for the recorded launches and
 * returns their count and summed duration in milliseconds. */
int swsgpu_profile(swsgpu_handle *h, int enable);
int swsgpu_profile_read(swsgpu_handle *h, int *launches, double *total_ms);

#ifdef __cplusplus
}
#endif

#endif /* SWSGPU_H */
