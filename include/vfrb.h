/*
 * vfrb.h -- C ABI of libvfrb, the B200 (sm_100a) implementation of the
 * vlite-frb FRB search chain (VDIF -> channelise -> bandpass -> dedisperse
 * -> statistics).
 *
 * The reference (paulray/vlite-frb) has no library or FFI: its boundary is
 * three command-line tools that keep all state in globals.  Each entry point
 * below names the reference code it replaces (file:line, paths relative to
 * the reference checkout; PIPE = vdifFILE2dedisp_PIPELINE.cu, STATS =
 * vdifDADA2stats.cu, TS = vdifDADA2timeseries.cu).  The drop-in tools built
 * on this ABI keep the reference's names, flags and output files.
 *
 * Conventions: plain pointers and sizes only.  Pointers documented "device"
 * are CUDA device pointers of the calling process; `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  Status
 * codes mirror the reference's reader (0 ok, 1 end of data, 2 error,
 * PIPE:829-883) and add checked CUDA/argument errors (>= 3): nothing here
 * calls exit().
 */
#ifndef VFRB_H
#define VFRB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define VFRB_OK 0
#define VFRB_EOD 1              /* end of data (reference FLAGEOF/FLAGEODADA) */
#define VFRB_ERR 2              /* data/stream error (reference return 2)     */
#define VFRB_ERR_CUDA 3         /* a CUDA call failed                         */
#define VFRB_ERR_ARG 4          /* invalid argument                           */
#define VFRB_ERR_UNSUPPORTED 5  /* configuration not supported by the kernels */
#define VFRB_ERR_NOMEM 6        /* allocation or admission failed             */
#define VFRB_ERR_TIMEOUT 7      /* a bounded device wait gave up              */
#define VFRB_ERR_DEVICE 8       /* a kernel flagged an out-of-range access    */

/* storage form of the bandpass-subtracted filterbank */
#define VFRB_F32 0   /* plain form: FP32 throughout                           */
#define VFRB_F16 1   /* z = (P - mean)/s_c stored FP16, FP32 accumulation    */
#define VFRB_I8 2    /* round(z*q) stored int8 with per-channel scale         */

/* Human-readable text for a status code. */
const char* vfrb_strerror(int status);

/* ---- VDIF header (replaces vdifio.h:53-95 getters) ------------------- */
typedef struct vfrb_hdr {
  uint32_t seconds, legacymode, invalid;
  uint32_t frame, epoch, unassigned;
  uint32_t framelength8, nchan_log2, version;
  uint32_t stationid, threadid, nbits_minus1, iscomplex;
  uint32_t eversion, extended1, extended2, extended3, extended4;
} vfrb_hdr;

/* Decode the 32-byte little-endian VDIF header (bit layout vdifio.h:53-72). */
int vfrb_decode_header(const uint8_t* hdr32, vfrb_hdr* out);

/* MJD of a frame, replacing getVDIFDMJD (vdifio.h:87; called PIPE:525). */
double vfrb_header_dmjd(const vfrb_hdr* h, int framespersec);

/* ---- derived parameters (PIPE:289-303, STATS:208-231, TS:277-298) ---- */
typedef struct vfrb_layout {
  int32_t twonchan, nchan, nfreq, nchanout, nskip, nave, nbundle, nloop;
  int32_t maxnt, nhalfcyc;
  double chanbw, fch1, foff, tchan;
  float maxtime;
} vfrb_layout;

/* nchanout_fixed > 0 forces NCHANOUT (TS hard-codes 3840, TS:282);
 * muoslowfreq 360 is the reference default, 384 the full band (PIPE:46-47). */
int vfrb_layout_init(vfrb_layout* L, int twonchan, int nave, int nbundle,
                     double muoslowfreq, int nchanout_fixed, float maxtime);

/* Delay table OFF[ndm][nchanout] in FB rows and max_delay, replacing the
 * OFFSET/max_delay code of TS:449-464 (PIPE:449-461). */
int vfrb_delay_table(const vfrb_layout* L, const float* dms, int ndm,
                     int32_t* off_out, int32_t* max_delay_out);

/* ---- K1: fused channeliser --------------------------------------------
 * Replaces, per bundle, the two H2D copies' consumers: convertarray x2,
 * cufftExecR2C x2 (N = TWONCHAN), sumpower, avepower and the 32 per-row
 * D2D channel-select copies (PIPE:574-632; STATS:377-405; TS:603-636).
 * Input is the raw VDIF stream: each pol's sample stream is the
 * concatenation of 5000-byte frame payloads named by a slot table.
 * Output row r (time-major, nchanout floats) is written at ring row
 * (out_row0 + r) & out_row_mask. */
typedef struct vfrb_chan_args {
  const uint8_t* frames;     /* device: raw VDIF bytes                          */
  const int64_t* slots0;     /* device: pol-0 payload byte offset per frame slot,
                                -1 = fill frame of zero bytes (PIPE:1044-1052)  */
  const int64_t* slots1;     /* device: same for pol 1                          */
  int64_t nslots;
  int64_t sample0;           /* stream position of row 0's first sample         */
  int32_t nrows;
  int32_t twonchan, nave, nfreq, nskip, nchanout;
  float* out;                /* device: time-major FB                           */
  int64_t out_row_stride;    /* floats between rows                             */
  int64_t out_row0;
  uint32_t out_row_mask;     /* rows-1 for a power-of-two ring, ~0 for linear   */
  int32_t* d_err;            /* device int (error bits) or NULL                 */
} vfrb_chan_args;
int vfrb_channelise(const vfrb_chan_args* a, void* stream);

/* ---- K2: bandpass + cal subtraction ------------------------------------
 * Replaces subtractbpCAL (PIPE:1427-1474; STATS:869-908; TS:1365-1407):
 * per (channel, window of `window` rows counted from in_row0) mean,
 * variance ("sig"), open-interval 3-sig clip, clipped mean subtracted.
 * Reads the raw time-major FB and writes the result channel-major
 * (the layout the dedisperser streams), in the chosen storage form. */
typedef struct vfrb_bp_args {
  const float* in;           /* device: raw time-major FB                       */
  int64_t in_row_stride;
  int64_t in_row0;
  uint32_t in_row_mask;
  int32_t nchan;
  int32_t nrows;             /* rows from in_row0; the last window may be short */
  int32_t window;            /* 128 (HALFCYCLE windows, PIPE:51,1433)           */
  int32_t storage;           /* VFRB_F32 / VFRB_F16 / VFRB_I8                   */
  void* out;                 /* device: channel-major result                    */
  int64_t out_chan_stride;   /* elements between channels                       */
  int64_t out_row0;
  uint32_t out_row_mask;
  const float* inv_scale;    /* device [nchan]: 1/s_c (F16, I8), NULL for F32   */
  float q_scale;             /* I8 only: stored = round(z*q_scale)              */
  float* win_mean;           /* device [nwin][nchan] subtracted mean, or NULL   */
  float* win_var;            /* device [nwin][nchan] window variance, or NULL   */
  float* tm_out;             /* device time-major F32 copy of the result, or NULL */
  int64_t tm_row_stride;
  int32_t* d_err;
  int32_t subtract_mode;     /* 0: cal windows (subtractbpCAL); 1: copy only,
                              * no subtraction (feeds vfrb_subtract_bp_full)  */
  void* out_shift1;          /* F16 only, or NULL (no reference counterpart):
                              * device copy of `out` shifted by one row, same
                              * strides and ring: absolute row R >= 1 of the
                              * result also goes to row R - 1 here, so that
                              * out_shift1[c][r] = out[c][r + 1]; pass it to
                              * vfrb_dedisperse as fb_shift1               */
} vfrb_bp_args;
int vfrb_bandpass(const vfrb_bp_args* a, void* stream);

/* ---- Optional RFI modes the reference keeps as dead code ----------------
 * Both work in place on a channel-major FP32 filterbank
 * fb_cm[c * chan_stride + ((row0 + t) & row_mask)], t < nrows; row_mask
 * 0xffffffff means a linear run (row0 + nrows <= chan_stride), otherwise a
 * power-of-two ring of row_mask + 1 <= chan_stride rows.  nchan, nrows >= 2.
 *
 * vfrb_subtract_bp_full replaces subtractbp (PIPE:1372-1424; its call is
 * commented out at PIPE:712): per channel, one clipped mean over the whole
 * block is subtracted.  The reference's arithmetic is kept: the first mean
 * divides the channel sum by NCHANOUT (nchan), not by the row count; the
 * clip is the open interval ave +- 3*sig with sig the variance about that
 * value; an empty clip gives NaN.
 *
 * vfrb_subtract_zero replaces subtractZERO (PIPE:1478-1515; commented out at
 * PIPE:661, after subtractbpCAL): per row, the clipped mean across channels
 * (count floored at 1) is subtracted from every channel (zero-DM removal). */
int vfrb_subtract_bp_full(float* fb_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask, int nchan,
                          int64_t nrows, void* stream);
int vfrb_subtract_zero(float* fb_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask, int nchan,
                       int64_t nrows, void* stream);

/* ---- K3: dedispersion + per-DM statistics ------------------------------
 * Replaces dedisp_execute (PIPE:671, dedisp library, semantics unpinned)
 * by the reference's in-tree brute-force sum (PIPE:1517-1537):
 *   out[d][t] = (sum_c w_c * FB[t + OFF[d][c]][c]) / nchan,  w_c = 1 (F32)
 * and fuses calcstats (PIPE:1337-1370).  With sigma_out set it computes
 * dedisperseSTATS instead (TS:1450-1481): the channel mean and the
 * per-sample channel sigma. */
typedef struct vfrb_ddplan vfrb_ddplan;

/* Copies the delay table (host, [ndm][nchan]) to the device and sizes the
 * shared-memory tiles.  ndm >= 1, nchan >= 2. */
int vfrb_ddplan_create(vfrb_ddplan** plan, const int32_t* h_offsets, int ndm, int nchan);
int vfrb_ddplan_destroy(vfrb_ddplan* plan);
int vfrb_ddplan_max_delay(const vfrb_ddplan* plan);
/* Trials per register group of the fast kernel (4, 2 or 1), 0 when only the
 * staged/direct kernels apply (no reference counterpart; introspection). */
int vfrb_ddplan_group_size(const vfrb_ddplan* plan);

/* Kernel variants of the dedisperser (no reference counterpart).  AUTO uses
 * the autotuned choice (or the largest register group that fits). */
#define VFRB_DD_AUTO 0
#define VFRB_DD_STAGED 1   /* shared-memory tile, one load per add           */
#define VFRB_DD_REG1 2     /* register window, 1 trial per thread            */
#define VFRB_DD_REG2 3     /* register window, 2 adjacent trials per thread  */
#define VFRB_DD_REG4 4     /* register window, 4 adjacent trials per thread  */
#define VFRB_DD_DIRECT 5   /* direct loads (delay spreads too wide to stage) */
#define VFRB_DD_PAT4 6     /* register window, 4 trials, runs of one delay pattern */
#define VFRB_DD_PAT2 7     /* register window, 2 trials, runs of one delay pattern */
#define VFRB_DD_NVARIANTS 8
int vfrb_ddplan_set_variant(vfrb_ddplan* plan, int storage, int variant);
int vfrb_ddplan_variant(const vfrb_ddplan* plan, int storage);
/* Times every applicable variant on scratch data of the given shape
 * (nt_out samples per trial, `storage` form) and keeps the fastest.  Writes
 * the per-variant times in ms to times[VFRB_DD_NVARIANTS] (index = variant,
 * < 0 = not applicable).  FP16 variants are timed without a shifted ring
 * (vfrb_dd_args.fb_shift1); given one, VFRB_DD_PAT4 runs its faster pair
 * form, so the choice of PAT4 stands. */
int vfrb_ddplan_autotune(vfrb_ddplan* plan, int storage, int64_t nt_out, float* times, void* stream);

typedef struct vfrb_dd_args {
  const void* fb;            /* device: channel-major FB in `storage` form       */
  int32_t storage;
  const float* chan_scale;   /* device [nchan]: w_c for F16/I8, NULL for F32     */
  float uniform_scale;       /* F16/I8 with chan_scale NULL: one w for all c     */
  int64_t chan_stride;
  int64_t row0;              /* ring row of output sample 0                      */
  uint32_t row_mask;
  int64_t nrows_valid;       /* rows readable from row0 (>= nt_out + max delay)  */
  int64_t nt_out;            /* output samples per DM                            */
  float* out;                /* device [ndm][out_stride]                         */
  int64_t out_stride;
  float* sigma_out;          /* device [ndm][out_stride] (TS mode) or NULL       */
  void* workspace;           /* device scratch, vfrb_dedisperse_workspace_bytes  */
  size_t workspace_bytes;
  /* calcstats outputs, device [ndm] each, any may be NULL */
  float* ave;
  float* sigma;
  float* peak;
  int32_t* frb;
  int32_t* argmax;
  int32_t* d_err;
  const void* fb_shift1;     /* F16 only, or NULL (no reference counterpart):
                              * `fb` shifted by one row (fb_shift1[c][r] =
                              * fb[c][r + 1] for every row but the last valid
                              * one; vfrb_bp_args.out_shift1 writes it).  The
                              * four-trial pattern kernel then reads windows of
                              * halves with 4-byte loads; results equal the
                              * plain FP16 form's up to FP32 summation order */
} vfrb_dd_args;
size_t vfrb_dedisperse_workspace_bytes(const vfrb_ddplan* plan, int64_t nt_out);
int vfrb_dedisperse(const vfrb_ddplan* plan, const vfrb_dd_args* a, void* stream);

/* vfrb_dedisperse without caller scratch (no counterpart in the reference,
 * whose dedisperse + calcstats write into buffers it allocated at start-up).
 * For callers that may not allocate device memory after start-up: the
 * per-DM statistics partials go to a fixed device array of
 * VFRB_NOALLOC_SCRATCH_BYTES per device instead of a->workspace, which is
 * ignored; this call allocates nothing.  Requests whose
 * vfrb_dedisperse_workspace_bytes exceed that size return VFRB_ERR_ARG and
 * launch nothing.  The first call on each device looks up the array's
 * address (make it before any stream capture); the address is looked up
 * again when the device's current CUDA context changes (another context
 * made current, the primary context re-created after cudaDeviceReset), and
 * the first call after such a change should likewise come before any
 * stream capture.  All calls on one device
 * share the array: calls whose work overlaps on the GPU (other streams,
 * other threads) race and corrupt each other's statistics, so order them
 * on one stream.  Nothing in the array needs to start at zero. */
#define VFRB_NOALLOC_SCRATCH_BYTES (4u << 20)
size_t vfrb_dedisperse_noalloc_scratch_bytes(void);
int vfrb_dedisperse_noalloc(const vfrb_ddplan* plan, const vfrb_dd_args* a, void* stream);

/* ---- candidate search (extension: the reference's calcstats peak,
 * PIPE:1337-1370, has no width) -------------------------------------------
 * Per trial d of a dedispersed series dd[d][0..nt) (row stride `stride`):
 * the best boxcar over widths 1, 2, 4, ..., max_width of
 *   snr_w(t) = (sum_{i<w} dd[d][t+i] - w*ave[d]) / (sigma[d]*sqrt(w)),
 * t = 0 .. nt-w, with the trial's calcstats ave/sigma (width 1 = peak).
 * Ties: smaller width, then earlier start.  All pointers device. */
int vfrb_boxcar(const float* dd, int ndm, int64_t nt, int64_t stride, const float* ave, const float* sigma,
                int max_width, float* snr, int32_t* start, int32_t* width, void* stream);

/* ---- K4: per-channel statistics (STATS:910-946) -------------------------
 * Per (channel, block of ncolstatblk rows): mean, variance ("sig") and the
 * outlier fraction count(x > ave + 5 sig)/npts with the reference's integer
 * division.  Outputs are [nstatblks][nchan] like CHANAVE/CHANSIGMA/
 * CHANOUTLIER. */
typedef struct vfrb_cs_args {
  const float* fb;           /* device: channel-major F32 FB                     */
  int64_t chan_stride;
  int64_t row0;
  uint32_t row_mask;
  int32_t nchan, nrows, ncolstatblk, nstatblks;
  float* ave;
  float* sig;
  float* outlier;
} vfrb_cs_args;
int vfrb_chan_stats(const vfrb_cs_args* a, void* stream);

/* Spectral kurtosis per (channel, block of ncolstatblk rows) of the RAW
 * time-major FB (before bandpass subtraction; no reference counterpart --
 * the reference's stats tool has none): the generalised estimator
 *   SK = (M*nsum + 1)/(M - 1) * (M*S2/S1^2 - 1),
 * M = rows in the block, S1 = sum x, S2 = sum x^2 (FP64), nsum = raw power
 * values summed per FB sample (2 pols x NAVE).  E[SK] = 1 for Gaussian
 * noise.  sk is [nstatblks][nchan]; every block needs a row (one row:
 * inf/NaN). */
int vfrb_chan_sk(const float* fb_tm, int64_t row_stride, int nchan, int nrows, int ncolstatblk, int nstatblks,
                 int nsum, float* sk, void* stream);

/* Channel-major -> time-major copy (the SIGPROC .nohead.fil layout,
 * PIPE:777). */
int vfrb_fb_to_time_major(const float* src_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask,
                          int nchan, int nrows, float* dst_tm, int64_t dst_row_stride, void* stream);

/* ======================================================================
 * Plan / stream API.  Replaces the main loops of the three tools
 * (PIPE:556-708, STATS:367-431, TS:589-746): raw VDIF bytes go in as they
 * arrive, results come out per block (reference semantics) or per chunk
 * (streaming).  The drop-in tools and the serving loop are built on it.
 * ====================================================================== */
#define VFRB_PENDING 9             /* vfrb_poll: nothing ready yet        */

#define VFRB_MODE_BLOCK 0          /* MAXTIME blocks, max_delay carry, block-relative
                                      bandpass windows (PIPE:649-704, TS:643-692,
                                      STATS:411-429)                       */
#define VFRB_MODE_STREAM 1         /* continuous: absolute 128-row bandpass windows,
                                      every output sample computed once    */

#define VFRB_READER_PIPE 0         /* gaps = frame-number difference mod 25600 */
#define VFRB_READER_TS 1           /* seconds-aware gaps (TS:895-937)      */

#define VFRB_OUT_DEDISP 1          /* dedispersed series [ndm][nt]          */
#define VFRB_OUT_DMSTATS 2         /* per-DM ave/sigma/peak/FRB/argmax      */
#define VFRB_OUT_SIGMA 4           /* per-sample channel sigma (TS)         */
#define VFRB_OUT_CHANSTATS 8       /* per-channel statistics (STATS); stream
                                      mode: FP32 form, one result per absolute
                                      TIMESTATS block (see vfrb_result)     */
#define VFRB_OUT_FB 16             /* bandpass-subtracted FB, time-major    */
#define VFRB_OUT_CANDS 32          /* candidate list                        */
#define VFRB_OUT_FLAGS 64          /* per-row data flags (VFRB_ROW_*)       */

/* Row flags: an FB row is flagged when any frame whose samples it holds (in
 * either pol) carried the VDIF invalid bit (the reference ignores the bit,
 * so the data are processed as usual), or was a zero-filled missing frame. */
#define VFRB_ROW_INVALID 1
#define VFRB_ROW_FILL 2

typedef struct vfrb_plan vfrb_plan;

typedef struct vfrb_params {
  int32_t twonchan, nave, nbundle; /* -nchan*2, -nave, -nb (PIPE:1245-1288)   */
  double muoslowfreq;              /* 360 (default) or 384 (full band)       */
  int32_t nchanout_fixed;          /* > 0 forces NCHANOUT (TS: 3840)         */
  float maxtime;                   /* block length in seconds (MAXTIME)      */
  float timestats;                 /* STATS statistics block (TIMESTATS)     */
  const float* dms;                /* DM trial list (DM101.txt), host        */
  int32_t ndm;
  int32_t mode;                    /* VFRB_MODE_*                            */
  int32_t reader;                  /* VFRB_READER_*                          */
  int32_t dada_skip;               /* skip NFRAMEDADAINIT pairs first (TS)   */
  int32_t storage;                 /* VFRB_F32 / VFRB_F16 / VFRB_I8          */
  float q_scale;                   /* int8 quantisation (z units -> counts)  */
  int32_t outputs;                 /* VFRB_OUT_* bits                        */
  int32_t fb_block;                /* block whose FB is returned (-1: all)   */
  int32_t nstreams;                /* streams opened at creation (0..4096; more
                                    * with vfrb_stream_open)               */
  float chunk_seconds;             /* streaming output chunk                 */
  float ring_seconds;              /* device raw-frame ring per stream       */
  float cand_snr;                  /* candidate threshold (peak SNR)         */
  int32_t device;
  int64_t device_bytes;            /* admission budget, 0 = 90% of free      */
  int32_t boxcar_max;              /* candidates: widest boxcar (1 = peak only) */
  int32_t bp_mode;                 /* VFRB_BP_CAL (subtractbpCAL) or VFRB_BP_FULL
                                    * (subtractbp, PIPE:1372); FULL: block
                                    * mode, FP32 storage only                 */
  int32_t zero_dm;                 /* 1: subtractZERO after the bandpass
                                    * (PIPE:1478); block mode, FP32 only      */
  int32_t batch_streams;           /* stream mode: 1 = the dedispersion of the
                                    * chunks that become ready in several
                                    * streams runs as one launch (up to 32
                                    * streams), issued at the next vfrb_poll
                                    * or when a stream needs its buffers
                                    * again; results are identical to
                                    * per-stream launches                  */
} vfrb_params;

#define VFRB_BP_CAL 0
#define VFRB_BP_FULL 1

/* Reference defaults: 12500-point FFT, NAVE 4, NBUNDLE 32, 3908 channels,
 * MAXTIME 70 s, block mode, FP32, one stream. */
void vfrb_params_default(vfrb_params* p);

typedef struct vfrb_cand {
  int32_t dm_index;
  int32_t width;                   /* boxcar width in samples (1 = none)     */
  int64_t t;                       /* absolute FB row of the peak (with the
                                    * boxcar search: of the box's first row) */
  float snr;
  float dm;
} vfrb_cand;

/* Friends-of-friends clustering of candidates across trials and time (no
 * reference counterpart).  Friends: |dm_index_a - dm_index_b| <= dm_tol and
 * max(t_a, t_b) - min(t_a + width_a, t_b + width_b) <= t_tol.  Writes one
 * entry per connected component to out[] (capacity n): its brightest member
 * (ties: lower dm_index, then earlier t), ordered by t then dm_index; *nout =
 * their count; cluster_of[i] (optional, n entries) = the cluster of in[i].
 * Candidates from several results can be concatenated and clustered together. */
int vfrb_cluster_cands(const vfrb_cand* in, int32_t n, int32_t dm_tol, int64_t t_tol, vfrb_cand* out,
                       int32_t* nout, int32_t* cluster_of);

typedef struct vfrb_result {
  int32_t stream;
  int64_t seq;                     /* block (block mode) or chunk index      */
  int64_t row0;                    /* absolute FB row of output sample 0 (block
                                    * mode: of block row 0; block rows from
                                    * (max_delay/NBUNDLE)*NBUNDLE on lie
                                    * max_delay mod NBUNDLE rows later, as the
                                    * reference's carry overwrites them)    */
  double tstart_mjd;               /* getVDIFDMJD of the first frame used    */
  int32_t ndm;
  int64_t nt;
  const float* dd;                 /* [ndm][nt] or NULL                      */
  const float* dd_sigma;           /* [ndm][nt] or NULL                      */
  const float* ave;                /* [ndm] each, or NULL                    */
  const float* sigma;
  const float* peak;
  const int32_t* frb;
  const int32_t* argmax;
  int32_t nchan;
  int64_t fb_rows;
  const float* fb;                 /* [fb_rows][nchan] or NULL               */
  int32_t nstatblks;               /* block mode: TIMESTATS blocks of the
                                    * block; stream mode: 1 in the result of
                                    * one statistics block (rows [row0, row0 +
                                    * nflag_rows or TIMESTATS rows), nt = 0),
                                    * 0 in series results                  */
  const float* chan_ave;           /* [nstatblks][nchan] each, or NULL       */
  const float* chan_sig;
  const float* chan_outlier;
  int32_t ncand;
  const vfrb_cand* cands;
  double latency_ms;               /* data complete -> result on the host    */
  int32_t device_errors;           /* kernel error bits seen (0 = none)      */
  const float* box_snr;            /* [ndm] best boxcar SNR, or NULL          */
  const int32_t* box_start;        /* [ndm] its start (row0-relative)         */
  const int32_t* box_width;        /* [ndm] its width in samples              */
  const float* chan_sk;            /* [nstatblks][nchan] spectral kurtosis of
                                    * the raw FB (with chan_ave), or NULL   */
  int64_t nflag_rows;
  const uint8_t* row_flags;        /* VFRB_OUT_FLAGS: VFRB_ROW_* per FB row;
                                    * block mode: block rows [0, MAXNT);
                                    * stream mode: rows [row0, row0 + nt)   */
} vfrb_result;

int vfrb_plan_create(vfrb_plan** plan, const vfrb_params* params);
int vfrb_plan_destroy(vfrb_plan* plan);
/* Derived layout and the max_delay in FB rows used for the overlap carry. */
int vfrb_plan_layout(const vfrb_plan* plan, vfrb_layout* L, int32_t* max_delay);
int64_t vfrb_plan_device_bytes(const vfrb_plan* plan);

/* Feed raw VDIF bytes of one stream (any split; frames may straddle calls).
 * nbytes == 0 marks end of data (the reference's EOF/EOD).  Page-locked
 * input is copied to the device directly, other host input through a
 * staging buffer; `bytes` may also be device memory of the plan's device
 * (frames already on the GPU, e.g. from a capture kernel): they are copied
 * device to device and only their 32-byte headers go to the host for the
 * pair reader.  Device input is read after all work queued before the call
 * on the legacy default stream (PyTorch's default stream); input written on
 * another stream must be complete (that stream synchronised) before the
 * call.  `bytes` may be reused as soon as the call returns. */
int vfrb_push_frames(vfrb_plan* plan, int stream, const uint8_t* bytes, size_t nbytes);

/* Streams opened and closed while others run (serving).  vfrb_stream_open
 * admits one more stream if its device bytes fit the budget (device_bytes,
 * or 90% of the free memory) beside the open streams, and returns its id
 * (ids are never reused); VFRB_ERR_NOMEM when it does not fit -- retry after
 * another stream has closed.  vfrb_stream_close ends the stream's data (as
 * vfrb_push_frames with nbytes 0) and, once all its results have been
 * polled, frees its memory and returns VFRB_OK; before that it returns
 * VFRB_PENDING.  A result of the stream returned by the last vfrb_poll is
 * invalid after the close. */
int vfrb_stream_open(vfrb_plan* plan, int* stream);
int vfrb_stream_close(vfrb_plan* plan, int stream);

/* Next completed result in submission order.  Returns VFRB_OK with *out
 * filled (host buffers owned by the plan, valid until the next poll),
 * VFRB_PENDING when work is in flight but not done (wait == 0), or
 * VFRB_EOD when every stream has ended and nothing is left. */
int vfrb_poll(vfrb_plan* plan, vfrb_result* out, int wait);

/* Host-only: run the pol-pair reader of the plan API over a byte buffer fed
 * in pieces of `split` bytes (0 = one piece), as initframe01 +
 * readtwoframe (PIPE:1031-1131; TS:767-1145 with reader VFRB_READER_TS).
 * Writes the pair sequence as frame indices into the input (-1 = zero fill
 * frame); entry 0 is the pair initframe01 leaves in the buffers.  Returns
 * VFRB_OK, or VFRB_ERR when initialisation fails (the reference exits 2). */
int vfrb_read_pairs(const uint8_t* bytes, size_t nbytes, int reader_mode, int dada_skip, size_t split,
                    int64_t* e0, int64_t* e1, int64_t cap, int64_t* npairs, double* tstart_mjd);

/* Reader log lines (frame skips, misalignment) of a stream, '\n'-joined;
 * valid until the next call.  Mirrors the reference's <OUT>.log messages. */
const char* vfrb_stream_log(vfrb_plan* plan, int stream);

/* MJD of the first frame pair a stream uses (getVDIFDMJD after initframe01,
 * PIPE:525, STATS:365, TS:535): VFRB_OK once the reader has started,
 * VFRB_PENDING before, VFRB_ERR when the stream failed to start. */
int vfrb_stream_tstart(vfrb_plan* plan, int stream, double* mjd);

/* ---- DADA-style input ring (host only) -----------------------------------
 * The STATS and TS tools read VDIF from a psrdada ring (ipcio_connect /
 * ipcio_open 'R' / ipcio_read / ipcbuf_eod: STATS:286-310, 444-462;
 * TS:383-404, 767-826).  psrdada is not part of this build; this is a
 * project-defined single-writer single-reader byte ring in POSIX shared
 * memory named after the DADA key, with the same reader-side operations.
 * All waits are bounded: reads and writes return -VFRB_ERR_TIMEOUT when
 * nothing moved for timeout_ms. */
typedef struct vfrb_dada vfrb_dada;
/* capacity: data bytes, a power of two >= 4096.  Fails if the key exists. */
int vfrb_dada_create(uint32_t key, uint64_t capacity, vfrb_dada** ring);
int vfrb_dada_connect(uint32_t key, vfrb_dada** ring);
/* Bytes written (all of them unless the wait ran out), or -status. */
int64_t vfrb_dada_write(vfrb_dada* ring, const void* bytes, uint64_t n, int timeout_ms);
int vfrb_dada_set_eod(vfrb_dada* ring);
/* Bytes read: n, fewer at end of data (like ipcio_read), or -status. */
int64_t vfrb_dada_read(vfrb_dada* ring, void* buf, uint64_t n, int timeout_ms);
/* 1 when the writer has ended and every byte was read (ipcbuf_eod). */
int vfrb_dada_eod(const vfrb_dada* ring);
/* In-place reading: waits (bounded) for readable bytes and points *ptr at
 * the longest contiguous run of them (at most max_n; it stops at the ring's
 * end) without consuming them; returns its length, 0 at end of data, or
 * -status.  vfrb_dada_release(n) consumes the first n acquired bytes. */
int64_t vfrb_dada_acquire(vfrb_dada* ring, const uint8_t** ptr, uint64_t max_n, int timeout_ms);
int vfrb_dada_release(vfrb_dada* ring, uint64_t n);
/* Page-locks this process's mapping of the ring (needs a CUDA device), so
 * vfrb_push_frames copies acquired bytes straight to the device. */
int vfrb_dada_pin(vfrb_dada* ring);
/* The header block beside the data block (as a DADA ring's): the writer sets
 * up to 4096 bytes of text; a reader waits (bounded) for it and copies at
 * most cap bytes.  Returns the header's length, or -status. */
int vfrb_dada_set_header(vfrb_dada* ring, const char* text, uint64_t n);
int64_t vfrb_dada_get_header(vfrb_dada* ring, char* buf, uint64_t cap, int timeout_ms);
/* Primary read client (ipcio_open 'R', STATS:294, TS:368): the ring's
 * `iread` names the reader holding the role, -1 = none.  vfrb_dada_open_read
 * takes it and returns VFRB_ERR while another reader holds it;
 * vfrb_dada_force_iread clears it (the reference's ipcbuf_force_iread,
 * STATS:127-134, TS:140-147) and returns the previous holder; closing a
 * handle gives its role back. */
int vfrb_dada_iread(const vfrb_dada* ring);
int vfrb_dada_force_iread(vfrb_dada* ring);
int vfrb_dada_open_read(vfrb_dada* ring);
int vfrb_dada_close(vfrb_dada* ring);
int vfrb_dada_destroy(uint32_t key);

/* ---- output formats (host only) -----------------------------------------
 * SIGPROC filterbank header as PIPE:529-540 writes it with the send_*
 * helpers of PIPE:1177-1201 (keyword = int32 length + text, values native
 * binary).  Returns the header length; writes it when cap is large enough. */
size_t vfrb_sigproc_header(uint8_t* buf, size_t cap, double fch1, double foff, int32_t nchans, int32_t nbits,
                           double tstart, double tsamp, int32_t nifs);
/* PRESTO .inf text of the TS time series (writeprestoheader, TS:1483-1515).
 * Returns the text length (excluding the NUL), writing it when cap > that;
 * -1 on a NULL basename. */
int vfrb_presto_inf(char* buf, size_t cap, const char* basename, double mjdstart, int32_t ntimes, double tsamp,
                    float dm, double fchanlo, double bw, int32_t nchan, double chanbw);

#ifdef __cplusplus
}
#endif
#endif /* VFRB_H */
