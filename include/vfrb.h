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
} vfrb_bp_args;
int vfrb_bandpass(const vfrb_bp_args* a, void* stream);

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

typedef struct vfrb_dd_args {
  const void* fb;            /* device: channel-major FB in `storage` form       */
  int32_t storage;
  const float* chan_scale;   /* device [nchan]: w_c for F16/I8, NULL for F32     */
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
} vfrb_dd_args;
size_t vfrb_dedisperse_workspace_bytes(const vfrb_ddplan* plan, int64_t nt_out);
int vfrb_dedisperse(const vfrb_ddplan* plan, const vfrb_dd_args* a, void* stream);

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

/* Channel-major -> time-major copy (the SIGPROC .nohead.fil layout,
 * PIPE:777). */
int vfrb_fb_to_time_major(const float* src_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask,
                          int nchan, int nrows, float* dst_tm, int64_t dst_row_stride, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VFRB_H */
