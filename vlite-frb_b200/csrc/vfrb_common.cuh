// Shared definitions for the vlite-frb B200 kernels (sm_100a only).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "../../include/vfrb.h"

namespace vfrb {

// VLITE VDIF geometry (PIPE:33-36).
constexpr int kFrameLen = 5032;
constexpr int kHdrLen = 32;
constexpr int kDataLen = 5000;

// The channeliser's transform length: TWONCHAN = 2*6250 (PIPE:1249).
constexpr int kFftN = 12500;

// Device-side error bits (the kernels never trap; they flag and skip).
constexpr int kErrSlotRange = 1;     // sample position outside the slot table
constexpr int kErrRowRange = 2;      // FB row outside the ring
constexpr int kErrOffsetRange = 4;   // delay outside the prepared window
constexpr int kErrTimeout = 8;       // a bounded device wait gave up

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? VFRB_OK : VFRB_ERR_CUDA; }

// One stream's share of a batched dedispersion launch (grid z = job): what
// differs between streams of a plan -- their filterbank ring, FP16 scale,
// rows and output.  The delay tables, ring geometry and trial grid are the
// plan's.
struct DdJob {
  const void* fb;
  const void* fb1;  // FP16: the same ring shifted by one row (fb1[c][r] = fb[c][r + 1]), or NULL
  float out_scale;
  long long row0;
  long long nrows_valid;
  long long nt_out;
  float* out;
  long long out_stride;
  int* err;
};
constexpr int kDdMaxJobs = 32;

// Launchers (host side, defined in the .cu files).
int launch_channelise(const vfrb_chan_args& a, cudaStream_t s);
int launch_bandpass(const vfrb_bp_args& a, cudaStream_t s);
int launch_chan_stats(const vfrb_cs_args& a, cudaStream_t s);
int launch_chan_sk(const float* fb_tm, long long row_stride, int nchan, int nrows, int ncolstatblk, int nstatblks,
                   int nsum, float* sk, cudaStream_t s);
int launch_chan_sk_ring(const float* fb_tm, long long row_stride, long long row0, unsigned long long row_mask,
                        int nchan, int nrows, int ncolstatblk, int nstatblks, int nsum, float* sk, cudaStream_t s);
int launch_fb_transpose(const float* src_cm, long long chan_stride, unsigned row_mask, long long row0,
                        int nchan, int nrows, float* dst_tm, long long dst_row_stride, cudaStream_t s);
int launch_subtract_bp_full(float* fb, long long chan_stride, long long row0, unsigned row_mask, int nchan,
                            long long nrows, cudaStream_t s);
int launch_subtract_zero(float* fb, long long chan_stride, long long row0, unsigned row_mask, int nchan,
                         long long nrows, cudaStream_t s);
}  // namespace vfrb
struct vfrb_ddplan;
namespace vfrb {
int launch_dedisperse_jobs(const vfrb_ddplan* pl, int storage, const DdJob* jobs, int njobs, long long chan_stride,
                           unsigned row_mask, cudaStream_t s, int* launched);

}  // namespace vfrb
