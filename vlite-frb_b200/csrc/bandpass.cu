// K2: bandpass + noise-cal subtraction, K4: per-channel statistics, and the
// channel-major -> time-major copy.  HBM-bound kernels for sm_100a.
//
// K2 replaces subtractbpCAL (PIPE:1427-1474; STATS:869-908; TS:1365-1407).
// A CTA takes one window of <=128 rows x 32 channels of the raw time-major
// filterbank (coalesced 128-byte row segments), transposes it in shared
// memory, and one warp per channel computes in FP64: mean, the variance the
// reference calls "sig", the open-interval clip ave +- 3 sig and the clipped
// mean (count floored at 1).  The subtracted rows are written channel-major
// (512-byte runs per channel), the layout the dedisperser streams, in FP32,
// FP16 (z = x/s_c) or int8 (round(z*q)) form.  subtract_mode 1 skips the
// statistics and writes the rows unchanged (the input of the whole-block
// subtractbp in rfi.cu).  The FP16 form can also write a copy shifted by one
// row, out1[c][r - 1] = out[c][r] (absolute rows, the same ring geometry):
// with both copies the dedisperser reads any window of halves with aligned
// 4-byte loads.
#include "vfrb_common.cuh"

namespace vfrb {

constexpr int kBpThreads = 256;  // 8 warps
constexpr int kBpChan = 32;      // channels per CTA
constexpr int kBpMaxWin = 128;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int STORAGE>
__global__ void __launch_bounds__(kBpThreads) k_bandpass(const vfrb_bp_args a, __half* __restrict__ out1) {
  __shared__ float tile[kBpChan][kBpMaxWin + 1];
  const int win = blockIdx.y;
  const int c0 = blockIdx.x * kBpChan;
  const long long r0 = (long long)win * a.window;
  const int npts = (int)min((long long)a.window, (long long)a.nrows - r0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int err = 0;

  // load rows (time-major) -> tile[ch][row]: a warp's 16 rows are loaded
  // into registers first, so all 16 row segments are in flight together
  {
    constexpr int kRowsPerWarp = kBpMaxWin / (kBpThreads / 32);
    float v[kRowsPerWarp];
    const int c = c0 + lane;
#pragma unroll
    for (int k = 0; k < kRowsPerWarp; ++k) {
      const int r = warp + (kBpThreads / 32) * k;
      const unsigned long long rr = (unsigned long long)(a.in_row0 + r0 + r) & (unsigned long long)a.in_row_mask;
      v[k] = (r < npts && c < a.nchan) ? a.in[(long long)rr * a.in_row_stride + c] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < kRowsPerWarp; ++k) {
      const int r = warp + (kBpThreads / 32) * k;
      if (r < npts) tile[lane][r] = v[k];
    }
  }
  __syncthreads();

  for (int cl = warp; cl < kBpChan; cl += kBpThreads / 32) {
    const int c = c0 + cl;
    if (c >= a.nchan) break;
    float x[kBpMaxWin / 32];
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kBpMaxWin / 32; ++k) {
      const int r = lane + 32 * k;
      x[k] = (r < npts) ? tile[cl][r] : 0.f;
      s += (r < npts) ? (double)x[k] : 0.0;
    }
    double cave = 0.0, sig = 0.0;  // subtract_mode 1: copy only (cave = 0)
    if (a.subtract_mode == 0) {
      const double n = (double)npts;
      const double ave = warp_sum(s) / n;
      double sd = 0.0, sd2 = 0.0;
#pragma unroll
      for (int k = 0; k < kBpMaxWin / 32; ++k) {
        const int r = lane + 32 * k;
        if (r < npts) {
          const double d = (double)x[k] - ave;
          sd += d;
          sd2 += d * d;
        }
      }
      sd = warp_sum(sd);
      sd2 = warp_sum(sd2);
      sig = (sd2 - (sd * sd) / n) / (n - 1.0);  // variance, NaN when npts == 1
      const double hi = ave + 3.0 * sig, lo = ave - 3.0 * sig;
      double cs = 0.0;
      int cnt = 0;
#pragma unroll
      for (int k = 0; k < kBpMaxWin / 32; ++k) {
        const int r = lane + 32 * k;
        const double xv = (double)x[k];
        if (r < npts && xv < hi && xv > lo) {
          cs += xv;
          ++cnt;
        }
      }
      cs = warp_sum(cs);
      cnt = warp_sum_i(cnt);
      if (cnt == 0) cnt = 1;
      cave = cs / (double)cnt;
    }
    if (lane == 0) {
      if (a.win_mean) a.win_mean[(long long)win * a.nchan + c] = (float)cave;
      if (a.win_var) a.win_var[(long long)win * a.nchan + c] = (float)sig;
    }
    const float inv = (STORAGE == VFRB_F32) ? 1.f : a.inv_scale[c];
#pragma unroll
    for (int k = 0; k < kBpMaxWin / 32; ++k) {
      const int r = lane + 32 * k;
      if (r < npts) {
        const float y = (float)((double)x[k] - cave);
        const unsigned long long orow =
            (unsigned long long)(a.out_row0 + r0 + r) & (unsigned long long)a.out_row_mask;
        const long long o = (long long)c * a.out_chan_stride + (long long)orow;
        if (STORAGE == VFRB_F32) {
          reinterpret_cast<float*>(a.out)[o] = y;
        } else if (STORAGE == VFRB_F16) {
          const __half h = __float2half_rn(y * inv);
          reinterpret_cast<__half*>(a.out)[o] = h;
          const long long ra = a.out_row0 + r0 + r;  // absolute row; row ra - 1 of the shifted copy
          if (out1 && ra >= 1)
            out1[(long long)c * a.out_chan_stride +
                 (long long)((unsigned long long)(ra - 1) & (unsigned long long)a.out_row_mask)] = h;
        } else {
          float q = rintf(y * inv * a.q_scale);
          q = fminf(fmaxf(q, -127.f), 127.f);
          reinterpret_cast<int8_t*>(a.out)[o] = (int8_t)q;
        }
        if (a.tm_out) tile[cl][r] = y;
      }
    }
  }
  if (a.tm_out) {
    __syncthreads();
    for (int r = warp; r < npts; r += kBpThreads / 32) {
      const int c = c0 + lane;
      if (c < a.nchan) a.tm_out[(r0 + r) * a.tm_row_stride + c] = tile[lane][r];
    }
  }
  if (err && a.d_err) atomicOr(a.d_err, err);
}

int launch_bandpass(const vfrb_bp_args& a, cudaStream_t s) {
  if (a.nrows <= 0) return a.nrows == 0 ? VFRB_OK : VFRB_ERR_ARG;
  if (a.out_shift1 && (a.storage != VFRB_F16 || a.out_row0 < 0 || ((uintptr_t)a.out_shift1 & 1))) return VFRB_ERR_ARG;
  if (!a.in || !a.out || a.nchan <= 0 || a.window <= 0 || a.window > kBpMaxWin) return VFRB_ERR_ARG;
  if (a.storage != VFRB_F32 && !a.inv_scale) return VFRB_ERR_ARG;
  if (a.subtract_mode != 0 && a.subtract_mode != 1) return VFRB_ERR_ARG;
  const int nwin = (a.nrows + a.window - 1) / a.window;
  dim3 grid((a.nchan + kBpChan - 1) / kBpChan, nwin);
  switch (a.storage) {
    case VFRB_F32: k_bandpass<VFRB_F32><<<grid, kBpThreads, 0, s>>>(a, nullptr); break;
    case VFRB_F16: k_bandpass<VFRB_F16><<<grid, kBpThreads, 0, s>>>(a, static_cast<__half*>(a.out_shift1)); break;
    case VFRB_I8: k_bandpass<VFRB_I8><<<grid, kBpThreads, 0, s>>>(a, nullptr); break;
    default: return VFRB_ERR_ARG;
  }
  return cuda_status(cudaGetLastError());
}

// ---- K4: per-channel statistics (STATS:910-946) ---------------------------
// One warp per (channel, statistics block); the block's rows are contiguous
// in the channel-major layout.  FP64 mean and variance; the outlier count
// uses the reference's float comparison x > ave + 5*sig and stores the
// integer quotient count/npts.
__global__ void __launch_bounds__(256) k_chan_stats(const vfrb_cs_args a) {
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (gw >= (long long)a.nchan * a.nstatblks) return;
  const int c = (int)(gw % a.nchan);
  const int k = (int)(gw / a.nchan);
  const long long colmin = (long long)a.ncolstatblk * k;
  long long colmax = colmin + a.ncolstatblk;
  if (colmax > a.nrows) colmax = a.nrows;
  const int npts = (int)(colmax - colmin);
  const float* base = a.fb + (long long)c * a.chan_stride;
  auto at = [&](long long r) {
    return base[(unsigned long long)(a.row0 + r) & (unsigned long long)a.row_mask];
  };
  double s = 0.0;
  for (long long r = colmin + lane; r < colmax; r += 32) s += (double)at(r);
  const double n = (double)npts;
  const double ave = warp_sum(s) / n;
  double sd = 0.0, sd2 = 0.0;
  for (long long r = colmin + lane; r < colmax; r += 32) {
    const double d = (double)at(r) - ave;
    sd += d;
    sd2 += d * d;
  }
  sd = warp_sum(sd);
  sd2 = warp_sum(sd2);
  const double sig = (sd2 - sd * sd / n) / (n - 1.0);
  const double hi = ave + 5.0 * sig;
  int cnt = 0;
  for (long long r = colmin + lane; r < colmax; r += 32) cnt += ((double)at(r) > hi) ? 1 : 0;
  cnt = warp_sum_i(cnt);
  if (lane == 0) {
    const long long o = (long long)k * a.nchan + c;
    a.ave[o] = (float)ave;
    a.sig[o] = (float)sig;
    a.outlier[o] = (float)(npts > 0 ? cnt / npts : 0);
  }
}

int launch_chan_stats(const vfrb_cs_args& a, cudaStream_t s) {
  if (!a.fb || !a.ave || !a.sig || !a.outlier || a.nchan <= 0 || a.nstatblks <= 0 || a.ncolstatblk <= 1)
    return VFRB_ERR_ARG;
  if ((long long)a.ncolstatblk * (a.nstatblks - 1) >= a.nrows) return VFRB_ERR_ARG;
  const long long nw = (long long)a.nchan * a.nstatblks;
  k_chan_stats<<<(unsigned)((nw + 7) / 8), 256, 0, s>>>(a);
  return cuda_status(cudaGetLastError());
}

// ---- spectral kurtosis per (channel, statistics block) ----------------------
// Generalised SK estimator (Nita & Gary 2010) of the raw (not bandpass-
// subtracted) power: with M rows in the block, S1 = sum x, S2 = sum x^2 and
// nsum = N*d raw power values per FB sample (2 pols x NAVE spectra, each an
// exponential variable for Gaussian noise),
//   SK = (M*nsum + 1)/(M - 1) * (M*S2/S1^2 - 1),
// whose expectation is 1 for Gaussian noise; narrowband RFI drives it below 1
// (steady tones) or far above it (bursts); a one-row block gives inf/NaN as
// M - 1 = 0.  FP64 sums.  The FB is time-major,
// so a warp reads 32 consecutive channels of a row: 128-byte segments.
__global__ void __launch_bounds__(256) k_chan_sk(const float* __restrict__ fb, long long row_stride, long long row0,
                                                 unsigned long long row_mask, int nchan, int nrows, int ncolstatblk,
                                                 int nstatblks, double nsum, float* __restrict__ sk) {
  const int c = blockIdx.x * 256 + threadIdx.x;
  const int k = blockIdx.y;
  if (c >= nchan || k >= nstatblks) return;
  const long long r0 = (long long)ncolstatblk * k;
  const long long r1 = min(r0 + ncolstatblk, (long long)nrows);
  double s1 = 0.0, s2 = 0.0;
  for (long long r = r0; r < r1; ++r) {
    const double x = (double)fb[(long long)((unsigned long long)(row0 + r) & row_mask) * row_stride + c];
    s1 += x;
    s2 += x * x;
  }
  const double m = (double)(r1 - r0);
  const double v = (m * nsum + 1.0) / (m - 1.0) * (m * s2 / (s1 * s1) - 1.0);
  sk[(long long)k * nchan + c] = (float)v;
}

// rows r < nrows of the block start at ring row (row0 + r) & row_mask
// (row_mask ~0: a linear array)
int launch_chan_sk_ring(const float* fb_tm, long long row_stride, long long row0, unsigned long long row_mask,
                        int nchan, int nrows, int ncolstatblk, int nstatblks, int nsum, float* sk, cudaStream_t s) {
  if (!fb_tm || !sk || nchan <= 0 || nstatblks <= 0 || ncolstatblk <= 1 || nsum < 1 || row_stride < nchan ||
      (long long)nrows - (long long)ncolstatblk * (nstatblks - 1) < 1 || nstatblks > 65535 || row0 < 0)
    return VFRB_ERR_ARG;
  dim3 grid((unsigned)((nchan + 255) / 256), (unsigned)nstatblks);
  k_chan_sk<<<grid, 256, 0, s>>>(fb_tm, row_stride, row0, row_mask, nchan, nrows, ncolstatblk, nstatblks,
                                 (double)nsum, sk);
  return cuda_status(cudaGetLastError());
}

int launch_chan_sk(const float* fb_tm, long long row_stride, int nchan, int nrows, int ncolstatblk, int nstatblks,
                   int nsum, float* sk, cudaStream_t s) {
  return launch_chan_sk_ring(fb_tm, row_stride, 0, ~0ULL, nchan, nrows, ncolstatblk, nstatblks, nsum, sk, s);
}

// ---- channel-major -> time-major copy ---------------------------------------
__global__ void __launch_bounds__(256) k_transpose(const float* __restrict__ src, long long chan_stride,
                                                   unsigned row_mask, long long row0, int nchan, int nrows,
                                                   float* __restrict__ dst, long long dst_row_stride) {
  __shared__ float t[32][33];
  const int cb = blockIdx.x * 32, rb = blockIdx.y * 32;
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
  for (int i = ly; i < 32; i += 8) {
    const int c = cb + i, r = rb + lx;
    t[i][lx] = (c < nchan && r < nrows)
                   ? src[(long long)c * chan_stride +
                         (long long)((unsigned long long)(row0 + r) & (unsigned long long)row_mask)]
                   : 0.f;
  }
  __syncthreads();
  for (int i = ly; i < 32; i += 8) {
    const int r = rb + i, c = cb + lx;
    if (c < nchan && r < nrows) dst[(long long)r * dst_row_stride + c] = t[lx][i];
  }
}

int launch_fb_transpose(const float* src_cm, long long chan_stride, unsigned row_mask, long long row0, int nchan,
                        int nrows, float* dst_tm, long long dst_row_stride, cudaStream_t s) {
  if (!src_cm || !dst_tm || nchan <= 0 || nrows < 0) return VFRB_ERR_ARG;
  if (nrows == 0) return VFRB_OK;
  dim3 grid((nchan + 31) / 32, (nrows + 31) / 32);
  k_transpose<<<grid, 256, 0, s>>>(src_cm, chan_stride, row_mask, row0, nchan, nrows, dst_tm, dst_row_stride);
  return cuda_status(cudaGetLastError());
}

}  // namespace vfrb
