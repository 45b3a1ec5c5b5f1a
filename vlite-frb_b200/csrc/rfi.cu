// Optional bandpass / zero-DM modes that the reference keeps as dead code
// (its calls are commented out), offered here for RFI-heavy data.  Both work
// in place on the channel-major FP32 filterbank fb[c * chan_stride + row].
//
//  * k_subtract_bp_full -- subtractbp (PIPE:1372-1424): one clipped mean per
//    channel over the whole block instead of per 128-row cal window.  Kept as
//    the reference computes it: the first mean divides the channel's sum by
//    NCHANOUT (the number of channels) rather than by the number of rows, the
//    variance ("sig") is taken about that value, the clip is the open interval
//    ave +- 3 sig, and an empty clip window divides by zero.
//  * k_subtract_zero -- subtractZERO (PIPE:1478-1515): per time row, the
//    clipped mean across channels (count floored at 1) is subtracted from
//    every channel, removing the zero-DM (undispersed) signal.
//
// Sums are FP64 (the reference sums sequentially in FP32).  Both kernels are
// HBM-bound: four passes over the data they touch.
#include "vfrb_common.cuh"

namespace vfrb {

__device__ __forceinline__ double rfi_wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// one CTA (256 threads) per channel
__global__ void __launch_bounds__(256) k_subtract_bp_full(float* __restrict__ fb, long long chan_stride, long long row0,
                                                          unsigned row_mask, int nchan, long long nrows) {
  __shared__ double red[8];
  __shared__ double bc;
  const int c = blockIdx.x;
  float* x = fb + (long long)c * chan_stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  auto at = [&](long long t) -> float& { return x[(unsigned long long)(row0 + t) & (unsigned long long)row_mask]; };
  auto block_sum = [&](double v) -> double {
    v = rfi_wsum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += red[w];
      bc = t;
    }
    __syncthreads();
    return bc;
  };
  double s = 0.0;
  for (long long t = threadIdx.x; t < nrows; t += 256) s += (double)at(t);
  const double ave = block_sum(s) / (double)nchan;  // the reference divides by NCHANOUT
  double d1 = 0.0, d2 = 0.0;
  for (long long t = threadIdx.x; t < nrows; t += 256) {
    const double d = (double)at(t) - ave;
    d1 += d;
    d2 += d * d;
  }
  const double sum = block_sum(d1);
  const double sum2 = block_sum(d2);
  const double n = (double)nrows;
  const double sig = (sum2 - sum * sum / n) / (n - 1.0);
  const double hi = ave + 3.0 * sig, lo = ave - 3.0 * sig;
  double cs = 0.0, cn = 0.0;
  for (long long t = threadIdx.x; t < nrows; t += 256) {
    const double v = (double)at(t);
    if (v < hi && v > lo) {
      cs += v;
      cn += 1.0;
    }
  }
  const double csum = block_sum(cs);
  const double cnt = block_sum(cn);
  const float m = (float)(csum / cnt);  // cnt == 0 gives NaN, as the reference's ave/=i
  for (long long t = threadIdx.x; t < nrows; t += 256) at(t) -= m;
}

// one thread per row; a warp covers 32 consecutive rows, so every channel's
// load is one 128-byte segment
__global__ void __launch_bounds__(256) k_subtract_zero(float* __restrict__ fb, long long chan_stride, long long row0,
                                                       unsigned row_mask, int nchan, long long nrows) {
  const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
  if (t >= nrows) return;
  float* x = fb + ((unsigned long long)(row0 + t) & (unsigned long long)row_mask);
  double s = 0.0;
  for (int c = 0; c < nchan; ++c) s += (double)x[(long long)c * chan_stride];
  const double ave = s / (double)nchan;
  double d1 = 0.0, d2 = 0.0;
  for (int c = 0; c < nchan; ++c) {
    const double d = (double)x[(long long)c * chan_stride] - ave;
    d1 += d;
    d2 += d * d;
  }
  const double n = (double)nchan;
  const double sig = (d2 - d1 * d1 / n) / (n - 1.0);
  const double hi = ave + 3.0 * sig, lo = ave - 3.0 * sig;
  double cs = 0.0;
  int cnt = 0;
  for (int c = 0; c < nchan; ++c) {
    const double v = (double)x[(long long)c * chan_stride];
    if (v < hi && v > lo) {
      cs += v;
      ++cnt;
    }
  }
  const float m = (float)(cs / (double)(cnt > 0 ? cnt : 1));
  for (int c = 0; c < nchan; ++c) x[(long long)c * chan_stride] -= m;
}

// rows [row0, row0 + nrows) of every channel must lie in its chan_stride
// elements: a power-of-two ring (row_mask + 1 <= chan_stride) or a linear run
static bool rfi_args_ok(const float* fb, long long chan_stride, long long row0, unsigned row_mask, int nchan,
                        long long nrows) {
  if (!fb || nchan < 2 || nrows < 2 || chan_stride < 1) return false;
  if (row_mask != 0xffffffffu) {
    const unsigned long long r = (unsigned long long)row_mask + 1ULL;
    if ((r & (r - 1)) != 0 || (long long)r < nrows || chan_stride < (long long)r) return false;
  } else if (row0 < 0 || row0 + nrows > chan_stride) {
    return false;
  }
  return true;
}

int launch_subtract_bp_full(float* fb, long long chan_stride, long long row0, unsigned row_mask, int nchan,
                            long long nrows, cudaStream_t s) {
  if (!rfi_args_ok(fb, chan_stride, row0, row_mask, nchan, nrows)) return VFRB_ERR_ARG;
  k_subtract_bp_full<<<nchan, 256, 0, s>>>(fb, chan_stride, row0, row_mask, nchan, nrows);
  return cuda_status(cudaGetLastError());
}

int launch_subtract_zero(float* fb, long long chan_stride, long long row0, unsigned row_mask, int nchan,
                         long long nrows, cudaStream_t s) {
  if (!rfi_args_ok(fb, chan_stride, row0, row_mask, nchan, nrows)) return VFRB_ERR_ARG;
  const long long nb = (nrows + 255) / 256;
  if (nb > 0x7fffffffLL) return VFRB_ERR_UNSUPPORTED;
  k_subtract_zero<<<(unsigned)nb, 256, 0, s>>>(fb, chan_stride, row0, row_mask, nchan, nrows);
  return cuda_status(cudaGetLastError());
}

}  // namespace vfrb

extern "C" int vfrb_subtract_bp_full(float* fb_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask, int nchan,
                                     int64_t nrows, void* stream) {
  return vfrb::launch_subtract_bp_full(fb_cm, chan_stride, row0, row_mask, nchan, nrows, (cudaStream_t)stream);
}

extern "C" int vfrb_subtract_zero(float* fb_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask, int nchan,
                                  int64_t nrows, void* stream) {
  return vfrb::launch_subtract_zero(fb_cm, chan_stride, row0, row_mask, nchan, nrows, (cudaStream_t)stream);
}
