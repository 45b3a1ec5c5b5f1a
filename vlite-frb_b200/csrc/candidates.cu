// Boxcar width search over dedispersed series (new-build extension of the
// reference's calcstats peak, PIPE:1337-1370, which has no width).
//
// Per DM trial: for widths w = 1, 2, 4, ..., max_width the window sums
// S_w(t) = sum_{i<w} x[t+i] (FP64 sliding sums, t = 0 .. nt-w) and
// snr_w(t) = (S_w(t) - w*ave) / (sigma*sqrt(w)) with the trial's calcstats
// ave and sigma, so width 1 is calcstats' peak.  The best (snr, start,
// width) is kept; ties go to the smaller width, then the earlier start.
//
// One CTA per trial; each thread slides over a contiguous stretch of the
// series (reads are L1/L2 resident: one series is a few kB to a few hundred
// kB), and the CTA reduces the per-thread bests.  The work is a few FP64
// adds per sample and width: negligible next to the dedispersion that
// produced the series.
#include "vfrb_common.cuh"

#include <cmath>

namespace vfrb {

constexpr int kBoxThreads = 256;

struct BoxBest {
  double snr;
  int t, w;
};

__device__ __forceinline__ bool box_better(const BoxBest& a, const BoxBest& b) {
  if (a.snr != b.snr) return a.snr > b.snr;
  if (a.w != b.w) return a.w < b.w;
  return a.t < b.t;
}

__global__ void __launch_bounds__(kBoxThreads) k_boxcar(const float* __restrict__ dd, long long nt, long long stride,
                                                         const float* __restrict__ ave, const float* __restrict__ sigma,
                                                         int max_width, float* __restrict__ snr_out,
                                                         int* __restrict__ t_out, int* __restrict__ w_out) {
  const int d = blockIdx.x;
  const float* x = dd + (long long)d * stride;
  const double a = (double)ave[d];
  const double s = (double)sigma[d];
  const long long per = (nt + kBoxThreads - 1) / kBoxThreads;
  const long long t_lo = (long long)threadIdx.x * per;
  BoxBest best{-INFINITY, 0x7fffffff, 0x7fffffff};
  for (int w = 1; w <= max_width && w <= nt; w *= 2) {
    const long long t_hi = min(t_lo + per, nt - w + 1);  // starts t in [t_lo, t_hi)
    if (t_lo >= t_hi) continue;
    const double inv = 1.0 / (s * sqrt((double)w));
    double S = 0.0;
    for (int i = 0; i < w; ++i) S += (double)x[t_lo + i];
    for (long long t = t_lo;; ++t) {
      const double v = (S - (double)w * a) * inv;
      if (v > best.snr) best = BoxBest{v, (int)t, w};
      if (t + 1 >= t_hi) break;
      S += (double)x[t + w] - (double)x[t];
    }
  }
  // CTA reduction with the tie rule
  __shared__ BoxBest red[kBoxThreads];
  red[threadIdx.x] = best;
  __syncthreads();
  for (int o = kBoxThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o && box_better(red[threadIdx.x + o], red[threadIdx.x])) red[threadIdx.x] = red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    snr_out[d] = (float)red[0].snr;
    t_out[d] = red[0].t;
    w_out[d] = red[0].w;
  }
}

int launch_boxcar(const float* dd, int ndm, long long nt, long long stride, const float* ave, const float* sigma,
                  int max_width, float* snr, int* t, int* w, cudaStream_t s) {
  if (!dd || !ave || !sigma || !snr || !t || !w || ndm < 1 || nt < 1 || stride < nt || max_width < 1)
    return VFRB_ERR_ARG;
  if (nt > 0x7fffffffLL) return VFRB_ERR_UNSUPPORTED;
  k_boxcar<<<ndm, kBoxThreads, 0, s>>>(dd, nt, stride, ave, sigma, max_width, snr, t, w);
  return cuda_status(cudaGetLastError());
}

}  // namespace vfrb

extern "C" int vfrb_boxcar(const float* dd, int ndm, int64_t nt, int64_t stride, const float* ave,
                           const float* sigma, int max_width, float* snr, int32_t* start, int32_t* width,
                           void* stream) {
  return vfrb::launch_boxcar(dd, ndm, nt, stride, ave, sigma, max_width, snr, start, width, (cudaStream_t)stream);
}
