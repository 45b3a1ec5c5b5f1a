// K3: brute-force incoherent dedispersion + fused per-DM statistics (sm_100a).
//
// Replaces dedisp_execute (PIPE:671) by the reference's in-tree sum
// (PIPE:1517-1537) and fuses calcstats (PIPE:1337-1370); the SIGMA variant
// is dedisperseSTATS (TS:1450-1481).
//
// Tiling: a CTA owns a block of 16 DM trials x 256 output samples.  For each
// chunk of channels it stages, per channel, the contiguous run of rows that
// any of its 16 DMs touches (256 + the chunk's delay spread) from the
// channel-major filterbank into shared memory with 16-byte vector loads; the
// 16 trials then all read their shifted windows from that one copy (reuse
// across neighbouring DM trials).  Lanes run along time, so every shared
// memory read of a warp is 32 consecutive elements (conflict free) and the
// per-channel delay is warp-uniform.  Accumulation is FP32 in registers; the
// FP16 / int8 forms apply the per-channel weight with an FMA.
#include "vfrb_common.cuh"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

namespace vfrb {

constexpr int kDdThreads = 256;
constexpr int kDdDm = 16;          // DM trials per CTA
constexpr int kDdDmPerWarp = kDdDm / (kDdThreads / 32);
constexpr int kDdPerLane = 8;      // output samples per lane
constexpr int kDdNt = 32 * kDdPerLane;  // 256 output samples per CTA
constexpr int kDdSmemBudget = 96 * 1024;
constexpr int kDdMaxChunk = 32;

struct DmPartial {
  double s, s2;
  float mx;
  int arg;
};

struct DdKParams {
  const void* fb;
  const float* chan_scale;
  float uniform_scale;  // weight of every channel when chan_scale is NULL (F16/I8)
  long long chan_stride;
  long long row0;
  unsigned row_mask;
  long long nrows_valid;
  int nchan;
  const int* off;
  int ndm;
  long long nt_out;
  float* out;
  long long out_stride;
  float* sig_out;
  DmPartial* part;
  int chunk;
  int lmax;
  int* err;
};

template <typename T> struct Vec;
template <> struct Vec<float> { static constexpr int n = 4; };
template <> struct Vec<__half> { static constexpr int n = 8; };
template <> struct Vec<int8_t> { static constexpr int n = 16; };

template <typename T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f<int8_t>(int8_t v) { return (float)v; }

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T, bool SIGMA>
__global__ void __launch_bounds__(kDdThreads) k_dedisperse(const DdKParams p) {
  constexpr int VEC = Vec<T>::n;
  extern __shared__ float4 sm4[];
  const int CH = p.chunk;
  int* s_off = reinterpret_cast<int*>(sm4);            // [kDdDm][CH]
  long long* s_abs = reinterpret_cast<long long*>(s_off + kDdDm * CH);  // [CH] first staged row (8-byte aligned: 16*CH ints)
  float* s_w = reinterpret_cast<float*>(s_abs + CH);    // [CH]
  T* tile = reinterpret_cast<T*>(sm4 + ((kDdDm * CH * 4 + CH * 8 + CH * 4 + 8 * 4 + 15) / 16));

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long t0 = (long long)blockIdx.x * kDdNt;
  const int d0 = blockIdx.y * kDdDm;
  const T* fb = reinterpret_cast<const T*>(p.fb);
  int err = 0;

  float acc[kDdDmPerWarp][kDdPerLane];
  float acc2[SIGMA ? kDdDmPerWarp : 1][SIGMA ? kDdPerLane : 1];
#pragma unroll
  for (int j = 0; j < kDdDmPerWarp; ++j)
#pragma unroll
    for (int k = 0; k < kDdPerLane; ++k) {
      acc[j][k] = 0.f;
      if (SIGMA) acc2[j][k] = 0.f;
    }

  for (int c0 = 0; c0 < p.nchan; c0 += CH) {
    const int nc = min(CH, p.nchan - c0);
    for (int i = tid; i < kDdDm * CH; i += kDdThreads) {
      const int dl = i / CH, cl = i - dl * CH;
      const int d = min(d0 + dl, p.ndm - 1);
      s_off[i] = (cl < nc) ? __ldg(p.off + (long long)d * p.nchan + c0 + cl) : 0;
    }
    __syncthreads();
    for (int cl = tid; cl < CH; cl += kDdThreads) {
      int mn = 0x7fffffff, mx = -0x7fffffff;
#pragma unroll
      for (int dl = 0; dl < kDdDm; ++dl) {
        const int o = s_off[dl * CH + cl];
        mn = min(mn, o);
        mx = max(mx, o);
      }
      const long long a0 = (p.row0 + t0 + mn) & ~(long long)(VEC - 1);
      if (p.row0 + t0 + mx + kDdNt - a0 > p.lmax) err |= kErrOffsetRange;
      s_abs[cl] = a0;
      s_w[cl] = (p.chan_scale && cl < nc) ? p.chan_scale[c0 + cl] : p.uniform_scale;
    }
    __syncthreads();
    // stage rows [s_abs, s_abs + lmax) of each channel of the chunk
    const int nvec = p.lmax / VEC;
    for (int cl = warp; cl < nc; cl += kDdThreads / 32) {
      const T* src = fb + (long long)(c0 + cl) * p.chan_stride;
      const long long a0 = s_abs[cl];
      uint4* dst = reinterpret_cast<uint4*>(tile + (long long)cl * p.lmax);
      for (int v = lane; v < nvec; v += 32) {
        const long long r = a0 + (long long)v * VEC;  // absolute (unmasked) row
        uint4 val = make_uint4(0, 0, 0, 0);
        if (r >= p.row0 && r + VEC <= p.row0 + p.nrows_valid) {
          const unsigned long long rr = (unsigned long long)r & (unsigned long long)p.row_mask;
          val = __ldg(reinterpret_cast<const uint4*>(src + rr));
        } else if (r + VEC > p.row0 && r < p.row0 + p.nrows_valid) {
          // partially valid vector at the edge of the valid rows
          union {
            uint4 u;
            T t[VEC];
          } tmp;
          tmp.u = make_uint4(0, 0, 0, 0);
#pragma unroll
          for (int e = 0; e < VEC; ++e) {
            const long long re = r + e;
            if (re >= p.row0 && re < p.row0 + p.nrows_valid)
              tmp.t[e] = src[(unsigned long long)re & (unsigned long long)p.row_mask];
          }
          val = tmp.u;
        }
        dst[v] = val;
      }
    }
    __syncthreads();
#pragma unroll 2
    for (int cl = 0; cl < nc; ++cl) {
      const T* trow = tile + (long long)cl * p.lmax;
      const float wc = s_w[cl];
#pragma unroll
      for (int j = 0; j < kDdDmPerWarp; ++j) {
        const int dl = warp * kDdDmPerWarp + j;
        int o = (int)(p.row0 + t0 + s_off[dl * CH + cl] - s_abs[cl]);
        o = min(max(o, 0), p.lmax - kDdNt) + lane;  // never leaves the tile, even for a bad table
#pragma unroll
        for (int k = 0; k < kDdPerLane; ++k) {
          const float v = to_f<T>(trow[o + 32 * k]);
          if (sizeof(T) == 4) {
            acc[j][k] += v;
          } else {
            acc[j][k] = fmaf(wc, v, acc[j][k]);
          }
          if (SIGMA) acc2[j][k] = fmaf(v, v, acc2[j][k]);
        }
      }
    }
    __syncthreads();
  }

  // epilogue: out = sum / NCHANOUT (PIPE:1534), and calcstats partials
  const float fn = (float)p.nchan;
#pragma unroll
  for (int j = 0; j < kDdDmPerWarp; ++j) {
    const int d = d0 + warp * kDdDmPerWarp + j;
    if (d >= p.ndm) continue;  // warp-uniform
    double s = 0.0, s2 = 0.0;
    float mx = -INFINITY;
    int arg = 0x7fffffff;
#pragma unroll
    for (int k = 0; k < kDdPerLane; ++k) {
      const long long t = t0 + lane + 32 * k;
      if (t < p.nt_out) {
        const float val = acc[j][k] / fn;
        p.out[(long long)d * p.out_stride + t] = val;
        if (SIGMA) {
          // sigma = sqrt((sum d^2 - (sum d)^2) / (N (N-1))), d = x - mean (TS:1468-1477)
          const double n = (double)p.nchan;
          const double sx = (double)acc[j][k], sxx = (double)acc2[j][k];
          double var = (sxx - sx * sx / n) / (n * (n - 1.0));
          p.sig_out[(long long)d * p.out_stride + t] = (float)sqrt(var > 0.0 ? var : 0.0);
        }
        s += (double)val;
        s2 += (double)val * (double)val;
        if (val > mx) {
          mx = val;
          arg = (int)t;
        }
      }
    }
    s = wsum(s);
    s2 = wsum(s2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float omx = __shfl_xor_sync(0xffffffffu, mx, o);
      const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
      if (omx > mx || (omx == mx && oarg < arg)) {
        mx = omx;
        arg = oarg;
      }
    }
    if (lane == 0 && p.part) {
      DmPartial q;
      q.s = s;
      q.s2 = s2;
      q.mx = mx;
      q.arg = arg;
      p.part[(long long)blockIdx.x * p.ndm + d] = q;
    }
  }
  if (err && p.err) atomicOr(p.err, err);
}

// calcstats from FP64 sums (PIPE:1337-1370): FP64 mean, corrected two-pass
// variance, both stored as float; peak = max(0, (max x - ave)/sigma) in float.
__device__ __forceinline__ void dm_finalize(int d, long long nt_out, double s, double s2, float mx, int arg,
                                            float* ave, float* sigma, float* peak, int* frb, int* argmax) {
  const double n = (double)nt_out;
  const double tave = s / n;
  const double tsig = (s2 - s * s / n) / (n - 1.0);  // == the reference's corrected two-pass form
  const float ave_f = (float)tave;
  const float sig_f = (float)sqrt(tsig);
  // max_t (x - ave)/sigma in float equals f(max_t x): the map is monotone.
  const float snr = (mx - ave_f) / sig_f;
  if (ave) ave[d] = ave_f;
  if (sigma) sigma[d] = sig_f;
  if (peak) peak[d] = (snr > 0.f) ? snr : 0.f;
  if (frb) frb[d] = (snr > 3.0f) ? 1 : 0;
  if (argmax) argmax[d] = arg;
}

// calcstats finalize: one warp per DM reduces the time-block partials.
__global__ void __launch_bounds__(256) k_dm_stats(const DmPartial* __restrict__ part, int ntb, int ndm,
                                                  long long nt_out, float* ave, float* sigma, float* peak,
                                                  int* frb, int* argmax) {
  const int lane = threadIdx.x & 31;
  const int d = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (d >= ndm) return;
  double s = 0.0, s2 = 0.0;
  float mx = -INFINITY;
  int arg = 0x7fffffff;
  for (int b = lane; b < ntb; b += 32) {
    const DmPartial q = part[(long long)b * ndm + d];
    s += q.s;
    s2 += q.s2;
    if (q.mx > mx || (q.mx == mx && q.arg < arg)) {
      mx = q.mx;
      arg = q.arg;
    }
  }
  s = wsum(s);
  s2 = wsum(s2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float omx = __shfl_xor_sync(0xffffffffu, mx, o);
    const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
    if (omx > mx || (omx == mx && oarg < arg)) {
      mx = omx;
      arg = oarg;
    }
  }
  if (lane != 0) return;
  dm_finalize(d, nt_out, s, s2, mx, arg, ave, sigma, peak, frb, argmax);
}

// calcstats of whole series: one warp per DM over dd[d][0..nt) (stream mode,
// where one dedispersion launch may cover several output chunks).
__global__ void __launch_bounds__(256) k_series_stats(const float* __restrict__ dd, long long nt, long long stride,
                                                      int ndm, float* ave, float* sigma, float* peak, int* frb,
                                                      int* argmax) {
  const int lane = threadIdx.x & 31;
  const int d = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (d >= ndm) return;
  const float* x = dd + (long long)d * stride;
  double s = 0.0, s2 = 0.0;
  float mx = -INFINITY;
  int arg = 0x7fffffff;
  for (long long t = lane; t < nt; t += 32) {
    const float v = x[t];
    s += (double)v;
    s2 += (double)v * (double)v;
    if (v > mx) {  // t grows: the first maximum is kept
      mx = v;
      arg = (int)t;
    }
  }
  s = wsum(s);
  s2 = wsum(s2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float omx = __shfl_xor_sync(0xffffffffu, mx, o);
    const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
    if (omx > mx || (omx == mx && oarg < arg)) {
      mx = omx;
      arg = oarg;
    }
  }
  if (lane != 0) return;
  dm_finalize(d, nt, s, s2, mx, arg, ave, sigma, peak, frb, argmax);
}

int launch_series_stats(const float* dd, int ndm, long long nt, long long stride, float* ave, float* sigma,
                        float* peak, int* frb, int* argmax, cudaStream_t s) {
  if (!dd || ndm < 1 || nt < 2 || stride < nt || nt > 0x7fffffffLL) return VFRB_ERR_ARG;
  k_series_stats<<<(ndm + 7) / 8, 256, 0, s>>>(dd, nt, stride, ndm, ave, sigma, peak, frb, argmax);
  return cuda_status(cudaGetLastError());
}

// Fallback for delay spreads too wide to stage: direct loads, one thread per
// output sample (lanes along time keep the loads coalesced).
template <typename T, bool SIGMA>
__global__ void __launch_bounds__(256) k_dedisperse_direct(const DdKParams p) {
  const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
  const int d = blockIdx.y;
  const T* fb = reinterpret_cast<const T*>(p.fb);
  float acc = 0.f, acc2 = 0.f;
  int err = 0;
  if (t < p.nt_out) {
    for (int c = 0; c < p.nchan; ++c) {
      const int o = __ldg(p.off + (long long)d * p.nchan + c);
      if (t + o >= p.nrows_valid || o < 0) {
        err |= kErrOffsetRange;
        continue;
      }
      const unsigned long long rr = (unsigned long long)(p.row0 + t + o) & (unsigned long long)p.row_mask;
      const float v = to_f<T>(fb[(long long)c * p.chan_stride + rr]);
      if (sizeof(T) == 4) acc += v;
      else acc = fmaf(p.chan_scale ? p.chan_scale[c] : p.uniform_scale, v, acc);
      if (SIGMA) acc2 = fmaf(v, v, acc2);
    }
    const float val = acc / (float)p.nchan;
    p.out[(long long)d * p.out_stride + t] = val;
    if (SIGMA) {
      const double n = (double)p.nchan;
      double var = ((double)acc2 - (double)acc * (double)acc / n) / (n * (n - 1.0));
      p.sig_out[(long long)d * p.out_stride + t] = (float)sqrt(var > 0.0 ? var : 0.0);
    }
  }
  // per-(DM, 256-sample block) partials
  const float val = (t < p.nt_out) ? acc / (float)p.nchan : -INFINITY;
  double s = (t < p.nt_out) ? (double)val : 0.0, s2 = s * s;
  float mx = val;
  int arg = (t < p.nt_out) ? (int)t : 0x7fffffff;
  __shared__ double ss[8], ss2[8];
  __shared__ float smx[8];
  __shared__ int sarg[8];
  s = wsum(s);
  s2 = wsum(s2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float omx = __shfl_xor_sync(0xffffffffu, mx, o);
    const int oarg = __shfl_xor_sync(0xffffffffu, arg, o);
    if (omx > mx || (omx == mx && oarg < arg)) {
      mx = omx;
      arg = oarg;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    ss[warp] = s;
    ss2[warp] = s2;
    smx[warp] = mx;
    sarg[warp] = arg;
  }
  __syncthreads();
  if (threadIdx.x == 0 && p.part) {
    DmPartial q{0.0, 0.0, -INFINITY, 0x7fffffff};
    for (int w = 0; w < 8; ++w) {
      q.s += ss[w];
      q.s2 += ss2[w];
      if (smx[w] > q.mx || (smx[w] == q.mx && sarg[w] < q.arg)) {
        q.mx = smx[w];
        q.arg = sarg[w];
      }
    }
    p.part[(long long)blockIdx.x * p.ndm + d] = q;
  }
  if (err && p.err) atomicOr(p.err, err);
}

}  // namespace vfrb

#include "dedisperse_reg.cuh"
#include "dedisperse_pat.cuh"


// ---- plan object --------------------------------------------------------------
namespace vfrb {
// Register-window grouping for one group size D: per (group, channel) the
// group's smallest delay and the D delay differences (8 bits each), and per
// CTA block of kRegWarps groups the smallest delay (tile start).
struct RegGroup {
  int D = 0;
  int smax = 0;  // largest in-group delay difference
  int span = 0;  // largest (max - min) delay over a CTA block's trials
  int ngroups = 0, nblocks = 0;
  int* d_gbase = nullptr;
  unsigned* d_gpack = nullptr;
  int* d_bmin = nullptr;
  int bmin_mid_max = 0;             // max over CTA blocks of bmin at the middle channel
  // the same three for CTAs of 16 warps (16*D trials), used by the pattern kernel's
  // one-CTA-per-SM form
  int nblocks16 = 0, span_16w = 0, bmin_mid_max16 = 0;
  int* d_bmin16 = nullptr;
  unsigned char* d_gpat = nullptr;  // pattern id per (group, channel), D = 4 and 2
  long long n_generic = 0;          // (group, channel) pairs outside the pattern table
};
}  // namespace vfrb

struct vfrb_ddplan {
  int ndm = 0, nchan = 0;
  int max_delay = 0;  // max over the table
  int span16 = 0;     // max over 16-trial blocks and channels of (max - min) delay
  int* d_off = nullptr;
  vfrb::RegGroup reg[3];            // D = 4, 2, 1 when applicable
  int variant[3] = {0, 0, 0};       // chosen variant per storage form (VFRB_DD_*)
};

namespace vfrb {

static const RegGroup* find_group(const vfrb_ddplan* pl, int D) {
  for (const auto& g : pl->reg)
    if (g.D == D) return &g;
  return nullptr;
}

size_t dedisperse_workspace_bytes_plan(const vfrb_ddplan* pl, long long nt_out) {
  const long long ntb = (nt_out + kDdNt - 1) / kDdNt;  // every kernel's time block is >= 256 samples
  return (size_t)ntb * (size_t)pl->ndm * sizeof(DmPartial);
}

static int dd_lmax(const vfrb_ddplan* pl, int vec) {
  const int need = kDdNt + pl->span16 + vec;  // + alignment slack
  return (need + 15) & ~15;
}

// staged (v1) or direct kernel; returns the number of time blocks in *ntb
template <typename T, bool SIGMA>
static int dd_launch_t(const vfrb_ddplan* pl, const vfrb_dd_args& a, DdKParams& k, cudaStream_t s, bool allow_staged,
                       int* ntb) {
  constexpr int VEC = Vec<T>::n;
  const int lmax = dd_lmax(pl, VEC);
  const size_t fixed = ((size_t)kDdDm * kDdMaxChunk * 4 + kDdMaxChunk * 8 + kDdMaxChunk * 4 + 8 * 4 + 15) / 16 * 16;
  int chunk = (int)((kDdSmemBudget - fixed) / ((size_t)lmax * sizeof(T)));
  chunk = std::min(chunk, kDdMaxChunk);
  const long long tb = (a.nt_out + kDdNt - 1) / kDdNt;
  const bool vec_ok = (a.chan_stride % VEC) == 0 && ((unsigned long long)a.row_mask + 1ULL) % VEC == 0 &&
                      ((uintptr_t)a.fb & 15) == 0;
  *ntb = (int)tb;
  if (allow_staged && chunk >= 4 && vec_ok) {
    k.chunk = chunk;
    k.lmax = lmax;
    const size_t smem = ((size_t)kDdDm * chunk * 4 + chunk * 8 + chunk * 4 + 8 * 4 + 15) / 16 * 16 +
                        (size_t)chunk * lmax * sizeof(T);
    cudaError_t e = cudaFuncSetAttribute(k_dedisperse<T, SIGMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return VFRB_ERR_CUDA;
    dim3 grid((unsigned)tb, (unsigned)((pl->ndm + kDdDm - 1) / kDdDm));
    k_dedisperse<T, SIGMA><<<grid, kDdThreads, smem, s>>>(k);
  } else {
    dim3 grid((unsigned)tb, (unsigned)pl->ndm);
    k_dedisperse_direct<T, SIGMA><<<grid, 256, 0, s>>>(k);
  }
  return cuda_status(cudaGetLastError());
}

template <typename T, int D, int TT, int SMAX>
static int reg_launch_t(const vfrb_ddplan* pl, const RegGroup& g, const vfrb_dd_args& a, DmPartial* part,
                        float out_scale, cudaStream_t s, int* ntb) {
  using Cfg = RegCfg<T, D, TT, SMAX>;
  constexpr int VEC = Cfg::VEC;
  *ntb = 0;
  if (g.D != D || g.smax > SMAX) return VFRB_OK;  // not applicable
  const int lm = (g.span + 2 * VEC + Cfg::NT + Cfg::NQ * VEC + 32 * VEC + VEC - 1) / VEC * VEC;
  const int per_ch = 2 * lm * (int)sizeof(T) + 2 * kRegWarps * 16;
  const int chunk = std::min(32, (int)(96 * 1024 / per_ch));
  if (chunk < 2) return VFRB_OK;
  DdRegParams k{};
  k.fb = a.fb;
  k.out_scale = out_scale;
  k.chan_stride = a.chan_stride;
  k.row0 = a.row0;
  k.row_mask = a.row_mask;
  k.nrows_valid = a.nrows_valid;
  k.nchan = pl->nchan;
  k.ndm = pl->ndm;
  k.ngroups = g.ngroups;
  k.nt_out = a.nt_out;
  k.out = a.out;
  k.out_stride = a.out_stride;
  k.part = part;
  k.gbase = g.d_gbase;
  k.gpack = g.d_gpack;
  k.bmin = g.d_bmin;
  k.chunk = chunk;
  k.lmax = lm;
  k.err = a.d_err;
  const size_t smem = (size_t)2 * kRegWarps * chunk * 16 + (size_t)2 * chunk * lm * sizeof(T);
  cudaError_t e = cudaFuncSetAttribute(k_dedisp_reg<T, D, TT, SMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return VFRB_ERR_CUDA;
  dim3 grid((unsigned)((a.nt_out + Cfg::NT - 1) / Cfg::NT), (unsigned)g.nblocks);
  k_dedisp_reg<T, D, TT, SMAX><<<grid, kRegWarps * 32, smem, s>>>(k);
  const int st = cuda_status(cudaGetLastError());
  if (st == VFRB_OK) *ntb = (int)grid.x;
  return st;
}

// Register-window variant `v` for this call; *ntb == 0 when it does not apply.
static int reg_launch(const vfrb_ddplan* pl, int v, const vfrb_dd_args& a, DmPartial* part, cudaStream_t s,
                      int* ntb) {
  *ntb = 0;
  if (((uintptr_t)a.fb & 15) != 0) return VFRB_OK;
  const int D = v == VFRB_DD_REG4 ? 4 : v == VFRB_DD_REG2 ? 2 : v == VFRB_DD_REG1 ? 1 : 0;
  const RegGroup* g = find_group(pl, D);
  if (!g) return VFRB_OK;
  if (a.storage == VFRB_F32) {
    if (a.chan_stride % 4 || ((unsigned long long)a.row_mask + 1ULL) % 4) return VFRB_OK;
    if (D == 4) return reg_launch_t<float, 4, 12, 20>(pl, *g, a, part, 1.f, s, ntb);
    if (D == 2) return reg_launch_t<float, 2, 20, 16>(pl, *g, a, part, 1.f, s, ntb);
    return reg_launch_t<float, 1, 20, 0>(pl, *g, a, part, 1.f, s, ntb);
  }
  if (a.storage == VFRB_F16) {
    // the mixed-precision add takes no per-channel weight: one scale for all channels
    if (a.chan_scale || !(a.uniform_scale > 0.f)) return VFRB_OK;
    if (a.chan_stride % 8 || ((unsigned long long)a.row_mask + 1ULL) % 8) return VFRB_OK;
    if (D == 4) return reg_launch_t<__half, 4, 8, 20>(pl, *g, a, part, a.uniform_scale, s, ntb);
    if (D == 2) return reg_launch_t<__half, 2, 24, 16>(pl, *g, a, part, a.uniform_scale, s, ntb);
    return reg_launch_t<__half, 1, 24, 0>(pl, *g, a, part, a.uniform_scale, s, ntb);
  }
  return VFRB_OK;
}

template <typename T, int D, int TT, int SMAX, int W, bool PAIR = false>
static int pat_launch_t(const vfrb_ddplan* pl, const RegGroup& g, const vfrb_dd_args& a, DmPartial* part,
                        float out_scale, cudaStream_t s, int* ntb, const DdJob* jobs = nullptr, int njobs = 0,
                        const void* fb1 = nullptr) {
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int NCOPY = PAIR ? 2 : 1;
  constexpr int NT = 32 * TT;
  *ntb = 0;
  if (g.D != D || g.smax > SMAX || !g.d_gpat) return VFRB_OK;  // not applicable
  // CTA blocks of W*D trials: the 8-warp tables, or the 16-warp ones
  const int span = W == 16 ? g.span_16w : g.span;
  const int nblocks = W == 16 ? g.nblocks16 : g.nblocks;
  const int* bmin = W == 16 ? g.d_bmin16 : g.d_bmin;
  const int mid_max = W == 16 ? g.bmin_mid_max16 : g.bmin_mid_max;
  if (!bmin) return VFRB_OK;
  const int lm = (span + VEC - 1 + NT + SMAX + VEC - 1) / VEC * VEC;
  // 8 warps: two CTAs per SM, each under ~110 KB of shared memory; 16 warps:
  // one CTA per SM with ~220 KB
  const int budget = (W == 16 ? 220 : 110) * 1024;
  const int per_ch = 2 * NCOPY * lm * (int)sizeof(T) + 3 * W * 4;
  const int chunk = std::min(32, (budget - W * 4 - 32) / per_ch);
  if (chunk < 4) return VFRB_OK;
  DdPatParams k{};
  k.fb = a.fb;
  k.fb1 = fb1;
  k.out_scale = out_scale;
  k.chan_stride = a.chan_stride;
  k.row0 = a.row0;
  k.row_mask = a.row_mask;
  k.nrows_valid = a.nrows_valid;
  k.nchan = pl->nchan;
  k.ndm = pl->ndm;
  k.ngroups = g.ngroups;
  k.nt_out = a.nt_out;
  k.out = a.out;
  k.out_stride = a.out_stride;
  k.part = part;
  k.gbase = g.d_gbase;
  k.gpack = g.d_gpack;
  k.gpat = g.d_gpat;
  k.bmin = bmin;
  k.chunk = chunk;
  k.lmax = lm;
  k.err = a.d_err;
  k.njobs = njobs;
  for (int i = 0; i < njobs; ++i) k.jobs[i] = jobs[i];
  const size_t meta = 16 + ((size_t)3 * W * chunk + W + 3) / 4 * 16;
  const size_t smem = meta + (size_t)2 * NCOPY * chunk * lm * sizeof(T);
  cudaError_t e = cudaFuncSetAttribute(k_dedisp_pat<T, D, TT, SMAX, W, PAIR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return VFRB_ERR_CUDA;
  const long long ntime = (a.nt_out + NT - 1) / NT;
  // grid y runs time blocks shifted by each DM block's delay at the middle
  // channel (see the kernel); the first and last rows hold empty CTAs
  const long long ny = ntime + mid_max / NT;
  if (ny > 65535) return VFRB_OK;
  dim3 grid((unsigned)nblocks, (unsigned)ny, (unsigned)std::max(1, njobs));
  k_dedisp_pat<T, D, TT, SMAX, W, PAIR><<<grid, W * 32, smem, s>>>(k);
  const int st = cuda_status(cudaGetLastError());
  if (st == VFRB_OK) *ntb = (int)ntime;
  return st;
}

// Pattern-run variant `v` for this call; *ntb == 0 when it does not apply.
// fb1 (FP16 only, or NULL): the ring shifted by one row, for the pair form.
static int pat_launch(const vfrb_ddplan* pl, int v, const vfrb_dd_args& a, DmPartial* part, cudaStream_t s,
                      int* ntb, const DdJob* jobs = nullptr, int njobs = 0, const void* fb1 = nullptr) {
  *ntb = 0;
  if (((uintptr_t)a.fb & 15) != 0) return VFRB_OK;
  const int D = v == VFRB_DD_PAT4 ? 4 : 2;
  const RegGroup* g = find_group(pl, D);
  if (!g) return VFRB_OK;
  if (a.storage == VFRB_F32) {
    if (a.chan_stride % 4 || ((unsigned long long)a.row_mask + 1ULL) % 4) return VFRB_OK;
    // FP32, four trials: 16-warp CTAs (one per SM) share each staged row
    // between twice as many trials (48.9 vs 55.2 ms at the 61,440-sample x
    // 2048-trial shape); FP16 tiles are half the size, and there the 8-warp
    // form is faster (47.7 vs 49.3 ms)
    if (D == 4) return pat_launch_t<float, 4, 15, VFRB_PAT4_SMAX, 16>(pl, *g, a, part, 1.f, s, ntb, jobs, njobs);
    return pat_launch_t<float, 2, 27, VFRB_PAT2_SMAX, 8>(pl, *g, a, part, 1.f, s, ntb, jobs, njobs);
  }
  if (a.storage == VFRB_F16) {
    if (a.chan_scale || !(a.uniform_scale > 0.f)) return VFRB_OK;
    if (a.chan_stride % 8 || ((unsigned long long)a.row_mask + 1ULL) % 8) return VFRB_OK;
    // with the shifted copy: the pair form (two staged copies per row, so the
    // 16-warp CTA's tiles are the FP32 form's size)
    if (D == 4 && fb1 && ((uintptr_t)fb1 & 15) == 0) {
      const int st = pat_launch_t<__half, 4, 14, VFRB_PAT4_SMAX, 16, true>(pl, *g, a, part, a.uniform_scale, s, ntb,
                                                                          jobs, njobs, fb1);
      if (st || *ntb) return st;  // else (tiles too large for the pair form) the plain FP16 form below
    }
    if (D == 4)
      return pat_launch_t<__half, 4, 14, VFRB_PAT4_SMAX, 8>(pl, *g, a, part, a.uniform_scale, s, ntb, jobs, njobs);
    return pat_launch_t<__half, 2, 26, VFRB_PAT2_SMAX, 8>(pl, *g, a, part, a.uniform_scale, s, ntb, jobs, njobs);
  }
  return VFRB_OK;
}

static int default_variant(const vfrb_ddplan* pl, int storage) {
  if (storage == VFRB_F32 || storage == VFRB_F16) {
    const RegGroup* g4 = find_group(pl, 4);
    const RegGroup* g2 = find_group(pl, 2);
    if (g4 && g4->d_gpat) return VFRB_DD_PAT4;
    if (g2 && g2->d_gpat) return VFRB_DD_PAT2;
  }
  if (storage == VFRB_F32) {
    if (find_group(pl, 4)) return VFRB_DD_REG4;
    if (find_group(pl, 2)) return VFRB_DD_REG2;
    if (find_group(pl, 1)) return VFRB_DD_REG1;
  } else if (storage == VFRB_F16) {
    if (find_group(pl, 2)) return VFRB_DD_REG2;
    if (find_group(pl, 4)) return VFRB_DD_REG4;
    if (find_group(pl, 1)) return VFRB_DD_REG1;
  }
  return VFRB_DD_STAGED;
}

static int launch_variant(const vfrb_ddplan* pl, int v, const vfrb_dd_args& a, cudaStream_t s,
                          const void* fb1 = nullptr) {
  const bool want_stats = a.ave || a.sigma || a.peak || a.frb || a.argmax;
  DdKParams k{};
  k.fb = a.fb;
  k.chan_scale = a.chan_scale;
  k.uniform_scale = a.uniform_scale > 0.f ? a.uniform_scale : 1.f;
  k.chan_stride = a.chan_stride;
  k.row0 = a.row0;
  k.row_mask = a.row_mask;
  k.nrows_valid = a.nrows_valid;
  k.nchan = pl->nchan;
  k.off = pl->d_off;
  k.ndm = pl->ndm;
  k.nt_out = a.nt_out;
  k.out = a.out;
  k.out_stride = a.out_stride;
  k.sig_out = a.sigma_out;
  k.part = want_stats ? reinterpret_cast<DmPartial*>(a.workspace) : nullptr;
  k.err = a.d_err;
  int ntb = 0, st = VFRB_OK;
  if (!a.sigma_out && (v == VFRB_DD_REG1 || v == VFRB_DD_REG2 || v == VFRB_DD_REG4))
    st = reg_launch(pl, v, a, k.part, s, &ntb);
  if (!a.sigma_out && (v == VFRB_DD_PAT4 || v == VFRB_DD_PAT2))
    st = pat_launch(pl, v, a, k.part, s, &ntb, nullptr, 0, a.storage == VFRB_F16 ? fb1 : nullptr);
  if (st) return st;
  if (ntb == 0) {
    const bool staged = v != VFRB_DD_DIRECT;
    if (a.sigma_out) {
      st = dd_launch_t<float, true>(pl, a, k, s, staged, &ntb);
    } else {
      switch (a.storage) {
        case VFRB_F32: st = dd_launch_t<float, false>(pl, a, k, s, staged, &ntb); break;
        case VFRB_F16: st = dd_launch_t<__half, false>(pl, a, k, s, staged, &ntb); break;
        case VFRB_I8: st = dd_launch_t<int8_t, false>(pl, a, k, s, staged, &ntb); break;
        default: return VFRB_ERR_ARG;
      }
    }
    if (st) return st;
  }
  if (!want_stats) return VFRB_OK;
  k_dm_stats<<<(pl->ndm + 7) / 8, 256, 0, s>>>(k.part, ntb, pl->ndm, a.nt_out, a.ave, a.sigma, a.peak, a.frb,
                                               a.argmax);
  return cuda_status(cudaGetLastError());
}

int launch_dedisperse_plan(const vfrb_ddplan* pl, const vfrb_dd_args& a, cudaStream_t s) {
  if (!pl || !a.fb || !a.out) return VFRB_ERR_ARG;
  if (a.nt_out <= 0) return a.nt_out == 0 ? VFRB_OK : VFRB_ERR_ARG;
  if (a.nrows_valid < a.nt_out + pl->max_delay) return VFRB_ERR_ARG;
  if (a.storage != VFRB_F32 && !a.chan_scale && !(a.uniform_scale > 0.f)) return VFRB_ERR_ARG;
  if (a.storage < VFRB_F32 || a.storage > VFRB_I8) return VFRB_ERR_ARG;
  if (a.sigma_out && a.storage != VFRB_F32) return VFRB_ERR_UNSUPPORTED;
  if ((unsigned long long)a.row_mask != 0xffffffffULL) {
    const unsigned long long r = (unsigned long long)a.row_mask + 1ULL;
    if ((r & (r - 1)) != 0) return VFRB_ERR_ARG;  // ring sizes are powers of two
    if ((long long)r < a.nrows_valid) return VFRB_ERR_ARG;
  }
  const bool want_stats = a.ave || a.sigma || a.peak || a.frb || a.argmax;
  if (want_stats && (!a.workspace || a.workspace_bytes < dedisperse_workspace_bytes_plan(pl, a.nt_out)))
    return VFRB_ERR_ARG;
  int v = pl->variant[a.storage];
  if (v == VFRB_DD_AUTO) v = default_variant(pl, a.storage);
  return launch_variant(pl, v, a, s, a.fb_shift1);
}

// One launch of the pattern kernel over several streams' chunks (grid z =
// job), the series only (no statistics partials).  Every job shares the
// plan's delay tables and the ring geometry (chan_stride, row_mask); the
// launch covers the longest job, the other jobs' surplus CTAs return at
// once.  *launched = 0 when the plan's kernel for this storage form is not
// a pattern kernel (or does not apply): the caller then dedisperses the
// jobs one by one.
int launch_dedisperse_jobs(const vfrb_ddplan* pl, int storage, const DdJob* jobs, int njobs, long long chan_stride,
                           unsigned row_mask, cudaStream_t s, int* launched) {
  *launched = 0;
  if (!pl || njobs < 1 || njobs > kDdMaxJobs || storage < VFRB_F32 || storage > VFRB_F16) return VFRB_ERR_ARG;
  int v = pl->variant[storage];
  if (v == VFRB_DD_AUTO) v = default_variant(pl, storage);
  if (v != VFRB_DD_PAT4 && v != VFRB_DD_PAT2) return VFRB_OK;
  vfrb_dd_args a{};
  a.fb = jobs[0].fb;
  a.storage = storage;
  a.uniform_scale = storage == VFRB_F16 ? jobs[0].out_scale : 0.f;
  a.chan_stride = chan_stride;
  a.row_mask = row_mask;
  a.nrows_valid = jobs[0].nrows_valid;
  long long nt = 0;
  bool pair = storage == VFRB_F16;  // every job has its shifted copy
  for (int i = 0; i < njobs; ++i) {
    pair = pair && jobs[i].fb1 != nullptr;
    nt = std::max(nt, jobs[i].nt_out);
    if (((uintptr_t)jobs[i].fb & 15) != 0 || (storage == VFRB_F16 && !(jobs[i].out_scale > 0.f)) ||
        jobs[i].nrows_valid < jobs[i].nt_out + pl->max_delay)
      return VFRB_OK;
  }
  a.nt_out = nt;
  a.out = jobs[0].out;
  a.out_stride = jobs[0].out_stride;
  int ntb = 0;
  const int st = pat_launch(pl, v, a, nullptr, s, &ntb, jobs, njobs, pair ? jobs[0].fb1 : nullptr);
  if (st) return st;
  *launched = ntb > 0;
  return VFRB_OK;
}

// Time every applicable variant on scratch data and keep the fastest.
int ddplan_autotune(vfrb_ddplan* pl, int storage, long long nt, float* times, cudaStream_t s) {
  if (!pl || storage < VFRB_F32 || storage > VFRB_I8 || nt <= 0) return VFRB_ERR_ARG;
  const size_t eb = storage == VFRB_F32 ? 4 : storage == VFRB_F16 ? 2 : 1;
  const long long rows = (nt + pl->max_delay + 15) / 16 * 16;
  void* fb = nullptr;
  float *out = nullptr, *st = nullptr, *w = nullptr;
  int* stb = nullptr;
  void* ws = nullptr;
  const size_t wsb = dedisperse_workspace_bytes_plan(pl, nt);
  auto cleanup = [&]() {
    cudaFree(fb);
    cudaFree(out);
    cudaFree(st);
    cudaFree(stb);
    cudaFree(ws);
    cudaFree(w);
  };
  if (cudaMalloc(&fb, (size_t)pl->nchan * rows * eb) != cudaSuccess ||
      cudaMalloc(&out, (size_t)pl->ndm * nt * 4) != cudaSuccess || cudaMalloc(&st, (size_t)pl->ndm * 12) != cudaSuccess ||
      cudaMalloc(&stb, (size_t)pl->ndm * 8) != cudaSuccess || cudaMalloc(&ws, wsb + 16) != cudaSuccess ||
      cudaMalloc(&w, (size_t)pl->nchan * 4) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return VFRB_ERR_NOMEM;
  }
  if (cudaMemsetAsync(fb, 0, (size_t)pl->nchan * rows * eb, s) != cudaSuccess ||
      cudaMemsetAsync(w, 0, (size_t)pl->nchan * 4, s) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return VFRB_ERR_CUDA;
  }
  vfrb_dd_args a{};
  a.fb = fb;
  a.storage = storage;
  a.chan_scale = storage == VFRB_I8 ? w : nullptr;
  a.uniform_scale = 1.f;
  a.chan_stride = rows;
  a.row_mask = 0xffffffffu;
  a.nrows_valid = rows;
  a.nt_out = nt;
  a.out = out;
  a.out_stride = nt;
  a.workspace = ws;
  a.workspace_bytes = wsb + 16;
  a.ave = st;
  a.sigma = st + pl->ndm;
  a.peak = st + 2 * pl->ndm;
  a.frb = stb;
  a.argmax = stb + pl->ndm;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    cleanup();
    return VFRB_ERR_CUDA;
  }
  float best = 1e30f;
  int bestv = VFRB_DD_STAGED;
  if (times) times[VFRB_DD_AUTO] = -1.f;
  // the direct variant last: it is timed only when nothing faster applies
  static const int order[] = {VFRB_DD_STAGED, VFRB_DD_REG1, VFRB_DD_REG2, VFRB_DD_REG4,
                              VFRB_DD_PAT2,   VFRB_DD_PAT4, VFRB_DD_DIRECT};
  for (int v : order) {
    if (times) times[v] = -1.f;
    if (v == VFRB_DD_DIRECT && bestv != VFRB_DD_STAGED) continue;
    const bool reg = v == VFRB_DD_REG1 || v == VFRB_DD_REG2 || v == VFRB_DD_REG4;
    const bool pat = v == VFRB_DD_PAT2 || v == VFRB_DD_PAT4;
    if (reg || pat) {
      const int D = v == VFRB_DD_REG4 || v == VFRB_DD_PAT4 ? 4 : v == VFRB_DD_REG2 || v == VFRB_DD_PAT2 ? 2 : 1;
      const RegGroup* g = find_group(pl, D);
      if (!g || storage == VFRB_I8 || (pat && !g->d_gpat)) continue;
    }
    if (launch_variant(pl, v, a, s) != VFRB_OK) continue;  // warm-up; also rejects what does not apply
    cudaEventRecord(e0, s);
    for (int r = 0; r < 2; ++r) launch_variant(pl, v, a, s);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms *= 0.5f;
    if (times) times[v] = ms;
    if (ms < best) {
      best = ms;
      bestv = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int err = cuda_status(cudaStreamSynchronize(s));
  cleanup();
  if (err) return err;
  pl->variant[storage] = bestv;
  return VFRB_OK;
}

int ddplan_set_variant(vfrb_ddplan* pl, int storage, int v) {
  if (!pl || storage < VFRB_F32 || storage > VFRB_I8 || v < VFRB_DD_AUTO || v >= VFRB_DD_NVARIANTS)
    return VFRB_ERR_ARG;
  pl->variant[storage] = v;
  return VFRB_OK;
}

int ddplan_variant(const vfrb_ddplan* pl, int storage) {
  if (!pl || storage < VFRB_F32 || storage > VFRB_I8) return -1;
  return pl->variant[storage] == VFRB_DD_AUTO ? default_variant(pl, storage) : pl->variant[storage];
}

// Pattern id of the packed in-group differences (8 bits per trial, trial 0
// first), kPatGeneric when the pattern has no straight-line code.
static unsigned char pattern_id(int D, unsigned pk) {
  static const std::vector<unsigned char> lut4 = [] {
    std::vector<unsigned char> t(1u << 15, kPatGeneric);
#define VFRB_L4(ID, A, B, C) t[(unsigned)(A) | ((unsigned)(B) << 5) | ((unsigned)(C) << 10)] = (unsigned char)(ID);
    VFRB_PAT4_LIST(VFRB_L4)
#undef VFRB_L4
    return t;
  }();
  static const std::vector<unsigned char> lut2 = [] {
    std::vector<unsigned char> t(256, kPatGeneric);
#define VFRB_L2(ID, A) t[(unsigned)(A)] = (unsigned char)(ID);
    VFRB_PAT2_LIST(VFRB_L2)
#undef VFRB_L2
    return t;
  }();
  if ((pk & 0xFFu) != 0) return kPatGeneric;  // trial 0 must have the smallest delay
  if (D == 4) {
    const unsigned a = (pk >> 8) & 0xFFu, b = (pk >> 16) & 0xFFu, c = pk >> 24;
    if (a > 31 || b > 31 || c > 31) return kPatGeneric;
    return lut4[a | (b << 5) | (c << 10)];
  }
  if (D == 2) return lut2[(pk >> 8) & 0xFFu];
  return kPatGeneric;
}

static int build_group(vfrb_ddplan* p, const int32_t* h_off, int D, int smax_allowed) {
  const int ndm = p->ndm, nchan = p->nchan;
  const int ng = (ndm + D - 1) / D;
  const int DB = kRegWarps * D;
  const int nb = (ndm + DB - 1) / DB;
  auto off = [&](int d, int c) { return (int)h_off[(long long)std::min(d, ndm - 1) * nchan + c]; };
  std::vector<int> gb((size_t)ng * nchan), bm((size_t)nb * nchan);
  std::vector<unsigned> gp((size_t)ng * nchan);
  int smax = 0, span = 0;
  for (int g = 0; g < ng; ++g)
    for (int c = 0; c < nchan; ++c) {
      int mn = 0x7fffffff, mx = 0;
      for (int j = 0; j < D; ++j) {
        mn = std::min(mn, off(g * D + j, c));
        mx = std::max(mx, off(g * D + j, c));
      }
      smax = std::max(smax, mx - mn);
      if (smax > smax_allowed) return VFRB_OK;  // this group size does not apply
      unsigned pk = 0;
      for (int j = 0; j < D; ++j) pk |= (unsigned)(off(g * D + j, c) - mn) << (8 * j);
      gb[(size_t)g * nchan + c] = mn;
      gp[(size_t)g * nchan + c] = pk;
    }
  for (int b = 0; b < nb; ++b)
    for (int c = 0; c < nchan; ++c) {
      int mn = 0x7fffffff, mx = 0;
      for (int d = b * DB; d < std::min(ndm, (b + 1) * DB); ++d) {
        mn = std::min(mn, off(d, c));
        mx = std::max(mx, off(d, c));
      }
      bm[(size_t)b * nchan + c] = mn;
      span = std::max(span, mx - mn);
    }
  // the same per-block table for 16-warp CTAs (the pattern kernel's
  // one-CTA-per-SM form)
  const int DB16 = 16 * D;
  const int nb16 = (ndm + DB16 - 1) / DB16;
  std::vector<int> bm16((size_t)nb16 * nchan);
  int span16 = 0;
  for (int b = 0; b < nb16; ++b)
    for (int c = 0; c < nchan; ++c) {
      int mn = 0x7fffffff, mx = 0;
      for (int d = b * DB16; d < std::min(ndm, (b + 1) * DB16); ++d) {
        mn = std::min(mn, off(d, c));
        mx = std::max(mx, off(d, c));
      }
      bm16[(size_t)b * nchan + c] = mn;
      span16 = std::max(span16, mx - mn);
    }
  RegGroup* slot = nullptr;
  for (auto& r : p->reg)
    if (r.D == 0) {
      slot = &r;
      break;
    }
  if (!slot) return VFRB_OK;
  RegGroup g;
  g.D = D;
  g.smax = smax;
  g.span = span;
  for (int b = 0; b < nb; ++b) g.bmin_mid_max = std::max(g.bmin_mid_max, bm[(size_t)b * nchan + nchan / 2]);
  g.ngroups = ng;
  g.nblocks = nb;
  g.nblocks16 = nb16;
  g.span_16w = span16;
  for (int b = 0; b < nb16; ++b) g.bmin_mid_max16 = std::max(g.bmin_mid_max16, bm16[(size_t)b * nchan + nchan / 2]);
  const bool with_pat = (D == 4 && smax <= VFRB_PAT4_SMAX) || (D == 2 && smax <= VFRB_PAT2_SMAX);
  std::vector<unsigned char> pt;
  if (with_pat) {
    pt.resize(gp.size());
    for (size_t i = 0; i < gp.size(); ++i) {
      pt[i] = pattern_id(D, gp[i]);
      g.n_generic += pt[i] == kPatGeneric;
    }
  }
  bool ok = cudaMalloc(&g.d_gbase, gb.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&g.d_gpack, gp.size() * sizeof(unsigned)) == cudaSuccess &&
            cudaMalloc(&g.d_bmin, bm.size() * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&g.d_bmin16, bm16.size() * sizeof(int)) == cudaSuccess &&
            (!with_pat || cudaMalloc(&g.d_gpat, pt.size()) == cudaSuccess);
  ok = ok && cudaMemcpy(g.d_gbase, gb.data(), gb.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(g.d_gpack, gp.data(), gp.size() * sizeof(unsigned), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(g.d_bmin, bm.data(), bm.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(g.d_bmin16, bm16.data(), bm16.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
       (!with_pat || cudaMemcpy(g.d_gpat, pt.data(), pt.size(), cudaMemcpyHostToDevice) == cudaSuccess);
  if (!ok) {
    cudaGetLastError();
    cudaFree(g.d_gbase);
    cudaFree(g.d_gpack);
    cudaFree(g.d_bmin);
    cudaFree(g.d_bmin16);
    cudaFree(g.d_gpat);
    return VFRB_ERR_NOMEM;
  }
  *slot = g;
  return VFRB_OK;
}

int ddplan_destroy(vfrb_ddplan* p) {
  if (!p) return VFRB_OK;
  if (p->d_off) cudaFree(p->d_off);
  for (auto& g : p->reg) {
    if (g.d_gbase) cudaFree(g.d_gbase);
    if (g.d_gpack) cudaFree(g.d_gpack);
    if (g.d_bmin) cudaFree(g.d_bmin);
    if (g.d_bmin16) cudaFree(g.d_bmin16);
    if (g.d_gpat) cudaFree(g.d_gpat);
  }
  delete p;
  return VFRB_OK;
}

int ddplan_create(vfrb_ddplan** out, const int32_t* h_off, int ndm, int nchan) {
  if (!out || !h_off || ndm < 1 || nchan < 2) return VFRB_ERR_ARG;
  vfrb_ddplan* p = new vfrb_ddplan();
  p->ndm = ndm;
  p->nchan = nchan;
  int mxd = 0, span = 0;
  for (long long i = 0; i < (long long)ndm * nchan; ++i) {
    if (h_off[i] < 0) {
      delete p;
      return VFRB_ERR_ARG;
    }
    mxd = std::max(mxd, (int)h_off[i]);
  }
  for (int d0 = 0; d0 < ndm; d0 += kDdDm)
    for (int c = 0; c < nchan; ++c) {
      int mn = 0x7fffffff, mx = 0;
      for (int d = d0; d < std::min(ndm, d0 + kDdDm); ++d) {
        mn = std::min(mn, (int)h_off[(long long)d * nchan + c]);
        mx = std::max(mx, (int)h_off[(long long)d * nchan + c]);
      }
      span = std::max(span, mx - mn);
    }
  p->max_delay = mxd;
  p->span16 = span;
  // register-window groups: D = 4 and 2 when their in-group shifts fit, else D = 1
  int st = build_group(p, h_off, 4, 20);
  if (!st) st = build_group(p, h_off, 2, 16);
  if (!st && !find_group(p, 2) && !find_group(p, 4)) st = build_group(p, h_off, 1, 0);
  if (st) {
    ddplan_destroy(p);
    return st;
  }
  const size_t bytes = sizeof(int) * (size_t)ndm * nchan;
  if (cudaMalloc(&p->d_off, bytes) != cudaSuccess ||
      cudaMemcpy(p->d_off, h_off, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    ddplan_destroy(p);
    return VFRB_ERR_NOMEM;
  }
  *out = p;
  return VFRB_OK;
}

int ddplan_max_delay(const vfrb_ddplan* p) { return p->max_delay; }
int ddplan_reg_group(const vfrb_ddplan* p) {
  const int v = ddplan_variant(p, VFRB_F32);
  return v == VFRB_DD_REG4 || v == VFRB_DD_PAT4 ? 4 : v == VFRB_DD_REG2 || v == VFRB_DD_PAT2 ? 2 : v == VFRB_DD_REG1 ? 1 : 0;
}

}  // namespace vfrb
