// K1: fused channeliser for sm_100a.
//
// A persistent CTA (512 threads, one per SM) produces filterbank rows in turn;
// each row is: NAVE consecutive 12500-sample windows
// of both polarisations.  Per window the two real 8-bit streams are packed
// into one complex sequence z[n] = (x0[n]-128) + i (x1[n]-128) and transformed
// by a hand-written 12500-point mixed-radix Stockham FFT (radices 25, 25, 20)
// that lives entirely in shared memory (100 kB).  Because
//   |X0[k]|^2 + |X1[k]|^2 = (|Z[k]|^2 + |Z[N-k]|^2) / 2,
// detection, the polarisation sum, /NFREQ, the NAVE average and the NSKIP
// channel slice are an epilogue on Z.  The -128 offset only changes bin 0,
// which no output channel uses (NSKIP >= 1), and keeps the FP32 transform
// well conditioned.  This replaces convertarray, cufftExecR2C, sumpower,
// avepower and the per-row D2D copies of PIPE:574-632 (STATS:377-405,
// TS:603-636).
#include "vfrb_common.cuh"
#include "dft_codelets.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace vfrb {

constexpr int kThreads = 512;
constexpr int kR1 = 25, kR2 = 25, kR3 = 20;
constexpr int kM1 = kFftN / kR1;  // 500 butterflies in passes 1 and 2
constexpr int kM3 = kFftN / kR3;  // 625 butterflies in pass 3
constexpr int kNs2 = kR1;         // 25
constexpr int kNs3 = kR1 * kR2;   // 625

// Twiddles, computed on the host in double precision and rounded to float
// (row r = 0 is all ones and is not stored):
//   g_tw2[r-1][m] = W_625^(m r),   m < 25,  1 <= r < 25   (pass 2, Ns = 25)
//   g_tw3[r-1][m] = W_12500^(m r), m < 625, 1 <= r < 20   (pass 3, Ns = 625)
// Each CTA copies both tables into shared memory once.
constexpr int kTw2 = (kR2 - 1) * kNs2;  // 600
constexpr int kTw3 = (kR3 - 1) * kNs3;  // 11875
constexpr int kAccFloats = kFftN / 2 + 2;  // 6252 >= any NCHANOUT
__device__ float2 g_tw2[kTw2];
__device__ float2 g_tw3[kTw3];
// shared-memory layout (bytes): Z | tw3 | tw2 | acc
constexpr size_t kSmZ = sizeof(float2) * kFftN;
constexpr size_t kSmTw3 = sizeof(float2) * kTw3;
constexpr size_t kSmTw2 = sizeof(float2) * kTw2;
constexpr size_t kSmem = kSmZ + kSmTw3 + kSmTw2 + sizeof(float) * kAccFloats;
static_assert(kSmem <= 227 * 1024, "channeliser shared memory");

static std::mutex g_tw_mu;
static bool g_tw_ready[64];

static int ensure_twiddles() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return VFRB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_tw_mu);
  if (g_tw_ready[dev]) return VFRB_OK;
  static float2 h2[kTw2], h3[kTw3];
  for (int r = 1; r < kR2; ++r)
    for (int m = 0; m < kNs2; ++m) {
      double a = -2.0 * M_PI * (double)((m * r) % 625) / 625.0;
      h2[(r - 1) * kNs2 + m] = make_float2((float)cos(a), (float)sin(a));
    }
  for (int r = 1; r < kR3; ++r)
    for (int m = 0; m < kNs3; ++m) {
      double a = -2.0 * M_PI * (double)((m * r) % kFftN) / (double)kFftN;
      h3[(r - 1) * kNs3 + m] = make_float2((float)cos(a), (float)sin(a));
    }
  if (cudaMemcpyToSymbol(g_tw2, h2, sizeof(h2)) != cudaSuccess) return VFRB_ERR_CUDA;
  if (cudaMemcpyToSymbol(g_tw3, h3, sizeof(h3)) != cudaSuccess) return VFRB_ERR_CUDA;
  g_tw_ready[dev] = true;
  return VFRB_OK;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// Load one 12500-sample window of both pols into Z as (x0-128) + i(x1-128).
// ALIGNED: every 4-sample group lies inside one payload at a 4-byte boundary
// (true whenever sample0 and TWONCHAN are multiples of 4).
template <bool ALIGNED>
__device__ __forceinline__ void load_window(float2* __restrict__ Z, const vfrb_chan_args& a, long long pos0,
                                            int& err) {
  const int tid = threadIdx.x;
  if (ALIGNED) {
    for (int g = tid; g < kFftN / 4; g += kThreads) {
      const long long pos = pos0 + 4LL * g;
      const long long slot = pos / kDataLen;
      const int off = (int)(pos - slot * kDataLen);
      uchar4 b0 = make_uchar4(0, 0, 0, 0), b1 = b0;
      if (pos < 0 || slot >= a.nslots) {
        err |= kErrSlotRange;
      } else {
        const long long s0 = __ldg(a.slots0 + slot), s1 = __ldg(a.slots1 + slot);
        if (((s0 | s1) & 3) != 0 && s0 >= 0 && s1 >= 0) {
          err |= kErrSlotRange;  // payloads must start on a 4-byte boundary
        } else {
          if (s0 >= 0 && (s0 & 3) == 0) b0 = __ldg(reinterpret_cast<const uchar4*>(a.frames + s0 + off));
          if (s1 >= 0 && (s1 & 3) == 0) b1 = __ldg(reinterpret_cast<const uchar4*>(a.frames + s1 + off));
        }
      }
      float4* z4 = reinterpret_cast<float4*>(Z + 4 * g);
      z4[0] = make_float4((float)b0.x - 128.f, (float)b1.x - 128.f, (float)b0.y - 128.f, (float)b1.y - 128.f);
      z4[1] = make_float4((float)b0.z - 128.f, (float)b1.z - 128.f, (float)b0.w - 128.f, (float)b1.w - 128.f);
    }
  } else {
    for (int n = tid; n < kFftN; n += kThreads) {
      const long long pos = pos0 + n;
      const long long slot = pos / kDataLen;
      const int off = (int)(pos - slot * kDataLen);
      unsigned char v0 = 0, v1 = 0;
      if (pos < 0 || slot >= a.nslots) {
        err |= kErrSlotRange;
      } else {
        const long long s0 = __ldg(a.slots0 + slot), s1 = __ldg(a.slots1 + slot);
        if (s0 >= 0) v0 = __ldg(a.frames + s0 + off);
        if (s1 >= 0) v1 = __ldg(a.frames + s1 + off);
      }
      Z[n] = make_float2((float)v0 - 128.f, (float)v1 - 128.f);
    }
  }
}

// In-place 12500-point forward FFT of Z (natural order in and out).
// Stockham passes: data1[(j/Ns)*Ns*R + j%Ns + r*Ns] = DFT_R(data0[j + r*N/R] * W^(r*(j%Ns)*N/(Ns*R))).
// Each pass holds its butterfly inputs in registers across a barrier, so one
// buffer suffices.
__device__ __forceinline__ void fft12500(float2* __restrict__ Z, const float2* __restrict__ tw2,
                                         const float2* __restrict__ tw3) {
  const int tid = threadIdx.x;
  {  // pass 1: R = 25, Ns = 1 (no twiddles); writes are stride 25 (odd -> no bank conflicts)
    float2 v[kR1];
    if (tid < kM1) {
#pragma unroll
      for (int r = 0; r < kR1; ++r) v[r] = Z[tid + r * kM1];
      dft25(v);
    }
    __syncthreads();
    if (tid < kM1) {
#pragma unroll
      for (int r = 0; r < kR1; ++r) Z[tid * kR1 + r] = v[dft25_pos(r)];
    }
    __syncthreads();
  }
  {  // pass 2: R = 25, Ns = 25
    float2 v[kR2];
    const int m = tid % kNs2;
    if (tid < kM1) {
#pragma unroll
      for (int r = 0; r < kR2; ++r) v[r] = Z[tid + r * kM1];
#pragma unroll
      for (int r = 1; r < kR2; ++r) v[r] = cmul(v[r], tw2[(r - 1) * kNs2 + m]);
      dft25(v);
    }
    __syncthreads();
    if (tid < kM1) {
      const int base = (tid / kNs2) * (kNs2 * kR2) + m;
#pragma unroll
      for (int r = 0; r < kR2; ++r) Z[base + r * kNs2] = v[dft25_pos(r)];
    }
    __syncthreads();
  }
  {  // pass 3: R = 20, Ns = 625.  The last Stockham pass writes exactly the
     // positions it reads (j + r*625), so butterflies are independent: no
     // barrier between read and write, and 512 threads loop over 625.
    for (int j = tid; j < kM3; j += kThreads) {
      float2 u[kR3];
#pragma unroll
      for (int r = 0; r < kR3; ++r) u[r] = Z[j + r * kM3];
#pragma unroll
      for (int r = 1; r < kR3; ++r) u[r] = cmul(u[r], tw3[(r - 1) * kNs3 + j]);
      dft20(u);
#pragma unroll
      for (int r = 0; r < kR3; ++r) Z[j + r * kNs3] = u[dft20_pos(r)];
    }
    __syncthreads();
  }
}

template <bool ALIGNED>
__global__ void __launch_bounds__(kThreads, 1) k_channelise(const vfrb_chan_args a) {
  extern __shared__ float4 smem_f4[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(smem_f4);
  float2* Z = reinterpret_cast<float2*>(sm);
  float2* tw3 = reinterpret_cast<float2*>(sm + kSmZ);
  float2* tw2 = reinterpret_cast<float2*>(sm + kSmZ + kSmTw3);
  // per-bin power accumulators live in shared memory (each thread owns the
  // same bins in every window), keeping registers for the butterflies
  float* acc = reinterpret_cast<float*>(sm + kSmZ + kSmTw3 + kSmTw2);
  const int tid = threadIdx.x;
  int err = 0;
  for (int i = tid; i < kTw3; i += kThreads) tw3[i] = g_tw3[i];
  for (int i = tid; i < kTw2; i += kThreads) tw2[i] = g_tw2[i];
  const float scale = 1.0f / (2.0f * (float)a.nfreq * (float)a.nave);

  // persistent CTAs: one per SM, striding over the rows
  for (long long row = blockIdx.x; row < a.nrows; row += gridDim.x) {
    for (int c = tid; c < a.nchanout; c += kThreads) acc[c] = 0.f;
    for (int w = 0; w < a.nave; ++w) {
      const long long pos0 = a.sample0 + (row * a.nave + w) * (long long)kFftN;
      load_window<ALIGNED>(Z, a, pos0, err);
      __syncthreads();
      fft12500(Z, tw2, tw3);
      // epilogue: |Z_k|^2 + |Z_{N-k}|^2 for the selected bins
      for (int c = tid; c < a.nchanout; c += kThreads) {
        const int k = a.nskip + c;
        const float2 z1 = Z[k];
        const float2 z2 = Z[kFftN - k];
        acc[c] += fmaf(z1.x, z1.x, z1.y * z1.y) + fmaf(z2.x, z2.x, z2.y * z2.y);
      }
      __syncthreads();
    }
    // (|X0|^2 + |X1|^2)/NFREQ averaged over NAVE spectra (PIPE:1296, 1310)
    const unsigned long long orow = (unsigned long long)(a.out_row0 + row) & (unsigned long long)a.out_row_mask;
    float* dst = a.out + (long long)orow * a.out_row_stride;
    for (int c = tid; c < a.nchanout; c += kThreads) dst[c] = acc[c] * scale;
  }
  if (err && a.d_err) atomicOr(a.d_err, err);
}

int launch_channelise(const vfrb_chan_args& a, cudaStream_t s) {
  if (a.nrows <= 0) return a.nrows == 0 ? VFRB_OK : VFRB_ERR_ARG;
  if (!a.frames || !a.slots0 || !a.slots1 || !a.out || a.nave <= 0) return VFRB_ERR_ARG;
  if (a.twonchan != kFftN || a.nfreq != kFftN / 2 + 1) return VFRB_ERR_UNSUPPORTED;
  if (a.nskip < 1 || a.nchanout < 1 || a.nskip + a.nchanout > kFftN / 2 + 1) return VFRB_ERR_ARG;
  int st = ensure_twiddles();
  if (st) return st;
  const size_t smem = kSmem;
  const bool aligned = (a.sample0 % 4) == 0;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<long long>(a.nrows, (long long)nsm);
  cudaError_t e;
  if (aligned) {
    e = cudaFuncSetAttribute(k_channelise<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_channelise<true><<<grid, kThreads, smem, s>>>(a);
  } else {
    e = cudaFuncSetAttribute(k_channelise<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_channelise<false><<<grid, kThreads, smem, s>>>(a);
  }
  if (e != cudaSuccess) return VFRB_ERR_CUDA;
  return cuda_status(cudaGetLastError());
}

}  // namespace vfrb
