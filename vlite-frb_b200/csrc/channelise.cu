// K1: fused channeliser for sm_100a.
//
// A persistent CTA (512 threads, one per SM) produces filterbank rows in turn;
// each row is NAVE consecutive 12500-sample windows of both polarisations.
// Per window the two real 8-bit streams are packed into one complex sequence
// z[n] = (x0[n]-128) + i (x1[n]-128) and transformed by a hand-written
// 12500-point mixed-radix Stockham FFT (radices 25, 25, 20) that lives
// entirely in shared memory (100 kB).  Because
//   |X0[k]|^2 + |X1[k]|^2 = (|Z[k]|^2 + |Z[N-k]|^2) / 2,
// detection, the polarisation sum, /NFREQ, the NAVE average and the NSKIP
// channel slice are an epilogue on Z.  The -128 offset only changes bin 0,
// which no output channel uses (NSKIP >= 1), and keeps the FP32 transform
// well conditioned.  This replaces convertarray, cufftExecR2C, sumpower,
// avepower and the per-row D2D copies of PIPE:574-632 (STATS:377-405,
// TS:603-636).
//
// Input staging: the raw bytes of the NEXT window (2 x 12500) are copied
// from the frame ring into a second shared-memory byte buffer with 4-byte
// cp.async while the current window is transformed, so the global-memory
// latency is hidden behind the FFT; the byte -> float conversion is fused
// into the first pass's loads.  Gap frames (slot -1) are zero-filled by the
// copy itself.
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

// Twiddles, computed on the host in double precision and rounded to float:
//   g_tw2[r-1][m] = W_625^(m r), m < 25, 1 <= r < 25   (pass 2, Ns = 25)
//   pass 3 needs W^(j r) = W_12500^(j r) for j < 625, 1 <= r < 20: with
//   r = 5a + b it is T_a[j] * (W^j)^b, from four tables of 625 entries
//   (T_0 = W^j, T_1 = W^5j, T_2 = W^10j, T_3 = W^15j) and at most three
//   multiplications for (W^j)^b -- 20 kB instead of a 95 kB table, four
//   table loads per butterfly instead of nineteen.
// Each CTA copies the tables into shared memory once.
constexpr int kTw2 = (kR2 - 1) * kNs2;  // 600
constexpr int kTw3 = 4 * kM3;           // 2500
constexpr int kAccFloats = kFftN / 2 + 2;  // 6252 >= any NCHANOUT
constexpr int kStage = 12512;              // one pol's window bytes, padded to 16
__device__ float2 g_tw2[kTw2];
__device__ float2 g_tw3[kTw3];
// shared-memory layout (bytes): Z | stage[2 buffers][2 pols] | tw2 | tw3 | acc
constexpr size_t kSmZ = sizeof(float2) * kFftN;
constexpr size_t kSmStage = (size_t)4 * kStage;
constexpr size_t kSmTw2 = sizeof(float2) * kTw2;
constexpr size_t kSmTw3 = sizeof(float2) * kTw3;
constexpr size_t kSmem = kSmZ + kSmStage + kSmTw2 + kSmTw3 + sizeof(float) * kAccFloats;
static_assert(kSmem <= 227 * 1024, "channeliser shared memory");
static_assert(kSmZ % 16 == 0 && kSmStage % 16 == 0 && kStage % 16 == 0 && kSmTw2 % 16 == 0 && kSmTw3 % 16 == 0,
              "16-byte aligned regions");

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
      const double a = -2.0 * M_PI * (double)((m * r) % 625) / 625.0;
      h2[(r - 1) * kNs2 + m] = make_float2((float)cos(a), (float)sin(a));
    }
  for (int t = 0; t < 4; ++t)
    for (int m = 0; m < kM3; ++m) {
      const double a = -2.0 * M_PI * (double)(((long long)(t == 0 ? 1 : 5 * t) * m) % kFftN) / (double)kFftN;
      h3[t * kM3 + m] = make_float2((float)cos(a), (float)sin(a));
    }
  if (cudaMemcpyToSymbol(g_tw2, h2, sizeof(h2)) != cudaSuccess) return VFRB_ERR_CUDA;
  if (cudaMemcpyToSymbol(g_tw3, h3, sizeof(h3)) != cudaSuccess) return VFRB_ERR_CUDA;
  g_tw_ready[dev] = true;
  return VFRB_OK;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(gsrc), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit_k1() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Stage the raw bytes of one 12500-sample window of both pols (stream
// positions pos0 ..) into st0 / st1.  ALIGNED (sample0 % 4 == 0): 4-byte
// asynchronous copies, each inside one payload; otherwise synchronous byte
// loads.  Positions outside the slot table and misaligned payloads set
// kErrSlotRange and read as zero bytes.
template <bool ALIGNED>
__device__ __forceinline__ void stage_window(unsigned char* __restrict__ st0, unsigned char* __restrict__ st1,
                                             const vfrb_chan_args& a, long long pos0, int& err) {
  const int tid = threadIdx.x;
  if (ALIGNED) {
    // one 64-bit division per window; 32-bit arithmetic per 4-byte group
    const long long slot0 = pos0 >= 0 ? pos0 / kDataLen : -1;
    const int off0 = pos0 >= 0 ? (int)(pos0 - slot0 * kDataLen) : 0;
    for (int g = tid; g < kFftN / 4; g += kThreads) {
      const int o = off0 + 4 * g;  // < 5000 + 12500
      const int q = o / kDataLen;
      const long long slot = slot0 + q;
      const int off = o - q * kDataLen;
      long long s0 = -1, s1 = -1;
      if (slot0 < 0 || slot >= a.nslots) {
        err |= kErrSlotRange;
      } else {
        s0 = __ldg(a.slots0 + slot);
        s1 = __ldg(a.slots1 + slot);
        if ((s0 >= 0 && (s0 & 3)) || (s1 >= 0 && (s1 & 3))) {  // payloads must start on a 4-byte boundary
          err |= kErrSlotRange;
          s0 = s1 = -1;
        }
      }
      cp_async4(st0 + 4 * g, s0 >= 0 ? a.frames + s0 + off : a.frames, s0 >= 0 ? 4 : 0);
      cp_async4(st1 + 4 * g, s1 >= 0 ? a.frames + s1 + off : a.frames, s1 >= 0 ? 4 : 0);
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
      st0[n] = v0;
      st1[n] = v1;
    }
  }
}

// Passes 1 and 2 of the 12500-point forward FFT of the staged window into Z.
// Stockham passes: data1[(j/Ns)*Ns*R + j%Ns + r*Ns] = DFT_R(data0[j + r*N/R] * W^(r*(j%Ns)*N/(Ns*R))).
// Pass 1 reads the staged bytes (not Z), so it needs no barrier between its
// reads and writes; pass 2 holds its inputs in registers across one barrier,
// so one Z buffer suffices.
__device__ __forceinline__ void fft_passes12(float2* __restrict__ Z, const unsigned char* __restrict__ st0,
                                             const unsigned char* __restrict__ st1, const float2* __restrict__ tw2) {
  const int tid = threadIdx.x;
  if (tid < kM1) {  // pass 1: R = 25, Ns = 1 (no twiddles); writes stride 25 (odd -> no bank conflicts)
    float2 v[kR1];
#pragma unroll
    for (int r = 0; r < kR1; ++r)
      v[r] = make_float2((float)st0[tid + r * kM1] - 128.f, (float)st1[tid + r * kM1] - 128.f);
    dft25(v);
#pragma unroll
    for (int r = 0; r < kR1; ++r) Z[tid * kR1 + r] = v[dft25_pos(r)];
  }
  __syncthreads();
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
}

// Pass 3 butterfly j (R = 20, Ns = 625): inputs Z[j + 625 r] times W^(j r),
// output index r in u[dft20_pos(r)] is spectrum bin j + 625 r.
__device__ __forceinline__ void pass3_butterfly(const float2* __restrict__ Z, const float2* __restrict__ tw3, int j,
                                                float2 (&u)[kR3]) {
#pragma unroll
  for (int r = 0; r < kR3; ++r) u[r] = Z[j + r * kM3];
  const float2 w1 = tw3[j];
  const float2 w2 = cmul(w1, w1);
  const float2 w3 = cmul(w2, w1);
  const float2 w4 = cmul(w3, w1);
  const float2 t5 = tw3[kM3 + j], t10 = tw3[2 * kM3 + j], t15 = tw3[3 * kM3 + j];
#pragma unroll
  for (int r = 1; r < kR3; ++r) {
    const int a = r / 5, b = r % 5;
    const float2 wb = b == 1 ? w1 : b == 2 ? w2 : b == 3 ? w3 : w4;
    const float2 ta = a == 1 ? t5 : a == 2 ? t10 : t15;
    const float2 w = a == 0 ? wb : (b == 0 ? ta : cmul(ta, wb));
    u[r] = cmul(u[r], w);
  }
  dft20(u);
}

__device__ __forceinline__ float pw(float2 z) { return fmaf(z.x, z.x, z.y * z.y); }

template <bool ALIGNED>
__global__ void __launch_bounds__(kThreads, 1) k_channelise(const vfrb_chan_args a) {
  extern __shared__ float4 smem_f4[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(smem_f4);
  float2* Z = reinterpret_cast<float2*>(sm);
  unsigned char* stage = sm + kSmZ;  // [2 buffers][2 pols][kStage]
  float2* tw2 = reinterpret_cast<float2*>(sm + kSmZ + kSmStage);
  float2* tw3 = reinterpret_cast<float2*>(sm + kSmZ + kSmStage + kSmTw2);
  // per-bin power accumulators in shared memory; thread j owns the bins of
  // pass-3 butterflies j and 625 - j in every window
  float* acc = reinterpret_cast<float*>(sm + kSmZ + kSmStage + kSmTw2 + kSmTw3);
  const int tid = threadIdx.x;
  int err = 0;
  for (int i = tid; i < kTw2; i += kThreads) tw2[i] = g_tw2[i];
  for (int i = tid; i < kTw3; i += kThreads) tw3[i] = g_tw3[i];
  for (int c = tid; c < a.nchanout; c += kThreads) acc[c] = 0.f;
  const float scale = 1.0f / (2.0f * (float)a.nfreq * (float)a.nave);

  // persistent CTAs: one per SM; this CTA's windows are (row, w) for rows
  // blockIdx.x + k*gridDim.x, w < NAVE, in that order
  const long long nrows_cta = (a.nrows - blockIdx.x + gridDim.x - 1) / gridDim.x;
  const long long nwin = nrows_cta * a.nave;
  auto win_pos = [&](long long i) {
    const long long row = blockIdx.x + (i / a.nave) * gridDim.x;
    return a.sample0 + (row * a.nave + i % a.nave) * (long long)kFftN;
  };
  if (nwin > 0) stage_window<ALIGNED>(stage, stage + kStage, a, win_pos(0), err);
  cp_async_commit_k1();
  for (long long i = 0; i < nwin; ++i) {
    unsigned char* cur = stage + (size_t)(i & 1) * 2 * kStage;
    unsigned char* nxt = stage + (size_t)((i + 1) & 1) * 2 * kStage;
    // the buffer of window i+1 was last read by pass 1 of window i-1, which
    // every thread has left (barriers after passes 1 and 2)
    if (i + 1 < nwin) stage_window<ALIGNED>(nxt, nxt + kStage, a, win_pos(i + 1), err);
    cp_async_commit_k1();
    cp_async_wait_1();  // this thread's copies of window i have landed
    __syncthreads();    // ... and everybody else's; pass 3 of window i-1 is done with Z
    fft_passes12(Z, cur, cur + kStage, tw2);
    // Pass 3 fused with detection.  Bins k = j + 625 r and N - k =
    // (625 - j) + 625 (19 - r) come from butterflies j and 625 - j, so thread
    // j computes both and adds |Z_k|^2 + |Z_{N-k}|^2 to the channel of
    // min(k, N - k) straight from registers (j = 0 pairs with itself):
    // pass 3 writes nothing back and there is no separate epilogue.
    if (tid <= kM3 / 2) {
      const int jj = tid, jp = (kM3 - jj) % kM3;
      const bool last = (i % a.nave) == a.nave - 1;
      const long long row = blockIdx.x + (i / a.nave) * gridDim.x;
      const unsigned long long orow = (unsigned long long)(a.out_row0 + row) & (unsigned long long)a.out_row_mask;
      float* dst = a.out + (long long)orow * a.out_row_stride;
      float mag[kR3];
      float2 u[kR3];
      if (jj != 0) {
        pass3_butterfly(Z, tw3, jp, u);
#pragma unroll
        for (int r = 0; r < kR3; ++r) mag[r] = pw(u[dft20_pos(r)]);
      }
      pass3_butterfly(Z, tw3, jj, u);
#pragma unroll
      for (int r = 0; r < kR3; ++r) {
        float p;
        int bin;
        if (jj == 0) {  // bins 625 r and 625 (20 - r); r = 10 is the Nyquist bin (counted twice, as N - k = k)
          if (r == 0 || r > kR3 / 2) continue;
          p = pw(u[dft20_pos(r)]) + pw(u[dft20_pos(kR3 - r)]);
          bin = kM3 * r;
        } else {
          p = pw(u[dft20_pos(r)]) + mag[kR3 - 1 - r];
          bin = r < kR3 / 2 ? jj + kM3 * r : jp + kM3 * (kR3 - 1 - r);
        }
        const int c = bin - a.nskip;
        if (c >= 0 && c < a.nchanout) {
          const float v = acc[c] + p;
          if (last) {
            // (|X0|^2 + |X1|^2)/NFREQ averaged over NAVE spectra (PIPE:1296, 1310)
            dst[c] = v * scale;
            acc[c] = 0.f;
          } else {
            acc[c] = v;
          }
        }
      }
    }
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
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) {
    cudaGetLastError();
    nsm = 148;
  }
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
