// K1: fused channeliser for sm_100a.
//
// Replaces convertarray, cufftExecR2C (x2), sumpower, avepower and the
// per-row D2D channel-select copies of PIPE:574-632 (STATS:377-405,
// TS:603-636): raw 8-bit VDIF payload bytes of both polarisations in, one
// NAVE-averaged, NFREQ-normalised, pol-summed power spectrum row out.
//
// The two polarisations' real 12500-sample windows are transformed together:
// each pol's window becomes a 6250-point complex sequence
// z[m] = (x[2m] - 128) + i (x[2m+1] - 128), and the two sequences run in
// lockstep as PolPairs (re = (pol0, pol1), im = (pol0, pol1)), so every
// butterfly step is one packed FP32 instruction (add/sub/mul/fma .f32x2)
// for both pols.  The 6250-point Stockham FFT has radices 25, 25, 10 and
// lives in 100 kB of shared memory.  With Z = FFT(z), H = 6250, N = 12500,
// W = W_N, the real spectrum of each pol is
//   X[k] = (A - iC)/2,  X[H-k] = conj(A + iC)/2,
//   A = Z[k] + conj(Z[H-k]),  B = Z[k] - conj(Z[H-k]),  C = W^k B,
// so bins k and H-k need only Z[k] and Z[H-k].  The last pass's butterflies
// j and 625-j hold exactly such pairs (bins j + 625 k and 625-j + 625 (9-k)),
// so one thread runs both and detects |X0|^2 + |X1|^2 for 20 bins straight
// from registers; the NAVE average accumulates in the output row itself (the
// first window of a row stores, later ones add with a reduction nothing waits
// for), each window pre-scaled by 1/(4 NFREQ NAVE).  The -128 offset only
// changes bin 0, which no output channel uses (NSKIP >= 1), and keeps the
// FP32 transform well conditioned.
//
// One persistent 256-thread CTA per SM (a radix-25 pol-pair butterfly holds
// 100 floats, so a thread needs up to 255 registers).  The raw bytes of the
// next window are copied from the frame ring into a shared-memory byte buffer
// with 4-byte cp.async while the current window is transformed.  The copies
// are issued by warps 2..7 only: pass 3 has 313 tasks for 256 threads, and
// the 57 second-round tasks of warps 0 and 1 run while the other six warps
// issue the copies (payload pieces with one source pointer each, so a copy
// costs a few instructions).  Frames sit 5032 bytes apart in the frame ring
// and a payload is 5000 bytes, both 8 mod 16, so the pieces of one window
// differ in alignment mod 16 and no single shared-memory offset makes every
// piece a legal 16-byte or bulk copy.
#include "vfrb_common.cuh"
#include "dft_pairs.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace vfrb {

constexpr int kH = kFftN / 2;          // 6250-point complex transform per pol
constexpr int kPThreads = 256;         // one CTA per SM, 8 warps (up to 255 registers)
constexpr int kPB = kH / 25;           // 250 butterflies in passes 1 and 2
constexpr int kPM3 = kH / 10;          // 625 butterflies in pass 3
constexpr int kPTasks = kPM3 / 2 + 1;  // 313 pass-3 tasks: pairs (j, 625 - j), and j = 0
constexpr int kStage = 12512;          // one pol's window bytes, padded to 16
// the staging copies are issued by warps 2..7: pass 3's second round (threads
// 0..56) then runs while they copy
constexpr int kStageT0 = 64;
constexpr int kStageThreads = kPThreads - kStageT0;

// Twiddle tables, computed on the host in double precision:
//   g_pw2[(r-1)*25 + m] = W_625^(m r) as (c, c, s, s), so a twiddle is one
//                         packed pair per component   (pass 2, Ns = 25)
//   g_pw12[m] = W_12500^m as (c, s), m < 6250: pass 3 reads its real-split
//                         twiddles W_12500^(j + 625 k) and its radix-10 seed
//                         W_6250^j = W_12500^(2 j) here instead of building
//                         them by repeated complex products
constexpr int kPTw2 = 24 * 25;
constexpr int kPT12 = kH;
__device__ float4 g_pw2[kPTw2];
__device__ float2 g_pw12[kPT12];

// shared memory: Z | tw2 | codelet constants | t12 | staged bytes
// [2 buffers][2 pols][kStage]
constexpr size_t kPSmZ = sizeof(float4) * kH;
constexpr size_t kPSmTab = sizeof(float4) * (kPTw2 + kPairTable) + sizeof(float2) * kPT12;
constexpr size_t kPSmem = kPSmZ + kPSmTab + 4 * kStage;
static_assert(kPSmem <= 227 * 1024, "channeliser shared memory");
static_assert(kPB <= kPThreads && kPTasks <= 2 * kPThreads, "pass-3 tasks in two rounds");
static_assert((kPSmZ + kPSmTab) % 16 == 0 && kStage % 16 == 0, "16-byte aligned staging");

static std::mutex g_tw_mu;
static bool g_tw_ready[64];

static int ensure_twiddles() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return VFRB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_tw_mu);
  if (g_tw_ready[dev]) return VFRB_OK;
  static float4 p2[kPTw2];
  static float2 p12[kPT12];
  auto quad = [](double num, double den) {
    const double a = -2.0 * M_PI * num / den;
    return make_float4((float)cos(a), (float)cos(a), (float)sin(a), (float)sin(a));
  };
  for (int r = 1; r < 25; ++r)
    for (int m = 0; m < 25; ++m) p2[(r - 1) * 25 + m] = quad((double)((m * r) % 625), 625.0);
  for (int j = 0; j < kPT12; ++j) {
    const double a = -2.0 * M_PI * (double)j / 12500.0;
    p12[j] = make_float2((float)cos(a), (float)sin(a));
  }
  if (cudaMemcpyToSymbol(g_pw2, p2, sizeof(p2)) != cudaSuccess) return VFRB_ERR_CUDA;
  if (cudaMemcpyToSymbol(g_pw12, p12, sizeof(p12)) != cudaSuccess) return VFRB_ERR_CUDA;
  g_tw_ready[dev] = true;
  return VFRB_OK;
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(gsrc), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit_k1() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// a twiddle c + i s held as packed pairs (both lanes equal); ns = -s
struct Rot {
  float2 c, s, ns;
};
__device__ __forceinline__ Rot rot_of(float4 q) {
  return Rot{make_float2(q.x, q.y), make_float2(q.z, q.w), make_float2(-q.z, -q.w)};
}
__device__ __forceinline__ Rot rot_of2(float2 q) {
  return Rot{make_float2(q.x, q.x), make_float2(q.y, q.y), make_float2(-q.y, -q.y)};
}
__device__ __forceinline__ Rot rot_mul(const Rot& a, const Rot& b) {
  return Rot{f2fma(a.s, b.ns, f2mul(a.c, b.c)), f2fma(a.s, b.c, f2mul(a.c, b.s)), f2fma(a.ns, b.c, f2mul(a.c, b.ns))};
}
// v *= w, and v *= conj(w)
__device__ __forceinline__ void pp_mul(PolPair& v, const Rot& w) {
  const float2 re = f2fma(v.im, w.ns, f2mul(v.re, w.c));
  v.im = f2fma(v.re, w.s, f2mul(v.im, w.c));
  v.re = re;
}
__device__ __forceinline__ void pp_mulc(PolPair& v, const Rot& w) {
  const float2 re = f2fma(v.im, w.s, f2mul(v.re, w.c));
  v.im = f2fma(v.re, w.ns, f2mul(v.im, w.c));
  v.re = re;
}
__device__ __forceinline__ float4 pp_pack(const PolPair& v) { return make_float4(v.re.x, v.re.y, v.im.x, v.im.y); }
__device__ __forceinline__ PolPair pp_unpack(float4 q) { return PolPair{make_float2(q.x, q.y), make_float2(q.z, q.w)}; }

// A packed point word holds bytes (pol0 sample 2m, pol0 2m+1, pol1 2m,
// pol1 2m+1).  0x4B0000xx is the float 2^23 + xx; subtracting 2^23 + 128
// leaves xx - 128 exactly.
__device__ __forceinline__ PolPair pp_from_word(unsigned w) {
  const float2 off = f2s(-8388736.0f);
  const float2 re = make_float2(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7550)),
                                __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7552)));
  const float2 im = make_float2(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7551)),
                                __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7553)));
  return PolPair{f2add(re, off), f2add(im, off)};
}

// Stage the raw bytes of one 12500-sample window of both pols (stream
// positions pos0 ..) into st0 / st1.  ALIGNED (pos0 % 4 == 0, payloads at
// 4-byte offsets): 4-byte asynchronous copies, each inside one payload,
// zero-filled for fill frames (slot -1); otherwise synchronous byte loads.
// Positions outside the slot table and misaligned payloads set
// kErrSlotRange and read as zero bytes.
template <bool ALIGNED>
__device__ __forceinline__ void pp_stage(unsigned char* __restrict__ st0, unsigned char* __restrict__ st1,
                                         const vfrb_chan_args& a, long long pos0, int& err) {
  const int tid = (int)threadIdx.x - kStageT0;  // staging thread index
  if (tid < 0) return;
  if (ALIGNED) {
    // the window's bytes [0, 12500) start at payload offset off0 of slot
    // slot0 and cover up to 4 payload pieces; the pieces' slot entries are
    // loaded together, then each piece is copied from one source pointer
    const long long slot0 = pos0 >= 0 ? pos0 / kDataLen : -1;
    const int off0 = pos0 >= 0 ? (int)(pos0 - slot0 * kDataLen) : 0;
    long long sv0[4], sv1[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long slot = slot0 + q;
      const bool in = slot0 >= 0 && slot < a.nslots && q * kDataLen - off0 < kFftN;
      sv0[q] = in ? __ldg(a.slots0 + slot) : -1;
      sv1[q] = in ? __ldg(a.slots1 + slot) : -1;
      if (!in && q * kDataLen - off0 < kFftN) err |= kErrSlotRange;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int lo = max(0, q * kDataLen - off0), hi = min(kFftN, (q + 1) * kDataLen - off0);
      long long s0 = sv0[q], s1 = sv1[q];
      if ((s0 >= 0 && (s0 & 3)) || (s1 >= 0 && (s1 & 3))) {  // payloads must start on a 4-byte boundary
        err |= kErrSlotRange;
        s0 = s1 = -1;
      }
      // window byte n of this piece is payload byte n + off0 - q * kDataLen
      const long long d = (long long)off0 - (long long)q * kDataLen;
      const int n0 = s0 >= 0 ? 4 : 0, n1 = s1 >= 0 ? 4 : 0;  // source bytes (0: zero fill)
      const int glo = lo / 4, ghi = hi / 4;
      int g = glo + ((tid - glo) % kStageThreads + kStageThreads) % kStageThreads;
      const unsigned char* q0 = s0 >= 0 ? a.frames + s0 + d + 4LL * g : a.frames;
      const unsigned char* q1 = s1 >= 0 ? a.frames + s1 + d + 4LL * g : a.frames;
      const int m0 = n0 * kStageThreads, m1 = n1 * kStageThreads;  // source step per copy (0 when zero filling)
      for (; g < ghi; g += kStageThreads) {
        cp_async4(st0 + 4 * g, q0, n0);
        cp_async4(st1 + 4 * g, q1, n1);
        q0 += m0;
        q1 += m1;
      }
    }
  } else {
    for (int n = tid; n < kFftN; n += kStageThreads) {
      const long long pos = pos0 + n;
      const long long slot = pos >= 0 ? pos / kDataLen : -1;
      unsigned char v0 = 0, v1 = 0;
      if (slot < 0 || slot >= a.nslots) {
        err |= kErrSlotRange;
      } else {
        const int off = (int)(pos - slot * kDataLen);
        const long long s0 = __ldg(a.slots0 + slot), s1 = __ldg(a.slots1 + slot);
        if (s0 >= 0) v0 = __ldg(a.frames + s0 + off);
        if (s1 >= 0) v1 = __ldg(a.frames + s1 + off);
      }
      st0[n] = v0;
      st1[n] = v1;
    }
  }
}

// Power of the pol pair into output channel bin - nskip: the first window of
// a row stores, later ones add (same-thread, same-address order keeps the
// store first)
__device__ __forceinline__ void pp_emit(float* dst, int bin, int nskip, int nchanout, bool first, float p) {
  const int c = bin - nskip;
  if ((unsigned)c < (unsigned)nchanout) {
    if (first)
      dst[c] = p;
    else
      atomicAdd(dst + c, p);  // result unused: a reduction, nothing waits for it
  }
}

// Pass 3 (radix 10, Ns = 625) of butterfly j and its mirror 625 - j, the
// real split and detection.  j = 0 is its own mirror.  t12[m] = W_12500^m.
__device__ __forceinline__ void pp_pass3(const float4* __restrict__ Z, const float2* __restrict__ t12,
                                         const float4* __restrict__ kt, int j, float* dst, int nskip, int nchanout,
                                         bool first, float scale) {
  PolPair u[10], d[10];
  if (j == 0) {
#pragma unroll
    for (int r = 0; r < 10; ++r) u[r] = pp_unpack(Z[kPM3 * r]);
    dft10p(u, kt);
  } else {
    const Rot w1 = rot_of2(t12[2 * j]);  // W_6250^j
    Rot wr = w1;
    u[0] = pp_unpack(Z[j]);
    d[0] = pp_unpack(Z[kPM3 - j]);
#pragma unroll
    for (int r = 1; r < 10; ++r) {
      u[r] = pp_unpack(Z[j + kPM3 * r]);
      d[r] = pp_unpack(Z[kPM3 - j + kPM3 * r]);
      // butterfly 625 - j has twiddles W_6250^((625 - j) r) = W_10^r conj(W_6250^(j r));
      // the W_10^r factor only moves its outputs by one index (below)
      pp_mul(u[r], wr);
      pp_mulc(d[r], wr);
      if (r < 9) wr = rot_mul(wr, w1);
    }
    dft10p(u, kt);
    dft10p(d, kt);
  }
  const int kend = j == 0 ? 6 : 10;
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    if (k < kend) {
      const Rot wk = rot_of2(t12[j + kPM3 * k]);  // W_12500^(j + 625 k), j + 625 k < 6250
      // Z[k'] with k' = j + 625 k, and Z[H - k'] (butterfly 625 - j, output
      // 9 - k, which its twiddle shift leaves at index 10 - k)
      const PolPair zk = u[dft10p_pos(k)];
      const PolPair zm = j == 0 ? u[dft10p_pos((10 - k) % 10)] : d[dft10p_pos((10 - k) % 10)];
      const float2 ar = f2add(zk.re, zm.re), ai = f2sub(zk.im, zm.im);
      const float2 br = f2sub(zk.re, zm.re), bi = f2add(zk.im, zm.im);
      const float2 cr = f2fma(bi, wk.ns, f2mul(br, wk.c));
      const float2 ci = f2fma(br, wk.s, f2mul(bi, wk.c));
      // |A - iC|^2 and |A + iC|^2, summed over the two pols
      const float2 ur = f2add(ar, ci), ui = f2sub(ai, cr);
      const float2 vr = f2sub(ar, ci), vi = f2add(ai, cr);
      const float2 pu = f2fma(ur, ur, f2mul(ui, ui));
      const float2 pv = f2fma(vr, vr, f2mul(vi, vi));
      const int bin = j + kPM3 * k;
      pp_emit(dst, bin, nskip, nchanout, first, (pu.x + pu.y) * scale);
      if (bin != kH - bin) pp_emit(dst, kH - bin, nskip, nchanout, first, (pv.x + pv.y) * scale);
    }
  }
}

template <bool ALIGNED>
__global__ void __launch_bounds__(kPThreads, 1) k_channelise(const vfrb_chan_args a) {
  extern __shared__ float4 smem_f4[];
  float4* Z = smem_f4;
  float4* tw2 = smem_f4 + kH;
  float4* ktab = tw2 + kPTw2;  // codelet constants
  float2* t12 = reinterpret_cast<float2*>(ktab + kPairTable);
  unsigned char* stage = reinterpret_cast<unsigned char*>(t12 + kPT12);  // [2 buffers][2 pols][kStage]
  const int tid = threadIdx.x;
  int err = 0;
  for (int i = tid; i < kPTw2; i += kPThreads) tw2[i] = g_pw2[i];
  for (int i = tid; i < kPT12; i += kPThreads) t12[i] = g_pw12[i];
  if (tid < kPairTable) ktab[tid] = c_pair_table[tid];
  // the staging buffers' padding (never written by the copies) holds the
  // zero read below: 3 ints in each of the 4 pol buffers
  if (tid < 4 * ((kStage - kFftN) / 4)) {
    const int b = tid / ((kStage - kFftN) / 4), e = tid % ((kStage - kFftN) / 4);
    reinterpret_cast<int*>(stage + (size_t)b * kStage + kFftN)[e] = 0;
  }
  // NFREQ-normalised pol-summed power, averaged over NAVE (PIPE:1296, 1310);
  // |X|^2 = |A -+ iC|^2 / 4
  const float scale = 0.25f / ((float)a.nfreq * (float)a.nave);
  // persistent CTAs: this CTA's windows are (row, w) for rows
  // blockIdx.x + k*gridDim.x, w < NAVE, in that order (32-bit bookkeeping:
  // a launch has fewer than 2^31 rows)
  const int nrows_cta = (a.nrows - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const long long win0 = a.sample0 + (long long)blockIdx.x * a.nave * kFftN;  // first window of row blockIdx.x
  const long long row_step = (long long)gridDim.x * a.nave * kFftN;            // to the CTA's next row
  if (nrows_cta > 0) pp_stage<ALIGNED>(stage, stage + kStage, a, win0, err);
  cp_async_commit_k1();
  int w = 0, rk = 0, buf = 0;  // window within the row, row of this CTA, staging buffer
#pragma unroll 1
  while (rk < nrows_cta) {
    const int row = (int)blockIdx.x + rk * (int)gridDim.x;
    const int wn = w + 1 < a.nave ? w + 1 : 0, rn = w + 1 < a.nave ? rk : rk + 1;
    const unsigned char* cur = stage + (size_t)buf * 2 * kStage;
    unsigned char* nxt = stage + (size_t)(buf ^ 1) * 2 * kStage;
    // the next window's buffer was last read by pass 1 of the previous
    // window, which every thread has left (barriers after passes 1 and 2)
    if (rn < nrows_cta) pp_stage<ALIGNED>(nxt, nxt + kStage, a, win0 + rn * row_step + (long long)wn * kFftN, err);
    cp_async_commit_k1();
    cp_async_wait_1();  // this thread's copies of the current window have landed
    __syncthreads();    // ... and everybody else's; pass 3 of the previous window is done with Z
    // The tables' addresses, offset by a zero the compiler cannot see through
    // (the staging padding, read each window): their entries -- constants,
    // and twiddles fixed per thread -- are then read where used instead of
    // being kept in registers across the whole loop, which would not fit.
    const int z = *reinterpret_cast<const volatile int*>(cur + kFftN);
    const float4* kt = ktab + z;
    const float4* tw = tw2 + z;
    const float2* tj = t12 + z;
    if (tid < kPB) {  // pass 1: R = 25, Ns = 1, from the staged bytes
      PolPair v[25];
#pragma unroll
      for (int r = 0; r < 25; ++r) {
        const int o = 2 * (tid + kPB * r);
        const unsigned w0 = *reinterpret_cast<const unsigned short*>(cur + o);
        const unsigned w1 = *reinterpret_cast<const unsigned short*>(cur + kStage + o);
        v[r] = pp_from_word(__byte_perm(w0, w1, 0x5410));
      }
      dft25p(v, kt);
#pragma unroll
      for (int k = 0; k < 25; ++k) Z[tid * 25 + k] = pp_pack(v[dft25p_pos(k)]);
    }
    __syncthreads();
    {  // pass 2: R = 25, Ns = 25 (inputs held in registers across the barrier)
      PolPair v[25];
      const int m = tid % 25;
      if (tid < kPB) {
#pragma unroll
        for (int r = 0; r < 25; ++r) v[r] = pp_unpack(Z[tid + kPB * r]);
#pragma unroll
        for (int r = 1; r < 25; ++r) pp_mul(v[r], rot_of(tw[(r - 1) * 25 + m]));
        dft25p(v, kt);
      }
      __syncthreads();
      if (tid < kPB) {
        const int base = (tid / 25) * 625 + m;
#pragma unroll
        for (int k = 0; k < 25; ++k) Z[base + 25 * k] = pp_pack(v[dft25p_pos(k)]);
      }
    }
    __syncthreads();
    const unsigned long long orow = (unsigned long long)(a.out_row0 + row) & (unsigned long long)a.out_row_mask;
    float* dst = a.out + (long long)orow * a.out_row_stride;
    // pass 3: butterflies 1..312 and the cheap self-mirror butterfly 0, one
    // task each (threads 0..56 take a second one)
    for (int t = tid; t < kPTasks; t += kPThreads)
      pp_pass3(Z, tj, kt, t + 1 < kPTasks ? t + 1 : 0, dst, a.nskip, a.nchanout, w == 0, scale);
    w = wn;
    rk = rn;
    buf ^= 1;
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
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) {
    cudaGetLastError();
    nsm = 148;
  }
  // persistent: one CTA per SM, rows dealt round robin
  const int grid = (int)std::min<long long>(a.nrows, (long long)nsm);
  const bool aligned = (a.sample0 % 4) == 0;
  auto kern = aligned ? k_channelise<true> : k_channelise<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPSmem);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return VFRB_ERR_CUDA;
  }
  kern<<<grid, kPThreads, kPSmem, s>>>(a);
  return cuda_status(cudaGetLastError());
}

}  // namespace vfrb
