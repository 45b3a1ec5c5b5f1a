// Register-window dedispersion kernel (included by dedisperse.cu).
//
// Each thread owns D adjacent DM trials (a "group") x TT consecutive output
// samples.  For every channel it loads ONE window of TT + S samples from the
// shared-memory tile into registers with 16-byte loads (S = the largest
// delay difference inside its group for that channel, plus the 16-byte
// alignment residual) and adds it, shifted by each trial's delay
// difference, into D accumulator rows.  The shift depends only on the group
// and the channel, so it is warp-uniform: a switch over statically indexed
// cases keeps the window in registers, and one shared-memory word feeds up
// to D additions.  That lifts the kernel above the shared-memory bandwidth
// bound of a one-load-per-add kernel.
//
// Lanes own consecutive TT-sample runs with TT/VEC odd (VEC = elements per
// 16 bytes), so the 16-byte loads of each quarter warp hit distinct banks.
// The per-(group, channel) metadata -- window start in 16-byte units, the D
// shifts (8 bits each) and the number of 16-byte loads -- is computed while
// a chunk of channels is staged, and read back with one broadcast load.  The
// tile of the next chunk is staged with cp.async (16-byte, zero-filled past
// the valid rows) into the other half of a double buffer while the current
// chunk is summed.
//
// FP16 form: z = (P - mean)/S with one scale S per stream, accumulated in
// FP32 with the sm_100 mixed-precision add (add.rn.f32.f16), so no
// per-element conversion; the result is scaled by S at the end.
#pragma once

namespace vfrb {

constexpr int kRegWarps = 8;

struct DdRegParams {
  const void* fb;
  float out_scale;  // multiplies sum/nchan (1 for FP32, S for FP16)
  long long chan_stride;
  long long row0;
  unsigned row_mask;
  long long nrows_valid;
  int nchan;
  int ndm;
  int ngroups;
  long long nt_out;
  float* out;
  long long out_stride;
  DmPartial* part;
  const int* gbase;        // [ngroups][nchan] smallest delay of the group
  const unsigned* gpack;   // [ngroups][nchan] D delay differences, 8 bits each
  const int* bmin;         // [nblocks][nchan] smallest delay of a CTA's DM block
  int chunk;
  int lmax;                // tile row length (elements, multiple of 16 bytes)
  int* err;
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// acc += half value (FP32 accumulate, sm_100 mixed-precision add)
__device__ __forceinline__ float add_h(float acc, unsigned short h) {
  float r;
  asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(r) : "h"(h), "f"(acc));
  return r;
}

// Window storage: one 32-bit register holds PER elements (1 float or 2 halves).
template <typename T>
struct RegWin;
template <>
struct RegWin<float> {
  using W = float;
  static constexpr int VEC = 4;  // elements per 16 bytes
  static constexpr int PER = 1;  // elements per register
  template <int E, int NR>
  __device__ __forceinline__ static float add(float acc, const W (&w)[NR]) {
    return acc + w[E];
  }
};
template <>
struct RegWin<__half> {
  using W = unsigned;  // a half2 word, low half = earlier sample
  static constexpr int VEC = 8;
  static constexpr int PER = 2;
  template <int E, int NR>
  __device__ __forceinline__ static float add(float acc, const W (&w)[NR]) {
    unsigned short lo, hi;
    asm("mov.b32 {%0,%1}, %2;" : "=h"(lo), "=h"(hi) : "r"(w[E >> 1]));
    return add_h(acc, (E & 1) ? hi : lo);
  }
};

template <typename T, int S, int TT, int NR, int I = 0>
__device__ __forceinline__ void add_at(float (&acc)[TT], const typename RegWin<T>::W (&w)[NR]) {
  if constexpr (I < TT) {
    acc[I] = RegWin<T>::template add<I + S, NR>(acc[I], w);
    add_at<T, S, TT, NR, I + 1>(acc, w);
  }
}

#define VFRB_CASES_0_31(X)                                                                                     \
  X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) \
      X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31)

template <typename T, int TT, int NR>
__device__ __forceinline__ void add_shift(float (&acc)[TT], const typename RegWin<T>::W (&w)[NR], int s) {
  switch (s) {
#define VFRB_C(S)                                                                 \
  case S:                                                                         \
    if constexpr (S + TT <= NR * RegWin<T>::PER) add_at<T, S, TT, NR>(acc, w);    \
    break;
    VFRB_CASES_0_31(VFRB_C)
#undef VFRB_C
    default:
      break;
  }
}

template <typename T, int D, int TT, int SMAX>
struct RegCfg {
  static constexpr int VEC = RegWin<T>::VEC;
  static constexpr int SHMAX = SMAX + VEC - 1;                 // largest shift incl. alignment residual
  static constexpr int NQ = (TT + SHMAX + VEC - 1) / VEC;      // 16-byte loads per window
  static constexpr int NW = NQ * VEC;                          // window elements
  static constexpr int NR = NQ * 4;                            // window registers (32-bit)
  static constexpr int NT = 32 * TT;                           // output samples per CTA
  static constexpr int DB = kRegWarps * D;                     // DM trials per CTA
  static_assert(TT % VEC == 0 && ((TT / VEC) & 1) == 1, "lane stride must be an odd number of 16-byte units");
  static_assert(SHMAX <= 31, "switch covers shifts 0..31");
  static_assert(D <= 4, "shifts are packed in one 32-bit word");
};

template <typename T, int D, int TT, int SMAX>
__global__ void __launch_bounds__(kRegWarps * 32, 2) k_dedisp_reg(const DdRegParams p) {
  using Cfg = RegCfg<T, D, TT, SMAX>;
  using W = typename RegWin<T>::W;
  static_assert(sizeof(W) == 4, "window registers are 32-bit");
  constexpr int VEC = Cfg::VEC, NQ = Cfg::NQ, NR = Cfg::NR, NT = Cfg::NT;
  extern __shared__ int4 smr4[];
  const int CH = p.chunk, LM = p.lmax;
  const int LMQ = LM / VEC;  // tile row length in 16-byte units
  // shared layout: meta[2][W][CH] int4 {window start (16-byte units), shifts, loads, 0}, then tile[2][CH][LM]
  int4* meta = smr4;
  int4* tiles = smr4 + 2 * kRegWarps * CH;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long t0 = (long long)blockIdx.x * NT;
  const int blk = blockIdx.y;
  const int g0 = blk * kRegWarps;
  const T* fb = reinterpret_cast<const T*>(p.fb);
  const int nchunks = (p.nchan + CH - 1) / CH;
  int err = 0;

  auto stage = [&](int k, int b) {
    const int c0 = k * CH;
    const int nc = min(CH, p.nchan - c0);
    int4* mb = meta + b * kRegWarps * CH;
    for (int i = tid; i < kRegWarps * CH; i += kRegWarps * 32) {
      const int w = i / CH, cl = i - w * CH;
      const int g = min(g0 + w, p.ngroups - 1);
      const int c = c0 + min(cl, nc - 1);
      const long long a0 = (p.row0 + t0 + __ldg(p.bmin + (long long)blk * p.nchan + c)) & ~(long long)(VEC - 1);
      int rel = (int)(p.row0 + t0 + __ldg(p.gbase + (long long)g * p.nchan + c) - a0);
      const unsigned pk = __ldg(p.gpack + (long long)g * p.nchan + c);
      const int res = rel & (VEC - 1);
      unsigned sh = 0;
      int smx = 0;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const int s = min((int)((pk >> (8 * j)) & 0xFFu), SMAX) + res;
        sh |= (unsigned)s << (8 * j);
        smx = max(smx, s);
      }
      int q0 = rel / VEC;
      if (rel < 0 || (q0 + 31 * (TT / VEC) + NQ) > LMQ) {  // cannot happen with a consistent plan
        err |= kErrOffsetRange;
        q0 = 0;
      }
      mb[i] = make_int4(q0, (int)sh, (TT + smx + VEC - 1) / VEC, 0);
    }
    for (int cl = warp; cl < nc; cl += kRegWarps) {
      const long long a = (p.row0 + t0 + __ldg(p.bmin + (long long)blk * p.nchan + c0 + cl)) & ~(long long)(VEC - 1);
      const T* src = fb + (long long)(c0 + cl) * p.chan_stride;
      int4* dst = tiles + ((long long)b * CH + cl) * LMQ;
      const long long vend = p.row0 + p.nrows_valid;
      for (int v = lane; v < LMQ; v += 32) {
        const long long r = a + (long long)v * VEC;
        int bytes = 0;
        if (r >= 0 && r < vend) bytes = (int)(min((long long)VEC, vend - r) * (long long)sizeof(T));
        const unsigned long long rr = (unsigned long long)(bytes ? r : 0) & (unsigned long long)p.row_mask;
        cp_async16(dst + v, src + rr, bytes);
      }
    }
    cp_async_commit();
  };

  float acc[D][TT];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < TT; ++i) acc[j][i] = 0.f;

  stage(0, 0);
  for (int k = 0; k < nchunks; ++k) {
    cp_async_wait_all();
    __syncthreads();
    if (k + 1 < nchunks) stage(k + 1, (k + 1) & 1);
    const int b = k & 1;
    const int nc = min(CH, p.nchan - k * CH);
    const int4* mb = meta + (b * kRegWarps + warp) * CH;
    const int4* tile = tiles + (long long)b * CH * LMQ + lane * (TT / VEC);
#pragma unroll 1
    for (int cl = 0; cl < nc; ++cl) {
      const int4 m = mb[cl];
      const int4* q = tile + (long long)cl * LMQ + m.x;
      // the whole window, unconditionally: tile rows are padded so every
      // load stays inside the row, and no register keeps an old value
      W w[NR];
#pragma unroll
      for (int qi = 0; qi < NQ; ++qi) {
        const int4 v = q[qi];
        if constexpr (sizeof(W) == 4 && RegWin<T>::PER == 1) {
          w[4 * qi + 0] = __int_as_float(v.x);
          w[4 * qi + 1] = __int_as_float(v.y);
          w[4 * qi + 2] = __int_as_float(v.z);
          w[4 * qi + 3] = __int_as_float(v.w);
        } else {
          w[4 * qi + 0] = (W)v.x;
          w[4 * qi + 1] = (W)v.y;
          w[4 * qi + 2] = (W)v.z;
          w[4 * qi + 3] = (W)v.w;
        }
      }
#pragma unroll
      for (int j = 0; j < D; ++j) add_shift<T, TT, NR>(acc[j], w, (int)(((unsigned)m.y >> (8 * j)) & 0xFFu));
    }
  }

  // epilogue: out = sum / NCHANOUT (PIPE:1534) x scale; calcstats partials per (DM, time block)
  const float fs = p.out_scale / (float)p.nchan;
  const bool plain = p.out_scale == 1.f;
  const float fn = (float)p.nchan;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const int d = (g0 + warp) * D + j;
    if (d >= p.ndm) continue;  // warp-uniform
    double s = 0.0, s2 = 0.0;
    float mx = -INFINITY;
    int arg = 0x7fffffff;
    float* orow = p.out + (long long)d * p.out_stride;
#pragma unroll
    for (int i = 0; i < TT; ++i) {
      const long long t = t0 + (long long)lane * TT + i;
      if (t < p.nt_out) {
        const float val = plain ? acc[j][i] / fn : acc[j][i] * fs;
        orow[t] = val;
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
      DmPartial pq;
      pq.s = s;
      pq.s2 = s2;
      pq.mx = mx;
      pq.arg = arg;
      p.part[(long long)blockIdx.x * p.ndm + d] = pq;
    }
  }
  if (err && p.err) atomicOr(p.err, err);
}

}  // namespace vfrb
