// Register-window dedispersion kernel (included by dedisperse.cu).
//
// Each thread owns D adjacent DM trials (a "group") x TT consecutive output
// samples.  For every channel it loads ONE window of TT + S samples from the
// shared-memory tile into registers (S = the largest delay difference inside
// its group for that channel) and adds it, shifted by each trial's delay
// difference, into D accumulator rows.  The shift is warp-uniform (it depends
// only on the group and the channel), so a switch over statically indexed
// cases keeps the window in registers: one shared-memory word feeds up to D
// additions, which is what lifts the kernel above the shared-memory
// bandwidth bound of a one-load-per-add kernel.
//
// Lanes own consecutive TT-sample runs; TT is odd for 4-byte words (FP32) and
// twice an odd number for FP16 (7 words), so the 32 window loads of a warp
// hit 32 different banks.  The tile of a chunk of channels is staged with
// cp.async (16-byte, zero-filled past the valid rows) into the other half of
// a double buffer while the current chunk is summed.
#pragma once

namespace vfrb {

constexpr int kRegWarps = 8;

struct DdRegParams {
  const void* fb;
  const float* chan_scale;
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
  int lmax;
  int* err;
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gsrc), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

template <int S, int TT, int NW, bool FMA>
__device__ __forceinline__ void add_at(float (&acc)[TT], const float (&w)[NW], float wc) {
#pragma unroll
  for (int i = 0; i < TT; ++i) {
    if (FMA) acc[i] = fmaf(wc, w[i + S], acc[i]);
    else acc[i] += w[i + S];
  }
}

#define VFRB_CASES_0_31(X)                                                                                     \
  X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) \
      X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31)

template <int TT, int NW, bool FMA>
__device__ __forceinline__ void add_shift(float (&acc)[TT], const float (&w)[NW], int s, float wc) {
  switch (s) {
#define VFRB_C(S)                                                  \
  case S:                                                          \
    if constexpr (S + TT <= NW) add_at<S, TT, NW, FMA>(acc, w, wc); \
    break;
    VFRB_CASES_0_31(VFRB_C)
#undef VFRB_C
    default:
      break;
  }
}

template <typename T, int D, int TT, int SMAX>
struct RegCfg {
  static constexpr bool HALF = sizeof(T) == 2;
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int NW = TT + SMAX + (HALF ? 2 : 0);  // window length in floats
  static constexpr int NT = 32 * TT;                     // output samples per CTA
  static constexpr int DB = kRegWarps * D;               // DM trials per CTA
  static_assert(NW <= 64, "window too long");
  static_assert(SMAX + (HALF ? 1 : 0) <= 31, "switch covers shifts 0..31");
};

template <typename T, int D, int TT, int SMAX>
__global__ void __launch_bounds__(kRegWarps * 32, 2) k_dedisp_reg(const DdRegParams p) {
  using Cfg = RegCfg<T, D, TT, SMAX>;
  constexpr bool HALF = Cfg::HALF;
  constexpr int VEC = Cfg::VEC, NW = Cfg::NW, NT = Cfg::NT;
  extern __shared__ float4 sm4[];
  const int CH = p.chunk, LM = p.lmax;
  // shared layout: meta[2] { int gb[W][CH]; unsigned gp[W][CH]; long long a0[CH] } then tile[2][CH][LM]
  const int meta_words = 2 * kRegWarps * CH + 2 * CH;  // 4-byte words per buffer
  int* meta = reinterpret_cast<int*>(sm4);
  T* tiles = reinterpret_cast<T*>(sm4 + (2 * meta_words * 4 + 15) / 16);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long t0 = (long long)blockIdx.x * NT;
  const int blk = blockIdx.y;
  const int g0 = blk * kRegWarps;
  const T* fb = reinterpret_cast<const T*>(p.fb);
  const int nchunks = (p.nchan + CH - 1) / CH;
  int err = 0;

  auto gbs = [&](int b) { return meta + b * meta_words; };
  auto gps = [&](int b) { return reinterpret_cast<unsigned*>(meta + b * meta_words + kRegWarps * CH); };
  auto a0s = [&](int b) { return reinterpret_cast<long long*>(meta + b * meta_words + 2 * kRegWarps * CH); };

  auto stage = [&](int k, int b) {
    const int c0 = k * CH;
    const int nc = min(CH, p.nchan - c0);
    int* gb = gbs(b);
    unsigned* gp = gps(b);
    long long* a0 = a0s(b);
    for (int i = tid; i < kRegWarps * CH; i += kRegWarps * 32) {
      const int w = i / CH, cl = i - w * CH;
      const int g = min(g0 + w, p.ngroups - 1);
      const int c = c0 + min(cl, nc - 1);
      gb[i] = __ldg(p.gbase + (long long)g * p.nchan + c);
      gp[i] = __ldg(p.gpack + (long long)g * p.nchan + c);
    }
    for (int cl = warp; cl < nc; cl += kRegWarps) {
      const long long a = (p.row0 + t0 + __ldg(p.bmin + (long long)blk * p.nchan + c0 + cl)) & ~(long long)(VEC - 1);
      if (lane == 0) a0[cl] = a;
      const T* src = fb + (long long)(c0 + cl) * p.chan_stride;
      T* dst = tiles + ((long long)b * CH + cl) * LM;
      const long long vend = p.row0 + p.nrows_valid;
      for (int v = lane; v < LM / VEC; v += 32) {
        const long long r = a + (long long)v * VEC;
        int bytes = 0;
        if (r >= 0 && r < vend) bytes = (int)(min((long long)VEC, vend - r) * (long long)sizeof(T));
        const unsigned long long rr = (unsigned long long)(bytes ? r : 0) & (unsigned long long)p.row_mask;
        cp_async16(dst + (long long)v * VEC, src + rr, bytes);
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
    const int c0 = k * CH;
    const int nc = min(CH, p.nchan - c0);
    const int* gb = gbs(b) + warp * CH;
    const unsigned* gp = gps(b) + warp * CH;
    const long long* a0 = a0s(b);
    const T* tile = tiles + (long long)b * CH * LM;
    for (int cl = 0; cl < nc; ++cl) {
      const unsigned pk = gp[cl];
      int sh[D];
      int smax = 0;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        sh[j] = min((int)((pk >> (8 * j)) & 0xFFu), SMAX);
        smax = max(smax, sh[j]);
      }
      int start = (int)(p.row0 + t0 + gb[cl] - a0[cl]);
      if (start < 0 || start + NT + NW > LM) {  // cannot happen with a consistent plan; never read outside the tile
        err |= kErrOffsetRange;
        start = min(max(start, 0), LM - NT - NW);
      }
      start += lane * TT;
      const T* trow = tile + (long long)cl * LM;
      float w[NW];
      float wc = 1.f;
      int par = 0;
      if constexpr (!HALF) {
#pragma unroll
        for (int i = 0; i < NW; ++i) w[i] = (i < TT + smax) ? trow[start + i] : 0.f;
      } else {
        wc = p.chan_scale[c0 + cl];
        par = start & 1;
        const __half2* hw = reinterpret_cast<const __half2*>(trow + (start - par));
        const int nwords = (TT + smax + par + 1) >> 1;
#pragma unroll
        for (int q = 0; q < NW / 2; ++q) {
          if (q < nwords) {
            const float2 f = __half22float2(hw[q]);
            w[2 * q] = f.x;
            w[2 * q + 1] = f.y;
          } else {
            w[2 * q] = 0.f;
            w[2 * q + 1] = 0.f;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < D; ++j) add_shift<TT, NW, HALF>(acc[j], w, sh[j] + par, wc);
    }
  }

  // epilogue: out = sum / NCHANOUT (PIPE:1534); calcstats partials per (DM, time block)
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
        const float val = acc[j][i] / fn;
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

}  // namespace vfrb
