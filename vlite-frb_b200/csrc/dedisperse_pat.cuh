// Pattern-run dedispersion kernel (included by dedisperse.cu, after
// dedisperse_reg.cuh).
//
// Like the register-window kernel, each thread owns D adjacent DM trials (a
// "group") x TT consecutive output samples and, per channel, loads ONE window
// of TT + Delta_max samples from the shared-memory tile into registers and
// adds it at each trial's delay difference Delta_j, so one shared load feeds
// up to D additions.  The difference is how the shifts reach the code:
//
//  * windows are read with 4-byte (FP32) or 2-byte (FP16) loads at any
//    element offset, so there is no 16-byte alignment residual and the shift
//    of trial j is exactly Delta_j(group, channel);
//  * for equally spaced DM trials Delta_j = floor(phi + j*y) takes only a
//    few dozen distinct patterns (dedisp_patterns.cuh), so the kernel has
//    straight-line code per pattern;
//  * when a chunk of channels is staged, each warp sorts its channels by
//    pattern (warp match + prefix sum) into runs, and the summation loop
//    dispatches once per run instead of once per (trial, channel).
//
// Lanes own TT-sample runs with TT odd (FP32) or TT = 2 mod 4 (FP16), so the
// 32 lanes of a load touch 32 different banks.  Groups whose pattern is not
// in the table take a generic path (one dispatch per trial and channel).
//
// FP16 pair form (PAIR): the bandpass also writes the FP16 ring shifted by
// one row (fb1[c][r] = fb[c][r + 1]), and each staged channel row is copied
// from both rings.  With TT even, a window's start parity is the channel's
// (warp-uniform), so the window is read from the copy that puts its start on
// a 4-byte boundary: one 32-bit load per two halves, which halves both the
// shared-load instructions and the shared-memory wavefronts of the 2-byte
// loads (a warp's 2-byte load moves 64 bytes, its 4-byte load 128).  The
// adds, their order and the FP32 accumulation are those of the plain FP16
// form.
#pragma once

#include "dedisp_patterns.cuh"

namespace vfrb {

constexpr int kPatWarps = 8;  // warps per CTA of the two-CTAs-per-SM form (the other: 16, one CTA)
constexpr unsigned char kPatGeneric = 255;


struct DdPatParams {
  int njobs;                   // 0: one launch with the fields below; else jobs[blockIdx.z] overrides them
  DdJob jobs[kDdMaxJobs];
  const void* fb;
  const void* fb1;             // PAIR form: fb shifted by one row
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
  const int* gbase;            // [ngroups][nchan] smallest delay of the group
  const unsigned* gpack;       // [ngroups][nchan] D delay differences, 8 bits each
  const unsigned char* gpat;   // [ngroups][nchan] pattern id, kPatGeneric if none
  const int* bmin;             // [nblocks][nchan] smallest delay of a CTA's trials
  int chunk;                   // channels per stage (<= 32)
  int lmax;                    // tile row length in elements (multiple of 16 bytes)
  int* err;
};

template <typename T>
struct PatElem;
template <>
struct PatElem<float> {
  using R = float;
  __device__ __forceinline__ static R load(const float* p) { return *p; }
  __device__ __forceinline__ static float add(float a, R v) { return a + v; }
};
template <>
struct PatElem<__half> {
  using R = unsigned short;
  __device__ __forceinline__ static R load(const __half* p) { return *reinterpret_cast<const unsigned short*>(p); }
  __device__ __forceinline__ static float add(float a, R v) { return add_h(a, v); }
};

template <int A, int... R>
struct PatMax {
  static constexpr int v = A > PatMax<R...>::v ? A : PatMax<R...>::v;
};
template <int A>
struct PatMax<A> {
  static constexpr int v = A;
};

// acc[J + i][t] += w[t + S_i] for the trials J, J+1, ... with shifts S...
// FP32 with an even shift: the samples t, t + 1 (t even) and the window
// elements t + S, t + S + 1 are both register pairs, so one packed add
// (add.rn.f32x2, two independent round-to-nearest adds: the same results as
// two scalar adds) serves two samples.  An odd shift would pair elements
// across register pairs and stays scalar.
template <typename T, int D, int TT, int NW, int J, int S0, int... SR>
__device__ __forceinline__ void pat_add(float (&acc)[D][TT], const typename PatElem<T>::R (&w)[NW]) {
  if constexpr (sizeof(T) == 4 && (S0 & 1) == 0) {
#pragma unroll
    for (int t = 0; t + 1 < TT; t += 2) {
      const float2 r = __fadd2_rn(make_float2(acc[J][t], acc[J][t + 1]), make_float2(w[t + S0], w[t + S0 + 1]));
      acc[J][t] = r.x;
      acc[J][t + 1] = r.y;
    }
    if constexpr ((TT & 1) != 0) acc[J][TT - 1] = acc[J][TT - 1] + w[TT - 1 + S0];
  } else {
#pragma unroll
    for (int t = 0; t < TT; ++t) acc[J][t] = PatElem<T>::add(acc[J][t], w[t + S0]);
  }
  if constexpr (sizeof...(SR) > 0) pat_add<T, D, TT, NW, J + 1, SR...>(acc, w);
}

// n channels of one run: window loads + static-shift adds
template <typename T, int D, int TT, int... S>
__device__ __forceinline__ void pat_run(float (&acc)[D][TT], const T* tile, const int* slot, int n, int lane_off) {
  constexpr int NW = TT + PatMax<S...>::v;
  using R = typename PatElem<T>::R;
  // slot[n] (read ahead on the last channel) is the next entry of the same
  // shared table, in bounds and unused
  int sl = slot[0];
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const T* src = tile + sl + lane_off;
    sl = slot[i + 1];
    R w[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) w[k] = PatElem<T>::load(src + k);
    pat_add<T, D, TT, NW, 0, S...>(acc, w);
  }
}

// PAIR form: window element m is half (m & 1) of word w[m >> 1]; a
// register split (mov.b32 {lo, hi}) rather than shifts, so the halves can
// feed the mixed-precision adds directly
template <int NW2>
__device__ __forceinline__ void split_halves(const unsigned (&w)[NW2], unsigned short (&h)[2 * NW2]) {
#pragma unroll
  for (int k = 0; k < NW2; ++k) asm("mov.b32 {%0, %1}, %2;" : "=h"(h[2 * k]), "=h"(h[2 * k + 1]) : "r"(w[k]));
}
template <int D, int TT, int NH, int J, int S0, int... SR>
__device__ __forceinline__ void pat_add_pair(float (&acc)[D][TT], const unsigned short (&h)[NH]) {
#pragma unroll
  for (int t = 0; t < TT; ++t) acc[J][t] = add_h(acc[J][t], h[t + S0]);
  if constexpr (sizeof...(SR) > 0) pat_add_pair<D, TT, NH, J + 1, SR...>(acc, h);
}
// n channels of one run, PAIR form: slot entries are even element offsets
// into the copy that aligns the window
template <int D, int TT, int... S>
__device__ __forceinline__ void pat_run_pair(float (&acc)[D][TT], const __half* tile, const int* slot, int n,
                                             int lane_off) {
  constexpr int NW2 = (TT + PatMax<S...>::v + 1) / 2;
  int sl = slot[0];
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const unsigned* src = reinterpret_cast<const unsigned*>(tile + sl + lane_off);
    sl = slot[i + 1];
    unsigned w[NW2];
#pragma unroll
    for (int k = 0; k < NW2; ++k) w[k] = src[k];
    unsigned short h[2 * NW2];
    split_halves<NW2>(w, h);
    pat_add_pair<D, TT, 2 * NW2, 0, S...>(acc, h);
  }
}
template <int TT, int NH, int S>
__device__ __forceinline__ void pat_add_one_pair(float (&acc)[TT], const unsigned short (&h)[NH]) {
#pragma unroll
  for (int t = 0; t < TT; ++t) acc[t] = add_h(acc[t], h[t + S]);
}
template <int D, int TT, int SMAX>
__device__ __forceinline__ void pat_run_generic_pair(float (&acc)[D][TT], const __half* tile, const int* slot,
                                                     const unsigned* pk, int n, int lane_off) {
  constexpr int NW2 = (TT + SMAX + 1) / 2;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const unsigned* src = reinterpret_cast<const unsigned*>(tile + slot[i] + lane_off);
    unsigned w[NW2];
#pragma unroll
    for (int k = 0; k < NW2; ++k) w[k] = src[k];
    unsigned short h[2 * NW2];
    split_halves<NW2>(w, h);
    const unsigned sh = pk[i];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      switch ((int)((sh >> (8 * j)) & 0xFFu)) {
#define VFRB_G(S)                                                          \
  case S:                                                                  \
    if constexpr (S <= SMAX) pat_add_one_pair<TT, 2 * NW2, S>(acc[j], h);  \
    break;
        VFRB_CASES_0_31(VFRB_G)
#undef VFRB_G
        default:
          break;
      }
    }
  }
}

template <typename T, int TT, int NW, int S>
__device__ __forceinline__ void pat_add_one(float (&acc)[TT], const typename PatElem<T>::R (&w)[NW]) {
#pragma unroll
  for (int t = 0; t < TT; ++t) acc[t] = PatElem<T>::add(acc[t], w[t + S]);
}

// generic path: per channel, one dispatch per trial on its shift
template <typename T, int D, int TT, int SMAX>
__device__ __forceinline__ void pat_run_generic(float (&acc)[D][TT], const T* tile, const int* slot, const unsigned* pk,
                                             int n, int lane_off) {
  constexpr int NW = TT + SMAX;
  using R = typename PatElem<T>::R;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const T* src = tile + slot[i] + lane_off;
    R w[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) w[k] = PatElem<T>::load(src + k);
    const unsigned sh = pk[i];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      switch ((int)((sh >> (8 * j)) & 0xFFu)) {
#define VFRB_G(S)                                                       \
  case S:                                                               \
    if constexpr (S <= SMAX) pat_add_one<T, TT, NW, S>(acc[j], w);      \
    break;
        VFRB_CASES_0_31(VFRB_G)
#undef VFRB_G
        default:
          break;
      }
    }
  }
}

template <typename T, int D, int TT, int SMAX, bool PAIR = false>
__device__ __forceinline__ void pat_dispatch(float (&acc)[D][TT], int pat, const T* tile, const int* slot,
                                             const unsigned* pk, int n, int lane_off) {
  if constexpr (PAIR) {
    static_assert(sizeof(T) == 2 && D == 4, "pair form: FP16, four trials");
    switch (pat) {
#define VFRB_P4(ID, A, B, C)                                                                  \
  case ID:                                                                                    \
    if constexpr (PatMax<A, B, C>::v <= SMAX) pat_run_pair<D, TT, 0, A, B, C>(acc, tile, slot, n, lane_off); \
    return;
      VFRB_PAT4_LIST(VFRB_P4)
#undef VFRB_P4
      default:
        break;
    }
    pat_run_generic_pair<D, TT, SMAX>(acc, tile, slot, pk, n, lane_off);
    return;
  } else if constexpr (D == 4) {
    switch (pat) {
#define VFRB_P4(ID, A, B, C)                                                           \
  case ID:                                                                             \
    if constexpr (PatMax<A, B, C>::v <= SMAX) pat_run<T, D, TT, 0, A, B, C>(acc, tile, slot, n, lane_off); \
    return;
      VFRB_PAT4_LIST(VFRB_P4)
#undef VFRB_P4
      default:
        break;
    }
  } else if constexpr (D == 2) {
    switch (pat) {
#define VFRB_P2(ID, A)                                                               \
  case ID:                                                                           \
    if constexpr (A <= SMAX) pat_run<T, D, TT, 0, A>(acc, tile, slot, n, lane_off);  \
    return;
      VFRB_PAT2_LIST(VFRB_P2)
#undef VFRB_P2
      default:
        break;
    }
  }
  pat_run_generic<T, D, TT, SMAX>(acc, tile, slot, pk, n, lane_off);
}

// mbarrier and bulk-copy helpers (sm_90+ PTX; no multicast)
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Waits for the barrier phase with the given parity; gives up (false) after
// a bounded number of polls instead of spinning for ever.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  const unsigned a = smem_u32(bar);
  for (int i = 0; i < (1 << 22); ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// bytes from global to this CTA's shared memory, completing on `bar` (16-byte
// aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// W warps per CTA: 8 (two CTAs per SM, ~110 KB of tiles each) or 16 (one
// CTA per SM sharing ~220 KB of tiles between twice as many DM trials).
// PAIR: the FP16 pair form (two staged copies of each row, 4-byte loads).
template <typename T, int D, int TT, int SMAX, int W, bool PAIR = false>
__global__ void __launch_bounds__(W * 32, 16 / W) k_dedisp_pat(const DdPatParams pp) {
  // a batched launch: this CTA's stream's fields from its job
  DdPatParams p;
  p.fb = pp.fb;
  p.fb1 = pp.fb1;
  p.out_scale = pp.out_scale;
  p.row0 = pp.row0;
  p.nrows_valid = pp.nrows_valid;
  p.nt_out = pp.nt_out;
  p.out = pp.out;
  p.out_stride = pp.out_stride;
  p.err = pp.err;
  p.part = pp.part;
  if (pp.njobs > 0) {
    const DdJob& j = pp.jobs[blockIdx.z];
    p.fb = j.fb;
    p.fb1 = j.fb1;
    p.out_scale = j.out_scale;
    p.row0 = j.row0;
    p.nrows_valid = j.nrows_valid;
    p.nt_out = j.nt_out;
    p.out = j.out;
    p.out_stride = j.out_stride;
    p.err = j.err;
    p.part = nullptr;  // batched launches are stream mode: statistics come from the series
  }
  p.chan_stride = pp.chan_stride;
  p.row_mask = pp.row_mask;
  p.nchan = pp.nchan;
  p.ndm = pp.ndm;
  p.ngroups = pp.ngroups;
  p.gbase = pp.gbase;
  p.gpack = pp.gpack;
  p.gpat = pp.gpat;
  p.bmin = pp.bmin;
  p.chunk = pp.chunk;
  p.lmax = pp.lmax;
  constexpr int VEC = 16 / (int)sizeof(T);
  constexpr int NT = 32 * TT;
  static_assert(sizeof(T) == 4 ? (TT & 1) == 1 : (TT & 3) == 2, "lane stride must spread loads over all banks");
  static_assert(!PAIR || (sizeof(T) == 2 && D == 4), "pair form: FP16, four trials");
  constexpr int NCOPY = PAIR ? 2 : 1;  // staged copies of each row: the row, and (PAIR) the row shifted by one
  extern __shared__ int4 smp4[];
  const int CH = p.chunk, LM = p.lmax;
  const int LMQ = LM / VEC;
  // shared layout: full[2] mbarriers (16 B) | slot[W][CH] int | pk[W][CH] unsigned | run[W][CH] int | nrun[W] int
  //                | tiles[2][NCOPY][CH][LM] (16-byte aligned)
  unsigned long long* s_full = reinterpret_cast<unsigned long long*>(smp4);
  int* s_slot = reinterpret_cast<int*>(smp4 + 1);
  unsigned* s_pk = reinterpret_cast<unsigned*>(s_slot + W * CH);
  int* s_run = reinterpret_cast<int*>(s_pk + W * CH);
  int* s_nrun = s_run + W * CH;
  const int meta_q = 1 + (3 * W * CH + W + 3) / 4;
  int4* tiles = smp4 + meta_q;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // DM blocks run along x (fastest); along y, DM block b takes time block
  // y - shift_b, shift_b = its smallest delay at the middle channel in time
  // blocks.  The CTAs resident together then read about the same rows of the
  // middle channels (the rows a DM block needs move with its delay), which
  // keeps the wave's working set near the L2 size; CTAs whose time block
  // falls outside the output return at once.
  const int blk = blockIdx.x;
  const int tb = (int)blockIdx.y - __ldg(p.bmin + (long long)blk * p.nchan + p.nchan / 2) / NT;
  if (tb < 0 || (long long)tb * NT >= p.nt_out) return;
  const long long t0 = (long long)tb * NT;
  const int g = min(blk * W + warp, p.ngroups - 1);
  const T* fb = reinterpret_cast<const T*>(p.fb);
  const T* fb1 = reinterpret_cast<const T*>(p.fb1);  // PAIR: fb1[c][r] = fb[c][r + 1]
  const int nchunks = (p.nchan + CH - 1) / CH;
  const long long vend = p.row0 + p.nrows_valid;
  const unsigned long long rmask = (unsigned long long)p.row_mask;
  int err = 0;
  if (tid == 0) {
    mbar_init(&s_full[0], W);
    mbar_init(&s_full[1], W);
    mbar_fence_init();
  }
  __syncthreads();

  // Staging, shared by the W warps: warp w copies its ceil(CH/W)
  // channels of chunk k into tile buffer b.  A channel's rows [a, a + LM) go
  // in one bulk asynchronous copy when they are all valid (two when they
  // wrap the ring: the split is at the ring end, a multiple of 16 bytes);
  // otherwise the warp copies them itself, with zeros outside
  // [0, row0 + nrows_valid), before announcing its bulk bytes.  Each warp
  // arrives once per buffer phase, so the barrier counts W arrivals.
  const int per = (CH + W - 1) / W;
  // bmin of this lane's staging channel of chunk k (loaded ahead of use)
  auto stage_bmin = [&](int k) -> int {
    if (k >= nchunks) return 0;
    const int c0 = k * CH;
    const int cb = warp * per;
    const int cn = max(0, min(per, min(CH, p.nchan - c0) - cb));
    return lane < cn ? __ldg(p.bmin + (long long)blk * p.nchan + c0 + cb + lane) : 0;
  };
  auto stage = [&](int k, int b, int sbmin) {
    const int c0 = k * CH;
    const int nc = min(CH, p.nchan - c0);
    const int cb = warp * per;                 // this warp's first channel of the chunk
    const int cn = max(0, min(per, nc - cb));  // and how many
    long long a = 0;
    unsigned long long ra = 0;
    int n1 = LM;  // rows before the ring end
    bool bulk = false;
    if (lane < cn) {
      a = (p.row0 + t0 + sbmin) & ~(long long)(VEC - 1);
      ra = (unsigned long long)a & rmask;
      bulk = a >= 0 && a + LM <= vend;
      if (ra + (unsigned long long)LM > rmask + 1ULL) n1 = (int)(rmask + 1ULL - ra);
    }
    unsigned slow = __ballot_sync(0xffffffffu, lane < cn && !bulk);
    while (slow) {
      const int cl = __ffs(slow) - 1;
      slow &= slow - 1;
      const long long ac = __shfl_sync(0xffffffffu, a, cl);
#pragma unroll
      for (int cp = 0; cp < NCOPY; ++cp) {
        // copy cp holds rows r + cp of the filterbank (read as row r of fb1 for cp = 1)
        const T* src = (cp ? fb1 : fb) + (long long)(c0 + cb + cl) * p.chan_stride;
        int4* dst = tiles + (((long long)b * NCOPY + cp) * CH + cb + cl) * LMQ;
        for (int v = lane; v < LMQ; v += 32) {
          const long long r = ac + (long long)v * VEC;
          int4 val = make_int4(0, 0, 0, 0);
          if (r + cp >= 0 && r + VEC + cp <= vend) {  // a VEC-aligned group never straddles the ring end
            val = *reinterpret_cast<const int4*>(src + ((unsigned long long)r & rmask));
          } else if (r + VEC + cp > 0 && r + cp < vend) {
            union {
              int4 u;
              T t[VEC];
            } tmp;
            tmp.u = make_int4(0, 0, 0, 0);
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
              const long long re = r + e;
              if (re + cp >= 0 && re + cp < vend) tmp.t[e] = src[(unsigned long long)re & rmask];
            }
            val = tmp.u;
          }
          dst[v] = val;
        }
      }
    }
    __syncwarp();
    const unsigned nbulk = __popc(__ballot_sync(0xffffffffu, bulk));
    fence_proxy_async_smem();  // earlier generic reads of this buffer before the async writes
    if (lane == 0) mbar_arrive_expect_tx(&s_full[b], nbulk * (unsigned)(NCOPY * LM * (int)sizeof(T)));
    __syncwarp();
    if (bulk) {
      // the shifted copy's last element (row a + LM of the filterbank) may
      // lie past the valid rows; no window reads it
#pragma unroll
      for (int cp = 0; cp < NCOPY; ++cp) {
        int4* dst = tiles + (((long long)b * NCOPY + cp) * CH + cb + lane) * LMQ;
        const T* src = (cp ? fb1 : fb) + (long long)(c0 + cb + lane) * p.chan_stride;
        bulk_g2s(dst, src + ra, (unsigned)(n1 * (int)sizeof(T)), &s_full[b]);
        if (n1 < LM) bulk_g2s(dst + n1 / VEC, src, (unsigned)((LM - n1) * (int)sizeof(T)), &s_full[b]);
      }
    }
  };

  // This warp's channels of chunk k, sorted into runs of one pattern.
  // The per-(group, channel) tables of chunk k for this lane's channel,
  // loaded one chunk ahead so that their global-load latency hides under the
  // previous chunk's sums.
  struct MetaIn {
    int bmin, gbase, pat;
    unsigned pk;
  };
  auto meta_in = [&](int k) -> MetaIn {
    MetaIn m{0, 0, 0, 0u};
    if (k < nchunks && lane < min(CH, p.nchan - k * CH)) {
      const int c = k * CH + lane;
      m.bmin = __ldg(p.bmin + (long long)blk * p.nchan + c);
      m.gbase = __ldg(p.gbase + (long long)g * p.nchan + c);
      m.pk = __ldg(p.gpack + (long long)g * p.nchan + c);
      m.pat = __ldg(p.gpat + (long long)g * p.nchan + c);
    }
    return m;
  };
  auto meta = [&](int k, const MetaIn& m) {
    const int c0 = k * CH;
    const int nc = min(CH, p.nchan - c0);
    int pat = 0x10000 + lane;  // inactive lanes: a pattern of their own
    int slot = 0;
    unsigned pk = 0;
    if (lane < nc) {
      const long long a0 = (p.row0 + t0 + m.bmin) & ~(long long)(VEC - 1);
      int rel = (int)(p.row0 + t0 + m.gbase - a0);
      if (rel < 0 || rel + NT + SMAX > LM) {  // cannot happen with a consistent plan
        err |= kErrOffsetRange;
        rel = 0;
      }
      slot = lane * LM + rel;
      if (PAIR) {  // the copy that puts the window's start (rel + lane * TT, TT even) on a 4-byte boundary
        const int par = rel & 1;
        slot += par * (CH * LM - 1);
      }
      pk = m.pk;
      pat = m.pat;
    }
    const unsigned same = __match_any_sync(0xffffffffu, pat);
    const int leader = __ffs(same) - 1;
    const bool lead = lane == leader && lane < nc;
    const int cnt = __popc(same);
    int incl = lead ? cnt : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int start_l = incl - (lead ? cnt : 0);
    const int start = __shfl_sync(0xffffffffu, start_l, leader);
    const unsigned below = (1u << lane) - 1u;
    const int rank = __popc(same & below);
    const int mb = warp * CH;
    const unsigned leads = __ballot_sync(0xffffffffu, lead);
    if (lane < nc) {
      s_slot[mb + start + rank] = slot;
      s_pk[mb + start + rank] = pk;
    }
    if (lead) s_run[mb + __popc(leads & below)] = (pat & 0xFF) | (start << 8) | (cnt << 16);
    if (lane == 0) s_nrun[warp] = __popc(leads);
    __syncwarp();
  };

  float acc[D][TT];
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int i = 0; i < TT; ++i) acc[j][i] = 0.f;

  stage(0, 0, stage_bmin(0));
  int sb_next = stage_bmin(1);
  MetaIn m_cur = meta_in(0);
  for (int k = 0; k < nchunks; ++k) {
    __syncthreads();  // every warp is done with chunk k-1: its buffer can be refilled
    if (k + 1 < nchunks) stage(k + 1, (k + 1) & 1, sb_next);
    sb_next = stage_bmin(k + 2);
    meta(k, m_cur);
    m_cur = meta_in(k + 1);
    if (!mbar_wait(&s_full[k & 1], (unsigned)(k >> 1) & 1u)) err |= kErrTimeout;
    const int b = k & 1;
    const T* tile = reinterpret_cast<const T*>(tiles + (long long)b * NCOPY * CH * LMQ);
    const int mb = warp * CH;
    const int nrun = s_nrun[warp];
#pragma unroll 1
    for (int r = 0; r < nrun; ++r) {
      const int rd = s_run[mb + r];
      const int s0 = (rd >> 8) & 0xFF;
      pat_dispatch<T, D, TT, SMAX, PAIR>(acc, rd & 0xFF, tile, s_slot + mb + s0, s_pk + mb + s0, rd >> 16, lane * TT);
    }
    __syncwarp();  // this warp's metadata is rewritten for the next chunk
  }

  // epilogue: out = sum / NCHANOUT (PIPE:1534) x scale; calcstats partials per (DM, time block)
  const float fs = p.out_scale / (float)p.nchan;
  const bool plain = p.out_scale == 1.f;
  const float fn = (float)p.nchan;
  const int gw = blk * W + warp;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const int d = gw * D + j;
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
      p.part[(long long)tb * p.ndm + d] = pq;
    }
  }
  if (err && p.err) atomicOr(p.err, err);
}

}  // namespace vfrb
