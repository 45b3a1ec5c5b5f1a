// Generated by gen_dft.py -- do not edit by hand.
// Forward DFT codelets (W = exp(-2*pi*i/N)) on pairs of polarisations: a
// PolPair holds one complex sample of pol 0 and pol 1 as re = (re0, re1),
// im = (im0, im1), so each step is one packed FP32 instruction (sm_100).
// This header is included by one .cu file only.
#pragma once
#include <cuda_runtime.h>

namespace vfrb {

struct PolPair {
  float2 re, im;
};

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  unsigned long long x, y, d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(y) : "f"(b.x), "f"(b.y));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(d));
  return r;
}
__device__ __forceinline__ float2 f2s(float c) { return make_float2(c, c); }

// Constants of the codelets, as float4 (x, x, y, y) pairs in a table the
// caller stages in shared memory (kPairTable entries, values in
// c_pair_table below) and passes as `kt`:
//   kt[0] = (c1, c1, c2, c2), kt[1] = (s1, s1, s2, s2), kt[2] = (-s1, -s1, 0, 0)
// (the DFT-5 constants), then kt[3 + k] = (c, c, s, s) of twiddle k.
// Reading them from memory where used keeps them out of registers between
// uses (in a persistent loop every constant would otherwise stay live).
constexpr int kPairTable = 16;
__device__ __forceinline__ float2 lo2(float4 q) { return make_float2(q.x, q.y); }
__device__ __forceinline__ float2 hi2(float4 q) { return make_float2(q.z, q.w); }

// v *= c + i*s, the same rotation for both pols: twiddle K of the table
template <int K>
__device__ __forceinline__ void pp_rot(PolPair& v, const float4* __restrict__ kt) {
  const float4 q = kt[3 + K];
  const float2 c = lo2(q), s = hi2(q);
  const float2 re = f2fma(v.im, make_float2(-s.x, -s.y), f2mul(v.re, c));
  const float2 im = f2fma(v.re, s, f2mul(v.im, c));
  v.re = re;
  v.im = im;
}

// forward DFT-2 in place
__device__ __forceinline__ void dft2p(PolPair& a, PolPair& b, const float4* __restrict__) {
  const PolPair s{f2add(a.re, b.re), f2add(a.im, b.im)};
  b = PolPair{f2sub(a.re, b.re), f2sub(a.im, b.im)};
  a = s;
}

// forward DFT-5 in place: (a,b,c,d,e) <- X0..X4
__device__ __forceinline__ void dft5p(PolPair& a, PolPair& b, PolPair& c, PolPair& d, PolPair& e,
                                      const float4* __restrict__ kt) {
  const float4 k0 = kt[0], k1 = kt[1], k2 = kt[2];
  const float2 c1 = lo2(k0), c2 = hi2(k0), s1 = lo2(k1), s2 = hi2(k1), ns1 = lo2(k2);
  const float2 t1r = f2add(b.re, e.re), t1i = f2add(b.im, e.im);
  const float2 t2r = f2add(c.re, d.re), t2i = f2add(c.im, d.im);
  const float2 t3r = f2sub(b.re, e.re), t3i = f2sub(b.im, e.im);
  const float2 t4r = f2sub(c.re, d.re), t4i = f2sub(c.im, d.im);
  const float2 m1r = f2fma(c1, t1r, f2fma(c2, t2r, a.re)), m1i = f2fma(c1, t1i, f2fma(c2, t2i, a.im));
  const float2 m2r = f2fma(c2, t1r, f2fma(c1, t2r, a.re)), m2i = f2fma(c2, t1i, f2fma(c1, t2i, a.im));
  const float2 n1r = f2fma(s1, t3r, f2mul(s2, t4r)), n1i = f2fma(s1, t3i, f2mul(s2, t4i));
  const float2 n2r = f2fma(s2, t3r, f2mul(ns1, t4r)), n2i = f2fma(s2, t3i, f2mul(ns1, t4i));
  a.re = f2add(a.re, f2add(t1r, t2r));
  a.im = f2add(a.im, f2add(t1i, t2i));
  // X1 = m1 - i*n1, X4 = m1 + i*n1, X2 = m2 - i*n2, X3 = m2 + i*n2
  b = PolPair{f2add(m1r, n1i), f2sub(m1i, n1r)};
  e = PolPair{f2sub(m1r, n1i), f2add(m1i, n1r)};
  c = PolPair{f2add(m2r, n2i), f2sub(m2i, n2r)};
  d = PolPair{f2sub(m2r, n2i), f2add(m2i, n2r)};
}

// forward DFT-25 = 5 x 5 on pol pairs; X[k1 + 5*k2] ends in v[5*k1 + k2]
__device__ __forceinline__ void dft25p(PolPair (&v)[25], const float4* __restrict__ kt) {
  dft5p(v[0], v[5], v[10], v[15], v[20], kt);
  dft5p(v[1], v[6], v[11], v[16], v[21], kt);
  dft5p(v[2], v[7], v[12], v[17], v[22], kt);
  dft5p(v[3], v[8], v[13], v[18], v[23], kt);
  dft5p(v[4], v[9], v[14], v[19], v[24], kt);
  pp_rot<0>(v[6], kt);  // W_25^1
  pp_rot<1>(v[7], kt);  // W_25^2
  pp_rot<2>(v[8], kt);  // W_25^3
  pp_rot<3>(v[9], kt);  // W_25^4
  pp_rot<1>(v[11], kt);  // W_25^2
  pp_rot<3>(v[12], kt);  // W_25^4
  pp_rot<4>(v[13], kt);  // W_25^6
  pp_rot<5>(v[14], kt);  // W_25^8
  pp_rot<2>(v[16], kt);  // W_25^3
  pp_rot<4>(v[17], kt);  // W_25^6
  pp_rot<6>(v[18], kt);  // W_25^9
  pp_rot<7>(v[19], kt);  // W_25^12
  pp_rot<3>(v[21], kt);  // W_25^4
  pp_rot<5>(v[22], kt);  // W_25^8
  pp_rot<7>(v[23], kt);  // W_25^12
  pp_rot<8>(v[24], kt);  // W_25^16
  dft5p(v[0], v[1], v[2], v[3], v[4], kt);
  dft5p(v[5], v[6], v[7], v[8], v[9], kt);
  dft5p(v[10], v[11], v[12], v[13], v[14], kt);
  dft5p(v[15], v[16], v[17], v[18], v[19], kt);
  dft5p(v[20], v[21], v[22], v[23], v[24], kt);
}
// output index r of dft25p lives in v[dft25p_pos(r)]
__host__ __device__ constexpr int dft25p_pos(int r) { return 5 * (r % 5) + r / 5; }

// forward DFT-10 = 2 x 5 on pol pairs; X[k1 + 2*k2] ends in v[5*k1 + k2]
__device__ __forceinline__ void dft10p(PolPair (&v)[10], const float4* __restrict__ kt) {
  dft2p(v[0], v[5], kt);
  dft2p(v[1], v[6], kt);
  dft2p(v[2], v[7], kt);
  dft2p(v[3], v[8], kt);
  dft2p(v[4], v[9], kt);
  pp_rot<9>(v[6], kt);  // W_10^1
  pp_rot<10>(v[7], kt);  // W_10^2
  pp_rot<11>(v[8], kt);  // W_10^3
  pp_rot<12>(v[9], kt);  // W_10^4
  dft5p(v[0], v[1], v[2], v[3], v[4], kt);
  dft5p(v[5], v[6], v[7], v[8], v[9], kt);
}
// output index r of dft10p lives in v[dft10p_pos(r)]
__host__ __device__ constexpr int dft10p_pos(int r) { return 5 * (r % 2) + r / 2; }

// values of the constant table kt[]
__constant__ float4 c_pair_table[kPairTable] = {
    {3.090169944e-01f, 3.090169944e-01f, -8.090169944e-01f, -8.090169944e-01f},
    {9.510565163e-01f, 9.510565163e-01f, 5.877852523e-01f, 5.877852523e-01f},
    {-9.510565163e-01f, -9.510565163e-01f, 0.0f, 0.0f},
    {9.685831611e-01f, 9.685831611e-01f, -2.486898872e-01f, -2.486898872e-01f},
    {8.763066800e-01f, 8.763066800e-01f, -4.817536741e-01f, -4.817536741e-01f},
    {7.289686274e-01f, 7.289686274e-01f, -6.845471059e-01f, -6.845471059e-01f},
    {5.358267950e-01f, 5.358267950e-01f, -8.443279255e-01f, -8.443279255e-01f},
    {6.279051953e-02f, 6.279051953e-02f, -9.980267284e-01f, -9.980267284e-01f},
    {-4.257792916e-01f, -4.257792916e-01f, -9.048270525e-01f, -9.048270525e-01f},
    {-6.374239897e-01f, -6.374239897e-01f, -7.705132428e-01f, -7.705132428e-01f},
    {-9.921147013e-01f, -9.921147013e-01f, -1.253332336e-01f, -1.253332336e-01f},
    {-6.374239897e-01f, -6.374239897e-01f, 7.705132428e-01f, 7.705132428e-01f},
    {8.090169944e-01f, 8.090169944e-01f, -5.877852523e-01f, -5.877852523e-01f},
    {3.090169944e-01f, 3.090169944e-01f, -9.510565163e-01f, -9.510565163e-01f},
    {-3.090169944e-01f, -3.090169944e-01f, -9.510565163e-01f, -9.510565163e-01f},
    {-8.090169944e-01f, -8.090169944e-01f, -5.877852523e-01f, -5.877852523e-01f}};

}  // namespace vfrb
