#!/usr/bin/env python3
"""Build step: writes dft_pairs.cuh, the in-register DFT-2/-5/-10/-25
codelets of the channeliser's 6250-point pol-pair FFT.

The codelets follow the textbook Cooley-Tukey split of a length N = N1*N2 DFT
(inner DFTs of length N1 over n1, twiddles W_N^(n2*k1), outer DFTs of length
N2 over n2).  All constants are cos/sin of rational multiples of 2*pi computed
here in double precision and written as float literals; nothing is taken from
a library.  Output order: the value X[k1 + N1*k2] is left in v[N2*k1 + k2]
(the caller's stores undo the permutation at compile time).

Run:  python gen_dft.py > dft_pairs.cuh

The codelets work on a PolPair: one complex sample of each of the two
polarisations, held as re = (pol0, pol1) and im = (pol0, pol1) in two float2
registers, so every arithmetic step is one packed FP32 instruction
(add/sub/mul/fma .f32x2, sm_100) covering both pols.  Their constants come
from a small table the caller stages in shared memory.
"""
import math


def lit(x: float) -> str:
    if abs(x) < 1e-300:
        return "0.0f"
    return f"{x:.9e}f"


def w(e: int, n: int):
    a = -2.0 * math.pi * e / n
    return math.cos(a), math.sin(a)


PAIRS_HEADER = """// Generated by gen_dft.py -- do not edit by hand.
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
constexpr int kPairTable = NPAIRTABLE;
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
"""

PAIR_TW = []  # (c, s) of every twiddle the pair codelets use, in order


def pair_tw(c: float, sn: float) -> int:
    for i, t in enumerate(PAIR_TW):
        if abs(t[0] - c) < 1e-12 and abs(t[1] - sn) < 1e-12:
            return i
    PAIR_TW.append((c, sn))
    return len(PAIR_TW) - 1


def pair_codelet(n1: int, n2: int) -> str:
    n = n1 * n2
    inner = {5: "dft5p", 2: "dft2p"}[n1]
    outer = {5: "dft5p", 2: "dft2p"}[n2]
    s = f"\n// forward DFT-{n} = {n1} x {n2} on pol pairs; X[k1 + {n1}*k2] ends in v[{n2}*k1 + k2]\n"
    s += f"__device__ __forceinline__ void dft{n}p(PolPair (&v)[{n}], const float4* __restrict__ kt) {{\n"
    for q in range(n2):
        args = ", ".join(f"v[{n2 * i + q}]" for i in range(n1))
        s += f"  {inner}({args}, kt);\n"
    for k1 in range(n1):
        for q in range(n2):
            e = (q * k1) % n
            if e:
                c, sn = w(e, n)
                s += f"  pp_rot<{pair_tw(c, sn)}>(v[{n2 * k1 + q}], kt);  // W_{n}^{e}\n"
    for k1 in range(n1):
        args = ", ".join(f"v[{n2 * k1 + q}]" for q in range(n2))
        s += f"  {outer}({args}, kt);\n"
    s += "}\n"
    s += (f"// output index r of dft{n}p lives in v[dft{n}p_pos(r)]\n"
          f"__host__ __device__ constexpr int dft{n}p_pos(int r) {{ return {n2} * (r % {n1}) + r / {n1}; }}\n")
    return s


def main():
    c1 = math.cos(2 * math.pi / 5)
    c2 = math.cos(4 * math.pi / 5)
    s1 = math.sin(2 * math.pi / 5)
    s2 = math.sin(4 * math.pi / 5)
    body = pair_codelet(5, 5) + pair_codelet(2, 5)
    quads = [(c1, c2), (s1, s2), (-s1, 0.0)] + PAIR_TW
    out = PAIRS_HEADER.replace("NPAIRTABLE", str(len(quads)))
    out += body
    out += "\n// values of the constant table kt[]\n"
    out += "__constant__ float4 c_pair_table[kPairTable] = {\n"
    out += ",\n".join(f"    {{{lit(x)}, {lit(x)}, {lit(y)}, {lit(y)}}}" for x, y in quads)
    out += "};\n"
    out += "\n}  // namespace vfrb\n"
    print(out, end="")


if __name__ == "__main__":
    main()
