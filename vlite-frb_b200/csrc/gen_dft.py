#!/usr/bin/env python3
"""Build step: writes dft_codelets.cuh, the in-register DFT-5/-4/-20/-25
codelets used by the channeliser's 12500-point FFT.

The codelets follow the textbook Cooley-Tukey split of a length N = N1*N2 DFT
(inner DFTs of length N1 over n1, twiddles W_N^(n2*k1), outer DFTs of length
N2 over n2).  All constants are cos/sin of rational multiples of 2*pi computed
here in double precision and written as float literals; nothing is taken from
a library.  Output order: the value X[k1 + N1*k2] is left in v[N2*k1 + k2]
(the caller's stores undo the permutation at compile time).

Run:  python gen_dft.py > dft_codelets.cuh
      python gen_dft.py --pairs > dft_pairs.cuh

--pairs writes the same codelets for a PolPair: one complex sample of each
of the two polarisations, held as re = (pol0, pol1) and im = (pol0, pol1)
in two float2 registers, so every arithmetic step is one packed FP32
instruction (add/sub/mul/fma .f32x2, sm_100) covering both pols.  Their
constants come from a small table the caller stages in shared memory.
"""
import math


def lit(x: float) -> str:
    if abs(x) < 1e-300:
        return "0.0f"
    return f"{x:.9e}f"


def w(e: int, n: int):
    a = -2.0 * math.pi * e / n
    return math.cos(a), math.sin(a)


def twiddle_line(var: str, e: int, n: int) -> str:
    """var *= W_n^e with trivial cases folded."""
    e %= n
    if e == 0:
        return ""
    if 4 * e == n:  # -i
        return f"  {{ float t = {var}.x; {var}.x = {var}.y; {var}.y = -t; }}\n"
    if 2 * e == n:
        return f"  {var}.x = -{var}.x; {var}.y = -{var}.y;\n"
    if 4 * e == 3 * n:  # +i
        return f"  {{ float t = {var}.x; {var}.x = -{var}.y; {var}.y = t; }}\n"
    c, s = w(e, n)
    return (f"  {{ float xr = {var}.x, xi = {var}.y;"
            f" {var}.x = fmaf(xr, {lit(c)}, -xi * {lit(s)});"
            f" {var}.y = fmaf(xr, {lit(s)}, xi * {lit(c)}); }}\n")


HEADER = """// Generated by gen_dft.py -- do not edit by hand.
// In-register forward DFT codelets (W = exp(-2*pi*i/N)) for the channeliser.
#pragma once
#include <cuda_runtime.h>

namespace vfrb {

// forward DFT-5 in place: (a,b,c,d,e) <- X0..X4
__host__ __device__ __forceinline__ void dft5(float2& a, float2& b, float2& c, float2& d, float2& e) {
  const float c1 = %s, c2 = %s, s1 = %s, s2 = %s;
  float t1r = b.x + e.x, t1i = b.y + e.y;
  float t2r = c.x + d.x, t2i = c.y + d.y;
  float t3r = b.x - e.x, t3i = b.y - e.y;
  float t4r = c.x - d.x, t4i = c.y - d.y;
  float x0r = a.x, x0i = a.y;
  float m1r = fmaf(c1, t1r, fmaf(c2, t2r, x0r)), m1i = fmaf(c1, t1i, fmaf(c2, t2i, x0i));
  float m2r = fmaf(c2, t1r, fmaf(c1, t2r, x0r)), m2i = fmaf(c2, t1i, fmaf(c1, t2i, x0i));
  float n1r = fmaf(s1, t3r, s2 * t4r), n1i = fmaf(s1, t3i, s2 * t4i);
  float n2r = fmaf(s2, t3r, -s1 * t4r), n2i = fmaf(s2, t3i, -s1 * t4i);
  a.x = x0r + t1r + t2r; a.y = x0i + t1i + t2i;
  // X1 = m1 - i*n1, X4 = m1 + i*n1, X2 = m2 - i*n2, X3 = m2 + i*n2
  b.x = m1r + n1i; b.y = m1i - n1r;
  e.x = m1r - n1i; e.y = m1i + n1r;
  c.x = m2r + n2i; c.y = m2i - n2r;
  d.x = m2r - n2i; d.y = m2i + n2r;
}

// forward DFT-4 in place
__host__ __device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d) {
  float s0r = a.x + c.x, s0i = a.y + c.y, d0r = a.x - c.x, d0i = a.y - c.y;
  float s1r = b.x + d.x, s1i = b.y + d.y, d1r = b.x - d.x, d1i = b.y - d.y;
  a.x = s0r + s1r; a.y = s0i + s1i;
  c.x = s0r - s1r; c.y = s0i - s1i;
  b.x = d0r + d1i; b.y = d0i - d1r;   // d0 - i*d1
  d.x = d0r - d1i; d.y = d0i + d1r;   // d0 + i*d1
}
"""


def codelet(n1: int, n2: int) -> str:
    n = n1 * n2
    inner = "dft5" if n1 == 5 else "dft4"
    outer = "dft5" if n2 == 5 else "dft4"
    s = f"\n// forward DFT-{n} = {n1} x {n2}; X[k1 + {n1}*k2] ends in v[{n2}*k1 + k2]\n"
    s += f"__host__ __device__ __forceinline__ void dft{n}(float2 (&v)[{n}]) {{\n"
    for q in range(n2):  # inner DFTs over n1 of x[n2*n1 + q]
        args = ", ".join(f"v[{n2 * i + q}]" for i in range(n1))
        s += f"  {inner}({args});\n"
    for k1 in range(n1):
        for q in range(n2):
            s += twiddle_line(f"v[{n2 * k1 + q}]", q * k1, n)
    for k1 in range(n1):
        args = ", ".join(f"v[{n2 * k1 + q}]" for q in range(n2))
        s += f"  {outer}({args});\n"
    s += "}\n"
    s += (f"// output index r of dft{n} lives in v[dft{n}_pos(r)]\n"
          f"__host__ __device__ constexpr int dft{n}_pos(int r) {{ return {n2} * (r % {n1}) + r / {n1}; }}\n")
    return s


PAIRS_HEADER = """// Generated by gen_dft.py --pairs -- do not edit by hand.
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


def main_pairs():
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


def main():
    import sys
    if "--pairs" in sys.argv[1:]:
        return main_pairs()
    c1 = math.cos(2 * math.pi / 5)
    c2 = math.cos(4 * math.pi / 5)
    s1 = math.sin(2 * math.pi / 5)
    s2 = math.sin(4 * math.pi / 5)
    out = HEADER % (lit(c1), lit(c2), lit(s1), lit(s2))
    out += codelet(5, 5)
    out += codelet(4, 5)
    out += "\n}  // namespace vfrb\n"
    print(out, end="")


if __name__ == "__main__":
    main()
