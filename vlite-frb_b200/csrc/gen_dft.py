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


def main():
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
