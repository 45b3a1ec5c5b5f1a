// Generated by gen_dft.py -- do not edit by hand.
// In-register forward DFT codelets (W = exp(-2*pi*i/N)) for the channeliser.
#pragma once
#include <cuda_runtime.h>

namespace vfrb {

// forward DFT-5 in place: (a,b,c,d,e) <- X0..X4
__host__ __device__ __forceinline__ void dft5(float2& a, float2& b, float2& c, float2& d, float2& e) {
  const float c1 = 3.090169944e-01f, c2 = -8.090169944e-01f, s1 = 9.510565163e-01f, s2 = 5.877852523e-01f;
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

// forward DFT-25 = 5 x 5; X[k1 + 5*k2] ends in v[5*k1 + k2]
__host__ __device__ __forceinline__ void dft25(float2 (&v)[25]) {
  dft5(v[0], v[5], v[10], v[15], v[20]);
  dft5(v[1], v[6], v[11], v[16], v[21]);
  dft5(v[2], v[7], v[12], v[17], v[22]);
  dft5(v[3], v[8], v[13], v[18], v[23]);
  dft5(v[4], v[9], v[14], v[19], v[24]);
  { float xr = v[6].x, xi = v[6].y; v[6].x = fmaf(xr, 9.685831611e-01f, -xi * -2.486898872e-01f); v[6].y = fmaf(xr, -2.486898872e-01f, xi * 9.685831611e-01f); }
  { float xr = v[7].x, xi = v[7].y; v[7].x = fmaf(xr, 8.763066800e-01f, -xi * -4.817536741e-01f); v[7].y = fmaf(xr, -4.817536741e-01f, xi * 8.763066800e-01f); }
  { float xr = v[8].x, xi = v[8].y; v[8].x = fmaf(xr, 7.289686274e-01f, -xi * -6.845471059e-01f); v[8].y = fmaf(xr, -6.845471059e-01f, xi * 7.289686274e-01f); }
  { float xr = v[9].x, xi = v[9].y; v[9].x = fmaf(xr, 5.358267950e-01f, -xi * -8.443279255e-01f); v[9].y = fmaf(xr, -8.443279255e-01f, xi * 5.358267950e-01f); }
  { float xr = v[11].x, xi = v[11].y; v[11].x = fmaf(xr, 8.763066800e-01f, -xi * -4.817536741e-01f); v[11].y = fmaf(xr, -4.817536741e-01f, xi * 8.763066800e-01f); }
  { float xr = v[12].x, xi = v[12].y; v[12].x = fmaf(xr, 5.358267950e-01f, -xi * -8.443279255e-01f); v[12].y = fmaf(xr, -8.443279255e-01f, xi * 5.358267950e-01f); }
  { float xr = v[13].x, xi = v[13].y; v[13].x = fmaf(xr, 6.279051953e-02f, -xi * -9.980267284e-01f); v[13].y = fmaf(xr, -9.980267284e-01f, xi * 6.279051953e-02f); }
  { float xr = v[14].x, xi = v[14].y; v[14].x = fmaf(xr, -4.257792916e-01f, -xi * -9.048270525e-01f); v[14].y = fmaf(xr, -9.048270525e-01f, xi * -4.257792916e-01f); }
  { float xr = v[16].x, xi = v[16].y; v[16].x = fmaf(xr, 7.289686274e-01f, -xi * -6.845471059e-01f); v[16].y = fmaf(xr, -6.845471059e-01f, xi * 7.289686274e-01f); }
  { float xr = v[17].x, xi = v[17].y; v[17].x = fmaf(xr, 6.279051953e-02f, -xi * -9.980267284e-01f); v[17].y = fmaf(xr, -9.980267284e-01f, xi * 6.279051953e-02f); }
  { float xr = v[18].x, xi = v[18].y; v[18].x = fmaf(xr, -6.374239897e-01f, -xi * -7.705132428e-01f); v[18].y = fmaf(xr, -7.705132428e-01f, xi * -6.374239897e-01f); }
  { float xr = v[19].x, xi = v[19].y; v[19].x = fmaf(xr, -9.921147013e-01f, -xi * -1.253332336e-01f); v[19].y = fmaf(xr, -1.253332336e-01f, xi * -9.921147013e-01f); }
  { float xr = v[21].x, xi = v[21].y; v[21].x = fmaf(xr, 5.358267950e-01f, -xi * -8.443279255e-01f); v[21].y = fmaf(xr, -8.443279255e-01f, xi * 5.358267950e-01f); }
  { float xr = v[22].x, xi = v[22].y; v[22].x = fmaf(xr, -4.257792916e-01f, -xi * -9.048270525e-01f); v[22].y = fmaf(xr, -9.048270525e-01f, xi * -4.257792916e-01f); }
  { float xr = v[23].x, xi = v[23].y; v[23].x = fmaf(xr, -9.921147013e-01f, -xi * -1.253332336e-01f); v[23].y = fmaf(xr, -1.253332336e-01f, xi * -9.921147013e-01f); }
  { float xr = v[24].x, xi = v[24].y; v[24].x = fmaf(xr, -6.374239897e-01f, -xi * 7.705132428e-01f); v[24].y = fmaf(xr, 7.705132428e-01f, xi * -6.374239897e-01f); }
  dft5(v[0], v[1], v[2], v[3], v[4]);
  dft5(v[5], v[6], v[7], v[8], v[9]);
  dft5(v[10], v[11], v[12], v[13], v[14]);
  dft5(v[15], v[16], v[17], v[18], v[19]);
  dft5(v[20], v[21], v[22], v[23], v[24]);
}
// output index r of dft25 lives in v[dft25_pos(r)]
__host__ __device__ constexpr int dft25_pos(int r) { return 5 * (r % 5) + r / 5; }

// forward DFT-20 = 4 x 5; X[k1 + 4*k2] ends in v[5*k1 + k2]
__host__ __device__ __forceinline__ void dft20(float2 (&v)[20]) {
  dft4(v[0], v[5], v[10], v[15]);
  dft4(v[1], v[6], v[11], v[16]);
  dft4(v[2], v[7], v[12], v[17]);
  dft4(v[3], v[8], v[13], v[18]);
  dft4(v[4], v[9], v[14], v[19]);
  { float xr = v[6].x, xi = v[6].y; v[6].x = fmaf(xr, 9.510565163e-01f, -xi * -3.090169944e-01f); v[6].y = fmaf(xr, -3.090169944e-01f, xi * 9.510565163e-01f); }
  { float xr = v[7].x, xi = v[7].y; v[7].x = fmaf(xr, 8.090169944e-01f, -xi * -5.877852523e-01f); v[7].y = fmaf(xr, -5.877852523e-01f, xi * 8.090169944e-01f); }
  { float xr = v[8].x, xi = v[8].y; v[8].x = fmaf(xr, 5.877852523e-01f, -xi * -8.090169944e-01f); v[8].y = fmaf(xr, -8.090169944e-01f, xi * 5.877852523e-01f); }
  { float xr = v[9].x, xi = v[9].y; v[9].x = fmaf(xr, 3.090169944e-01f, -xi * -9.510565163e-01f); v[9].y = fmaf(xr, -9.510565163e-01f, xi * 3.090169944e-01f); }
  { float xr = v[11].x, xi = v[11].y; v[11].x = fmaf(xr, 8.090169944e-01f, -xi * -5.877852523e-01f); v[11].y = fmaf(xr, -5.877852523e-01f, xi * 8.090169944e-01f); }
  { float xr = v[12].x, xi = v[12].y; v[12].x = fmaf(xr, 3.090169944e-01f, -xi * -9.510565163e-01f); v[12].y = fmaf(xr, -9.510565163e-01f, xi * 3.090169944e-01f); }
  { float xr = v[13].x, xi = v[13].y; v[13].x = fmaf(xr, -3.090169944e-01f, -xi * -9.510565163e-01f); v[13].y = fmaf(xr, -9.510565163e-01f, xi * -3.090169944e-01f); }
  { float xr = v[14].x, xi = v[14].y; v[14].x = fmaf(xr, -8.090169944e-01f, -xi * -5.877852523e-01f); v[14].y = fmaf(xr, -5.877852523e-01f, xi * -8.090169944e-01f); }
  { float xr = v[16].x, xi = v[16].y; v[16].x = fmaf(xr, 5.877852523e-01f, -xi * -8.090169944e-01f); v[16].y = fmaf(xr, -8.090169944e-01f, xi * 5.877852523e-01f); }
  { float xr = v[17].x, xi = v[17].y; v[17].x = fmaf(xr, -3.090169944e-01f, -xi * -9.510565163e-01f); v[17].y = fmaf(xr, -9.510565163e-01f, xi * -3.090169944e-01f); }
  { float xr = v[18].x, xi = v[18].y; v[18].x = fmaf(xr, -9.510565163e-01f, -xi * -3.090169944e-01f); v[18].y = fmaf(xr, -3.090169944e-01f, xi * -9.510565163e-01f); }
  { float xr = v[19].x, xi = v[19].y; v[19].x = fmaf(xr, -8.090169944e-01f, -xi * 5.877852523e-01f); v[19].y = fmaf(xr, 5.877852523e-01f, xi * -8.090169944e-01f); }
  dft5(v[0], v[1], v[2], v[3], v[4]);
  dft5(v[5], v[6], v[7], v[8], v[9]);
  dft5(v[10], v[11], v[12], v[13], v[14]);
  dft5(v[15], v[16], v[17], v[18], v[19]);
}
// output index r of dft20 lives in v[dft20_pos(r)]
__host__ __device__ constexpr int dft20_pos(int r) { return 5 * (r % 4) + r / 4; }

}  // namespace vfrb
