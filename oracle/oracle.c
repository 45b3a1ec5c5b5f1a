/*
 * C restatement of the vlite-frb hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Used by the tests as a fast checker at sizes numpy cannot reach, and by
 * bench.py as the timed CPU baseline.  Built twice by build_oracle.py:
 * liboracle64.so (REAL = double, the FP64 checker) and liboracle32.so
 * (REAL = float, the C++/OpenMP-style host transcription that is timed).
 * Each function cites the reference code it restates (PIPE =
 * vdifFILE2dedisp_PIPELINE.cu, STATS = vdifDADA2stats.cu, TS =
 * vdifDADA2timeseries.cu).  FFTW is not available, so the transform is a
 * project-written mixed-radix Stockham FFT; the two polarisations share one
 * complex transform (z = x0 + i x1, |X0_k|^2 + |X1_k|^2 = (|Z_k|^2 +
 * |Z_{N-k}|^2)/2, an exact identity).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif

typedef struct { REAL re, im; } cpx;

/* ---- mixed-radix Stockham FFT (radices 2..7 + generic) -------------------- */
typedef struct {
  int n, npass;
  int radix[32];
  cpx* tw;   /* per pass: R * Ns twiddles */
  int twoff[32];
  cpx* dm;   /* per pass: R x R DFT matrix (generic radices) */
  int dmoff[32];
} fftplan;

static int factorize(int n, int* r) {
  int k = 0;
  const int pref[] = {4, 5, 2, 3, 7};
  for (int i = 0; i < 5; ++i)
    while (n % pref[i] == 0) { r[k++] = pref[i]; n /= pref[i]; }
  for (int p = 11; n > 1; p += 2)
    while (n % p == 0) { r[k++] = p; n /= p; }
  return k;
}

static fftplan* plan_new(int n) {
  fftplan* p = (fftplan*)calloc(1, sizeof(fftplan));
  p->n = n;
  p->npass = factorize(n, p->radix);
  size_t tot = 0;
  int ns = 1;
  for (int i = 0; i < p->npass; ++i) { p->twoff[i] = (int)tot; tot += (size_t)(p->radix[i]) * ns; ns *= p->radix[i]; }
  p->tw = (cpx*)malloc(sizeof(cpx) * (tot + 1));
  size_t dtot = 0;
  for (int i = 0; i < p->npass; ++i) { p->dmoff[i] = (int)dtot; dtot += (size_t)p->radix[i] * p->radix[i]; }
  p->dm = (cpx*)malloc(sizeof(cpx) * (dtot + 1));
  for (int i = 0; i < p->npass; ++i) {
    const int R = p->radix[i];
    for (int u = 0; u < R; ++u)
      for (int r = 0; r < R; ++r) {
        const double a = -2.0 * M_PI * (double)((u * r) % R) / R;
        p->dm[p->dmoff[i] + u * R + r].re = (REAL)cos(a);
        p->dm[p->dmoff[i] + u * R + r].im = (REAL)sin(a);
      }
  }
  ns = 1;
  for (int i = 0; i < p->npass; ++i) {
    const int R = p->radix[i];
    for (int r = 0; r < R; ++r)
      for (int k = 0; k < ns; ++k) {
        const double a = -2.0 * M_PI * (double)r * k / ((double)ns * R);
        p->tw[p->twoff[i] + r * ns + k].re = (REAL)cos(a);
        p->tw[p->twoff[i] + r * ns + k].im = (REAL)sin(a);
      }
    ns *= R;
  }
  return p;
}

static void plan_free(fftplan* p) { if (p) { free(p->tw); free(p->dm); free(p); } }

/* forward transform of x (length n) using scratch y; result left in x */
static void fft(const fftplan* p, cpx* x, cpx* y) {
  const int n = p->n;
  int ns = 1;
  cpx* a = x; cpx* b = y;
  cpx v[64], w[64];
  for (int s = 0; s < p->npass; ++s) {
    const int R = p->radix[s], M = n / R;
    const cpx* tw = p->tw + p->twoff[s];
    for (int j = 0; j < M; ++j) {
      const int k = j % ns;
      for (int r = 0; r < R; ++r) {
        const cpx t = a[j + r * M], q = tw[r * ns + k];
        v[r].re = t.re * q.re - t.im * q.im;
        v[r].im = t.re * q.im + t.im * q.re;
      }
      if (R == 4) {
        const cpx s0 = {v[0].re + v[2].re, v[0].im + v[2].im}, d0 = {v[0].re - v[2].re, v[0].im - v[2].im};
        const cpx s1 = {v[1].re + v[3].re, v[1].im + v[3].im}, d1 = {v[1].re - v[3].re, v[1].im - v[3].im};
        w[0].re = s0.re + s1.re; w[0].im = s0.im + s1.im;
        w[2].re = s0.re - s1.re; w[2].im = s0.im - s1.im;
        w[1].re = d0.re + d1.im; w[1].im = d0.im - d1.re;
        w[3].re = d0.re - d1.im; w[3].im = d0.im + d1.re;
      } else if (R == 5) {
        const REAL c1 = (REAL)0.30901699437494745, c2 = (REAL)-0.8090169943749475;
        const REAL s1 = (REAL)0.9510565162951535, s2 = (REAL)0.5877852522924731;
        const REAL t1r = v[1].re + v[4].re, t1i = v[1].im + v[4].im, t2r = v[2].re + v[3].re, t2i = v[2].im + v[3].im;
        const REAL t3r = v[1].re - v[4].re, t3i = v[1].im - v[4].im, t4r = v[2].re - v[3].re, t4i = v[2].im - v[3].im;
        const REAL m1r = v[0].re + c1 * t1r + c2 * t2r, m1i = v[0].im + c1 * t1i + c2 * t2i;
        const REAL m2r = v[0].re + c2 * t1r + c1 * t2r, m2i = v[0].im + c2 * t1i + c1 * t2i;
        const REAL n1r = s1 * t3r + s2 * t4r, n1i = s1 * t3i + s2 * t4i;
        const REAL n2r = s2 * t3r - s1 * t4r, n2i = s2 * t3i - s1 * t4i;
        w[0].re = v[0].re + t1r + t2r; w[0].im = v[0].im + t1i + t2i;
        w[1].re = m1r + n1i; w[1].im = m1i - n1r;
        w[4].re = m1r - n1i; w[4].im = m1i + n1r;
        w[2].re = m2r + n2i; w[2].im = m2i - n2r;
        w[3].re = m2r - n2i; w[3].im = m2i + n2r;
      } else {
        const cpx* m = p->dm + p->dmoff[s];
        for (int u = 0; u < R; ++u) {
          REAL sr = 0, si = 0;
          for (int r = 0; r < R; ++r) {
            const cpx q = m[u * R + r];
            sr += v[r].re * q.re - v[r].im * q.im;
            si += v[r].re * q.im + v[r].im * q.re;
          }
          w[u].re = sr; w[u].im = si;
        }
      }
      const int base = (j / ns) * ns * R + k;
      for (int u = 0; u < R; ++u) b[base + u * ns] = w[u];
    }
    cpx* t = a; a = b; b = t;
    ns *= R;
  }
  if (a != x) memcpy(x, a, sizeof(cpx) * n);
}

/* ---- a5-a9: channeliser (PIPE:574-632, 1292-1322) ------------------------ */
/* out[nrows][nchanout], time-major; no -128 offset in the reference
 * (PIPE:1316) -- it only changes bin 0, which no channel uses, so it is
 * removed here for conditioning, as the GPU kernel does. */
int oc_channelise(const uint8_t* p0, const uint8_t* p1, int64_t nrows, int twonchan, int nave, int nfreq, int nskip,
                  int nchanout, REAL* out) {
  fftplan* pl = plan_new(twonchan);
  int bad = 0;
#pragma omp parallel
  {
    cpx* x = (cpx*)malloc(sizeof(cpx) * twonchan);
    cpx* y = (cpx*)malloc(sizeof(cpx) * twonchan);
    REAL* acc = (REAL*)malloc(sizeof(REAL) * nchanout);
    if (!x || !y || !acc) bad = 1;
#pragma omp for schedule(dynamic, 4)
    for (int64_t r = 0; r < nrows; ++r) {
      if (bad) continue;
      for (int c = 0; c < nchanout; ++c) acc[c] = 0;
      for (int w = 0; w < nave; ++w) {
        const int64_t s0 = (r * nave + w) * (int64_t)twonchan;
        for (int i = 0; i < twonchan; ++i) {
          x[i].re = (REAL)p0[s0 + i] - (REAL)128;
          x[i].im = (REAL)p1[s0 + i] - (REAL)128;
        }
        fft(pl, x, y);
        for (int c = 0; c < nchanout; ++c) {
          const int k = nskip + c;
          const cpx a = x[k], b = x[twonchan - k];
          acc[c] += a.re * a.re + a.im * a.im + b.re * b.re + b.im * b.im;
        }
      }
      const REAL sc = (REAL)1 / ((REAL)2 * (REAL)nfreq * (REAL)nave);
      for (int c = 0; c < nchanout; ++c) out[r * nchanout + c] = acc[c] * sc;
    }
    free(x); free(y); free(acc);
  }
  plan_free(pl);
  return bad;
}

/* ---- a11: subtractbpCAL (PIPE:1427-1474) on a time-major FB, in place ----- */
void oc_bandpass(REAL* fb, int64_t nrows, int nchan, int window) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nchan; ++c) {
    for (int64_t r0 = 0; r0 < nrows; r0 += window) {
      const int64_t r1 = (r0 + window < nrows) ? r0 + window : nrows;
      const double n = (double)(r1 - r0);
      double s = 0;
      for (int64_t r = r0; r < r1; ++r) s += fb[r * nchan + c];
      const double ave = s / n;
      double sd = 0, sd2 = 0;
      for (int64_t r = r0; r < r1; ++r) { const double d = fb[r * nchan + c] - ave; sd += d; sd2 += d * d; }
      const double sig = (sd2 - sd * sd / n) / (n - 1.0);
      const double hi = ave + 3.0 * sig, lo = ave - 3.0 * sig;
      double cs = 0; int64_t cnt = 0;
      for (int64_t r = r0; r < r1; ++r) {
        const double x = fb[r * nchan + c];
        if (x < hi && x > lo) { cs += x; ++cnt; }
      }
      if (cnt == 0) cnt = 1;
      const double cave = cs / (double)cnt;
      for (int64_t r = r0; r < r1; ++r) fb[r * nchan + c] = (REAL)((double)fb[r * nchan + c] - cave);
    }
  }
}

/* time-major -> channel-major copy (the CPU dedisperser streams channels) */
void oc_transpose(const REAL* tm, int64_t nrows, int nchan, REAL* cm) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nchan; ++c)
    for (int64_t r = 0; r < nrows; ++r) cm[(int64_t)c * nrows + r] = tm[r * nchan + c];
}

/* ---- a13: dedisperse (PIPE:1517-1537) on a channel-major FB -------------- */
void oc_dedisperse(const REAL* cm, int64_t nrows, int nchan, const int32_t* off, int ndm, int64_t nt, REAL* out) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int d = 0; d < ndm; ++d) {
    REAL* o = out + (int64_t)d * nt;
    for (int64_t t = 0; t < nt; ++t) o[t] = 0;
    for (int c = 0; c < nchan; ++c) {
      const REAL* src = cm + (int64_t)c * nrows + off[(int64_t)d * nchan + c];
      for (int64_t t = 0; t < nt; ++t) o[t] += src[t];
    }
    for (int64_t t = 0; t < nt; ++t) o[t] /= (REAL)nchan;
  }
}

/* ---- a14: calcstats per DM (PIPE:1337-1370) ------------------------------ */
void oc_calcstats_dm(const REAL* out, int ndm, int64_t nt, float* ave, float* sigma, float* peak, int* frb,
                     int* argmax) {
#pragma omp parallel for schedule(static)
  for (int d = 0; d < ndm; ++d) {
    const REAL* x = out + (int64_t)d * nt;
    double s = 0;
    for (int64_t t = 0; t < nt; ++t) s += (double)x[t];
    const double tave = s / (double)nt;
    double sd = 0, sd2 = 0;
    for (int64_t t = 0; t < nt; ++t) { const double v = (double)x[t] - tave; sd += v; sd2 += v * v; }
    const double tsig = (sd2 - sd * sd / (double)nt) / ((double)nt - 1.0);
    const float af = (float)tave, sf = (float)sqrt(tsig);
    float pk = 0.f; int f = 0, am = 0; float best = -INFINITY;
    for (int64_t t = 0; t < nt; ++t) {
      const float v = ((float)x[t] - af) / sf;
      if (v > 3.0f) f = 1;
      if (v > pk) pk = v;
      if (v > best) { best = v; am = (int)t; }
    }
    ave[d] = af; sigma[d] = sf; peak[d] = pk; frb[d] = f; argmax[d] = am;
  }
}

/* ---- a15: dedisperseSTATS (TS:1450-1481), channel-major FB --------------- */
void oc_dedisperse_sigma(const REAL* cm, int64_t nrows, int nchan, const int32_t* off, int ndm, int64_t nt,
                         REAL* ave, REAL* sig) {
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < nt; ++t)
    for (int d = 0; d < ndm; ++d) {
      double s = 0;
      for (int c = 0; c < nchan; ++c) s += cm[(int64_t)c * nrows + off[(int64_t)d * nchan + c] + t];
      const double a = s / nchan;
      double sd = 0, sd2 = 0;
      for (int c = 0; c < nchan; ++c) {
        const double v = cm[(int64_t)c * nrows + off[(int64_t)d * nchan + c] + t] - a;
        sd += v; sd2 += v * v;
      }
      ave[(int64_t)d * nt + t] = (REAL)a;
      sig[(int64_t)d * nt + t] = (REAL)sqrt((sd2 - sd * sd) / ((double)nchan * (nchan - 1.0)));
    }
}

/* ---- a16: calcstats per channel (STATS:910-946), channel-major FB -------- */
void oc_chan_stats(const REAL* cm, int64_t nrows, int nchan, int ncol, int nblk, float* ave, float* sg, float* outl) {
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nchan; ++c)
    for (int k = 0; k < nblk; ++k) {
      const int64_t r0 = (int64_t)ncol * k;
      const int64_t r1 = (r0 + ncol < nrows) ? r0 + ncol : nrows;
      const double n = (double)(r1 - r0);
      const REAL* x = cm + (int64_t)c * nrows;
      double s = 0;
      for (int64_t r = r0; r < r1; ++r) s += x[r];
      const double a = s / n;
      double sd = 0, sd2 = 0;
      for (int64_t r = r0; r < r1; ++r) { const double v = x[r] - a; sd += v; sd2 += v * v; }
      const double sig = (sd2 - sd * sd / n) / (n - 1.0);
      int64_t cnt = 0;
      for (int64_t r = r0; r < r1; ++r) cnt += ((double)x[r] > a + 5.0 * sig);
      ave[(int64_t)k * nchan + c] = (float)a;
      sg[(int64_t)k * nchan + c] = (float)sig;
      outl[(int64_t)k * nchan + c] = (float)(cnt / (int64_t)n);
    }
}

int oc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oc_real_bytes(void) { return (int)sizeof(REAL); }
