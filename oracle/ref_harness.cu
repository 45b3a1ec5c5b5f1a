// Harness around the reference's own code -- TEST INFRASTRUCTURE ONLY.
//
// build_ref.py compiles one reference tool (vdifFILE2dedisp_PIPELINE.cu,
// vdifDADA2stats.cu or vdifDADA2timeseries.cu, in place, with main renamed)
// together with this file into oracle/_ref/libref_<tool>.so.  The functions
// below set the reference's globals and call its functions exactly as its
// main() does, so the outputs are the reference's own:
//   * ref_read_bundles: initframe01 / initskip01 / filltimebufferHOST on a
//     VDIF file (PIPE:505-565) or a file standing in for the DADA ring
//     (STATS:346-374; TS:384-599), CPU only;
//   * ref_gpu_*: the per-bundle channeliser (convertarray, cuFFT R2C,
//     sumpower, avepower, the per-row D2D copies, PIPE:574-632), subtractbpCAL,
//     the in-tree dedisperse + calcstats (PIPE), dedisperseSTATS (TS) and the
//     per-channel calcstats (STATS), launched with the reference's own grid
//     shapes, on the GPU.
#include <cufft.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vdifio.h"
#if defined(REF_STATS) || defined(REF_TS)
#include "ipcio.h"
#endif

// ---- the reference's globals and functions (defined in the tool's .cu) ----
extern FILE* outflog;
extern int TWONCHAN, NAVE, NBUNDLE;
extern int NPARTFILL, NPARTLEFT, NSKIP0, NSKIP1, INDREAD;
extern unsigned char *data0, *data1, *skip0, *skip1, *tmpdata0, *tmpdata1;
extern vdif_header hdr0, hdr1;
int initframe01();
int initskip01();
int filltimebufferHOST(unsigned char* timein0, unsigned char* timein1);
#if defined(REF_PIPE)
extern FILE* ft;
extern int FLAGEOF;
extern int NLOOP;
#else
extern ipcio_t dadain;
extern key_t keyin;
extern int FLAGEODADA;
extern char *tmphdr0, *tmphdr1;
#if defined(REF_STATS)
extern int NFFT;
#else
extern int NLOOP;
int initDADA();
#endif
#endif

extern __constant__ int CSTRIDEAVE, CNFREQ, CNAVE, CNTOT_SUM, CNTOT_AVE, CNTOT_CONVERT, CNCHANOUT, CMAXNT, CNHALFCYC;
__global__ void sumpower(cufftComplex* freqout0, cufftComplex* freqout1, cufftReal* powTOT);
__global__ void avepower(cufftReal* powTOT, cufftReal* powAVE);
__global__ void convertarray(cufftReal* time, unsigned char* utime);
__global__ void subtractbpCAL(cufftReal* FULLFB);
#if defined(REF_PIPE) || defined(REF_TS)
__global__ void subtractbp(cufftReal* FULLFB);
__global__ void subtractZERO(cufftReal* FULLFB);
#endif
#if defined(REF_PIPE)
typedef float dedisp_float_t;
extern __constant__ int CNTIME_OUTDD, CNDM;
__global__ void dedisperse(cufftReal* FULLFB, dedisp_float_t* outDD, int* OFFSET);
__global__ void calcstats(dedisp_float_t* outDD, int* FRB, float* ave, float* sigma, float* peak);
#elif defined(REF_TS)
extern __constant__ int CNTIME_OUTDD, CNDM;
__global__ void dedisperseSTATS(cufftReal* FULLFB, float* outDD, float* sigDD, int* OFFSET);
#else
extern __constant__ int CNSTATBLKS, CNCOLSTATBLK;
__global__ void calcstats(cufftReal* FULLFB, float* CHANAVE, float* CHANSIGMA, float* CHANOUTLIER);
#endif

#define DATALEN_H 5000
#define CKR(x)                                         \
  do {                                                 \
    cudaError_t e_ = (x);                              \
    if (e_ != cudaSuccess) {                           \
      fprintf(stderr, "ref harness: %s\n", cudaGetErrorString(e_)); \
      return 10;                                       \
    }                                                  \
  } while (0)

static void alloc_frame_buffers() {
  data0 = (unsigned char*)malloc(DATALEN_H);
  data1 = (unsigned char*)malloc(DATALEN_H);
  skip0 = (unsigned char*)malloc(DATALEN_H);
  skip1 = (unsigned char*)malloc(DATALEN_H);
  tmpdata0 = (unsigned char*)malloc(DATALEN_H);
  tmpdata1 = (unsigned char*)malloc(DATALEN_H);
}

static void free_frame_buffers() {
  free(data0); free(data1); free(skip0); free(skip1); free(tmpdata0); free(tmpdata1);
}

// Runs the reference reader over `path`; returns 0 and the bundles, 2 when
// initialisation fails (the reference exits with 2), 1 at end of data
// during TS initialisation, 3 when the file cannot be opened.
extern "C" int ref_read_bundles(const char* path, int twonchan, int nave, int nbundle, int max_bundles,
                                unsigned char* out0, unsigned char* out1, int* nbund, double* tstart, int dada_skip) {
  TWONCHAN = twonchan;
  NAVE = nave;
  NBUNDLE = nbundle;
  const long nl = (long)nbundle * nave * twonchan;
  outflog = fopen("/dev/null", "w");
  alloc_frame_buffers();
  NSKIP0 = NSKIP1 = 0;
  INDREAD = 0;
  NPARTLEFT = 0;
  *nbund = 0;
#if defined(REF_PIPE)
  (void)dada_skip;
  NLOOP = (int)nl;
  ft = fopen(path, "rb");
  if (!ft) return 3;
  FLAGEOF = 1;
  if (initframe01() != 0) return 2;
#else
#if defined(REF_STATS)
  (void)dada_skip;
  NFFT = (int)nl;
#else
  NLOOP = (int)nl;
#endif
  ref_shim_set_dada_file(path);
  if (ipcio_connect(&dadain, keyin) < 0 || ipcio_open(&dadain, 'R') < 0) return 3;
  tmphdr0 = (char*)malloc(32);
  tmphdr1 = (char*)malloc(32);
  FLAGEODADA = 1;
#if defined(REF_TS)
  if (dada_skip && initDADA() != 0) return 1;
  int f = initframe01();
  while (f != 0) {  // TS:516-523; the reference spins for ever at end of data -- stop there
    if (f == 2) return 2;
    if (ipcbuf_eod((ipcbuf_t*)&dadain)) return 1;
    f = initframe01();
  }
#else
  if (initframe01() != 0) return 2;
#endif
#endif
  initskip01();
  *tstart = getVDIFDMJD(&hdr0, 25600);
  int nb = 0;
#if defined(REF_PIPE)
  while (FLAGEOF && nb < max_bundles) {
#else
  while (FLAGEODADA && nb < max_bundles) {
#endif
    if (filltimebufferHOST(out0 + (size_t)nb * nl, out1 + (size_t)nb * nl)) break;
    ++nb;
  }
  *nbund = nb;
#if defined(REF_PIPE)
  fclose(ft);
#else
  ipcio_close(&dadain);
#endif
  fclose(outflog);
  free_frame_buffers();
  return 0;
}

// ---- GPU: the reference's per-bundle channeliser (PIPE:574-632) ------------
// h0/h1: nbundles * NLOOP bytes per pol; h_fb: nbundles*nbundle rows of
// nchanout floats (time-major).  *ms: device time of the loop (events).
extern "C" int ref_gpu_channelise(const unsigned char* h0, const unsigned char* h1, int nbundles, int twonchan,
                                  int nave, int nbundle, int nskip, int nchanout, float* h_fb, float* ms) {
  const int nchan = twonchan / 2, nfreq = nchan + 1;
  const int nloop = nbundle * nave * twonchan;
  const int ntot_sum = nfreq * nave * nbundle, ntot_ave = nfreq * nbundle, stride = nave * nfreq;
  CKR(cudaMemcpyToSymbol(CNTOT_SUM, &ntot_sum, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNTOT_AVE, &ntot_ave, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNTOT_CONVERT, &nloop, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNFREQ, &nfreq, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNAVE, &nave, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CSTRIDEAVE, &stride, sizeof(int)));
  unsigned char *u0, *u1;
  cufftReal *t0, *t1, *ptot, *pave, *fb;
  cufftComplex *f0, *f1;
  CKR(cudaMalloc(&u0, nloop));
  CKR(cudaMalloc(&u1, nloop));
  CKR(cudaMalloc(&t0, sizeof(cufftReal) * nloop));
  CKR(cudaMalloc(&t1, sizeof(cufftReal) * nloop));
  CKR(cudaMalloc(&f0, sizeof(cufftComplex) * (size_t)nfreq * nave * nbundle));
  CKR(cudaMalloc(&f1, sizeof(cufftComplex) * (size_t)nfreq * nave * nbundle));
  CKR(cudaMalloc(&ptot, sizeof(cufftReal) * (size_t)nfreq * nave * nbundle));
  CKR(cudaMalloc(&pave, sizeof(cufftReal) * (size_t)nfreq * nbundle));
  CKR(cudaMalloc(&fb, sizeof(float) * (size_t)nbundles * nbundle * nchanout));
  cufftHandle plan;
  if (cufftPlan1d(&plan, twonchan, CUFFT_R2C, nave * nbundle) != CUFFT_SUCCESS) return 11;
  const int nthr = 512;
  const int nblk_sum = ntot_sum / nthr + 1, nblk_ave = ntot_ave / nthr + 1, nblk_conv = nloop / nthr + 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  for (int b = 0; b < nbundles; ++b) {
    CKR(cudaMemcpy(u0, h0 + (size_t)b * nloop, nloop, cudaMemcpyHostToDevice));
    CKR(cudaMemcpy(u1, h1 + (size_t)b * nloop, nloop, cudaMemcpyHostToDevice));
    convertarray<<<nblk_conv, nthr>>>(t0, u0);
    convertarray<<<nblk_conv, nthr>>>(t1, u1);
    if (cufftExecR2C(plan, t0, f0) != CUFFT_SUCCESS) return 12;
    if (cufftExecR2C(plan, t1, f1) != CUFFT_SUCCESS) return 12;
    sumpower<<<nblk_sum, nthr>>>(f0, f1, ptot);
    avepower<<<nblk_ave, nthr>>>(ptot, pave);
    for (int j = 0; j < nbundle; ++j)
      CKR(cudaMemcpy(fb + ((size_t)b * nbundle + j) * nchanout, pave + nskip + (size_t)j * nfreq,
                     sizeof(float) * nchanout, cudaMemcpyDeviceToDevice));
  }
  cudaEventRecord(e1, 0);
  CKR(cudaEventSynchronize(e1));
  CKR(cudaGetLastError());
  cudaEventElapsedTime(ms, e0, e1);
  CKR(cudaMemcpy(h_fb, fb, sizeof(float) * (size_t)nbundles * nbundle * nchanout, cudaMemcpyDeviceToHost));
  cufftDestroy(plan);
  cudaFree(u0); cudaFree(u1); cudaFree(t0); cudaFree(t1); cudaFree(f0); cudaFree(f1);
  cudaFree(ptot); cudaFree(pave); cudaFree(fb);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}

// ---- GPU: subtractbpCAL in place on a [maxnt][nchanout] block -------------
extern "C" int ref_gpu_bandpass(float* h_fb, int maxnt, int nchanout, float* ms) {
  int nhalfcyc = maxnt / 128 + ((maxnt % 128) ? 1 : 0);
  CKR(cudaMemcpyToSymbol(CNCHANOUT, &nchanout, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CMAXNT, &maxnt, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNHALFCYC, &nhalfcyc, sizeof(int)));
  float* fb;
  const size_t bytes = sizeof(float) * (size_t)maxnt * nchanout;
  CKR(cudaMalloc(&fb, bytes));
  CKR(cudaMemcpy(fb, h_fb, bytes, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
#if defined(REF_TS)
  const int nthr = 512, ntot = nchanout * nhalfcyc;  // TS:321-328
  subtractbpCAL<<<ntot / nthr + 1, nthr>>>(fb);
#else
  if (nhalfcyc > 1024) return 5;  // <<<NCHANOUT, NHALFCYC>>> (PIPE:658) cannot launch
  subtractbpCAL<<<nchanout, nhalfcyc>>>(fb);
#endif
  cudaEventRecord(e1, 0);
  CKR(cudaEventSynchronize(e1));
  CKR(cudaGetLastError());
  cudaEventElapsedTime(ms, e0, e1);
  CKR(cudaMemcpy(h_fb, fb, bytes, cudaMemcpyDeviceToHost));
  cudaFree(fb);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}

#if defined(REF_PIPE) || defined(REF_TS)
// ---- GPU: in-tree dedisperse + calcstats (PIPE) / dedisperseSTATS (TS) -----
// h_fb: [maxnt][nchanout]; h_off: [ndm][nchanout]; outputs [ndm][ntime_out].
extern "C" int ref_gpu_dedisperse(const float* h_fb, int maxnt, int nchanout, const int* h_off, int ndm,
                                  int ntime_out, float* h_out, float* h_sig, int* frb, float* ave, float* sigma,
                                  float* peak, float* ms) {
  CKR(cudaMemcpyToSymbol(CNCHANOUT, &nchanout, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CMAXNT, &maxnt, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNDM, &ndm, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNTIME_OUTDD, &ntime_out, sizeof(int)));
  float *fb, *out, *sig = nullptr;
  int* off;
  const size_t fbb = sizeof(float) * (size_t)maxnt * nchanout, ob = sizeof(float) * (size_t)ndm * ntime_out;
  CKR(cudaMalloc(&fb, fbb));
  CKR(cudaMalloc(&out, ob));
  CKR(cudaMalloc(&off, sizeof(int) * (size_t)ndm * nchanout));
  CKR(cudaMemcpy(fb, h_fb, fbb, cudaMemcpyHostToDevice));
  CKR(cudaMemcpy(off, h_off, sizeof(int) * (size_t)ndm * nchanout, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
#if defined(REF_PIPE)
  (void)h_sig;
  int* dfrb;
  float *dave, *dsig, *dpeak;
  CKR(cudaMalloc(&dfrb, sizeof(int) * ndm));
  CKR(cudaMalloc(&dave, sizeof(float) * ndm));
  CKR(cudaMalloc(&dsig, sizeof(float) * ndm));
  CKR(cudaMalloc(&dpeak, sizeof(float) * ndm));
  cudaEventRecord(e0, 0);
  dedisperse<<<(int)((long)ndm * ntime_out / 512) + 1, 512>>>(fb, out, off);  // PIPE:551, 678
  calcstats<<<ndm, 1>>>(out, dfrb, dave, dsig, dpeak);                       // PIPE:546-547, 685
  cudaEventRecord(e1, 0);
  CKR(cudaEventSynchronize(e1));
  CKR(cudaGetLastError());
  CKR(cudaMemcpy(frb, dfrb, sizeof(int) * ndm, cudaMemcpyDeviceToHost));
  CKR(cudaMemcpy(ave, dave, sizeof(float) * ndm, cudaMemcpyDeviceToHost));
  CKR(cudaMemcpy(sigma, dsig, sizeof(float) * ndm, cudaMemcpyDeviceToHost));
  CKR(cudaMemcpy(peak, dpeak, sizeof(float) * ndm, cudaMemcpyDeviceToHost));
  cudaFree(dfrb); cudaFree(dave); cudaFree(dsig); cudaFree(dpeak);
#else
  (void)frb; (void)ave; (void)sigma; (void)peak;
  CKR(cudaMalloc(&sig, ob));
  const int sq = (int)sqrt((double)((long)ndm * ntime_out / 256)) + 1;  // TS:496-499
  cudaEventRecord(e0, 0);
  dedisperseSTATS<<<dim3(sq, sq), dim3(16, 16)>>>(fb, out, sig, off);
  cudaEventRecord(e1, 0);
  CKR(cudaEventSynchronize(e1));
  CKR(cudaGetLastError());
  CKR(cudaMemcpy(h_sig, sig, ob, cudaMemcpyDeviceToHost));
  cudaFree(sig);
#endif
  cudaEventElapsedTime(ms, e0, e1);
  CKR(cudaMemcpy(h_out, out, ob, cudaMemcpyDeviceToHost));
  cudaFree(fb); cudaFree(out); cudaFree(off);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}
#endif

#if defined(REF_STATS)
// ---- GPU: per-channel calcstats <<<NCHANOUT, NSTATBLKS>>> (STATS:416) -------
extern "C" int ref_gpu_chanstats(const float* h_fb, int maxnt, int nchanout, int ncolstatblk, int nstatblks,
                                 float* cave, float* csig, float* cout, float* ms) {
  CKR(cudaMemcpyToSymbol(CNCHANOUT, &nchanout, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CMAXNT, &maxnt, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNSTATBLKS, &nstatblks, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CNCOLSTATBLK, &ncolstatblk, sizeof(int)));
  float *fb, *a, *s, *o;
  const size_t fbb = sizeof(float) * (size_t)maxnt * nchanout, sb = sizeof(float) * (size_t)nstatblks * nchanout;
  CKR(cudaMalloc(&fb, fbb));
  CKR(cudaMalloc(&a, sb));
  CKR(cudaMalloc(&s, sb));
  CKR(cudaMalloc(&o, sb));
  CKR(cudaMemcpy(fb, h_fb, fbb, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  calcstats<<<nchanout, nstatblks>>>(fb, a, s, o);
  cudaEventRecord(e1, 0);
  CKR(cudaEventSynchronize(e1));
  CKR(cudaGetLastError());
  cudaEventElapsedTime(ms, e0, e1);
  CKR(cudaMemcpy(cave, a, sb, cudaMemcpyDeviceToHost));
  CKR(cudaMemcpy(csig, s, sb, cudaMemcpyDeviceToHost));
  CKR(cudaMemcpy(cout, o, sb, cudaMemcpyDeviceToHost));
  cudaFree(fb); cudaFree(a); cudaFree(s); cudaFree(o);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}
#endif

#if defined(REF_PIPE) || defined(REF_TS)
// ---- GPU: the dead-code modes subtractbp (kind 0) / subtractZERO (kind 1)
// in place on a [maxnt][nchanout] block.  Both kernels give each thread one
// independent channel (subtractbp) or row (subtractZERO), so any grid that
// covers them computes what the reference's launch would.
extern "C" int ref_gpu_subtract_mode(float* h_fb, int maxnt, int nchanout, int kind, float* ms) {
  CKR(cudaMemcpyToSymbol(CNCHANOUT, &nchanout, sizeof(int)));
  CKR(cudaMemcpyToSymbol(CMAXNT, &maxnt, sizeof(int)));
  float* fb;
  const size_t bytes = sizeof(float) * (size_t)maxnt * nchanout;
  CKR(cudaMalloc(&fb, bytes));
  CKR(cudaMemcpy(fb, h_fb, bytes, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  if (kind == 0)
    subtractbp<<<(nchanout + 127) / 128, 128>>>(fb);
  else
    subtractZERO<<<(maxnt + 127) / 128, 128>>>(fb);
  cudaEventRecord(e1, 0);
  CKR(cudaEventSynchronize(e1));
  CKR(cudaGetLastError());
  cudaEventElapsedTime(ms, e0, e1);
  CKR(cudaMemcpy(h_fb, fb, bytes, cudaMemcpyDeviceToHost));
  cudaFree(fb);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}
#endif
