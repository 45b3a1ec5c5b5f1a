// Host side of the libvfrb C ABI: header decode, parameter derivation,
// delay table and the stage entry points (argument checks + launches).
#include <cmath>
#include <cstring>

#include "vfrb_common.cuh"

namespace vfrb {
size_t dedisperse_workspace_bytes_plan(const vfrb_ddplan* pl, long long nt_out);
int launch_dedisperse_plan(const vfrb_ddplan* pl, const vfrb_dd_args& a, cudaStream_t s);
int ddplan_create(vfrb_ddplan** out, const int32_t* h_off, int ndm, int nchan);
int ddplan_destroy(vfrb_ddplan* p);
int ddplan_max_delay(const vfrb_ddplan* p);
int ddplan_reg_group(const vfrb_ddplan* p);
int ddplan_autotune(vfrb_ddplan* pl, int storage, long long nt, float* times, cudaStream_t s);
int ddplan_set_variant(vfrb_ddplan* pl, int storage, int v);
int ddplan_variant(const vfrb_ddplan* pl, int storage);
}  // namespace vfrb

extern "C" {

const char* vfrb_strerror(int st) {
  switch (st) {
    case VFRB_OK: return "ok";
    case VFRB_EOD: return "end of data";
    case VFRB_ERR: return "data or stream error";
    case VFRB_ERR_CUDA: return "CUDA error";
    case VFRB_ERR_ARG: return "invalid argument";
    case VFRB_ERR_UNSUPPORTED: return "configuration not supported";
    case VFRB_ERR_NOMEM: return "out of memory / not admitted";
    case VFRB_ERR_TIMEOUT: return "bounded device wait timed out";
    case VFRB_ERR_DEVICE: return "kernel flagged an out-of-range access";
    default: return "unknown status";
  }
}

int vfrb_decode_header(const uint8_t* b, vfrb_hdr* h) {
  if (!b || !h) return VFRB_ERR_ARG;
  uint32_t w[8];
  for (int i = 0; i < 8; ++i)
    w[i] = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 | (uint32_t)b[4 * i + 2] << 16 |
           (uint32_t)b[4 * i + 3] << 24;
  // gcc allocates bitfields from the least significant bit (vdifio.h:53-72)
  h->seconds = w[0] & 0x3FFFFFFFu;
  h->legacymode = (w[0] >> 30) & 1u;
  h->invalid = (w[0] >> 31) & 1u;
  h->frame = w[1] & 0xFFFFFFu;
  h->epoch = (w[1] >> 24) & 0x3Fu;
  h->unassigned = (w[1] >> 30) & 3u;
  h->framelength8 = w[2] & 0xFFFFFFu;
  h->nchan_log2 = (w[2] >> 24) & 0x1Fu;
  h->version = (w[2] >> 29) & 7u;
  h->stationid = w[3] & 0xFFFFu;
  h->threadid = (w[3] >> 16) & 0x3FFu;
  h->nbits_minus1 = (w[3] >> 26) & 0x1Fu;
  h->iscomplex = (w[3] >> 31) & 1u;
  h->eversion = w[4] & 0xFFu;
  h->extended1 = (w[4] >> 8) & 0xFFFFFFu;
  h->extended2 = w[5];
  h->extended3 = w[6];
  h->extended4 = w[7];
  return VFRB_OK;
}

// Days from 1970-01-01 of a proleptic Gregorian date (civil calendar arithmetic).
static long long days_from_civil(long long y, unsigned m, unsigned d) {
  y -= m <= 2;
  const long long era = (y >= 0 ? y : y - 399) / 400;
  const unsigned yoe = (unsigned)(y - era * 400);
  const unsigned doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  const unsigned doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + (long long)doe - 719468;
}

double vfrb_header_dmjd(const vfrb_hdr* h, int fps) {
  // VDIF: epoch = 6-month periods since 2000-01-01 00:00 UTC; seconds from the epoch start.
  if (!h || fps <= 0) return 0.0;
  const long long year = 2000 + h->epoch / 2;
  const unsigned month = 1 + 6 * (h->epoch % 2);
  const long long mjd_epoch = days_from_civil(year, month, 1) + 40587;  // MJD of 1970-01-01
  const int imjd = (int)(mjd_epoch + h->seconds / 86400);
  return (double)imjd + (double)(h->seconds % 86400) / 86400.0 + (double)h->frame / (fps * 86400.0);
}

int vfrb_layout_init(vfrb_layout* L, int twonchan, int nave, int nbundle, double muoslowfreq, int nchanout_fixed,
                     float maxtime) {
  if (!L || twonchan < 4 || nave < 1 || nbundle < 1 || maxtime <= 0.f) return VFRB_ERR_ARG;
  std::memset(L, 0, sizeof(*L));
  L->twonchan = twonchan;
  L->nave = nave;
  L->nbundle = nbundle;
  L->maxtime = maxtime;
  L->nchan = (int)(0.5 * twonchan);
  L->nfreq = L->nchan + 1;
  L->chanbw = 64.0 / L->nchan;
  if (nchanout_fixed > 0) {
    L->nchanout = nchanout_fixed;
  } else {
    L->nchanout = (int)((muoslowfreq - 320.0) / L->chanbw) + 1;
    if (L->nchanout % 2 == 1) L->nchanout++;
  }
  L->nskip = (L->nchan - L->nchanout) + 1;
  if (L->nskip < 1 || L->nchanout < 2 || L->nskip + L->nchanout > L->nfreq) return VFRB_ERR_ARG;
  L->nloop = nbundle * nave * twonchan;
  L->foff = -1.0 * L->chanbw;
  L->fch1 = (320.0 + (L->nchanout * L->chanbw)) - (0.5 * L->chanbw);
  L->tchan = (double)(nave * twonchan) / 128e6;
  L->maxnt = (int)((double)maxtime / L->tchan);
  L->nhalfcyc = L->maxnt / 128 + ((L->maxnt % 128) ? 1 : 0);
  return VFRB_OK;
}

int vfrb_delay_table(const vfrb_layout* L, const float* dms, int ndm, int32_t* off, int32_t* max_delay) {
  if (!L || !dms || ndm < 1 || !off) return VFRB_ERR_ARG;
  const double pf = std::pow(L->fch1, -2);
  for (int i = 0; i < ndm; ++i) {
    off[(long long)i * L->nchanout] = 0;  // highest frequency channel is the reference
    for (int j = 1; j < L->nchanout; ++j) {
      const double dt = 4.148808e3 * (double)dms[i] * (std::pow(L->fch1 - (j * L->chanbw), -2) - pf);
      off[(long long)i * L->nchanout + j] = (int32_t)(dt / L->tchan);
    }
  }
  if (max_delay)
    *max_delay = (int32_t)((4.148808e3 * (double)dms[ndm - 1] *
                            (std::pow(L->fch1 - (L->nchanout * L->chanbw), -2) - pf)) /
                           L->tchan);
  return VFRB_OK;
}

int vfrb_channelise(const vfrb_chan_args* a, void* stream) {
  if (!a) return VFRB_ERR_ARG;
  return vfrb::launch_channelise(*a, (cudaStream_t)stream);
}

int vfrb_bandpass(const vfrb_bp_args* a, void* stream) {
  if (!a) return VFRB_ERR_ARG;
  return vfrb::launch_bandpass(*a, (cudaStream_t)stream);
}

int vfrb_ddplan_create(vfrb_ddplan** plan, const int32_t* h_offsets, int ndm, int nchan) {
  return vfrb::ddplan_create(plan, h_offsets, ndm, nchan);
}

int vfrb_ddplan_destroy(vfrb_ddplan* plan) { return vfrb::ddplan_destroy(plan); }

int vfrb_ddplan_max_delay(const vfrb_ddplan* plan) { return plan ? vfrb::ddplan_max_delay(plan) : -1; }

int vfrb_ddplan_group_size(const vfrb_ddplan* plan) { return plan ? vfrb::ddplan_reg_group(plan) : -1; }

int vfrb_ddplan_set_variant(vfrb_ddplan* plan, int storage, int variant) {
  return vfrb::ddplan_set_variant(plan, storage, variant);
}

int vfrb_ddplan_variant(const vfrb_ddplan* plan, int storage) { return vfrb::ddplan_variant(plan, storage); }

int vfrb_ddplan_autotune(vfrb_ddplan* plan, int storage, int64_t nt_out, float* times, void* stream) {
  return vfrb::ddplan_autotune(plan, storage, nt_out, times, (cudaStream_t)stream);
}

size_t vfrb_dedisperse_workspace_bytes(const vfrb_ddplan* plan, int64_t nt_out) {
  return plan ? vfrb::dedisperse_workspace_bytes_plan(plan, nt_out) : 0;
}

int vfrb_dedisperse(const vfrb_ddplan* plan, const vfrb_dd_args* a, void* stream) {
  if (!a) return VFRB_ERR_ARG;
  return vfrb::launch_dedisperse_plan(plan, *a, (cudaStream_t)stream);
}

int vfrb_chan_stats(const vfrb_cs_args* a, void* stream) {
  if (!a) return VFRB_ERR_ARG;
  return vfrb::launch_chan_stats(*a, (cudaStream_t)stream);
}

int vfrb_chan_sk(const float* fb_tm, int64_t row_stride, int nchan, int nrows, int ncolstatblk, int nstatblks,
                 int nsum, float* sk, void* stream) {
  return vfrb::launch_chan_sk(fb_tm, row_stride, nchan, nrows, ncolstatblk, nstatblks, nsum, sk,
                              (cudaStream_t)stream);
}

int vfrb_fb_to_time_major(const float* src_cm, int64_t chan_stride, int64_t row0, uint32_t row_mask, int nchan,
                          int nrows, float* dst_tm, int64_t dst_row_stride, void* stream) {
  return vfrb::launch_fb_transpose(src_cm, chan_stride, row_mask, row0, nchan, nrows, dst_tm, dst_row_stride,
                                   (cudaStream_t)stream);
}

}  // extern "C"
