// Plan / stream engine behind vfrb_plan_* (the reference's main loops,
// PIPE:556-708, STATS:367-431, TS:589-746), B200 style:
//
//  * raw VDIF bytes are copied once to a per-stream device frame ring on a
//    copy stream; only headers are parsed on the host, by the reference's
//    pol-pair state machine (vdif_reader.h), which emits payload references;
//  * complete rows are channelised straight from the ring (K1), bandpassed
//    into the layout/precision the dedisperser wants (K2), dedispersed with
//    fused statistics (K3) or reduced to per-channel statistics (K4), all on
//    the stream's compute stream, overlapping the next copy;
//  * results are copied to page-locked host memory and handed out by
//    vfrb_poll() as they complete; a host callback stamps completion time
//    for latency accounting.
//
// Block mode reproduces the reference's block manager: a MAXNT-row
// filterbank filled NBUNDLE rows at a time, the raw last max_delay rows
// carried to the next block with new data written from row
// (max_delay/NBUNDLE)*NBUNDLE (PIPE:649-704; TS:643-692), bandpass windows
// counted from the block's first row; STATS restarts at row 0 (STATS:428).
// Stream mode keeps a max_delay overlap ring per stream, bandpasses absolute
// 128-row windows and emits every output sample once.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "vdif_reader.h"
#include "vfrb_common.cuh"

namespace vfrb {

// NVTX range for profilers' timelines (header-only NVTX 3: a no-op unless a
// tool is attached)
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

size_t dedisperse_workspace_bytes_plan(const vfrb_ddplan* pl, long long nt_out);
int launch_dedisperse_plan(const vfrb_ddplan* pl, const vfrb_dd_args& a, cudaStream_t s);
int ddplan_create(vfrb_ddplan** out, const int32_t* h_off, int ndm, int nchan);
int ddplan_destroy(vfrb_ddplan* p);
int ddplan_max_delay(const vfrb_ddplan* p);
int ddplan_autotune(vfrb_ddplan* pl, int storage, long long nt, float* times, cudaStream_t s);
int launch_boxcar(const float* dd, int ndm, long long nt, long long stride, const float* ave, const float* sigma,
                  int max_width, float* snr, int* t, int* w, cudaStream_t s);
int launch_series_stats(const float* dd, int ndm, long long nt, long long stride, float* ave, float* sigma,
                        float* peak, int* frb, int* argmax, cudaStream_t s);

static double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

#define CK(x)                                     \
  do {                                            \
    if ((x) != cudaSuccess) {                     \
      cudaGetLastError();                         \
      return VFRB_ERR_CUDA;                       \
    }                                             \
  } while (0)
#define ST(x)            \
  do {                   \
    const int st_ = (x); \
    if (st_) return st_; \
  } while (0)

constexpr int kStash = 1024;       // gap-revealing frames kept aside per stream
constexpr int kMaxStreams = 4096;  // stream ids over a plan's life
constexpr int kSlotBufs = 32;  // rotating slot-table uploads in flight (host runs ahead of the GPU)
constexpr int kStageBufs = 2;  // rotating staging buffers for pageable input

static unsigned long long pow2_at_least(unsigned long long v) {
  unsigned long long r = 1;
  while (r < v) r <<= 1;
  return r;
}

// Per-channel weights of the FP16 / int8 forms from the first bandpass
// window's variance: s_c = sqrt(var_c); stored z = x/s_c (times q for int8);
// the dedisperser weights channel c by s_c (s_c/q for int8).
__global__ void k_init_scale(const float* var, int nchan, float q, int storage, float* w, float* inv) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchan) return;
  float s = sqrtf(fmaxf(var[c], 0.f));
  if (!(s > 1e-30f)) s = 1.f;
  inv[c] = 1.f / s;
  w[c] = (storage == VFRB_I8) ? s / q : s;
}

// FP16 form: one scale per stream, S = sqrt(mean_c var_c) of the first
// window (FP16 keeps its relative precision at any scale; S only keeps the
// values well inside the FP16 range).  w[0] = S, inv[c] = 1/S.
__global__ void k_uniform_scale(const float* var, int nchan, float* w, float* inv) {
  __shared__ double part[256];
  double s = 0.0;
  for (int c = threadIdx.x; c < nchan; c += blockDim.x) s += (double)fmaxf(var[c], 0.f);
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  float S = (float)sqrt(part[0] / (double)nchan);
  if (!(S > 1e-30f)) S = 1.f;
  if (threadIdx.x == 0) w[0] = S;
  for (int c = threadIdx.x; c < nchan; c += blockDim.x) inv[c] = 1.f / S;
}

// Device and page-locked host memory, events and CUDA streams one stream
// owns; released together when the stream is closed or the plan destroyed.
struct Owned {
  std::vector<void*> dev, host;
  std::vector<cudaEvent_t> ev;
  std::vector<cudaStream_t> cs;
  int64_t dev_bytes = 0;
  void release() {
    for (auto s : cs) cudaStreamSynchronize(s);
    for (auto s : cs) cudaStreamDestroy(s);
    for (auto e : ev) cudaEventDestroy(e);
    for (auto p : dev) cudaFree(p);
    for (auto p : host) cudaFreeHost(p);
    cs.clear();
    ev.clear();
    dev.clear();
    host.clear();
    dev_bytes = 0;
  }
};

struct ResultSlot {
  vfrb_result r{};
  float *dd = nullptr, *dds = nullptr, *ave = nullptr, *sig = nullptr, *peak = nullptr, *fb = nullptr;
  int32_t *frb = nullptr, *arg = nullptr, *err = nullptr;
  float* bsnr = nullptr;  // boxcar search: best SNR, start, width per trial
  int32_t *bt = nullptr, *bw = nullptr;
  float *cave = nullptr, *csig = nullptr, *cout = nullptr, *csk = nullptr;
  std::vector<vfrb_cand> cands;
  std::vector<uint8_t> flags;  // VFRB_ROW_* of the result's rows
  cudaEvent_t ev = nullptr;
  double t_data = 0.0;
  volatile double t_done = 0.0;
  int state = 0;  // 0 free, 1 in flight, 2 held by the caller
};

static void CUDART_CB mark_done(void* p) { static_cast<ResultSlot*>(p)->t_done = now_ms(); }

struct SlotBuf {
  int64_t* h = nullptr;
  int64_t* d = nullptr;
  cudaEvent_t ev = nullptr;       // upload h -> d done
  cudaEvent_t ev_used = nullptr;  // the channeliser reading d done
};

struct StreamSt {
  int id = 0;
  Owned res;
  cudaStream_t cs = nullptr;   // compute
  cudaStream_t xs = nullptr;   // host-to-device copies
  cudaStream_t hs = nullptr;   // header copies of device-resident input
  cudaEvent_t ev_copied = nullptr, ev_consumed = nullptr;
  // Release events: one per channeliser launch, with the oldest frame any
  // later work still reads (frames below it are free once the event has
  // completed).  A copy into the ring waits only for the launch that freed
  // the slots it overwrites, so copies run ahead of the compute stream.
  static constexpr int kRelEv = 32;
  cudaEvent_t rel_ev[kRelEv] = {};
  int64_t rel_after[kRelEv] = {};
  int rel_head = 0, rel_n = 0;
  std::unique_ptr<PairReader> reader;
  std::vector<uint8_t> part;   // bytes of an incomplete frame
  uint8_t* d_frames = nullptr; // frame ring followed by the stash
  int64_t ring_frames = 0;
  int64_t frames_in = 0;       // frames received (ring position)
  int stash_next = 0;
  uint8_t* h_stage[kStageBufs] = {};
  // device input: each batch's 32-byte frame headers, packed in
  // page-locked host memory by one strided copy
  uint8_t* h_hdr = nullptr;
  // device input is read after the work queued before the push on the
  // legacy default stream (where, e.g., PyTorch queues the kernels that
  // produced it): the stream's own CUDA streams are non-blocking
  cudaEvent_t ev_input = nullptr;
  cudaEvent_t stage_ev[kStageBufs] = {};
  int stage_i = 0;
  size_t stage_frames = 0;
  SlotBuf sb[kSlotBufs];
  int sb_i = 0;
  int64_t slots_cap = 0;
  std::vector<int64_t> e0, e1;  // pair entries: frame index, -1 fill, <= -2 stash slot
  std::vector<uint8_t> finv;    // VDIF invalid bit of each ring frame slot
  uint8_t stash_flag[kStash] = {};
  std::vector<uint8_t> rflags;  // VFRB_ROW_* per FB row: block rows, or a ring of rows (stream)
  int64_t fmask = 0;
  size_t ehead = 0;             // consumed entries at the front of e0/e1
  int64_t ebase = 0;            // global index of e0[ehead]
  bool ended = false;
  bool started = false;
  int reader_error = 0;
  double tstart_mjd = 0.0;
  std::string logtext;
  double t_push = 0.0;
  int32_t* d_err = nullptr;
  // block mode
  float* d_fb_tm = nullptr;
  float* d_left = nullptr;
  int64_t bundles_done = 0;
  int loopcnt = 0;
  int64_t blocks = 0;
  // stream mode
  float* d_raw = nullptr;
  int64_t R1 = 0;
  int64_t rows_chan = 0, rows_bp = 0, rows_out = 0;
  int64_t chunks = 0;
  int64_t stat_blocks = 0;     // TIMESTATS blocks emitted (VFRB_OUT_CHANSTATS)
  // batch_streams: chunks whose dedispersion waits for the plan's shared
  // launch (rows, output chunks, and when their data were complete)
  bool job = false;
  int64_t job_row0 = 0, job_nvalid = 0, job_k = 0, job_nt = 0, job_seq0 = 0;
  double job_t_push = 0.0;
  cudaEvent_t ev_ready = nullptr;
  // both
  void* d_cm = nullptr;  // channel-major bandpassed FB (storage form)
  // FP16 with dedispersion: the same ring shifted by one row,
  // d_cm1[c][r] = d_cm[c][r + 1] (written by the bandpass beside d_cm), so
  // the dedisperser reads its windows of halves with aligned 4-byte loads
  void* d_cm1 = nullptr;
  int64_t cm_stride = 0;
  unsigned cm_mask = 0xffffffffu;
  float *d_w = nullptr, *d_inv = nullptr, *d_var = nullptr, *d_scr = nullptr;
  bool scale_ready = false;
  float uscale = 1.f;  // FP16 form: the stream's single scale S
  float *d_out = nullptr, *d_sig = nullptr, *d_ave = nullptr, *d_sgm = nullptr, *d_peak = nullptr;
  int32_t *d_frb = nullptr, *d_arg = nullptr;
  float* d_bsnr = nullptr;
  int32_t *d_bt = nullptr, *d_bw = nullptr;
  void* d_ws = nullptr;
  size_t ws_bytes = 0;
  float *d_cave = nullptr, *d_csig = nullptr, *d_cout = nullptr, *d_csk = nullptr, *d_fbt = nullptr;
  int64_t out_stride = 0;
  std::vector<std::unique_ptr<ResultSlot>> slots;
};

}  // namespace vfrb

using namespace vfrb;

struct vfrb_plan {
  vfrb_params P{};
  vfrb_layout L{};
  std::vector<float> dms;
  std::vector<int32_t> off;
  int max_delay = 0;
  int ndm = 0;
  vfrb_ddplan* dd = nullptr;
  bool want_dd = false;
  int64_t chunk_rows = 0;
  int64_t nt_block = 0;
  int64_t launch_rows = 0;  // most rows one channelise launch produces
  int64_t batch_chunks = 1; // stream mode: most output chunks one dedispersion launch covers
  int ncolstatblk = 0, nstatblks = 0;
  int64_t ring_frames = 0, R1 = 0, R2 = 0;  // per-stream geometry (admission, open)
  std::vector<std::unique_ptr<StreamSt>> st;  // by stream id; null once closed
  std::deque<ResultSlot*> queue;  // submission order
  ResultSlot* held = nullptr;     // returned by the last poll
  std::string logtmp;
  // stream mode, batch_streams: streams whose chunks wait for one shared
  // dedispersion launch on bs
  std::vector<StreamSt*> pending;
  cudaStream_t bs = nullptr;
  cudaEvent_t ev_batch = nullptr;
};

namespace {

// Where pushed bytes live: pageable host memory (copied through staging
// buffers), page-locked host memory (copied to the device in place), or
// device memory (copied device to device; only headers go to the host).
enum MemKind { kPageable = 0, kPinned = 1, kDevice = 2 };
MemKind mem_kind(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return kPageable;
  }
  if (a.type == cudaMemoryTypeHost) return kPinned;
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return kDevice;
  return kPageable;
}

template <typename T>
int dmalloc(Owned& o, T** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (cudaMalloc((void**)p, bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return VFRB_ERR_NOMEM;
  }
  o.dev.push_back((void*)*p);
  o.dev_bytes += (int64_t)bytes;
  return VFRB_OK;
}

template <typename T>
int hmalloc(Owned& o, T** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (cudaHostAlloc((void**)p, bytes, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return VFRB_ERR_NOMEM;
  }
  o.host.push_back((void*)*p);
  return VFRB_OK;
}

int mkevent(Owned& o, cudaEvent_t* e) {
  CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  o.ev.push_back(*e);
  return VFRB_OK;
}

int mkstream(Owned& o, cudaStream_t* s) {
  CK(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
  o.cs.push_back(*s);
  return VFRB_OK;
}

size_t storage_bytes(int s) { return s == VFRB_F32 ? 4 : (s == VFRB_F16 ? 2 : 1); }

bool want(const vfrb_plan* pl, int bit) { return (pl->P.outputs & bit) != 0; }

// device bytes one stream needs (admission control)
// FP16 storage with dedispersion keeps the channel-major ring twice (the
// second copy shifted by one row)
bool shifted_copy(const vfrb_plan* pl) { return pl->P.storage == VFRB_F16 && pl->want_dd; }

int64_t stream_bytes(const vfrb_plan* pl, int64_t ring_frames, int64_t R1, int64_t R2) {
  const vfrb_params& P = pl->P;
  const int64_t nch = pl->L.nchanout;
  int64_t b = ring_frames * kFrameLen + (int64_t)kStash * kDataLen + kSlotBufs * 2 * 16 * pl->launch_rows * 64;
  const int64_t nt = P.mode == VFRB_MODE_BLOCK ? pl->nt_block : pl->chunk_rows * pl->batch_chunks;
  if (P.mode == VFRB_MODE_BLOCK) {
    b += (int64_t)pl->L.maxnt * nch * 4;                                    // raw block
    b += (int64_t)pl->max_delay * nch * 4;                                  // leftover
    b += nch * (((int64_t)pl->L.maxnt + 15) / 16 * 16) * (int64_t)storage_bytes(P.storage) * (shifted_copy(pl) ? 2 : 1);
    if (want(pl, VFRB_OUT_FB)) b += (int64_t)pl->L.maxnt * nch * 4;
    if (want(pl, VFRB_OUT_CHANSTATS)) b += 3LL * pl->nstatblks * nch * 4;
  } else {
    b += R1 * nch * 4 + R2 * nch * (int64_t)storage_bytes(P.storage) * (shifted_copy(pl) ? 2 : 1);
    if (want(pl, VFRB_OUT_CHANSTATS)) b += 4LL * nch * 4;
  }
  if (pl->want_dd) {
    b += (int64_t)pl->ndm * nt * 4 * (want(pl, VFRB_OUT_SIGMA) ? 2 : 1);
    b += (int64_t)dedisperse_workspace_bytes_plan(pl->dd, nt) + 5LL * pl->ndm * 4;
  }
  return b;
}

// boxcar width search on: candidates wanted and widths beyond 1 requested
bool boxcar_on(const vfrb_plan* pl) {
  return (pl->P.outputs & VFRB_OUT_CANDS) && pl->P.boxcar_max > 1;
}

int alloc_slot(vfrb_plan* pl, StreamSt* s, ResultSlot** out) {
  for (auto& r : s->slots)
    if (r->state == 0) {
      *out = r.get();
      return VFRB_OK;
    }
  auto r = std::make_unique<ResultSlot>();
  const vfrb_params& P = pl->P;
  const int64_t nch = pl->L.nchanout;
  const int64_t nt = P.mode == VFRB_MODE_BLOCK ? pl->nt_block : pl->chunk_rows;
  if (pl->want_dd) {
    if (want(pl, VFRB_OUT_DEDISP)) ST(hmalloc(s->res, &r->dd, (size_t)pl->ndm * nt * 4));
    if (want(pl, VFRB_OUT_SIGMA)) ST(hmalloc(s->res, &r->dds, (size_t)pl->ndm * nt * 4));
    ST(hmalloc(s->res, &r->ave, (size_t)pl->ndm * 4));
    ST(hmalloc(s->res, &r->sig, (size_t)pl->ndm * 4));
    ST(hmalloc(s->res, &r->peak, (size_t)pl->ndm * 4));
    ST(hmalloc(s->res, &r->frb, (size_t)pl->ndm * 4));
    ST(hmalloc(s->res, &r->arg, (size_t)pl->ndm * 4));
    if (boxcar_on(pl)) {
      ST(hmalloc(s->res, &r->bsnr, (size_t)pl->ndm * 4));
      ST(hmalloc(s->res, &r->bt, (size_t)pl->ndm * 4));
      ST(hmalloc(s->res, &r->bw, (size_t)pl->ndm * 4));
    }
  }
  if (P.mode == VFRB_MODE_BLOCK && want(pl, VFRB_OUT_FB)) ST(hmalloc(s->res, &r->fb, (size_t)pl->L.maxnt * nch * 4));
  if (want(pl, VFRB_OUT_CHANSTATS)) {
    ST(hmalloc(s->res, &r->cave, (size_t)pl->nstatblks * nch * 4));
    ST(hmalloc(s->res, &r->csig, (size_t)pl->nstatblks * nch * 4));
    ST(hmalloc(s->res, &r->cout, (size_t)pl->nstatblks * nch * 4));
    ST(hmalloc(s->res, &r->csk, (size_t)pl->nstatblks * nch * 4));
  }
  ST(hmalloc(s->res, &r->err, 4));
  ST(mkevent(s->res, &r->ev));
  *out = r.get();
  s->slots.push_back(std::move(r));
  return VFRB_OK;
}

// Translate a pair entry into a payload byte offset within d_frames.
inline int64_t entry_offset(const StreamSt* s, int64_t v) {
  if (v >= 0) return (v % s->ring_frames) * kFrameLen + kHdrLen;
  if (v == -1) return -1;
  return s->ring_frames * kFrameLen + (-2 - v) * (int64_t)kDataLen;
}

// VFRB_ROW_* contribution of one pol's entry
inline uint8_t entry_flag(const StreamSt* s, int64_t v) {
  if (v >= 0) return s->finv[(size_t)(v % s->ring_frames)];
  if (v == -1) return VFRB_ROW_FILL;
  return s->stash_flag[-2 - v];
}

int64_t npairs(const StreamSt* s) { return s->ebase + (int64_t)(s->e0.size() - s->ehead); }

int64_t oldest_ref(const StreamSt* s);

void consume_entries(StreamSt* s, int64_t first_needed) {
  while (s->ebase < first_needed && s->ehead < s->e0.size()) {
    ++s->ehead;
    ++s->ebase;
  }
  // the newest channeliser launch consumed these entries
  if (s->rel_n > 0) s->rel_after[(s->rel_head + s->rel_n - 1) % StreamSt::kRelEv] = oldest_ref(s);
  if (s->ehead > 65536 && s->ehead * 2 > s->e0.size()) {
    s->e0.erase(s->e0.begin(), s->e0.begin() + (long)s->ehead);
    s->e1.erase(s->e1.begin(), s->e1.begin() + (long)s->ehead);
    s->ehead = 0;
  }
}

// Channelise `nrows` FB rows starting at stream row `row_first` into `out`
// (ring row out_row0, mask).  Samples of row r are stream positions
// [r*S, (r+1)*S) of each pol, S = NAVE*TWONCHAN.
int launch_rows(vfrb_plan* pl, StreamSt* s, int64_t row_first, int64_t nrows, float* out, int64_t out_row0,
                unsigned mask) {
  const Range nvtx_range("vfrb channelise");
  const vfrb_layout& L = pl->L;
  const int64_t S = (int64_t)L.nave * L.twonchan;
  const int64_t p0 = row_first * S, p1 = (row_first + nrows) * S;
  const int64_t e_lo = p0 / kDataLen, e_hi = (p1 + kDataLen - 1) / kDataLen;
  const int64_t n = e_hi - e_lo;
  if (n > s->slots_cap || e_lo < s->ebase || e_hi > npairs(s)) return VFRB_ERR;
  SlotBuf& b = s->sb[s->sb_i];
  s->sb_i = (s->sb_i + 1) % kSlotBufs;
  CK(cudaEventSynchronize(b.ev));  // the upload from this buffer kSlotBufs launches ago is done
  for (int64_t i = 0; i < n; ++i) {
    const size_t k = s->ehead + (size_t)(e_lo - s->ebase + i);
    b.h[i] = entry_offset(s, s->e0[k]);
    b.h[s->slots_cap + i] = entry_offset(s, s->e1[k]);
  }
  if (want(pl, VFRB_OUT_FLAGS)) {
    // row r holds pol bytes [r*S, (r+1)*S): the entries that cover them
    const bool blk = pl->P.mode == VFRB_MODE_BLOCK;
    for (int64_t r = 0; r < nrows; ++r) {
      const int64_t a0 = (row_first + r) * S / kDataLen, a1 = ((row_first + r + 1) * S - 1) / kDataLen;
      uint8_t f = 0;
      for (int64_t e = a0; e <= a1; ++e) {
        const size_t k = s->ehead + (size_t)(e - s->ebase);
        f |= entry_flag(s, s->e0[k]) | entry_flag(s, s->e1[k]);
      }
      s->rflags[(size_t)(blk ? out_row0 + r : (row_first + r) & s->fmask)] = f;
    }
  }
  // The upload goes on the copy stream: host-to-device copies queued on the
  // compute stream would sit in the copy engine's queue until the compute
  // stream reached them and hold up the frame copies behind them.  It waits
  // for the channeliser that last read this device buffer.
  CK(cudaStreamWaitEvent(s->xs, b.ev_used, 0));
  CK(cudaMemcpyAsync(b.d, b.h, sizeof(int64_t) * 2 * s->slots_cap, cudaMemcpyHostToDevice, s->xs));
  CK(cudaEventRecord(b.ev, s->xs));
  CK(cudaStreamWaitEvent(s->cs, b.ev, 0));
  vfrb_chan_args a{};
  a.frames = s->d_frames;
  a.slots0 = b.d;
  a.slots1 = b.d + s->slots_cap;
  a.nslots = n;
  a.sample0 = p0 - e_lo * kDataLen;
  a.nrows = (int32_t)nrows;
  a.twonchan = L.twonchan;
  a.nave = L.nave;
  a.nfreq = L.nfreq;
  a.nskip = L.nskip;
  a.nchanout = L.nchanout;
  a.out = out;
  a.out_row_stride = L.nchanout;
  a.out_row0 = out_row0;
  a.out_row_mask = mask;
  a.d_err = s->d_err;
  ST(launch_channelise(a, s->cs));
  CK(cudaEventRecord(b.ev_used, s->cs));
  CK(cudaEventRecord(s->ev_consumed, s->cs));
  if (s->rel_n == StreamSt::kRelEv) {  // drop the oldest: later copies wait on newer (later) launches
    s->rel_head = (s->rel_head + 1) % StreamSt::kRelEv;
    --s->rel_n;
  }
  const int k = (s->rel_head + s->rel_n) % StreamSt::kRelEv;
  CK(cudaEventRecord(s->rel_ev[k], s->cs));
  s->rel_after[k] = INT64_MIN;  // set when this launch's entries are consumed
  ++s->rel_n;
  return VFRB_OK;
}

// FP16/int8: weights from the variance of the first window (one extra F32
// bandpass pass of 128 rows into scratch).
int init_scale(vfrb_plan* pl, StreamSt* s, const float* raw, int64_t row0, unsigned mask) {
  if (s->scale_ready || pl->P.storage == VFRB_F32) return VFRB_OK;
  vfrb_bp_args a{};
  a.in = raw;
  a.in_row_stride = pl->L.nchanout;
  a.in_row0 = row0;
  a.in_row_mask = mask;
  a.nchan = pl->L.nchanout;
  a.nrows = 128;
  a.window = 128;
  a.storage = VFRB_F32;
  a.out = s->d_scr;
  a.out_chan_stride = 128;
  a.out_row_mask = 0xffffffffu;
  a.win_var = s->d_var;
  ST(launch_bandpass(a, s->cs));
  const int nch = pl->L.nchanout;
  if (pl->P.storage == VFRB_F16) {
    k_uniform_scale<<<1, 256, 0, s->cs>>>(s->d_var, nch, s->d_w, s->d_inv);
    CK(cudaGetLastError());
    // the dedisperser takes S by value: read it once per stream
    CK(cudaMemcpyAsync(&s->uscale, s->d_w, sizeof(float), cudaMemcpyDeviceToHost, s->cs));
    CK(cudaStreamSynchronize(s->cs));
  } else {
    k_init_scale<<<(nch + 255) / 256, 256, 0, s->cs>>>(s->d_var, nch, pl->P.q_scale, pl->P.storage, s->d_w,
                                                        s->d_inv);
    CK(cudaGetLastError());
  }
  s->scale_ready = true;
  return VFRB_OK;
}

int run_bandpass(vfrb_plan* pl, StreamSt* s, const float* raw, int64_t in_row0, unsigned in_mask, int64_t nrows,
                 int64_t out_row0, float* tm_out, int subtract_mode = 0) {
  const Range nvtx_range("vfrb bandpass");
  ST(init_scale(pl, s, raw, in_row0, in_mask));
  vfrb_bp_args a{};
  a.in = raw;
  a.in_row_stride = pl->L.nchanout;
  a.in_row0 = in_row0;
  a.in_row_mask = in_mask;
  a.nchan = pl->L.nchanout;
  a.nrows = (int32_t)nrows;
  a.window = 128;
  a.storage = pl->P.storage;
  a.out = s->d_cm;
  a.out_chan_stride = s->cm_stride;
  a.out_row0 = out_row0;
  a.out_row_mask = s->cm_mask;
  a.inv_scale = pl->P.storage == VFRB_F32 ? nullptr : s->d_inv;
  a.q_scale = pl->P.q_scale;
  a.tm_out = tm_out;
  a.tm_row_stride = pl->L.nchanout;
  a.d_err = s->d_err;
  a.subtract_mode = subtract_mode;
  a.out_shift1 = pl->P.storage == VFRB_F16 ? s->d_cm1 : nullptr;
  return launch_bandpass(a, s->cs);
}

// Dedisperse nt samples into d_out.  kernel_stats: calcstats (and the boxcar
// search) of the whole launch, fused (block mode); otherwise each output
// chunk gets its statistics from chunk_stats (stream mode).
int run_dedisp(vfrb_plan* pl, StreamSt* s, int64_t row0, int64_t nrows_valid, int64_t nt, bool kernel_stats,
               cudaStream_t on = nullptr) {
  const Range nvtx_range("vfrb dedisperse");
  vfrb_dd_args a{};
  a.fb = s->d_cm;
  a.storage = pl->P.storage;
  a.chan_scale = pl->P.storage == VFRB_I8 ? s->d_w : nullptr;
  a.uniform_scale = pl->P.storage == VFRB_F16 ? s->uscale : 0.f;
  a.chan_stride = s->cm_stride;
  a.row0 = row0;
  a.row_mask = s->cm_mask;
  a.nrows_valid = nrows_valid;
  a.nt_out = nt;
  a.out = s->d_out;
  a.out_stride = s->out_stride;
  a.sigma_out = want(pl, VFRB_OUT_SIGMA) ? s->d_sig : nullptr;
  a.workspace = s->d_ws;
  a.workspace_bytes = s->ws_bytes;
  const bool stats = kernel_stats && (want(pl, VFRB_OUT_DMSTATS) || want(pl, VFRB_OUT_CANDS));
  a.ave = stats ? s->d_ave : nullptr;
  a.sigma = stats ? s->d_sgm : nullptr;
  a.peak = stats ? s->d_peak : nullptr;
  a.frb = stats ? s->d_frb : nullptr;
  a.argmax = stats ? s->d_arg : nullptr;
  a.d_err = s->d_err;
  a.fb_shift1 = pl->P.storage == VFRB_F16 ? s->d_cm1 : nullptr;
  ST(launch_dedisperse_plan(pl->dd, a, on ? on : s->cs));
  if (kernel_stats && boxcar_on(pl))
    ST(launch_boxcar(s->d_out, pl->ndm, nt, s->out_stride, s->d_ave, s->d_sgm, pl->P.boxcar_max, s->d_bsnr, s->d_bt,
                     s->d_bw, s->cs));
  return VFRB_OK;
}

// Copy this result's outputs to the host and queue it.
int emit(vfrb_plan* pl, StreamSt* s, int64_t seq, int64_t row0, int64_t nt, bool with_fb, int64_t col0 = 0,
         double t_data = -1.0) {
  ResultSlot* r = nullptr;
  ST(alloc_slot(pl, s, &r));
  const int64_t nch = pl->L.nchanout;
  if (pl->want_dd && nt > 0) {
    if (want(pl, VFRB_OUT_DEDISP))
      CK(cudaMemcpy2DAsync(r->dd, nt * 4, s->d_out + col0, s->out_stride * 4, nt * 4, pl->ndm, cudaMemcpyDeviceToHost,
                           s->cs));
    if (want(pl, VFRB_OUT_SIGMA))
      CK(cudaMemcpy2DAsync(r->dds, nt * 4, s->d_sig + col0, s->out_stride * 4, nt * 4, pl->ndm, cudaMemcpyDeviceToHost,
                           s->cs));
    if (want(pl, VFRB_OUT_DMSTATS) || want(pl, VFRB_OUT_CANDS)) {
      CK(cudaMemcpyAsync(r->ave, s->d_ave, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
      CK(cudaMemcpyAsync(r->sig, s->d_sgm, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
      CK(cudaMemcpyAsync(r->peak, s->d_peak, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
      CK(cudaMemcpyAsync(r->frb, s->d_frb, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
      CK(cudaMemcpyAsync(r->arg, s->d_arg, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
    }
    if (boxcar_on(pl)) {
      CK(cudaMemcpyAsync(r->bsnr, s->d_bsnr, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
      CK(cudaMemcpyAsync(r->bt, s->d_bt, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
      CK(cudaMemcpyAsync(r->bw, s->d_bw, pl->ndm * 4, cudaMemcpyDeviceToHost, s->cs));
    }
  }
  if (with_fb && r->fb) CK(cudaMemcpyAsync(r->fb, s->d_fbt, (size_t)pl->L.maxnt * nch * 4, cudaMemcpyDeviceToHost, s->cs));
  const bool cst = pl->P.mode == VFRB_MODE_BLOCK && want(pl, VFRB_OUT_CHANSTATS);
  if (cst) {
    const size_t b = (size_t)pl->nstatblks * nch * 4;
    CK(cudaMemcpyAsync(r->cave, s->d_cave, b, cudaMemcpyDeviceToHost, s->cs));
    CK(cudaMemcpyAsync(r->csig, s->d_csig, b, cudaMemcpyDeviceToHost, s->cs));
    CK(cudaMemcpyAsync(r->cout, s->d_cout, b, cudaMemcpyDeviceToHost, s->cs));
    CK(cudaMemcpyAsync(r->csk, s->d_csk, b, cudaMemcpyDeviceToHost, s->cs));
  }
  r->flags.clear();
  if (want(pl, VFRB_OUT_FLAGS)) {
    if (pl->P.mode == VFRB_MODE_BLOCK) {
      r->flags = s->rflags;
    } else {
      r->flags.resize((size_t)nt);
      for (int64_t i = 0; i < nt; ++i) r->flags[(size_t)i] = s->rflags[(size_t)((row0 + i) & s->fmask)];
    }
  }
  CK(cudaMemcpyAsync(r->err, s->d_err, 4, cudaMemcpyDeviceToHost, s->cs));
  CK(cudaMemsetAsync(s->d_err, 0, 4, s->cs));
  r->t_done = 0.0;
  CK(cudaLaunchHostFunc(s->cs, mark_done, r));
  CK(cudaEventRecord(r->ev, s->cs));
  vfrb_result& o = r->r;
  o = vfrb_result{};
  o.stream = s->id;
  o.seq = seq;
  o.row0 = row0;
  o.tstart_mjd = s->tstart_mjd;
  o.ndm = pl->want_dd ? pl->ndm : 0;
  o.nt = pl->want_dd ? nt : 0;
  const bool stats = pl->want_dd && (want(pl, VFRB_OUT_DMSTATS) || want(pl, VFRB_OUT_CANDS));
  o.dd = (pl->want_dd && want(pl, VFRB_OUT_DEDISP)) ? r->dd : nullptr;
  o.dd_sigma = (pl->want_dd && want(pl, VFRB_OUT_SIGMA)) ? r->dds : nullptr;
  o.ave = stats ? r->ave : nullptr;
  o.sigma = stats ? r->sig : nullptr;
  o.peak = stats ? r->peak : nullptr;
  o.frb = stats ? r->frb : nullptr;
  o.argmax = stats ? r->arg : nullptr;
  o.box_snr = (stats && r->bsnr) ? r->bsnr : nullptr;
  o.box_start = (stats && r->bt) ? r->bt : nullptr;
  o.box_width = (stats && r->bw) ? r->bw : nullptr;
  o.nchan = (int32_t)nch;
  o.fb_rows = (with_fb && r->fb) ? pl->L.maxnt : 0;
  o.fb = (with_fb && r->fb) ? r->fb : nullptr;
  o.nstatblks = cst ? pl->nstatblks : 0;
  o.chan_ave = cst ? r->cave : nullptr;
  o.chan_sig = cst ? r->csig : nullptr;
  o.chan_outlier = cst ? r->cout : nullptr;
  o.chan_sk = cst ? r->csk : nullptr;
  o.nflag_rows = (int64_t)r->flags.size();
  o.row_flags = r->flags.empty() ? nullptr : r->flags.data();
  r->t_data = t_data >= 0.0 ? t_data : s->t_push;
  r->state = 1;
  pl->queue.push_back(r);
  return VFRB_OK;
}

int block_complete(vfrb_plan* pl, StreamSt* s) {
  const Range nvtx_range("vfrb block");
  const vfrb_layout& L = pl->L;
  const int64_t nch = L.nchanout;
  if (pl->want_dd && pl->max_delay > 0)
    CK(cudaMemcpyAsync(s->d_left, s->d_fb_tm + (int64_t)(L.maxnt - pl->max_delay) * nch,
                       (size_t)pl->max_delay * nch * 4, cudaMemcpyDeviceToDevice, s->cs));
  const bool with_fb = want(pl, VFRB_OUT_FB) && (pl->P.fb_block < 0 || pl->P.fb_block == s->blocks);
  const bool full_bp = pl->P.bp_mode == VFRB_BP_FULL;
  if (!full_bp && !pl->P.zero_dm) {
    ST(run_bandpass(pl, s, s->d_fb_tm, 0, 0xffffffffu, L.maxnt, 0, with_fb ? s->d_fbt : nullptr));
  } else {
    // subtractbp (whole block, PIPE:1372) in place of subtractbpCAL, and/or
    // subtractZERO after it (PIPE:661): in place on the FP32 block
    ST(run_bandpass(pl, s, s->d_fb_tm, 0, 0xffffffffu, L.maxnt, 0, nullptr, full_bp ? 1 : 0));
    float* cm = (float*)s->d_cm;
    if (full_bp) ST(launch_subtract_bp_full(cm, s->cm_stride, 0, 0xffffffffu, (int)nch, L.maxnt, s->cs));
    if (pl->P.zero_dm) ST(launch_subtract_zero(cm, s->cm_stride, 0, 0xffffffffu, (int)nch, L.maxnt, s->cs));
    if (with_fb) ST(launch_fb_transpose(cm, s->cm_stride, 0xffffffffu, 0, (int)nch, L.maxnt, s->d_fbt, nch, s->cs));
  }
  if (want(pl, VFRB_OUT_CHANSTATS)) {
    vfrb_cs_args c{};
    c.fb = (const float*)s->d_cm;
    c.chan_stride = s->cm_stride;
    c.row_mask = 0xffffffffu;
    c.nchan = (int32_t)nch;
    c.nrows = L.maxnt;
    c.ncolstatblk = pl->ncolstatblk;
    c.nstatblks = pl->nstatblks;
    c.ave = s->d_cave;
    c.sig = s->d_csig;
    c.outlier = s->d_cout;
    ST(launch_chan_stats(c, s->cs));
    // spectral kurtosis of the raw block (d_fb_tm is not modified by the bandpass)
    ST(launch_chan_sk(s->d_fb_tm, nch, (int)nch, L.maxnt, pl->ncolstatblk, pl->nstatblks, 2 * L.nave, s->d_csk,
                      s->cs));
  }
  if (pl->want_dd) ST(run_dedisp(pl, s, 0, L.maxnt, pl->nt_block, true));
  // absolute FB row of block row 0: block 0 starts at row 0; each later block
  // begins with the previous block's last max_delay rows, and its new rows
  // (from row `first` on) follow the previous block's last row
  const int64_t first = (int64_t)(pl->max_delay / L.nbundle) * L.nbundle;
  const int64_t row0 =
      s->blocks == 0 ? 0 : (int64_t)L.maxnt - pl->max_delay + (s->blocks - 1) * ((int64_t)L.maxnt - first);
  ST(emit(pl, s, s->blocks, row0, pl->want_dd ? pl->nt_block : 0, with_fb));
  if (pl->want_dd && pl->max_delay > 0) {
    CK(cudaMemcpyAsync(s->d_fb_tm, s->d_left, (size_t)pl->max_delay * nch * 4, cudaMemcpyDeviceToDevice, s->cs));
    std::memmove(s->rflags.data(), s->rflags.data() + (L.maxnt - pl->max_delay), (size_t)pl->max_delay);
    s->loopcnt = pl->max_delay / L.nbundle;
  } else {
    s->loopcnt = 0;
  }
  ++s->blocks;
  return VFRB_OK;
}

// calcstats (and the boxcar search) of one output chunk held in d_out
// columns [col0, col0 + nt): always computed per chunk from the series, so
// the statistics do not depend on how chunks were batched.
int chunk_stats(vfrb_plan* pl, StreamSt* s, int64_t col0, int64_t nt) {
  if (!(want(pl, VFRB_OUT_DMSTATS) || want(pl, VFRB_OUT_CANDS))) return VFRB_OK;
  ST(launch_series_stats(s->d_out + col0, pl->ndm, nt, s->out_stride, s->d_ave, s->d_sgm, s->d_peak, s->d_frb,
                         s->d_arg, s->cs));
  if (boxcar_on(pl))
    ST(launch_boxcar(s->d_out + col0, pl->ndm, nt, s->out_stride, s->d_ave, s->d_sgm, pl->P.boxcar_max, s->d_bsnr,
                     s->d_bt, s->d_bw, s->cs));
  return VFRB_OK;
}

// Stream mode, VFRB_OUT_CHANSTATS: statistics of TIMESTATS block k (rows
// [k*ncol, (k+1)*ncol) of the stream), once the bandpass has covered it, as
// a result of its own (nstatblks = 1, no series): calcstats per channel
// (STATS:910-946) of the bandpassed FP32 rows in the channel-major ring, and
// the spectral kurtosis of the raw rows still in the raw ring.
int stream_stats_block(vfrb_plan* pl, StreamSt* s, int64_t k) {
  const Range nvtx_range("vfrb stream stats");
  const vfrb_layout& L = pl->L;
  const int64_t nch = L.nchanout;
  const int64_t row0 = k * pl->ncolstatblk;
  vfrb_cs_args c{};
  c.fb = (const float*)s->d_cm;
  c.chan_stride = s->cm_stride;
  c.row0 = row0;
  c.row_mask = s->cm_mask;
  c.nchan = (int32_t)nch;
  c.nrows = pl->ncolstatblk;
  c.ncolstatblk = pl->ncolstatblk;
  c.nstatblks = 1;
  c.ave = s->d_cave;
  c.sig = s->d_csig;
  c.outlier = s->d_cout;
  ST(launch_chan_stats(c, s->cs));
  ST(launch_chan_sk_ring(s->d_raw, nch, row0, (unsigned long long)(s->R1 - 1), (int)nch, pl->ncolstatblk,
                         pl->ncolstatblk, 1, 2 * L.nave, s->d_csk, s->cs));
  ResultSlot* r = nullptr;
  ST(alloc_slot(pl, s, &r));
  const size_t b = (size_t)nch * 4;
  CK(cudaMemcpyAsync(r->cave, s->d_cave, b, cudaMemcpyDeviceToHost, s->cs));
  CK(cudaMemcpyAsync(r->csig, s->d_csig, b, cudaMemcpyDeviceToHost, s->cs));
  CK(cudaMemcpyAsync(r->cout, s->d_cout, b, cudaMemcpyDeviceToHost, s->cs));
  CK(cudaMemcpyAsync(r->csk, s->d_csk, b, cudaMemcpyDeviceToHost, s->cs));
  r->flags.clear();
  if (want(pl, VFRB_OUT_FLAGS)) {
    r->flags.resize((size_t)pl->ncolstatblk);
    for (int64_t i = 0; i < pl->ncolstatblk; ++i) r->flags[(size_t)i] = s->rflags[(size_t)((row0 + i) & s->fmask)];
  }
  CK(cudaMemcpyAsync(r->err, s->d_err, 4, cudaMemcpyDeviceToHost, s->cs));
  CK(cudaMemsetAsync(s->d_err, 0, 4, s->cs));
  r->t_done = 0.0;
  CK(cudaLaunchHostFunc(s->cs, mark_done, r));
  CK(cudaEventRecord(r->ev, s->cs));
  vfrb_result& o = r->r;
  o = vfrb_result{};
  o.stream = s->id;
  o.seq = k;
  o.row0 = row0;
  o.tstart_mjd = s->tstart_mjd;
  o.nchan = (int32_t)nch;
  o.nstatblks = 1;
  o.chan_ave = r->cave;
  o.chan_sig = r->csig;
  o.chan_outlier = r->cout;
  o.chan_sk = r->csk;
  o.nflag_rows = (int64_t)r->flags.size();
  o.row_flags = r->flags.empty() ? nullptr : r->flags.data();
  r->t_data = s->t_push;
  r->state = 1;
  pl->queue.push_back(r);
  return VFRB_OK;
}

// k output chunks of nt samples each with one dedispersion launch
bool batching(const vfrb_plan* pl) {
  return pl->P.batch_streams && pl->P.mode == VFRB_MODE_STREAM && !want(pl, VFRB_OUT_SIGMA) && pl->bs;
}

// The pending streams' chunks dedispersed by one launch on the plan's batch
// stream (after each stream's bandpass, recorded in its ev_ready), then each
// stream's per-chunk statistics and results on its own stream after the
// launch.  Results are the per-stream launch's bit for bit: the same kernel
// with the same inputs.
int flush_batch(vfrb_plan* pl) {
  if (pl->pending.empty()) return VFRB_OK;
  const Range nvtx_range("vfrb batched dedisperse");
  std::vector<DdJob> jobs;
  for (StreamSt* s : pl->pending) {
    CK(cudaStreamWaitEvent(pl->bs, s->ev_ready, 0));
    DdJob j{};
    j.fb = s->d_cm;
    j.fb1 = s->d_cm1;
    j.out_scale = pl->P.storage == VFRB_F16 ? s->uscale : 1.f;
    j.row0 = s->job_row0;
    j.nrows_valid = s->job_nvalid;
    j.nt_out = s->job_k * s->job_nt;
    j.out = s->d_out;
    j.out_stride = s->out_stride;
    j.err = s->d_err;
    jobs.push_back(j);
  }
  StreamSt* s0 = pl->pending.front();
  int launched = 0;
  ST(launch_dedisperse_jobs(pl->dd, pl->P.storage, jobs.data(), (int)jobs.size(), s0->cm_stride, s0->cm_mask, pl->bs,
                            &launched));
  if (!launched)  // the plan's kernel has no batched form: one launch per stream, on the batch stream
    for (StreamSt* s : pl->pending) ST(run_dedisp(pl, s, s->job_row0, s->job_nvalid, s->job_k * s->job_nt, false, pl->bs));
  CK(cudaEventRecord(pl->ev_batch, pl->bs));
  std::vector<StreamSt*> done;
  done.swap(pl->pending);
  for (StreamSt* s : done) {
    CK(cudaStreamWaitEvent(s->cs, pl->ev_batch, 0));
    for (int64_t i = 0; i < s->job_k; ++i) {
      ST(chunk_stats(pl, s, i * s->job_nt, s->job_nt));
      ST(emit(pl, s, s->job_seq0 + i, s->job_row0 + i * s->job_nt, s->job_nt, false, i * s->job_nt, s->job_t_push));
    }
    s->job = false;
  }
  return VFRB_OK;
}

int stream_chunks(vfrb_plan* pl, StreamSt* s, int64_t k, int64_t nt) {
  const Range nvtx_range("vfrb stream chunks");
  if (batching(pl)) {
    // a stream's output buffer holds one job: a second one waits for the first's launch
    if (s->job || (int)pl->pending.size() >= kDdMaxJobs) ST(flush_batch(pl));
    CK(cudaEventRecord(s->ev_ready, s->cs));
    s->job = true;
    s->job_row0 = s->rows_out;
    s->job_nvalid = s->rows_bp - s->rows_out;
    s->job_k = k;
    s->job_nt = nt;
    s->job_seq0 = s->chunks;
    s->job_t_push = s->t_push;
    s->rows_out += k * nt;
    s->chunks += k;
    pl->pending.push_back(s);
    return VFRB_OK;
  }
  ST(run_dedisp(pl, s, s->rows_out, s->rows_bp - s->rows_out, k * nt, false));
  for (int64_t i = 0; i < k; ++i) {
    ST(chunk_stats(pl, s, i * nt, nt));
    ST(emit(pl, s, s->chunks, s->rows_out, nt, false, i * nt));
    s->rows_out += nt;
    ++s->chunks;
  }
  return VFRB_OK;
}

// Turn every complete bundle / row / window into work.
int process(vfrb_plan* pl, StreamSt* s, bool final_flush) {
  const vfrb_layout& L = pl->L;
  const int64_t S = (int64_t)L.nave * L.twonchan;
  if (pl->P.mode == VFRB_MODE_BLOCK) {
    const int64_t per_block = L.maxnt / L.nbundle;
    for (;;) {
      // bundle b is complete once the pair read after its last byte exists (PIPE:1143-1158)
      int64_t nb = 0;
      const int64_t have = npairs(s);
      while (true) {
        const int64_t b = s->bundles_done + nb;
        const int64_t need = ((b + 1) * (int64_t)L.nloop) / kDataLen;
        if (need >= have) break;
        if (s->loopcnt + nb + 1 > per_block) break;
        if ((nb + 1) * L.nbundle > pl->launch_rows) break;
        ++nb;
      }
      if (nb == 0) break;
      ST(launch_rows(pl, s, s->bundles_done * L.nbundle, nb * L.nbundle, s->d_fb_tm, (int64_t)s->loopcnt * L.nbundle,
                     0xffffffffu));
      s->bundles_done += nb;
      s->loopcnt += (int)nb;
      consume_entries(s, (s->bundles_done * (int64_t)L.nloop) / kDataLen);
      if (s->loopcnt == per_block) ST(block_complete(pl, s));
    }
    return VFRB_OK;
  }
  const bool stats = want(pl, VFRB_OUT_CHANSTATS);
  for (;;) {
    const int64_t avail = npairs(s) * kDataLen / S;
    int64_t n = std::min(avail - s->rows_chan, pl->launch_rows);
    n = std::min(n, s->R1 - 256 - (s->rows_chan - s->rows_bp));
    // the raw rows of the statistics block in progress stay in the raw ring
    if (stats) n = std::min(n, s->R1 - (s->rows_chan - s->stat_blocks * pl->ncolstatblk));
    if (n <= 0) break;
    ST(launch_rows(pl, s, s->rows_chan, n, s->d_raw, s->rows_chan, (unsigned)(s->R1 - 1)));
    s->rows_chan += n;
    consume_entries(s, (s->rows_chan * S) / kDataLen);
    const int64_t w1 = (s->rows_chan / 128) * 128;
    // a pending job's rows stay in the channel-major ring until its launch
    if (s->job && w1 > s->job_row0 + (int64_t)s->cm_mask + 1) ST(flush_batch(pl));
    if (w1 > s->rows_bp) {
      ST(run_bandpass(pl, s, s->d_raw, s->rows_bp, (unsigned)(s->R1 - 1), w1 - s->rows_bp, s->rows_bp, nullptr));
      s->rows_bp = w1;
    }
    // statistics results stay after the stream's earlier series results
    if (stats && s->job && (s->stat_blocks + 1) * pl->ncolstatblk <= s->rows_bp) ST(flush_batch(pl));
    while (stats && (s->stat_blocks + 1) * pl->ncolstatblk <= s->rows_bp) {
      ST(stream_stats_block(pl, s, s->stat_blocks));
      ++s->stat_blocks;
    }
    if (pl->want_dd)
      for (;;) {  // a backlog of chunks is dedispersed in one launch (fills the GPU better)
        const int64_t k = (s->rows_bp - pl->max_delay - s->rows_out) / pl->chunk_rows;
        if (k < 1) break;
        ST(stream_chunks(pl, s, std::min(k, pl->batch_chunks), pl->chunk_rows));
      }
  }
  if (final_flush && pl->want_dd) {
    const int64_t rem = s->rows_bp - pl->max_delay - s->rows_out;
    if (rem > 0) ST(stream_chunks(pl, s, 1, rem));
  }
  return VFRB_OK;
}

int run_reader(vfrb_plan* pl, StreamSt* s) {
  const auto r = s->reader->run(s->e0, s->e1);
  if (!s->started && s->reader->initialised()) {
    s->started = true;
    vfrb_hdr h = s->reader->start_header();
    s->tstart_mjd = vfrb_header_dmjd(&h, kFramesPerSec);
  }
  for (auto& l : s->reader->log()) {
    s->logtext += l;
    s->logtext += '\n';
  }
  s->reader->log().clear();
  if (r == PairReader::STEP_ERROR) s->reader_error = VFRB_ERR;
  (void)pl;
  return VFRB_OK;
}

// Oldest frame index still referenced by unconsumed entries or queued frames.
int64_t oldest_ref(const StreamSt* s) {
  int64_t o = s->frames_in - (int64_t)s->reader->queued();
  for (size_t k = s->ehead; k < s->e0.size(); ++k) {
    if (s->e0[k] >= 0) o = std::min(o, s->e0[k]);
    if (s->e1[k] >= 0) o = std::min(o, s->e1[k]);
    if (s->e0[k] >= 0 && s->e1[k] >= 0) break;  // entries are in read order
  }
  return o;
}

// Copy `nf` whole frames to the ring, queue their headers, advance.
int feed_frames(vfrb_plan* pl, StreamSt* s, const uint8_t* in, int64_t nf, MemKind kind) {
  const Range nvtx_range("vfrb feed frames");
  const bool pinned = kind == kPinned, device = kind == kDevice;
  // page-locked input is copied in place, in quarters of the ring; other
  // input goes through the (smaller) staging buffers, whose frame count also
  // bounds a batch of device input (its headers are brought there)
  const int64_t batch_max = std::max<int64_t>(
      1, pinned || device ? s->ring_frames / 4 : std::min<int64_t>(s->ring_frames / 4, (int64_t)s->stage_frames));
  size_t pitch = kFrameLen;  // of the headers the reader reads
  for (int64_t done = 0; done < nf;) {
    const int64_t nb = std::min(batch_max, nf - done);
    const uint8_t* src = in + done * kFrameLen;  // host bytes, or device bytes (device input)
    // frames about to be overwritten must have been consumed by launched work
    if (oldest_ref(s) < s->frames_in + nb - s->ring_frames) {
      ST(process(pl, s, false));
      if (oldest_ref(s) < s->frames_in + nb - s->ring_frames) return VFRB_ERR_NOMEM;  // ring too small
    }
    // the ring slots of this batch held frames below X; wait for the first
    // channeliser launch after which none of them is read again
    const int64_t X = s->frames_in + nb - s->ring_frames;
    if (X > 0) {
      cudaEvent_t wait_ev = s->ev_consumed;  // the latest launch, if no recorded one suffices
      while (s->rel_n > 0) {
        const int k = s->rel_head;
        if (s->rel_after[k] >= X) {
          wait_ev = s->rel_ev[k];
          break;
        }
        s->rel_head = (s->rel_head + 1) % StreamSt::kRelEv;  // frees too little now, and X only grows
        --s->rel_n;
      }
      CK(cudaStreamWaitEvent(s->xs, wait_ev, 0));
    }
    const uint8_t* from = src;
    if (device) {
      // headers to the host packed (32 bytes a frame) by one strided copy on
      // the copy engine, where the reader reads them; frames device to
      // device.  Measured on B200 per data-second of frames: 0.08 ms for this
      // copy against 0.23 ms into a 5032-byte pitch, and host reads of
      // headers 5032 bytes apart (a page each) cost ~1.3 ms.  A gather
      // kernel would wait for the channeliser's persistent CTAs to leave the
      // SMs.
      CK(cudaMemcpy2DAsync(s->h_hdr, kHdrLen, src, kFrameLen, kHdrLen, (size_t)nb, cudaMemcpyDeviceToHost, s->hs));
      const int64_t slot0 = s->frames_in % s->ring_frames;
      const int64_t n1 = std::min(nb, s->ring_frames - slot0);
      CK(cudaMemcpyAsync(s->d_frames + slot0 * kFrameLen, src, (size_t)n1 * kFrameLen, cudaMemcpyDeviceToDevice, s->xs));
      if (nb > n1)
        CK(cudaMemcpyAsync(s->d_frames, src + n1 * kFrameLen, (size_t)(nb - n1) * kFrameLen, cudaMemcpyDeviceToDevice,
                           s->xs));
      CK(cudaStreamSynchronize(s->hs));
      src = s->h_hdr;  // the reader and the flags below read the headers only
      pitch = kHdrLen;
    } else if (!pinned) {
      const int k = s->stage_i;
      s->stage_i = (s->stage_i + 1) % kStageBufs;
      CK(cudaEventSynchronize(s->stage_ev[k]));
      std::memcpy(s->h_stage[k], src, (size_t)nb * kFrameLen);
      from = s->h_stage[k];
      // the staging event is recorded after the copies below
      const int64_t slot0 = s->frames_in % s->ring_frames;
      const int64_t n1 = std::min(nb, s->ring_frames - slot0);
      CK(cudaMemcpyAsync(s->d_frames + slot0 * kFrameLen, from, (size_t)n1 * kFrameLen, cudaMemcpyHostToDevice, s->xs));
      if (nb > n1)
        CK(cudaMemcpyAsync(s->d_frames, from + n1 * kFrameLen, (size_t)(nb - n1) * kFrameLen, cudaMemcpyHostToDevice,
                           s->xs));
      CK(cudaEventRecord(s->stage_ev[k], s->xs));
    } else {
      const int64_t slot0 = s->frames_in % s->ring_frames;
      const int64_t n1 = std::min(nb, s->ring_frames - slot0);
      CK(cudaMemcpyAsync(s->d_frames + slot0 * kFrameLen, from, (size_t)n1 * kFrameLen, cudaMemcpyHostToDevice, s->xs));
      if (nb > n1)
        CK(cudaMemcpyAsync(s->d_frames, from + n1 * kFrameLen, (size_t)(nb - n1) * kFrameLen, cudaMemcpyHostToDevice,
                           s->xs));
    }
    CK(cudaEventRecord(s->ev_copied, s->xs));
    CK(cudaStreamWaitEvent(s->cs, s->ev_copied, 0));
    // the VDIF invalid bit (word 0, bit 31) of each frame, for row flags
    {
      int64_t slot = s->frames_in % s->ring_frames;
      for (int64_t f = 0; f < nb; ++f) {
        s->finv[(size_t)slot] = (src[f * pitch + 3] >> 7) & 1;
        if (++slot == s->ring_frames) slot = 0;
      }
    }
    // in-order pairs go straight to pair entries; the rest through the queue
    int64_t i = (int64_t)s->reader->run_fast(src, s->frames_in, (size_t)nb, s->e0, s->e1, pitch);
    for (; i < nb; ++i) {
      QFrame q;
      vfrb_decode_header(src + i * pitch, &q.h);
      q.payload = s->frames_in + i;
      s->reader->push(q);
    }
    s->frames_in += nb;
    ST(run_reader(pl, s));
    ST(process(pl, s, false));
    done += nb;
  }
  if (pinned || device) CK(cudaEventSynchronize(s->ev_copied));  // the caller may reuse its buffer on return
  return VFRB_OK;
}

int free_plan(vfrb_plan* pl) {
  if (!pl) return VFRB_OK;
  for (auto& s : pl->st)
    if (s) s->res.release();
  if (pl->bs) {
    cudaStreamSynchronize(pl->bs);
    cudaStreamDestroy(pl->bs);
  }
  if (pl->ev_batch) cudaEventDestroy(pl->ev_batch);
  if (pl->dd) ddplan_destroy(pl->dd);
  delete pl;
  return VFRB_OK;
}

// Appends stream `id` to pl->st first, so a failure part-way leaves its
// allocations where free_plan (or vfrb_stream_open) releases them.
int create_stream(vfrb_plan* pl, int id, int64_t ring_frames, int64_t R1, int64_t R2) {
  pl->st.push_back(std::make_unique<StreamSt>());
  StreamSt* s = pl->st.back().get();
  const vfrb_params& P = pl->P;
  const vfrb_layout& L = pl->L;
  const int64_t nch = L.nchanout;
  s->id = id;
  s->reader = std::make_unique<PairReader>(P.reader == VFRB_READER_TS ? PairReader::TS : PairReader::PIPE,
                                           P.dada_skip != 0);
  ST(mkstream(s->res, &s->cs));
  ST(mkstream(s->res, &s->xs));
  ST(mkstream(s->res, &s->hs));
  ST(mkevent(s->res, &s->ev_copied));
  ST(mkevent(s->res, &s->ev_consumed));
  ST(mkevent(s->res, &s->ev_ready));
  ST(mkevent(s->res, &s->ev_input));
  for (auto& e : s->rel_ev) ST(mkevent(s->res, &e));
  CK(cudaEventRecord(s->ev_consumed, s->cs));
  s->ring_frames = ring_frames;
  s->finv.assign((size_t)ring_frames, 0);
  ST(dmalloc(s->res, &s->d_frames, (size_t)ring_frames * kFrameLen + (size_t)kStash * kDataLen));
  s->stage_frames = (size_t)std::min<int64_t>(ring_frames / 4, 8192);
  ST(hmalloc(s->res, &s->h_hdr, (size_t)std::max<int64_t>(1, ring_frames / 4) * kHdrLen));
  for (int k = 0; k < kStageBufs; ++k) {
    ST(hmalloc(s->res, &s->h_stage[k], s->stage_frames * kFrameLen));
    ST(mkevent(s->res, &s->stage_ev[k]));
    CK(cudaEventRecord(s->stage_ev[k], s->xs));
  }
  s->slots_cap = (pl->launch_rows * L.nave * (int64_t)L.twonchan) / kDataLen + 4;
  for (auto& b : s->sb) {
    ST(hmalloc(s->res, &b.h, sizeof(int64_t) * 2 * s->slots_cap));
    ST(dmalloc(s->res, &b.d, sizeof(int64_t) * 2 * s->slots_cap));
    ST(mkevent(s->res, &b.ev));
    ST(mkevent(s->res, &b.ev_used));
    CK(cudaEventRecord(b.ev, s->cs));
    CK(cudaEventRecord(b.ev_used, s->cs));
  }
  ST(dmalloc(s->res, &s->d_err, 4));
  CK(cudaMemsetAsync(s->d_err, 0, 4, s->cs));
  ST(dmalloc(s->res, &s->d_w, nch * 4));
  ST(dmalloc(s->res, &s->d_inv, nch * 4));
  ST(dmalloc(s->res, &s->d_var, nch * 4));
  ST(dmalloc(s->res, &s->d_scr, nch * 128 * 4));
  const size_t sb = storage_bytes(P.storage);
  int64_t nt = 0;
  if (P.mode == VFRB_MODE_BLOCK) {
    ST(dmalloc(s->res, &s->d_fb_tm, (size_t)L.maxnt * nch * 4));
    CK(cudaMemsetAsync(s->d_fb_tm, 0, (size_t)L.maxnt * nch * 4, s->cs));
    if (pl->want_dd && pl->max_delay > 0) ST(dmalloc(s->res, &s->d_left, (size_t)pl->max_delay * nch * 4));
    s->cm_stride = ((int64_t)L.maxnt + 15) / 16 * 16;
    s->cm_mask = 0xffffffffu;
    ST(dmalloc(s->res, &s->d_cm, (size_t)nch * s->cm_stride * sb));
    if (shifted_copy(pl)) {
      ST(dmalloc(s->res, &s->d_cm1, (size_t)nch * s->cm_stride * sb));
      CK(cudaMemsetAsync(s->d_cm1, 0, (size_t)nch * s->cm_stride * sb, s->cs));
    }
    if (want(pl, VFRB_OUT_FB)) ST(dmalloc(s->res, &s->d_fbt, (size_t)L.maxnt * nch * 4));
    if (want(pl, VFRB_OUT_CHANSTATS)) {
      ST(dmalloc(s->res, &s->d_cave, (size_t)pl->nstatblks * nch * 4));
      ST(dmalloc(s->res, &s->d_csig, (size_t)pl->nstatblks * nch * 4));
      ST(dmalloc(s->res, &s->d_cout, (size_t)pl->nstatblks * nch * 4));
      ST(dmalloc(s->res, &s->d_csk, (size_t)pl->nstatblks * nch * 4));
    }
    nt = pl->nt_block;
    s->rflags.assign((size_t)L.maxnt, 0);
  } else {
    s->R1 = R1;
    ST(dmalloc(s->res, &s->d_raw, (size_t)R1 * nch * 4));
    s->cm_stride = R2;
    s->cm_mask = (unsigned)(R2 - 1);
    ST(dmalloc(s->res, &s->d_cm, (size_t)nch * R2 * sb));
    CK(cudaMemsetAsync(s->d_cm, 0, (size_t)nch * R2 * sb, s->cs));
    if (shifted_copy(pl)) {
      ST(dmalloc(s->res, &s->d_cm1, (size_t)nch * R2 * sb));
      CK(cudaMemsetAsync(s->d_cm1, 0, (size_t)nch * R2 * sb, s->cs));
    }
    if (want(pl, VFRB_OUT_CHANSTATS)) {
      ST(dmalloc(s->res, &s->d_cave, (size_t)nch * 4));
      ST(dmalloc(s->res, &s->d_csig, (size_t)nch * 4));
      ST(dmalloc(s->res, &s->d_cout, (size_t)nch * 4));
      ST(dmalloc(s->res, &s->d_csk, (size_t)nch * 4));
    }
    nt = pl->chunk_rows * pl->batch_chunks;
    // rows from the oldest not yet emitted to the newest channelised: at
    // most R2 (channel-major ring) + R1 (raw ring)
    s->rflags.assign((size_t)(2 * std::max(R1, R2)), 0);
    s->fmask = 2 * std::max(R1, R2) - 1;
  }
  if (pl->want_dd) {
    s->out_stride = nt;
    ST(dmalloc(s->res, &s->d_out, (size_t)pl->ndm * nt * 4));
    if (want(pl, VFRB_OUT_SIGMA)) ST(dmalloc(s->res, &s->d_sig, (size_t)pl->ndm * nt * 4));
    ST(dmalloc(s->res, &s->d_ave, pl->ndm * 4));
    ST(dmalloc(s->res, &s->d_sgm, pl->ndm * 4));
    ST(dmalloc(s->res, &s->d_peak, pl->ndm * 4));
    ST(dmalloc(s->res, &s->d_frb, pl->ndm * 4));
    ST(dmalloc(s->res, &s->d_arg, pl->ndm * 4));
    if (boxcar_on(pl)) {
      ST(dmalloc(s->res, &s->d_bsnr, pl->ndm * 4));
      ST(dmalloc(s->res, &s->d_bt, pl->ndm * 4));
      ST(dmalloc(s->res, &s->d_bw, pl->ndm * 4));
    }
    s->ws_bytes = dedisperse_workspace_bytes_plan(pl->dd, nt);
    ST(dmalloc(s->res, &s->d_ws, s->ws_bytes));
  }
  StreamSt* sp = s;
  // a gap-revealing frame is copied aside: it is used again NSKIP pairs later
  s->reader->on_gap = [pl, sp](int64_t v) -> int64_t {
    if (v < 0) return v;
    const int k = sp->stash_next;
    sp->stash_next = (sp->stash_next + 1) % kStash;
    sp->stash_flag[k] = sp->finv[(size_t)(v % sp->ring_frames)];
    const uint8_t* from = sp->d_frames + (v % sp->ring_frames) * kFrameLen + kHdrLen;
    uint8_t* to = sp->d_frames + sp->ring_frames * kFrameLen + (int64_t)k * kDataLen;
    if (cudaMemcpyAsync(to, from, kDataLen, cudaMemcpyDeviceToDevice, sp->cs) != cudaSuccess) {
      cudaGetLastError();
      sp->reader_error = VFRB_ERR_CUDA;
    }
    (void)pl;
    return -2 - k;
  };
  return VFRB_OK;
}

}  // namespace

extern "C" {

void vfrb_params_default(vfrb_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->twonchan = 12500;
  p->nave = 4;
  p->nbundle = 32;
  p->muoslowfreq = 360.0;
  p->maxtime = 70.f;
  p->timestats = 1.f;
  p->mode = VFRB_MODE_BLOCK;
  p->reader = VFRB_READER_PIPE;
  p->storage = VFRB_F32;
  p->q_scale = 16.f;
  p->outputs = VFRB_OUT_DEDISP | VFRB_OUT_DMSTATS;
  p->fb_block = -1;
  p->nstreams = 1;
  p->chunk_seconds = 1.f;
  p->ring_seconds = 1.f;
  p->cand_snr = 6.f;
  p->boxcar_max = 1;
}

int vfrb_plan_create(vfrb_plan** out, const vfrb_params* prm) {
  if (!out || !prm) return VFRB_ERR_ARG;
  *out = nullptr;
  vfrb_plan* pl = new vfrb_plan();
  pl->P = *prm;
  vfrb_params& P = pl->P;
  auto fail = [&](int st) {
    free_plan(pl);
    return st;
  };
  if (P.nstreams < 0 || P.nstreams > kMaxStreams || (P.mode != VFRB_MODE_BLOCK && P.mode != VFRB_MODE_STREAM) ||
      P.storage < VFRB_F32 || P.storage > VFRB_I8 || P.ring_seconds <= 0.f || P.q_scale <= 0.f ||
      P.boxcar_max < 0 || P.boxcar_max > 65536 || (P.bp_mode != VFRB_BP_CAL && P.bp_mode != VFRB_BP_FULL) ||
      (P.zero_dm != 0 && P.zero_dm != 1))
    return fail(VFRB_ERR_ARG);
  // the whole-block bandpass and zero-DM modes work in place on the FP32
  // channel-major block
  if ((P.bp_mode == VFRB_BP_FULL || P.zero_dm) && (P.mode != VFRB_MODE_BLOCK || P.storage != VFRB_F32))
    return fail(VFRB_ERR_UNSUPPORTED);
  if (cudaSetDevice(P.device) != cudaSuccess) return fail(VFRB_ERR_CUDA);
  int st = vfrb_layout_init(&pl->L, P.twonchan, P.nave, P.nbundle, P.muoslowfreq, P.nchanout_fixed, P.maxtime);
  if (st) return fail(st);
  const vfrb_layout& L = pl->L;
  if (L.twonchan != kFftN) return fail(VFRB_ERR_UNSUPPORTED);
  pl->want_dd = (P.outputs & (VFRB_OUT_DEDISP | VFRB_OUT_DMSTATS | VFRB_OUT_SIGMA | VFRB_OUT_CANDS)) != 0;
  if (pl->want_dd) {
    if (P.ndm < 1 || !P.dms) return fail(VFRB_ERR_ARG);
    pl->ndm = P.ndm;
    pl->dms.assign(P.dms, P.dms + P.ndm);
    pl->off.resize((size_t)P.ndm * L.nchanout);
    int32_t mdf = 0;
    st = vfrb_delay_table(&L, pl->dms.data(), P.ndm, pl->off.data(), &mdf);
    if (st) return fail(st);
    st = ddplan_create(&pl->dd, pl->off.data(), P.ndm, L.nchanout);
    if (st) return fail(st);
    const int tmax = ddplan_max_delay(pl->dd);
    if (P.mode == VFRB_MODE_BLOCK) {
      // the reference's carry uses the TS:464 formula with the LAST list entry
      if (mdf < tmax) return fail(VFRB_ERR_ARG);  // DM list must end with its largest trial
      pl->max_delay = mdf;
    } else {
      pl->max_delay = tmax;
    }
  }
  if (P.mode == VFRB_MODE_BLOCK) {
    if (L.maxnt % L.nbundle != 0) return fail(VFRB_ERR_UNSUPPORTED);  // rows past the last bundle are never written
    if (pl->want_dd && L.maxnt <= pl->max_delay) return fail(VFRB_ERR_ARG);
    pl->nt_block = pl->want_dd ? L.maxnt - pl->max_delay : 0;
    if (P.outputs & VFRB_OUT_CHANSTATS) {
      pl->nstatblks = (int)(P.maxtime / P.timestats);          // STATS:210
      pl->ncolstatblk = (int)((double)P.timestats / L.tchan);  // STATS:211
      if (pl->nstatblks < 1 || pl->ncolstatblk < 2 || (int64_t)pl->ncolstatblk * (pl->nstatblks - 1) >= L.maxnt)
        return fail(VFRB_ERR_ARG);
      if (P.storage != VFRB_F32) return fail(VFRB_ERR_UNSUPPORTED);
    }
  } else {
    pl->chunk_rows = std::max<int64_t>(32, (int64_t)llround(P.chunk_seconds / L.tchan));
    if (P.outputs & VFRB_OUT_CHANSTATS) {
      // absolute TIMESTATS blocks of the stream, one result each
      pl->nstatblks = 1;
      pl->ncolstatblk = (int)((double)P.timestats / L.tchan);  // STATS:211
      if (pl->ncolstatblk < 2) return fail(VFRB_ERR_ARG);
      if (P.storage != VFRB_F32) return fail(VFRB_ERR_UNSUPPORTED);
    }
  }
  const int64_t S = (int64_t)L.nave * L.twonchan;
  int64_t ring_frames = std::max<int64_t>(4 * (2 * kFramesPerCal + 16), (int64_t)(P.ring_seconds * kFramesPerSec * 2));
  ring_frames += ring_frames & 1;
  pl->launch_rows = std::max<int64_t>(L.nbundle, ((ring_frames / 8) * kDataLen) / S / L.nbundle * L.nbundle);
  if (P.mode == VFRB_MODE_STREAM) {
    // whole rows per persistent channeliser CTA: a multiple of the SM count
    int nsm = 148;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P.device) != cudaSuccess || nsm < 1) {
      cudaGetLastError();
      nsm = 148;
    }
    if (pl->launch_rows >= nsm) pl->launch_rows = pl->launch_rows / nsm * nsm;
    // a backlog of chunks is dedispersed in launches of about 4096 samples
    pl->batch_chunks = std::min<int64_t>(8, std::max<int64_t>(1, (4096 + pl->chunk_rows - 1) / pl->chunk_rows));
  }
  // stream mode with statistics: both rings also hold a statistics block
  // and the rows channelised past it
  const int64_t stat_rows = (P.mode == VFRB_MODE_STREAM && pl->ncolstatblk > 0) ? pl->ncolstatblk + pl->launch_rows : 0;
  const int64_t R1 = (int64_t)pow2_at_least((unsigned long long)std::max(pl->launch_rows + 512, stat_rows + 512));
  const int64_t R2 = (int64_t)pow2_at_least((unsigned long long)std::max(
      pl->max_delay + pl->chunk_rows * pl->batch_chunks + pl->launch_rows + 512, stat_rows + 512));
  pl->ring_frames = ring_frames;
  pl->R1 = R1;
  pl->R2 = R2;
  // admission by device memory
  const int64_t need = stream_bytes(pl, ring_frames, R1, R2) * P.nstreams;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return fail(VFRB_ERR_CUDA);
  const int64_t budget = P.device_bytes > 0 ? P.device_bytes : (int64_t)(0.9 * (double)fr);
  if (need > budget) return fail(VFRB_ERR_NOMEM);
  if (P.batch_streams && P.mode == VFRB_MODE_STREAM) {
    if (cudaStreamCreateWithFlags(&pl->bs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&pl->ev_batch, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return fail(VFRB_ERR_CUDA);
    }
  }
  for (int i = 0; i < P.nstreams; ++i) {
    st = create_stream(pl, i, ring_frames, R1, R2);
    if (st) return fail(st);
  }
  for (auto& s : pl->st)
    if (cudaStreamSynchronize(s->cs) != cudaSuccess || cudaStreamSynchronize(s->xs) != cudaSuccess)
      return fail(VFRB_ERR_CUDA);
  if (pl->want_dd && !(P.outputs & VFRB_OUT_SIGMA)) {
    // pick the fastest dedispersion kernel variant for this grid and chunk
    const int64_t nt = P.mode == VFRB_MODE_BLOCK ? pl->nt_block : pl->chunk_rows;
    cudaStream_t ts = nullptr;
    if (cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking) != cudaSuccess) return fail(VFRB_ERR_CUDA);
    st = ddplan_autotune(pl->dd, P.storage, nt, nullptr, ts);
    cudaStreamDestroy(ts);
    if (st) return fail(st);
  }
  *out = pl;
  return VFRB_OK;
}

int vfrb_plan_destroy(vfrb_plan* pl) { return free_plan(pl); }

int vfrb_plan_layout(const vfrb_plan* pl, vfrb_layout* L, int32_t* max_delay) {
  if (!pl) return VFRB_ERR_ARG;
  if (L) *L = pl->L;
  if (max_delay) *max_delay = pl->max_delay;
  return VFRB_OK;
}

int64_t vfrb_plan_device_bytes(const vfrb_plan* pl) {
  if (!pl) return -1;
  int64_t b = 0;
  for (auto& s : pl->st)
    if (s) b += s->res.dev_bytes;
  return b;
}

int vfrb_stream_open(vfrb_plan* pl, int* stream) {
  if (!pl || !stream) return VFRB_ERR_ARG;
  if ((int)pl->st.size() >= kMaxStreams) return VFRB_ERR_NOMEM;
  if (cudaSetDevice(pl->P.device) != cudaSuccess) return VFRB_ERR_CUDA;
  // admission: the new stream's device bytes must fit the budget beside the
  // streams already open (the caller retries once others have closed)
  const int64_t need = stream_bytes(pl, pl->ring_frames, pl->R1, pl->R2);
  const int64_t used = vfrb_plan_device_bytes(pl);
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return VFRB_ERR_CUDA;
  const int64_t budget = pl->P.device_bytes > 0 ? pl->P.device_bytes : used + (int64_t)(0.9 * (double)fr);
  if (used + need > budget) return VFRB_ERR_NOMEM;
  const int id = (int)pl->st.size();
  int st = create_stream(pl, id, pl->ring_frames, pl->R1, pl->R2);
  StreamSt* s = pl->st.back().get();
  if (st == VFRB_OK &&
      (cudaStreamSynchronize(s->cs) != cudaSuccess || cudaStreamSynchronize(s->xs) != cudaSuccess))
    st = VFRB_ERR_CUDA;
  if (st != VFRB_OK) {
    s->res.release();
    pl->st.pop_back();
    return st;
  }
  *stream = id;
  return VFRB_OK;
}

int vfrb_stream_close(vfrb_plan* pl, int stream) {
  if (!pl || stream < 0 || stream >= (int)pl->st.size() || !pl->st[stream]) return VFRB_ERR_ARG;
  StreamSt* s = pl->st[stream].get();
  if (!s->ended) vfrb_push_frames(pl, stream, nullptr, 0);  // end of data; a reader error closes all the same
  for (const ResultSlot* r : pl->queue)
    if (r->r.stream == stream) return VFRB_PENDING;  // results still to be polled
  if (pl->held && pl->held->r.stream == stream) {  // the last poll's result of this stream ends here
    pl->held->state = 0;
    pl->held = nullptr;
  }
  s->res.release();
  pl->st[stream].reset();
  return VFRB_OK;
}

int vfrb_push_frames(vfrb_plan* pl, int stream, const uint8_t* bytes, size_t nbytes) {
  if (!pl || stream < 0 || stream >= (int)pl->st.size() || !pl->st[stream]) return VFRB_ERR_ARG;
  StreamSt* s = pl->st[stream].get();
  if (s->ended) return VFRB_ERR_ARG;
  if (s->reader_error) return s->reader_error;
  if (cudaSetDevice(pl->P.device) != cudaSuccess) return VFRB_ERR_CUDA;
  s->t_push = now_ms();
  if (nbytes == 0 || !bytes) {  // end of data: the incomplete frame is dropped, as fread would fail on it
    s->part.clear();
    s->reader->end_of_data();
    ST(run_reader(pl, s));
    ST(process(pl, s, true));
    ST(flush_batch(pl));
    s->ended = true;
    return s->reader_error;
  }
  const MemKind kind = mem_kind(bytes);
  if (kind == kDevice) {
    CK(cudaEventRecord(s->ev_input, cudaStreamLegacy));
    CK(cudaStreamWaitEvent(s->hs, s->ev_input, 0));
    CK(cudaStreamWaitEvent(s->xs, s->ev_input, 0));
  }
  // bytes of a frame split across calls are assembled on the host (device
  // input: the few bytes of the head and tail are copied down first)
  auto host_bytes = [&](size_t off, size_t n, std::vector<uint8_t>& dst) -> int {
    const size_t at = dst.size();
    dst.resize(at + n);
    if (kind == kDevice) {
      CK(cudaMemcpy(dst.data() + at, bytes + off, n, cudaMemcpyDeviceToHost));
    } else {
      std::memcpy(dst.data() + at, bytes + off, n);
    }
    return VFRB_OK;
  };
  size_t pos = 0;
  if (!s->part.empty()) {
    const size_t take = std::min(nbytes, (size_t)kFrameLen - s->part.size());
    ST(host_bytes(0, take, s->part));
    pos = take;
    if (s->part.size() == (size_t)kFrameLen) {
      ST(feed_frames(pl, s, s->part.data(), 1, kPageable));
      s->part.clear();
    }
  }
  const int64_t whole = (int64_t)((nbytes - pos) / kFrameLen);
  if (whole > 0) ST(feed_frames(pl, s, bytes + pos, whole, kind));
  pos += (size_t)whole * kFrameLen;
  if (pos < nbytes) {
    s->part.clear();
    ST(host_bytes(pos, nbytes - pos, s->part));
  }
  return s->reader_error;
}

int vfrb_poll(vfrb_plan* pl, vfrb_result* out, int wait) {
  if (!pl || !out) return VFRB_ERR_ARG;
  if (pl->held) {
    pl->held->state = 0;
    pl->held = nullptr;
  }
  ST(flush_batch(pl));  // the chunks that became ready since the last poll, as one launch
  if (pl->queue.empty()) {
    for (auto& s : pl->st)
      if (s && !s->ended && !s->reader_error) return VFRB_PENDING;  // a failed stream produces nothing more
    return VFRB_EOD;
  }
  auto it = pl->queue.begin();
  for (; it != pl->queue.end(); ++it) {
    const cudaError_t q = cudaEventQuery((*it)->ev);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) return VFRB_ERR_CUDA;
  }
  if (it == pl->queue.end()) {
    if (!wait) return VFRB_PENDING;
    it = pl->queue.begin();
    if (cudaEventSynchronize((*it)->ev) != cudaSuccess) return VFRB_ERR_CUDA;
  }
  ResultSlot* r = *it;
  pl->queue.erase(it);
  r->state = 2;
  pl->held = r;
  vfrb_result& o = r->r;
  o.latency_ms = r->t_done - r->t_data;
  o.device_errors = *r->err;
  r->cands.clear();
  if (o.peak && o.argmax && (pl->P.outputs & VFRB_OUT_CANDS)) {
    // candidates: per trial the chunk's best SNR -- the calcstats peak, or
    // the best boxcar over widths 1 .. boxcar_max -- above the threshold,
    // kept where it is a local maximum over neighbouring trials
    const bool box = o.box_snr && o.box_start && o.box_width;
    const float* best = box ? o.box_snr : o.peak;
    // block mode: rows from `first` on were read after the carried rows
    // [first, max_delay) that they overwrote, so they sit max_delay - first
    // rows later in the stream than their block index says
    const bool blk = pl->P.mode == VFRB_MODE_BLOCK;
    const int64_t first = (int64_t)(pl->max_delay / pl->L.nbundle) * pl->L.nbundle;
    auto abs_row = [&](int64_t i) {
      return o.row0 + i + ((blk && o.seq > 0 && i >= first) ? (int64_t)pl->max_delay - first : 0);
    };
    for (int d = 0; d < o.ndm; ++d) {
      const float p = best[d];
      if (!(p >= pl->P.cand_snr)) continue;
      if (d > 0 && best[d - 1] > p) continue;
      if (d + 1 < o.ndm && best[d + 1] >= p) continue;
      vfrb_cand c;
      c.dm_index = d;
      c.width = box ? o.box_width[d] : 1;
      c.t = abs_row(box ? o.box_start[d] : o.argmax[d]);
      c.snr = p;
      c.dm = pl->dms[d];
      r->cands.push_back(c);
    }
  }
  o.ncand = (int32_t)r->cands.size();
  o.cands = r->cands.empty() ? nullptr : r->cands.data();
  *out = o;
  return VFRB_OK;
}

const char* vfrb_stream_log(vfrb_plan* pl, int stream) {
  if (!pl || stream < 0 || stream >= (int)pl->st.size() || !pl->st[stream]) return "";
  pl->logtmp = pl->st[stream]->logtext;
  return pl->logtmp.c_str();
}

int vfrb_stream_tstart(vfrb_plan* pl, int stream, double* mjd) {
  if (!pl || !mjd || stream < 0 || stream >= (int)pl->st.size() || !pl->st[stream]) return VFRB_ERR_ARG;
  const StreamSt* s = pl->st[stream].get();
  if (s->started) {
    *mjd = s->tstart_mjd;
    return VFRB_OK;
  }
  return s->reader_error ? s->reader_error : VFRB_PENDING;
}

}  // extern "C"
