// Pol-pair reader state machine (see vdif_reader.h).
#include "vdif_reader.h"
#include "vfrb_common.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace vfrb {

bool PairReader::read_raw(int p) {
  if (q_.empty()) return false;
  hdr_[p] = q_.front().h;
  cur_[p] = q_.front().payload;
  q_.pop_front();
  return true;
}

// checkframeskip0/1: PIPE:888-930 (frame number mod 25600) and TS:895-937
// (seconds-aware; a negative gap leaves the pol on fill frames for good, as
// the reference's NSKIP countdown never reaches zero).
void PairReader::checkframeskip(int p) {
  const int fnum = (int)hdr_[p].frame;
  if (mode_ == TS) {
    const long long fsec = hdr_[p].seconds;
    if (fnum != expected_[p] || fsec != expsec_[p]) {
      nskip_[p] = (long long)fnum - expected_[p] + (fsec - expsec_[p]) * kFramesPerSec;
      tmp_[p] = on_gap ? on_gap(cur_[p]) : cur_[p];
      cur_[p] = kFill;
      char b[160];
      snprintf(b, sizeof b, "FRAME SKIP %d: expected %lld %d, read %lld %d (NSKIP=%lld)", p, expsec_[p], expected_[p],
               fsec, fnum, nskip_[p]);
      log_.emplace_back(b);
    }
    expected_[p] = (fnum + 1) % kFramesPerSec;
    expsec_[p] = fsec + (expected_[p] == 0 ? 1 : 0);
  } else {
    if (fnum != expected_[p]) {
      long long n = (long long)fnum - expected_[p];
      if (n < 0) n += kFramesPerSec;
      nskip_[p] = n;
      tmp_[p] = on_gap ? on_gap(cur_[p]) : cur_[p];
      cur_[p] = kFill;
      char b[160];
      snprintf(b, sizeof b, "FRAME SKIP %d: expected %d, read %d (NSKIP=%lld)", p, expected_[p], fnum, n);
      log_.emplace_back(b);
    }
    expected_[p] = (fnum + 1) % kFramesPerSec;
  }
}

// readoneframePOL0/1 (PIPE:934-1025)
bool PairReader::readone(int p) {
  if (nskip_[p]) {
    nskip_[p]--;
    if (nskip_[p] == 0) cur_[p] = tmp_[p];
    return true;
  }
  if (!read_raw(p)) return false;
  checkframeskip(p);
  return true;
}

// initframe01 (PIPE:1058-1131; TS:1070-1145).  0 ok, 1 abort/retry, 2 error.
int PairReader::initframe01() {
  if (!read_raw(0)) return 1;
  if (hdr_[0].threadid != 0) {
    log_.emplace_back("VDIF Threads misaligned, skipping forward 1 frame");
    if (!read_raw(0)) return 1;
  }
  if (hdr_[0].threadid != 0) return 1;
  if (!read_raw(1)) return 1;
  if (hdr_[1].threadid != 1) return 1;
  const bool ts = mode_ == TS;
  int fnum0 = (int)hdr_[0].frame;
  int fnum1 = (int)hdr_[1].frame;
  if (fnum0 != fnum1 || (ts && hdr_[0].seconds != hdr_[1].seconds)) return ts ? 2 : 1;
  long long ncal = 0;
  while (fnum0 % kFramesPerCal != 0) {  // fmod((float)fnum0, 2560.f) < 1e-4, exact below 2^24
    if (!read_raw(0)) return 1;
    if (!read_raw(1)) return 1;
    fnum0 = (int)hdr_[0].frame;
    ++ncal;
  }
  fnum1 = (int)hdr_[1].frame;
  if (fnum0 != fnum1 || (ts && hdr_[0].seconds != hdr_[1].seconds)) return ts ? 2 : 1;
  char b[96];
  snprintf(b, sizeof b, "Skipped %lld frames to begin at noise cal cycle", ncal);
  log_.emplace_back(b);
  for (int p = 0; p < 2; ++p) {
    expected_[p] = ((int)hdr_[p].frame + 1) % kFramesPerSec;
    expsec_[p] = (long long)hdr_[p].seconds + (expected_[p] == 0 ? 1 : 0);
  }
  return 0;
}

PairReader::Status PairReader::run(std::vector<int64_t>& e0, std::vector<int64_t>& e1) {
  if (phase_ == DONE) return failed_ ? STEP_EOD : STEP_ERROR;
  if (phase_ == INIT && dada_skip_ && skipped_ == 0) phase_ = DADA_SKIP;
  if (phase_ == DADA_SKIP) {  // initDADA: discard NFRAMEDADAINIT frame pairs (TS:767-826)
    while (skipped_ < kDadaInitFrames) {
      if (q_.size() < 2) {
        if (!eod_) return STEP_NEED;
        phase_ = DONE;
        failed_ = true;
        return STEP_EOD;
      }
      q_.pop_front();
      q_.pop_front();
      ++skipped_;
    }
    phase_ = INIT;
    dada_skip_ = false;
  }
  if (phase_ == INIT) {
    // initframe01 consumes at most 2 + 1 + 2*2559 + 1 frames: wait until they are queued.
    constexpr size_t kInitNeed = 2 * kFramesPerCal + 8;
    for (;;) {
      if (q_.size() < kInitNeed && !eod_) return STEP_NEED;
      const int r = initframe01();
      if (r == 0) {
        phase_ = RUNNING;
        start_hdr_ = hdr_[0];
        e0.push_back(cur_[0]);
        e1.push_back(cur_[1]);
        break;
      }
      // PIPE/STATS exit with 2 on any failure (PIPE:513-516); TS retries on 1 (TS:516-523) and
      // would spin for ever at end of data -- here the retry stops there.
      if (mode_ != TS || r == 2) {
        phase_ = DONE;
        return STEP_ERROR;
      }
      if (q_.empty() && eod_) {
        phase_ = DONE;
        failed_ = true;
        return STEP_EOD;
      }
    }
  }
  for (;;) {  // readtwoframe (PIPE:1031-1040), one pair per step
    if (q_.size() < 2 && !eod_) return STEP_NEED;
    if (!readone(0) || !readone(1)) {
      phase_ = DONE;
      failed_ = true;
      return STEP_EOD;
    }
    e0.push_back(cur_[0]);
    e1.push_back(cur_[1]);
  }
}

size_t PairReader::run_fast(const uint8_t* fr, int64_t pay0, size_t n, std::vector<int64_t>& e0,
                            std::vector<int64_t>& e1, size_t pitch) {
  if (phase_ != RUNNING || !q_.empty() || nskip_[0] || nskip_[1]) return 0;
  const bool ts = mode_ == TS;
  // Scan the pairs that continue the expected frame (and, TS, second)
  // sequence; the state after the scan is that of the last pair, as the
  // pair-by-pair path would leave it.
  int x0 = expected_[0], x1 = expected_[1];
  long long es0 = expsec_[0], es1 = expsec_[1];
  int lf0 = 0, lf1 = 0;
  long long ls0 = 0, ls1 = 0;
  size_t k = 0;
  for (; k + 1 < n; k += 2) {
    const uint8_t* h0 = fr + k * pitch;
    const uint8_t* h1 = h0 + pitch;
    uint32_t a0, b0, a1, b1;
    std::memcpy(&a0, h0, 4);  // seconds:30 | legacy | invalid (little-endian, vdifio.h:53-72)
    std::memcpy(&b0, h0 + 4, 4);  // frame:24 | epoch:6 | unassigned:2
    std::memcpy(&a1, h1, 4);
    std::memcpy(&b1, h1 + 4, 4);
    const int f0 = (int)(b0 & 0xFFFFFFu), f1 = (int)(b1 & 0xFFFFFFu);
    if (f0 != x0 || f1 != x1) break;  // a gap: checkframeskip decides
    const long long s0 = a0 & 0x3FFFFFFFu, s1 = a1 & 0x3FFFFFFFu;
    if (ts && (s0 != es0 || s1 != es1)) break;
    // checkframeskip with no skip: advance the expected frame (and second)
    x0 = f0 + 1 == kFramesPerSec ? 0 : f0 + 1;
    x1 = f1 + 1 == kFramesPerSec ? 0 : f1 + 1;
    if (ts) {
      es0 = s0 + (x0 == 0 ? 1 : 0);
      es1 = s1 + (x1 == 0 ? 1 : 0);
    }
    lf0 = f0;
    lf1 = f1;
    ls0 = s0;
    ls1 = s1;
  }
  if (k == 0) return 0;
  expected_[0] = x0;
  expected_[1] = x1;
  if (ts) {
    expsec_[0] = es0;
    expsec_[1] = es1;
  }
  hdr_[0].frame = (uint32_t)lf0;
  hdr_[1].frame = (uint32_t)lf1;
  hdr_[0].seconds = (uint32_t)ls0;
  hdr_[1].seconds = (uint32_t)ls1;
  cur_[0] = pay0 + (int64_t)k - 2;
  cur_[1] = pay0 + (int64_t)k - 1;
  // pair j uses payloads pay0 + 2j (pol 0) and pay0 + 2j + 1 (pol 1)
  const size_t np = k / 2, at = e0.size();
  e0.resize(at + np);
  e1.resize(at + np);
  int64_t* o0 = e0.data() + at;
  int64_t* o1 = e1.data() + at;
  for (size_t j = 0; j < np; ++j) {
    o0[j] = pay0 + 2 * (int64_t)j;
    o1[j] = pay0 + 2 * (int64_t)j + 1;
  }
  return k;
}

}  // namespace vfrb

extern "C" int vfrb_read_pairs(const uint8_t* bytes, size_t nbytes, int reader_mode, int dada_skip, size_t split,
                               int64_t* e0, int64_t* e1, int64_t cap, int64_t* npairs, double* tstart_mjd) {
  using namespace vfrb;
  if ((!bytes && nbytes) || !npairs || (cap > 0 && (!e0 || !e1))) return VFRB_ERR_ARG;
  PairReader r(reader_mode == VFRB_READER_TS ? PairReader::TS : PairReader::PIPE, dada_skip != 0);
  std::vector<int64_t> a, b;
  const size_t nfr = nbytes / kFrameLen;  // a trailing partial frame cannot be read
  if (split == 0) split = nbytes ? nbytes : 1;
  const size_t per = std::max<size_t>(1, split / kFrameLen);
  PairReader::Status st = PairReader::STEP_NEED;
  // pieces of `per` frames, as they would arrive: fast path first, the rest
  // queued for the general state machine
  for (size_t k0 = 0; k0 < nfr && st != PairReader::STEP_ERROR; k0 += per) {
    const size_t k1 = std::min(nfr, k0 + per);
    size_t k = k0 + r.run_fast(bytes + k0 * kFrameLen, (int64_t)k0, k1 - k0, a, b, kFrameLen);
    for (; k < k1; ++k) {
      QFrame q;
      vfrb_decode_header(bytes + k * kFrameLen, &q.h);
      q.payload = (int64_t)k;
      r.push(q);
    }
    st = r.run(a, b);
  }
  if (st != PairReader::STEP_ERROR) {
    r.end_of_data();
    st = r.run(a, b);
  }
  const int64_t n = (int64_t)a.size();
  *npairs = n;
  for (int64_t i = 0; i < n && i < cap; ++i) {
    e0[i] = a[i];
    e1[i] = b[i];
  }
  if (tstart_mjd) {
    vfrb_hdr h = r.start_header();
    *tstart_mjd = r.initialised() || r.failed() ? vfrb_header_dmjd(&h, kFramesPerSec) : 0.0;
  }
  return st == PairReader::STEP_ERROR ? VFRB_ERR : VFRB_OK;
}
