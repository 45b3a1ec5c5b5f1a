// Host-side VDIF pol-pair reader with the reference's semantics.
//
// The reference reads one file/ring sequentially (PIPE:829-1171; STATS:456-791;
// TS:767-1180): 32-byte header then 5000-byte payload per frame, threads 0/1
// alternating, start on a 10 Hz noise-cal boundary (frame % 2560 == 0), and a
// frame-number gap of g frames becomes g zero-byte fill frames followed by
// the frame that revealed the gap.  Instead of copying payload bytes into
// per-pol buffers, this reader emits, per pair, a reference to each pol's
// payload (its byte offset in the device frame ring, or -1 for a fill frame);
// the channeliser reads samples through those references.
//
// The state machine is resumable: frames arrive in any number of pushes and a
// step is only taken when the frames it may consume are queued (or the stream
// has ended), so results do not depend on how the input was split.
#pragma once
#include <cstdint>
#include <deque>
#include <functional>
#include <string>
#include <vector>

#include "../../include/vfrb.h"

namespace vfrb {

constexpr int kFramesPerSec = 25600;  // FRAMESPERSEC (PIPE:36)
constexpr int kFramesPerCal = 2560;   // 10 Hz cal half-period in frames (PIPE:1101)
constexpr int kDadaInitFrames = 256000;  // NFRAMEDADAINIT pairs skipped by TS (TS:74)

struct QFrame {
  vfrb_hdr h;
  int64_t payload;  // device byte offset of the 5000-byte payload
};

class PairReader {
 public:
  enum Mode { PIPE = 0, TS = 1 };
  enum Status { STEP_OK = 0, STEP_NEED = 1, STEP_EOD = 2, STEP_ERROR = 3 };

  explicit PairReader(Mode m = PIPE, bool dada_skip = false) : mode_(m), dada_skip_(dada_skip) {}

  void push(const QFrame& f) { q_.push_back(f); }
  void end_of_data() { eod_ = true; }
  bool ended() const { return eod_; }
  size_t queued() const { return q_.size(); }

  // Advances the state machine as far as the queued frames allow, appending
  // the produced pairs (entry 0 is the pair initframe01 leaves in the
  // buffers).  Returns STEP_NEED when more frames are needed, STEP_EOD when
  // the stream has ended, STEP_ERROR on a hard initialisation error (the
  // reference's return 2).
  Status run(std::vector<int64_t>& e0, std::vector<int64_t>& e1);

  // Fast path of the RUNNING phase: with nothing queued and no fill frames
  // pending, consumes in-order frame pairs straight from `frames` (nframes
  // whole frames whose payloads are numbered pay0, pay0+1, ...) as long as
  // each frame has the expected frame number (and second, TS), appending
  // their pairs exactly as run() would.  Stops before the first frame that
  // needs the general state machine; returns the frames consumed (even).
  // Frame k's header starts at frames + k * pitch: the frames themselves
  // (pitch 5032) or their 32-byte headers packed (pitch 32).
  size_t run_fast(const uint8_t* frames, int64_t pay0, size_t nframes, std::vector<int64_t>& e0,
                  std::vector<int64_t>& e1, size_t pitch);

  bool initialised() const { return phase_ == RUNNING; }
  // header of the first pol-0 frame used (tstart for getVDIFDMJD, PIPE:525)
  const vfrb_hdr& start_header() const { return start_hdr_; }
  // pairs the reader could not complete (the failed pair at end of data)
  bool failed() const { return failed_; }
  std::vector<std::string>& log() { return log_; }
  // Called with the frame that revealed a gap (its payload is used again
  // NSKIP pairs later); returns the reference to use for it then.
  std::function<int64_t(int64_t)> on_gap;

 private:
  enum Phase { DADA_SKIP, INIT, RUNNING, DONE };
  bool read_raw(int p);             // fread/ipcio_read of one frame into pol p
  int initframe01();                // 0 ok, 1 retry/EOD, 2 error
  void checkframeskip(int p);
  bool readone(int p);              // false on end of data
  static constexpr int64_t kFill = -1;

  Mode mode_;
  bool dada_skip_;
  bool eod_ = false;
  bool failed_ = false;
  Phase phase_ = INIT;
  long long skipped_ = 0;
  std::deque<QFrame> q_;
  vfrb_hdr hdr_[2]{};
  int64_t cur_[2]{kFill, kFill};
  int64_t tmp_[2]{kFill, kFill};
  long long nskip_[2]{0, 0};
  int expected_[2]{0, 0};
  long long expsec_[2]{0, 0};
  vfrb_hdr start_hdr_{};
  std::vector<std::string> log_;
};

}  // namespace vfrb
