// Shared host code of the drop-in command-line tools (built on libvfrb's
// plan API; see include/vfrb.h).
#pragma once

#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "vfrb.h"

namespace tool {

inline bool eq(const char* a, const char* b) { return std::strcmp(a, b) == 0; }

inline double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The reference opens DM101.txt in the working directory, counts its lines and
// reads one float per line with sscanf("%f") (PIPE:355-376, 420-431).
inline int read_dm_list(const char* path, std::vector<float>& dms) {
  FILE* f = std::fopen(path, "r");
  if (!f) return -1;
  char line[256];
  int n = 0;
  while (std::fgets(line, sizeof line, f)) ++n;
  std::rewind(f);
  dms.assign((size_t)n, 0.f);
  for (int i = 0; i < n; ++i) {
    if (!std::fgets(line, sizeof line, f)) break;
    std::sscanf(line, "%f", &dms[(size_t)i]);
  }
  std::fclose(f);
  return n;
}

inline bool file_exists(const char* p) { return access(p, F_OK) != -1; }

inline bool write_all(FILE* f, const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }

// Byte source the tools read VDIF from: a file ("-" = standard input) or a
// DADA-style ring named by its key (vfrb_dada_*).
struct Source {
  FILE* f = nullptr;
  bool own = false;
  vfrb_dada* ring = nullptr;
  int timeout_ms = 300000;
  bool failed = false;
  bool pinned = false;
  bool open(const char* path) {
    if (eq(path, "-")) {
      f = stdin;
      return true;
    }
    f = std::fopen(path, "rb");
    own = f != nullptr;
    return f != nullptr;
  }
  // ipcio_connect, then the reference's iread force and ipcio_open('R')
  // (STATS:284-298, TS:357-372) with its log lines; waits (bounded) for the
  // writer's ring.  Returns 0, 1 (could not connect) or 2 (could not open
  // as the primary reader).
  int connect(uint32_t key, FILE* log, int wait_ms = 30000) {
    const double t0 = now_s();
    while (vfrb_dada_connect(key, &ring) != VFRB_OK) {
      if ((now_s() - t0) * 1e3 > wait_ms) return 1;
      usleep(20000);
    }
    // iread = -1 is required to open as the primary read client
    const int iread = vfrb_dada_iread(ring);
    if (iread != -1) {
      std::fprintf(log, " iread= %d != -1, setting to -1\n", iread);
      vfrb_dada_force_iread(ring);
    } else {
      std::fprintf(log, " iread= %d, do not need to force\n", iread);
    }
    if (vfrb_dada_open_read(ring) != VFRB_OK) return 2;
    pinned = vfrb_dada_pin(ring) == VFRB_OK;  // else pushes go through the staging copy
    return 0;
  }
  // ring input: the next contiguous readable bytes in place (0 at end of data)
  size_t acquire(const uint8_t** p, size_t max_n) {
    const int64_t k = vfrb_dada_acquire(ring, p, max_n, timeout_ms);
    if (k < 0) {
      failed = true;
      return 0;
    }
    return (size_t)k;
  }
  void release(size_t n) { vfrb_dada_release(ring, n); }
  size_t read(void* buf, size_t n) {
    if (ring) {
      const int64_t k = vfrb_dada_read(ring, buf, n, timeout_ms);
      if (k < 0) {
        failed = true;
        return 0;
      }
      return (size_t)k;
    }
    return std::fread(buf, 1, n, f);
  }
  ~Source() {
    if (own) std::fclose(f);
    if (ring) vfrb_dada_close(ring);
  }
};

// Feeds a source through a plan, calling on_result for every completed
// result and on_start once the reader has found its first frame pair.
// Returns 0, or the reference's exit code for the failure (2).
template <typename OnStart, typename OnResult>
int run_stream(vfrb_plan* plan, Source& src, FILE* log, OnStart on_start, OnResult on_result) {
  std::vector<uint8_t> buf((size_t)64 << 20);
  bool started = false;
  auto drain = [&](int wait) -> int {
    for (;;) {
      vfrb_result r;
      const int st = vfrb_poll(plan, &r, wait);
      if (st == VFRB_PENDING || st == VFRB_EOD) return st;
      if (st != VFRB_OK) return st;
      on_result(r);
    }
  };
  auto check_start = [&]() {
    if (started) return;
    double mjd = 0.0;
    if (vfrb_stream_tstart(plan, 0, &mjd) == VFRB_OK) {
      started = true;
      on_start(mjd);
    }
  };
  for (;;) {
    // ring input is pushed in place (page-locked: copied straight to the
    // device), file input through the read buffer
    const uint8_t* p = buf.data();
    const size_t n = src.ring ? src.acquire(&p, buf.size()) : src.read(buf.data(), buf.size());
    if (n == 0) break;
    int st = vfrb_push_frames(plan, 0, p, n);
    if (src.ring) src.release(n);
    if (st != VFRB_OK) {
      std::fprintf(log, "%s\n", vfrb_stream_log(plan, 0));
      std::fprintf(log, "processing stopped: %s\n", vfrb_strerror(st));
      return 2;
    }
    check_start();
    st = drain(0);
    if (st != VFRB_PENDING && st != VFRB_EOD) {
      std::fprintf(log, "processing stopped: %s\n", vfrb_strerror(st));
      return 2;
    }
  }
  if (src.failed) {
    std::fprintf(log, "no data from the input ring for %d ms\n", src.timeout_ms);
    return 2;
  }
  int st = vfrb_push_frames(plan, 0, nullptr, 0);  // end of data (FLAGEOF / FLAGEODADA)
  check_start();
  if (st != VFRB_OK && st != VFRB_EOD) {
    std::fprintf(log, "%s\n", vfrb_stream_log(plan, 0));
    std::fprintf(log, "processing stopped: %s\n", vfrb_strerror(st));
    return 2;
  }
  st = drain(1);
  if (st != VFRB_EOD && st != VFRB_PENDING) {
    std::fprintf(log, "processing stopped: %s\n", vfrb_strerror(st));
    return 2;
  }
  std::fputs(vfrb_stream_log(plan, 0), log);
  if (!started) {
    std::fprintf(log, "initframe01 returned in error!\n");
    return 2;
  }
  return 0;
}

}  // namespace tool
