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

#ifdef VFRB_WITH_PSRDADA
// psrdada's reader API (ipcio.h from psrdada; build.py adds it when
// PSRDADA_DIR is set): the DADA tools then read the capture's own ring
#include "ipcio.h"
#endif

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
// ring named by its DADA key.  The ring is psrdada's own when the tools are
// built with psrdada (VFRB_WITH_PSRDADA), otherwise the project's ring
// (vfrb_dada_*, same reader-side behaviour).
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
#ifdef VFRB_WITH_PSRDADA
  ipcio_t dada{};  // zero-initialised, as the reference's global ipcio_t
  bool psrdada = false;
  // psrdada's ring: ipcio_connect, the iread force on the ipcbuf_t that the
  // ipcio_t begins with (iread = -1 is required to open as the primary read
  // client), ipcio_open('R') and the ring's counters in the log, as the
  // reference does (STATS:123-134, 284-304; TS:136-147, 357-382).  Returns
  // 0, 1 (could not connect) or 2 (could not open as the primary reader).
  int connect_psrdada(uint32_t key, FILE* log) {
    if (ipcio_connect(&dada, (key_t)key) < 0) return 1;
    ipcbuf_t* b = reinterpret_cast<ipcbuf_t*>(&dada);
    if (b->iread != -1) {
      std::fprintf(log, " iread= %d != -1, setting to -1\n", b->iread);
      b->iread = -1;
    } else {
      std::fprintf(log, " iread= %d, do not need to force\n", b->iread);
    }
    if (ipcio_open(&dada, 'R') < 0) {
      ipcio_disconnect(&dada);
      return 2;
    }
    psrdada = true;
    std::fprintf(log, " nbufs= %lu\n", (unsigned long)ipcbuf_get_nbufs(b));
    std::fprintf(log, " bufsz= %lu\n", (unsigned long)ipcbuf_get_bufsz(b));
    std::fprintf(log, " nfull= %lu\n", (unsigned long)ipcbuf_get_nfull(b));
    std::fprintf(log, " nclear= %lu\n", (unsigned long)ipcbuf_get_nclear(b));
    std::fprintf(log, " write count= %lu\n", (unsigned long)ipcbuf_get_write_count(b));
    std::fprintf(log, " read count = %lu\n", (unsigned long)ipcbuf_get_read_count(b));
    return 0;
  }
#endif
  // ipcio_connect, then the reference's iread force and ipcio_open('R')
  // (STATS:284-298, TS:357-372) with its log lines; waits (bounded) for the
  // writer's ring.  Returns 0, 1 (could not connect) or 2 (could not open
  // as the primary reader).
  int connect(uint32_t key, FILE* log, int wait_ms = 30000) {
#ifdef VFRB_WITH_PSRDADA
    (void)wait_ms;
    return connect_psrdada(key, log);
#endif
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
#ifdef VFRB_WITH_PSRDADA
    // a short read is the end of data (the reference then checks ipcbuf_eod)
    if (psrdada) {
      const long k = (long)ipcio_read(&dada, static_cast<char*>(buf), n);
      if (k < 0) {
        failed = true;
        return 0;
      }
      return (size_t)k;
    }
#endif
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
#ifdef VFRB_WITH_PSRDADA
    if (psrdada) {
      ipcio_close(&dada);
      ipcio_disconnect(&dada);
    }
#endif
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
