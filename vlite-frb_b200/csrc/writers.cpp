// Output formats of the three tools (host only, byte-exact):
//   * SIGPROC filterbank header (PIPE:529-540, written with the send_* helpers
//     of PIPE:1177-1201: int32 length + text for a keyword, then the value in
//     native little-endian binary);
//   * PRESTO .inf text header of the TS time series (TS:1483-1515).
// The data files themselves (.nohead.fil, OUTDD.bin, .stats, .dat,
// _SIGMA.dat) are raw native float arrays and are written by the tools.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "vfrb.h"

namespace {

struct Sink {
  uint8_t* buf;
  size_t cap;
  size_t n = 0;
  void put(const void* p, size_t k) {
    if (buf && n + k <= cap) std::memcpy(buf + n, p, k);
    n += k;
  }
  void key(const char* s) {
    const int32_t len = (int32_t)std::strlen(s);
    put(&len, 4);
    put(s, (size_t)len);
  }
  void i32(const char* k, int32_t v) {
    key(k);
    put(&v, 4);
  }
  void f64(const char* k, double v) {
    key(k);
    put(&v, 8);
  }
};

}  // namespace

extern "C" size_t vfrb_sigproc_header(uint8_t* buf, size_t cap, double fch1, double foff, int32_t nchans,
                                      int32_t nbits, double tstart, double tsamp, int32_t nifs) {
  Sink s{buf, cap};
  s.key("HEADER_START");
  s.i32("barycentric", 1);
  s.i32("telescope_id", 12);  // the reference's choice: SIGPROC has no VLA id
  s.i32("data_type", 1);
  s.f64("fch1", fch1);
  s.f64("foff", foff);
  s.i32("nchans", nchans);
  s.i32("nbits", nbits);
  s.f64("tstart", tstart);
  s.f64("tsamp", tsamp);
  s.i32("nifs", nifs);
  s.key("HEADER_END");
  return s.n;
}

extern "C" int vfrb_presto_inf(char* buf, size_t cap, const char* basename, double mjdstart, int32_t ntimes,
                               double tsamp, float dm, double fchanlo, double bw, int32_t nchan, double chanbw) {
  if (!basename) return -1;
  std::string t;
  char line[512];
  auto add = [&](const char* fmt, auto... v) {
    std::snprintf(line, sizeof line, fmt, v...);
    t += line;
  };
  add(" Data file name without suffix          = %s\n", basename);
  t += " Telescope used                         = VLA\n";
  t += " Instrument used                        = VLITE-FAST\n";
  t += " Object being observed                  = Unknown\n";
  t += " J2000 Right Ascension (hh:mm:ss.ssss)  = 00:00:00.0000\n";
  t += " J2000 Declination     (dd:mm:ss.ssss)  = 00:00:00.0000\n";
  t += " Data observed by                       = vdifDADA2timeseries\n";
  add(" Epoch of observation (MJD)             = %.15lf\n", mjdstart);
  t += " Barycentered?                          = 1\n";
  add(" Number of bins in the time series      = %d\n", ntimes);
  add(" Width of each time series bin (sec)    = %.9lf\n", tsamp);
  t += " Any breaks in the data? (1=yes, 0=no)  = 0\n";
  t += " Type of observation (EM band)          = Radio\n";
  t += " Beam diameter (arcsec)                 = 3600\n";
  add(" Dispersion measure (cm-3 pc)           = %f\n", (double)dm);
  add(" Central freq of low channel (MHz)      = %f\n", fchanlo);
  add(" Total bandwidth (MHz)                  = %f\n", bw);
  add(" Number of channels                     = %d\n", nchan);
  add(" Channel bandwidth (MHz)                = %f\n", chanbw);
  t += " Data analyzed by                       = vdifDADA2timeseries\n";
  t += " Any additional notes:\n    \n\n";
  if (buf && cap > t.size()) std::memcpy(buf, t.c_str(), t.size() + 1);
  return (int)t.size();
}
