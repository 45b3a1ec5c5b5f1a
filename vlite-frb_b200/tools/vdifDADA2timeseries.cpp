// vdifDADA2timeseries: drop-in for the reference tool of the same name
// (vdifDADA2timeseries.cu), running on libvfrb's plan API.
//
// Reference behaviour kept (TS:240-760, 1215-1258, 1483-1515): flags -d,
// -nchan N, -nave N, -nb N, -k KEY (hex), -o NAME; skips the first 256000
// frames of each pol (initDADA), 3840 channels, 30-s blocks with the
// max_delay carry, DM trials {0, 119.3}; per block the channel mean and the
// per-sample channel sigma of both trials are appended to
//   DM0.0_<UTC>.dat, DM0.0_<UTC>_SIGMA.dat, DM119.3_<UTC>.dat, DM119.3_<UTC>_SIGMA.dat
// (<UTC> = start time, %F_%T); on the first block after each UTC hour the
// PRESTO .inf headers of the finished files are written and new files
// begun.  Logs: NAME.log until the start, then NAME_<UTC>.log.
//
// Extensions: -i FILE (read a VDIF file or "-" instead of the ring),
// -noskip (do not skip the first 256000 frames), -maxtime S,
// -infatend (also write the .inf headers of the files open at the end),
// -flags (NAME.flags: one byte per time-series sample, appended with the
// series, bit 0 = a frame with the VDIF invalid bit, bit 1 = zero fill).
#include <ctime>

#include "tool_common.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "***************************************************************************\n"
               "This program reads VDIF data from a DADA ring buffer and writes the\n"
               "  DM 0 and DM 119.3 time series (channel mean and sigma) in PRESTO format.\n\n"
               "  Usage:\n./vdifDADA2timeseries -d:\t    use default values (unless other values given)\n"
               "\t             -k (hex):      DADA key,\n"
               "\t             -o (string):   base name of ouput files to write,\n"
               "\t             -nave (int):   number of time samples to average over,\n"
               "\t             -nchan (int):  number of frequency channels,\n"
               "\t             -nb (int):     number of bundles of size (2*2*nchan*nave) to send in 1 memcpy\n"
               "  Extensions:\n"
               "\t             -i (string)    read a VDIF file instead of the ring (- = stdin)\n"
               "\t             -noskip        do not skip the first 256000 frames per pol\n"
               "\t             -maxtime (s)   block length (default 30)\n"
               "\t             -infatend      write .inf headers for the files open at the end\n"
               "\t             -flags         write per-sample data flags to NAME.flags\n\n"
               "  DEFAULTS:\n"
               "\t             -k     dada\n"
               "\t             -o     testTIMESERIES\n"
               "\t             -nave  4\n"
               "\t             -nchan 6250\n"
               "\t             -nb    32\n\n");
}

std::string utc_stamp() {
  const std::time_t t = std::time(nullptr);
  std::tm u;
  gmtime_r(&t, &u);
  char b[64];
  std::strftime(b, sizeof b, "%F_%T", &u);
  return b;
}

int utc_hour() {
  const std::time_t t = std::time(nullptr);
  std::tm u;
  gmtime_r(&t, &u);
  return u.tm_hour;
}

bool write_inf(const std::string& base, double mjd, int64_t ntimes, double tsamp, float dm, double fchlo, double bw,
               int nchan, double chanbw) {
  const int n = vfrb_presto_inf(nullptr, 0, base.c_str(), mjd, (int32_t)ntimes, tsamp, dm, fchlo, bw, nchan, chanbw);
  std::string t((size_t)n + 1, '\0');
  vfrb_presto_inf(&t[0], t.size(), base.c_str(), mjd, (int32_t)ntimes, tsamp, dm, fchlo, bw, nchan, chanbw);
  FILE* f = std::fopen((base + ".inf").c_str(), "w");
  if (!f) return false;
  std::fwrite(t.data(), 1, (size_t)n, f);
  std::fclose(f);
  return true;
}

bool append(const std::string& name, const float* p, size_t n) {
  FILE* f = std::fopen(name.c_str(), "ab");
  if (!f) return false;
  const bool ok = tool::write_all(f, p, n * 4);
  std::fclose(f);
  return ok;
}

bool create_empty(const std::string& name) {
  if (tool::file_exists(name.c_str())) std::remove(name.c_str());
  FILE* f = std::fopen(name.c_str(), "wb");
  if (!f) return false;
  std::fclose(f);
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    usage();
    return 1;
  }
  int twonchan = 0, nave = 0, nbundle = 0;
  unsigned key = 0xdada;
  std::string in, out;
  bool skip = true, inf_at_end = false, want_flags = false;
  float maxtime = 30.f;
  int i = 1;
  if (tool::eq(argv[i], "-d")) {
    twonchan = 12500;
    nave = 4;
    nbundle = 32;
    out = "testTIMESERIES";
    ++i;
  }
  for (; i < argc; ++i) {
    const bool more = i + 1 < argc;
    if (tool::eq(argv[i], "-nchan") && more) {
      twonchan = 2 * std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-nave") && more) {
      nave = std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-nb") && more) {
      nbundle = std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-k") && more) {
      std::sscanf(argv[++i], "%x", &key);
    } else if (tool::eq(argv[i], "-o") && more) {
      out = argv[++i];
    } else if (tool::eq(argv[i], "-i") && more) {
      in = argv[++i];
    } else if (tool::eq(argv[i], "-noskip")) {
      skip = false;
    } else if (tool::eq(argv[i], "-maxtime") && more) {
      maxtime = (float)std::atof(argv[++i]);
    } else if (tool::eq(argv[i], "-infatend")) {
      inf_at_end = true;
    } else if (tool::eq(argv[i], "-flags")) {
      want_flags = true;
    } else {
      std::fprintf(stderr, "Error! Unknown argument: %s\n\n", argv[i]);
      usage();
      return 1;
    }
  }
  std::string logname = out + ".log";
  if (tool::file_exists(logname.c_str())) std::remove(logname.c_str());
  FILE* log = std::fopen(logname.c_str(), "w");
  if (!log) {
    std::fprintf(stderr, "Unable to open output log file: %s\n", logname.c_str());
    return 2;
  }
  std::fprintf(log, "Running vdifDADA2timeseries (libvfrb, sm_100a)\n");
  if (want_flags) std::remove((out + ".flags").c_str());

  const float dms[2] = {0.0f, 119.3f};  // 119.3 gives a 1-s sweep across the lower 39.3216 MHz (TS:437-438)
  vfrb_params p;
  vfrb_params_default(&p);
  p.twonchan = twonchan;
  p.nave = nave;
  p.nbundle = nbundle;
  p.nchanout_fixed = 3840;
  p.maxtime = maxtime;
  p.dms = dms;
  p.ndm = 2;
  p.mode = VFRB_MODE_BLOCK;
  p.reader = VFRB_READER_TS;
  p.dada_skip = skip ? 1 : 0;
  p.outputs = VFRB_OUT_DEDISP | VFRB_OUT_SIGMA | (want_flags ? VFRB_OUT_FLAGS : 0);
  vfrb_plan* plan = nullptr;
  int st = vfrb_plan_create(&plan, &p);
  if (st != VFRB_OK) {
    std::fprintf(log, "Error creating the processing plan: %s\n", vfrb_strerror(st));
    return 1;
  }
  vfrb_layout L;
  int32_t max_delay = 0;
  vfrb_plan_layout(plan, &L, &max_delay);
  const int64_t ntime_outdd = (int64_t)L.maxnt - max_delay;
  const double tsamp = (double)L.nave * L.twonchan / 128e6;
  const double bandw = L.nchanout * L.chanbw, fchlo = 320.0 + 0.5 * L.chanbw;
  std::fprintf(log, "NCHANOUT= %d\nMAXNT= %d\ndm_count= 2  max_delay= %d\nNTIME_OUTDD= %lld\n", L.nchanout, L.maxnt,
               max_delay, (long long)ntime_outdd);

  tool::Source src;
  if (!in.empty()) {
    if (!src.open(in.c_str())) {
      std::fprintf(log, " Could not open %s\n", in.c_str());
      return 255;
    }
  } else {
    std::fprintf(log, " Connecting to DADA buffer with key: %x ...\n", key);
    const int cst = src.connect(key, log);
    if (cst == 1) {
      std::fprintf(log, " Could not connect to DADA buffer!\n");
      return 255;  // the reference returns -1
    }
    if (cst == 2) {
      std::fprintf(log, " Could not open for reading DADA buffer!\n");
      return 255;
    }
  }

  std::string base[2], stamp;
  double mjdstart = 0.0;
  int64_t ntimes = 0;
  int hrnext = 0;
  bool files_ok = true;
  auto open_files = [&]() {
    stamp = utc_stamp();
    for (int d = 0; d < 2; ++d) {
      char b[64];
      std::snprintf(b, sizeof b, "DM%.1f_%s", (double)dms[d], stamp.c_str());
      base[d] = b;
      files_ok = files_ok && create_empty(base[d] + ".dat") && create_empty(base[d] + "_SIGMA.dat");
      if (tool::file_exists(base[d].c_str())) std::remove(base[d].c_str());
    }
  };
  st = tool::run_stream(
      plan, src, log,
      [&](double mjd) {
        mjdstart = mjd;
        std::fprintf(log, "tstart= %.15lf   tsamp= %le\n", mjd, tsamp);
        hrnext = (utc_hour() + 1) % 24;
        open_files();
        std::fclose(log);
        logname = out + "_" + stamp + ".log";
        log = std::fopen(logname.c_str(), "w");
        std::fprintf(log, "begin main loop...\n");
      },
      [&](const vfrb_result& r) {
        if (r.dd && r.dd_sigma && r.nt == ntime_outdd) {
          for (int d = 0; d < 2; ++d) {
            files_ok = files_ok && append(base[d] + ".dat", r.dd + (size_t)d * r.nt, (size_t)r.nt) &&
                       append(base[d] + "_SIGMA.dat", r.dd_sigma + (size_t)d * r.nt, (size_t)r.nt);
          }
          ntimes += r.nt;
          if (want_flags && r.row_flags && r.nflag_rows >= r.nt) {
            FILE* ff = std::fopen((out + ".flags").c_str(), "ab");
            files_ok = files_ok && ff && tool::write_all(ff, r.row_flags, (size_t)r.nt);
            if (ff) std::fclose(ff);
          }
        }
        if (utc_hour() == hrnext) {  // TS:696-739
          for (int d = 0; d < 2; ++d)
            write_inf(base[d], mjdstart, ntimes, tsamp, dms[d], fchlo, bandw, L.nchanout, L.chanbw);
          open_files();
          std::fprintf(log, "Log file closed at %s\n", stamp.c_str());
          std::fclose(log);
          logname = out + "_" + stamp + ".log";
          log = std::fopen(logname.c_str(), "w");
          std::fprintf(log, "New log file opened at %s\n", stamp.c_str());
          mjdstart += (double)ntimes * tsamp / 86400.0;
          ntimes = 0;
          hrnext = (hrnext + 1) % 24;
        }
        std::fflush(log);
      });
  if (inf_at_end && !base[0].empty())
    for (int d = 0; d < 2; ++d) write_inf(base[d], mjdstart, ntimes, tsamp, dms[d], fchlo, bandw, L.nchanout, L.chanbw);
  vfrb_plan_destroy(plan);
  if (!files_ok) {
    std::fprintf(log, "Error writing the time series files\n");
    st = 2;
  }
  std::fprintf(log, "\nfinished!\n");
  std::fclose(log);
  return st;
}
