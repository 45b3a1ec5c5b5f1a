// vdifDADA2stats: drop-in for the reference tool of the same name
// (vdifDADA2stats.cu), running on libvfrb's plan API.
//
// Reference behaviour kept (STATS:138-431, 811-834): no parameters but -h
// (any other argument: usage, exit 1); reads VDIF from the DADA ring with key
// 0xdada; 60-s blocks (MAXTIME) without overlap, bandpass + cal subtraction,
// then per channel and per 1-s statistics block (TIMESTATS) the mean, the
// variance and the outlier fraction; appends each block's three arrays
// [NSTATBLKS][NCHANOUT] float32 (CHANAVE, CHANSIGMA, CHANOUTLIER) to
// vdifDADA2stats_.stats, after truncating it at start; log in
// vdifDADA2stats_.log.
//
// Extensions: -k KEY (hex DADA key), -i FILE (read a VDIF file or "-"
// instead of a ring), -o NAME (output base name), -maxtime S, -timestats S,
// -nchan N / -nave N / -nb N (the reference fixes 6250 / 4 / 32),
// -fullband (MUOSLOWFREQ 384), -sk (NAME.sk: per block the spectral kurtosis
// of the raw filterbank, [NSTATBLKS][NCHANOUT] float32), -flags (NAME.flags:
// per block one byte per row, bit 0 = a frame with the VDIF invalid bit,
// bit 1 = a zero-filled missing frame).
#include "tool_common.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "***************************************************************************\n"
               "This program reads VDIF data from a DADA ring buffer and writes frequency\n"
               "  channel statistics (mean, variance, outlier fraction) per TIMESTATS block.\n\n"
               "  Usage:\n./vdifDADA2stats [-h]\n"
               "  Extensions:\n"
               "\t  -k (hex)        DADA key (default dada)\n"
               "\t  -i (string)     read a VDIF file instead of the ring (- = stdin)\n"
               "\t  -o (string)     base name of output files (default vdifDADA2stats_)\n"
               "\t  -maxtime (s)    block length (default 60)\n"
               "\t  -timestats (s)  statistics block (default 1)\n"
               "\t  -nchan/-nave/-nb (int)  channelisation (default 6250/4/32)\n"
               "\t  -fullband       all 6250 channels (MUOSLOWFREQ 384)\n"
               "\t  -sk             write the spectral kurtosis per block to NAME.sk\n"
               "\t  -flags          write the per-row data flags per block to NAME.flags\n\n");
}

}  // namespace

int main(int argc, char** argv) {
  int twonchan = 12500, nave = 4, nbundle = 32;
  unsigned key = 0xdada;
  std::string in, out = "vdifDADA2stats_";
  float maxtime = 60.f, timestats = 1.f;
  double muos = 360.0;
  bool want_sk = false, want_flags = false;
  for (int i = 1; i < argc; ++i) {
    const bool more = i + 1 < argc;
    if (tool::eq(argv[i], "-h")) {
      usage();
      return 1;
    } else if (tool::eq(argv[i], "-k") && more) {
      std::sscanf(argv[++i], "%x", &key);
    } else if (tool::eq(argv[i], "-i") && more) {
      in = argv[++i];
    } else if (tool::eq(argv[i], "-o") && more) {
      out = argv[++i];
    } else if (tool::eq(argv[i], "-maxtime") && more) {
      maxtime = (float)std::atof(argv[++i]);
    } else if (tool::eq(argv[i], "-timestats") && more) {
      timestats = (float)std::atof(argv[++i]);
    } else if (tool::eq(argv[i], "-nchan") && more) {
      twonchan = 2 * std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-nave") && more) {
      nave = std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-nb") && more) {
      nbundle = std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-fullband")) {
      muos = 384.0;
    } else if (tool::eq(argv[i], "-sk")) {
      want_sk = true;
    } else if (tool::eq(argv[i], "-flags")) {
      want_flags = true;
    } else {
      std::fprintf(stderr, "Error! Unknown argument: %s\n\n", argv[i]);
      usage();
      return 1;
    }
  }
  const std::string logname = out + ".log", statsname = out + ".stats";
  FILE* log = std::fopen(logname.c_str(), "w");
  if (!log) {
    std::fprintf(stderr, "Unable to open output log file: %s\n", logname.c_str());
    return 2;
  }
  FILE* stats = std::fopen(statsname.c_str(), "wb");
  if (!stats) {
    std::fprintf(stderr, "Unable to open output STATS file: %s\n", statsname.c_str());
    return 2;
  }
  FILE* skf = want_sk ? std::fopen((out + ".sk").c_str(), "wb") : nullptr;
  FILE* flf = want_flags ? std::fopen((out + ".flags").c_str(), "wb") : nullptr;
  if ((want_sk && !skf) || (want_flags && !flf)) {
    std::fprintf(stderr, "Unable to open the output SK / flags file\n");
    return 2;
  }
  std::fprintf(log, "Running vdifDADA2stats (libvfrb, sm_100a)\n");

  vfrb_params p;
  vfrb_params_default(&p);
  p.twonchan = twonchan;
  p.nave = nave;
  p.nbundle = nbundle;
  p.muoslowfreq = muos;
  p.maxtime = maxtime;
  p.timestats = timestats;
  p.mode = VFRB_MODE_BLOCK;
  p.reader = VFRB_READER_PIPE;
  p.outputs = VFRB_OUT_CHANSTATS | (want_flags ? VFRB_OUT_FLAGS : 0);
  p.dms = nullptr;
  p.ndm = 0;
  vfrb_plan* plan = nullptr;
  int st = vfrb_plan_create(&plan, &p);
  if (st != VFRB_OK) {
    std::fprintf(log, "Error creating the processing plan: %s\n", vfrb_strerror(st));
    return 1;
  }
  vfrb_layout L;
  vfrb_plan_layout(plan, &L, nullptr);
  std::fprintf(log, "NFREQ   = %d\nNCHAN   = %d\nNCHANOUT= %d\nNAVE    = %d\nNBUNDLE = %d\n", L.nfreq, L.nchan,
               L.nchanout, L.nave, L.nbundle);
  std::fprintf(log, "CHANBW  = %lf [MHz]  (foffNEG= %lf)\nfch1    = %lf [MHz]\n", L.chanbw, L.foff, L.fch1);

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
  int64_t nblocks = 0;
  st = tool::run_stream(
      plan, src, log, [&](double mjd) { std::fprintf(log, "tstart= %.15lf\n", mjd); },
      [&](const vfrb_result& r) {
        const size_t n = (size_t)r.nstatblks * (size_t)r.nchan;
        if (r.chan_ave && r.chan_sig && r.chan_outlier) {
          tool::write_all(stats, r.chan_ave, n * 4);
          tool::write_all(stats, r.chan_sig, n * 4);
          tool::write_all(stats, r.chan_outlier, n * 4);
          std::fflush(stats);
        }
        if (skf && r.chan_sk) tool::write_all(skf, r.chan_sk, n * 4);
        if (flf && r.row_flags) tool::write_all(flf, r.row_flags, (size_t)r.nflag_rows);
        ++nblocks;
      });
  std::fclose(stats);
  if (skf) std::fclose(skf);
  if (flf) std::fclose(flf);
  vfrb_plan_destroy(plan);
  std::fprintf(log, "Processed %f [sec] of data\n", (double)nblocks * L.maxnt * L.tchan);
  std::fprintf(log, "\nfinished!\n");
  std::fclose(log);
  return st;
}
