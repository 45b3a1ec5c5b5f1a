// vdifFILE2dedisp_PIPELINE: drop-in for the reference tool of the same name
// (vdifFILE2dedisp_PIPELINE.cu), running on libvfrb's plan API.
//
// Same command line (PIPE:1244-1288): -d (defaults), -nchan N, -nave N,
// -nb N, -i FILE, -o NAME; an unknown argument prints the usage and exits 1.
// Same inputs: the VDIF file and DM101.txt in the working directory.  Same
// outputs (PIPE:253-284, 529-540, 732-739, 777):
//   NAME.log           run log
//   NAME.head          SIGPROC header (tstart = MJD of the first frame pair)
//   NAME.nohead.fil    the bandpass-subtracted filterbank of the fifth block
//                      (MAXNT rows x NCHANOUT float32, time-major)
//   OUTDD.bin          per DM trial: the DM (float32) then the fifth block's
//                      dedispersed series (NTIME_OUTDD float32)
// The reference keeps the fifth block (its `q==4` debug copies); with fewer
// blocks those buffers were never filled, here they are written as zeros.
//
// Extensions (not in the reference; the reference fixes these at compile
// time): -fullband (MUOSLOWFREQ 384 MHz: all 6250 channels), -maxtime S
// (block length, default 70 s), -dmfile PATH (default DM101.txt),
// -fp16 (FP16 storage form of the filterbank for dedispersion),
// -filall (NAME.fil: SIGPROC header + the bandpassed filterbank of every
// block, appended as each block completes; block 0 whole, later blocks from
// row (max_delay/NBUNDLE)*NBUNDLE, the first row the reader refilled, so the
// file is one continuous time series), -bpfull / -zerodm (the reference's
// commented-out subtractbp, PIPE:1372, and subtractZERO, PIPE:1478),
// -cands SNR [-boxcar W] (NAME.cands: per block the trials whose best
// boxcar SNR reaches SNR and is a local maximum over trials, clustered
// across trials and blocks; one text line per cluster).
#include "tool_common.h"

namespace {

struct Opts {
  int twonchan = 0, nave = 0, nbundle = 0;
  std::string in, out;
  double muos = 360.0;
  float maxtime = 70.f;
  std::string dmfile = "DM101.txt";
  bool fp16 = false;
  bool filall = false, bpfull = false, zerodm = false;
  float cand_snr = 0.f;  // 0: no candidate file
  int boxcar = 1;
};

void usage() {
  std::fprintf(stderr,
               "***************************************************************************\n"
               "This program reads time series data from a file with VDIF format data,\n"
               "  dedisperses it over the DM trials in DM101.txt and writes a filterbank\n"
               "  file in SIGPROC format.\n\n"
               "  Usage:\n./vdifFILE2dedisp_PIPELINE -d:\t    use default values (unless other values given)\n"
               "\t             -i (string):   name of input file to read VDIF data from,\n"
               "\t             -o (string):   base name of ouput files to write,\n"
               "\t             -nave (int):   number of time samples to average over,\n"
               "\t             -nchan (int):  number of frequency channels,\n"
               "\t             -nb (int):     number of bundles of size (2*2*nchan*nave) to send in 1 memcpy\n"
               "  Extensions:\n"
               "\t             -fullband      write the full 320-384 MHz band (MUOSLOWFREQ 384)\n"
               "\t             -maxtime (s)   block length (default 70)\n"
               "\t             -dmfile (path) DM trial list (default DM101.txt)\n"
               "\t             -fp16          FP16 storage form for dedispersion\n"
               "\t             -filall        write every block's filterbank to NAME.fil (with header)\n"
               "\t             -bpfull        whole-block bandpass (subtractbp) instead of cal windows\n"
               "\t             -zerodm        subtract the zero-DM signal (subtractZERO)\n"
               "\t             -cands (float) write clustered candidates above this SNR to NAME.cands\n"
               "\t             -boxcar (int)  widest boxcar of the candidate search (default 1)\n\n"
               "  DEFAULTS:\n"
               "\t             -o     testDEDISP\n"
               "\t             -nave  4\n"
               "\t             -nchan 6250\n"
               "\t             -nb    32\n\n");
}

// PIPE:1244-1288, plus the extensions above
int parse(int argc, char** argv, Opts& o) {
  int i = 1;
  if (tool::eq(argv[i], "-d")) {
    o.twonchan = 6250 * 2;
    o.nave = 4;
    o.nbundle = 32;
    o.out = "testDEDISP";
    ++i;
  }
  for (; i < argc; ++i) {
    const bool more = i + 1 < argc;
    if (tool::eq(argv[i], "-nchan") && more) {
      o.twonchan = 2 * std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-nave") && more) {
      o.nave = std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-nb") && more) {
      o.nbundle = std::atoi(argv[++i]);
    } else if (tool::eq(argv[i], "-i") && more) {
      o.in = argv[++i];
    } else if (tool::eq(argv[i], "-o") && more) {
      o.out = argv[++i];
    } else if (tool::eq(argv[i], "-fullband")) {
      o.muos = 384.0;
    } else if (tool::eq(argv[i], "-maxtime") && more) {
      o.maxtime = (float)std::atof(argv[++i]);
    } else if (tool::eq(argv[i], "-dmfile") && more) {
      o.dmfile = argv[++i];
    } else if (tool::eq(argv[i], "-fp16")) {
      o.fp16 = true;
    } else if (tool::eq(argv[i], "-filall")) {
      o.filall = true;
    } else if (tool::eq(argv[i], "-bpfull")) {
      o.bpfull = true;
    } else if (tool::eq(argv[i], "-zerodm")) {
      o.zerodm = true;
    } else if (tool::eq(argv[i], "-cands") && more) {
      o.cand_snr = (float)std::atof(argv[++i]);
    } else if (tool::eq(argv[i], "-boxcar") && more) {
      o.boxcar = std::atoi(argv[++i]);
    } else {
      std::fprintf(stderr, "Error! Unknown argument: %s\n\n", argv[i]);
      usage();
      return 3;
    }
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  const double t_begin = tool::now_s();
  if (argc < 2) {
    usage();
    return 1;
  }
  Opts o;
  if (parse(argc, argv, o)) return 1;

  const std::string logname = o.out + ".log", headname = o.out + ".head", filname = o.out + ".nohead.fil";
  FILE* log = std::fopen(logname.c_str(), "w");
  if (!log) {
    std::fprintf(stderr, "Unable to open output log file: %s\n", logname.c_str());
    return 2;
  }
  FILE* head = std::fopen(headname.c_str(), "wb");
  if (!head) {
    std::fprintf(stderr, "Unable to open output SIGPROC header file: %s\n", headname.c_str());
    return 2;
  }
  if (tool::file_exists(filname.c_str())) std::remove(filname.c_str());
  FILE* fil = std::fopen(filname.c_str(), "wb");
  if (!fil) {
    std::fprintf(stderr, "Unable to open output SIGPROC headerless filterbank file: %s\n", filname.c_str());
    return 2;
  }
  if (tool::file_exists("OUTDD.bin")) std::remove("OUTDD.bin");
  FILE* outdd = std::fopen("OUTDD.bin", "wb");
  if (!outdd) {
    std::fprintf(stderr, "Unable to open output for dedispersion debugging\n");
    return 2;
  }
  std::fprintf(log, "Running vdifFILE2dedisp_PIPELINE (libvfrb, sm_100a)\n");

  vfrb_params p;
  vfrb_params_default(&p);
  p.twonchan = o.twonchan;
  p.nave = o.nave;
  p.nbundle = o.nbundle;
  p.muoslowfreq = o.muos;
  p.maxtime = o.maxtime;
  p.mode = VFRB_MODE_BLOCK;
  p.reader = VFRB_READER_PIPE;
  p.outputs = VFRB_OUT_DEDISP | VFRB_OUT_DMSTATS | VFRB_OUT_FB;
  p.fb_block = o.filall ? -1 : 4;  // the block the reference copies out (q == 4), or all
  p.storage = o.fp16 ? VFRB_F16 : VFRB_F32;
  p.bp_mode = o.bpfull ? VFRB_BP_FULL : VFRB_BP_CAL;
  p.zero_dm = o.zerodm ? 1 : 0;
  if (o.cand_snr > 0.f) {
    p.outputs |= VFRB_OUT_CANDS;
    p.cand_snr = o.cand_snr;
    p.boxcar_max = o.boxcar;
  }
  FILE* filall = nullptr;
  if (o.filall) {
    const std::string n = o.out + ".fil";
    if (tool::file_exists(n.c_str())) std::remove(n.c_str());
    filall = std::fopen(n.c_str(), "wb");
    if (!filall) {
      std::fprintf(stderr, "Unable to open output SIGPROC filterbank file: %s\n", n.c_str());
      return 2;
    }
  }

  tool::Source src;
  if (o.in.empty() || !src.open(o.in.c_str())) {
    std::fprintf(stderr, "Unable to open input VDIF file: %s\n", o.in.c_str());
    return 2;
  }
  std::vector<float> dms;
  std::fprintf(log, "counting number of DM trials in %s...\n", o.dmfile.c_str());
  if (tool::read_dm_list(o.dmfile.c_str(), dms) < 0) {
    std::fprintf(log, "ERROR opening file %s!\n", o.dmfile.c_str());
    return 2;
  }
  std::fprintf(log, "found %d DM trials.\n", (int)dms.size());
  p.dms = dms.data();
  p.ndm = (int32_t)dms.size();

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
  std::fprintf(log, "NFREQ= %d\nNCHAN= %d\nNCHANOUT= %d\nNAVE= %d\nNBUNDLE= %d\n", L.nfreq, L.nchan, L.nchanout,
               L.nave, L.nbundle);
  std::fprintf(log, "CHANBW= %lf [MHz]  (foffNEG= %lf)\nfch1= %lf [MHz]\n", L.chanbw, L.foff, L.fch1);
  std::fprintf(log, "MAXNT= %d\nNHALFCYC= %d\n", L.maxnt, L.nhalfcyc);
  std::fprintf(log, "dm_count = %d\nmax_delay= %d [samples]\nNTIME_OUTDD= %lld\n", (int)dms.size(), max_delay,
               (long long)ntime_outdd);

  std::vector<float> keep_dd((size_t)dms.size() * (size_t)std::max<int64_t>(ntime_outdd, 0), 0.f);
  std::vector<float> keep_fb((size_t)L.maxnt * L.nchanout, 0.f);
  int64_t nblocks = 0;
  bool files_ok = true;
  std::vector<vfrb_cand> cands;
  const double tsamp = (double)L.nave * L.twonchan / 128e6;
  st = tool::run_stream(
      plan, src, log,
      [&](double mjd) {
        std::vector<uint8_t> h(vfrb_sigproc_header(nullptr, 0, L.fch1, L.foff, L.nchanout, 32, mjd, tsamp, 1));
        vfrb_sigproc_header(h.data(), h.size(), L.fch1, L.foff, L.nchanout, 32, mjd, tsamp, 1);
        tool::write_all(head, h.data(), h.size());
        if (filall) files_ok = tool::write_all(filall, h.data(), h.size()) && files_ok;
      },
      [&](const vfrb_result& r) {
        std::fprintf(log, "block %lld: %lld samples x %d DM trials, device errors %d\n", (long long)r.seq,
                     (long long)r.nt, r.ndm, r.device_errors);
        if (r.seq == 4) {
          if (r.dd && r.nt == ntime_outdd) std::memcpy(keep_dd.data(), r.dd, keep_dd.size() * 4);
          if (r.fb && r.fb_rows == L.maxnt) std::memcpy(keep_fb.data(), r.fb, keep_fb.size() * 4);
        }
        if (filall && r.fb && r.fb_rows == L.maxnt) {
          const int64_t first = r.seq == 0 ? 0 : (int64_t)(max_delay / L.nbundle) * L.nbundle;
          files_ok = tool::write_all(filall, r.fb + (size_t)first * L.nchanout,
                                     (size_t)(L.maxnt - first) * L.nchanout * 4) && files_ok;
        }
        for (int32_t k = 0; k < r.ncand; ++k) cands.push_back(r.cands[k]);
        ++nblocks;
      });
  if (filall) std::fclose(filall);
  if (o.cand_snr > 0.f) {
    // one pulse: within 8 trials and 50 samples
    std::vector<vfrb_cand> cl(cands.size());
    int32_t ncl = 0;
    vfrb_cluster_cands(cands.data(), (int32_t)cands.size(), 8, 50, cl.data(), &ncl, nullptr);
    FILE* cf = std::fopen((o.out + ".cands").c_str(), "w");
    if (cf) {
      std::fprintf(cf, "# sample  time_s  dm  snr  width  dm_index\n");
      for (int32_t k = 0; k < ncl; ++k)
        std::fprintf(cf, "%lld %.6f %.3f %.3f %d %d\n", (long long)cl[(size_t)k].t, cl[(size_t)k].t * tsamp,
                     (double)cl[(size_t)k].dm, (double)cl[(size_t)k].snr, cl[(size_t)k].width,
                     cl[(size_t)k].dm_index);
      std::fclose(cf);
    } else {
      files_ok = false;
    }
    std::fprintf(log, "%d candidates in %d clusters\n", (int)cands.size(), (int)ncl);
  }
  // OUTDD.bin (PIPE:734-739) and the headerless filterbank (PIPE:777)
  for (size_t i = 0; i < dms.size(); ++i) {
    tool::write_all(outdd, &dms[i], 4);
    tool::write_all(outdd, keep_dd.data() + i * (size_t)std::max<int64_t>(ntime_outdd, 0),
                    (size_t)std::max<int64_t>(ntime_outdd, 0) * 4);
  }
  tool::write_all(fil, keep_fb.data(), keep_fb.size() * 4);
  std::fclose(head);
  std::fclose(fil);
  std::fclose(outdd);
  vfrb_plan_destroy(plan);
  std::fprintf(log, "Processed %lld blocks (q= %lld)\n", (long long)nblocks, (long long)nblocks);
  if (!files_ok) {
    std::fprintf(log, "Error writing the output files\n");
    if (st == 0) st = 2;
  }
  const double t = tool::now_s() - t_begin;
  std::fprintf(log, "Total run time = %f [sec]\n", t);
  std::fprintf(log, "\nfinished!\n");
  std::fclose(log);
  std::fprintf(stdout, "TOTAL TIME = %f [sec]\n", t);
  return st;
}
