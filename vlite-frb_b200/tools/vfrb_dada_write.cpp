// vfrb_dada_write: feeds a VDIF file into the DADA-style ring (vfrb_dada_*)
// that vdifDADA2stats and vdifDADA2timeseries read, standing in for the
// psrdada writer of a live VLITE system (dada_junkdb / the capture process).
//
//   vfrb_dada_write -k KEY -i FILE [-cap BYTES] [-chunk BYTES] [-timeout S]
//
// Creates the ring (capacity a power of two, default 256 MiB), sets its
// header block (DADA-style "KEY value" lines: header version and size, the
// source file, the VDIF frame geometry), writes the file, marks end of data, waits (bounded) until the reader has taken every
// byte, and removes the ring.  Exit 0 on success, 2 on an I/O error, 3 when
// the reader stalled past the timeout.
#include "tool_common.h"

int main(int argc, char** argv) {
  unsigned key = 0xdada;
  std::string in;
  uint64_t cap = 256ull << 20, chunk = 16ull << 20;
  int timeout_s = 300;
  for (int i = 1; i < argc; ++i) {
    const bool more = i + 1 < argc;
    if (tool::eq(argv[i], "-k") && more) {
      std::sscanf(argv[++i], "%x", &key);
    } else if (tool::eq(argv[i], "-i") && more) {
      in = argv[++i];
    } else if (tool::eq(argv[i], "-cap") && more) {
      cap = std::strtoull(argv[++i], nullptr, 10);
    } else if (tool::eq(argv[i], "-chunk") && more) {
      chunk = std::strtoull(argv[++i], nullptr, 10);
    } else if (tool::eq(argv[i], "-timeout") && more) {
      timeout_s = std::atoi(argv[++i]);
    } else {
      std::fprintf(stderr, "usage: vfrb_dada_write -k KEY -i FILE [-cap BYTES] [-chunk BYTES] [-timeout S]\n");
      return 1;
    }
  }
  tool::Source src;
  if (in.empty() || !src.open(in.c_str())) {
    std::fprintf(stderr, "cannot open %s\n", in.c_str());
    return 2;
  }
  vfrb_dada* ring = nullptr;
  int st = vfrb_dada_create(key, cap, &ring);
  if (st != VFRB_OK) {
    std::fprintf(stderr, "cannot create ring %x: %s\n", key, vfrb_strerror(st));
    return 2;
  }
  char hdr[1024];
  const int hn = std::snprintf(hdr, sizeof hdr,
                               "HDR_VERSION 1.0\nHDR_SIZE 4096\nFILE_NAME %s\nENCODING VDIF\nFRAME_SIZE 5032\n"
                               "NPOL 2\nNBIT 8\nBW 64\nTSAMP 0.0078125\n",
                               in.c_str());
  vfrb_dada_set_header(ring, hdr, (uint64_t)std::min(hn, (int)sizeof hdr - 1));
  std::vector<uint8_t> buf((size_t)chunk);
  int rc = 0;
  for (;;) {
    const size_t n = src.read(buf.data(), buf.size());
    if (n == 0) break;
    const int64_t w = vfrb_dada_write(ring, buf.data(), n, timeout_s * 1000);
    if (w != (int64_t)n) {
      std::fprintf(stderr, "reader stalled\n");
      rc = 3;
      break;
    }
  }
  vfrb_dada_set_eod(ring);
  const double t0 = tool::now_s();
  while (rc == 0 && !vfrb_dada_eod(ring)) {
    if (tool::now_s() - t0 > timeout_s) {
      rc = 3;
      break;
    }
    usleep(10000);
  }
  vfrb_dada_close(ring);
  vfrb_dada_destroy(key);
  return rc;
}
