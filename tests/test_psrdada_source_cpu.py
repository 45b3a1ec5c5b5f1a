"""The DADA tools' psrdada input (tool::Source built with VFRB_WITH_PSRDADA).

psrdada itself is not installed here, so the probe below is compiled
against the oracle's file-backed stand-in for psrdada's reader API
(oracle/ref_shim: ipcio_connect / ipcio_open / ipcio_read / ipcbuf_* with
the ipcbuf_t first in the ipcio_t, as the reference relies on).  It checks
the tools' side: the reference's connect sequence and log lines (the iread
force, STATS:123-134, 284-304), every byte read back in order through reads
of an odd size, a short read at the end of data, and the failure code when
the ring cannot be opened.  No GPU is used.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "ref_shim")
LIB = os.path.join(ROOT, "vlite-frb_b200", "lib")

PROBE = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "tool_common.h"
#include "ipcio.h"
int main(int argc, char** argv) {
  if (argc != 5) return 100;
  ref_shim_set_dada_file(argv[1]);
  ref_shim_set_iread(std::atoi(argv[4]));
  FILE* log = std::fopen(argv[2], "w");
  int rc = 0;
  {
    tool::Source src;
    const int st = src.connect(0xdada, log);
    if (st) {
      rc = 10 + st;
    } else {
      FILE* out = std::fopen(argv[3], "wb");
      std::vector<char> b(4999);  // not a whole number of frames
      size_t n;
      while ((n = src.read(b.data(), b.size())) > 0) std::fwrite(b.data(), 1, n, out);
      std::fclose(out);
      if (src.failed) rc = 3;
    }
  }
  std::fclose(log);
  return rc;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if shutil.which("g++") is None or shutil.which("gcc") is None:
        pytest.skip("no C/C++ compiler")
    if not os.path.exists(os.path.join(LIB, "libvfrb.so")):
        pytest.skip("libvfrb.so not built")
    d = tmp_path_factory.mktemp("psrdada")
    shim_o = d / "shim.o"
    subprocess.run(["gcc", "-O2", "-DREF_SHIM_DADA_ONLY", "-I" + SHIM, "-c", os.path.join(SHIM, "ref_shim.c"),
                    "-o", str(shim_o)], check=True)
    src = d / "probe.cpp"
    src.write_text(PROBE)
    exe = d / "probe"
    subprocess.run(["g++", "-std=c++17", "-O1", "-DVFRB_WITH_PSRDADA", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "vlite-frb_b200", "tools"), "-I" + SHIM, str(src), str(shim_o),
                    "-L" + LIB, "-lvfrb", "-Wl,-rpath," + LIB, "-o", str(exe)], check=True)
    return d, exe


def _run(probe, data, iread):
    d, exe = probe
    fin, flog, fout = d / "ring.bin", d / f"log{iread}.txt", d / f"out{iread}.bin"
    if fout.exists():
        fout.unlink()
    if data is not None:
        fin.write_bytes(data)
    elif fin.exists():
        fin.unlink()
    r = subprocess.run([str(exe), str(fin), str(flog), str(fout), str(iread)], timeout=60)
    return r.returncode, flog.read_text(), (fout.read_bytes() if fout.exists() else None)


@pytest.mark.parametrize("iread", [-1, 3])
def test_psrdada_source_reads_every_byte(probe, iread):
    data = np.random.default_rng(5).integers(0, 256, 7 * 5032 + 1234, dtype=np.uint8).tobytes()
    rc, log, out = _run(probe, data, iread)
    assert rc == 0, log
    assert out == data
    if iread == -1:
        assert " iread= -1, do not need to force\n" in log
    else:
        assert " iread= 3 != -1, setting to -1\n" in log
    for line in (" nbufs= 1\n", " nfull= 0\n", " read count = 0\n"):
        assert line in log, log


def test_psrdada_source_cannot_open(probe):
    rc, log, out = _run(probe, None, -1)
    assert rc == 12  # connect returned 2: not opened as the primary reader
    assert out is None
