#!/usr/bin/env python3
"""Builds libvfrb.so (sm_100a) and the drop-in command-line tools in-tree.

    python vlite-frb_b200/build.py [--clean] [-j N]

Objects go to vlite-frb_b200/_build/, the library to vlite-frb_b200/lib/ and
the tools to vlite-frb_b200/bin/.  Rebuilds only what changed.

With PSRDADA_DIR set (a psrdada install: include/ipcio.h, lib/libpsrdada),
the DADA tools (vdifDADA2stats, vdifDADA2timeseries) are built against
psrdada and read the capture's own ring, as the reference tools do; without
it they read the project's ring (vfrb_dada_*).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
TOOLS = os.path.join(HERE, "tools")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-Wall,-Wno-unused-function",
          "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include"), "-I" + CSRC]

LIB_SOURCES = ["channelise.cu", "bandpass.cu", "rfi.cu", "dedisperse.cu", "vfrb_api.cpp"]
LIB_SOURCES_OPTIONAL = ["engine.cu", "vdif_reader.cpp", "writers.cpp", "dada.cpp", "noalloc.cu", "candidates.cu", "cluster.cpp"]
TOOL_MAINS = ["vdifFILE2dedisp_PIPELINE.cpp", "vdifDADA2stats.cpp", "vdifDADA2timeseries.cpp", "vfrb_dada_write.cpp"]
DADA_TOOLS = ("vdifDADA2stats.cpp", "vdifDADA2timeseries.cpp")


def psrdada_flags(main: str) -> list:
    """Compile and link flags that put a DADA tool on psrdada's own ring
    (PSRDADA_DIR set), else none."""
    d = os.environ.get("PSRDADA_DIR")
    if not d or main not in DADA_TOOLS:
        return []
    lib = os.path.join(d, "lib")
    return ["-DVFRB_WITH_PSRDADA", "-I" + os.path.join(d, "include"), "-L" + lib, "-lpsrdada",
            "-Xlinker", "-rpath," + lib]


def _newer(src: str, dst: str, deps=()) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in (src, *deps) if os.path.exists(p))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def gen_codelets():
    gen = os.path.join(CSRC, "gen_dft.py")
    out = os.path.join(CSRC, "dft_pairs.cuh")
    if _newer(gen, out):
        txt = subprocess.run([sys.executable, gen], capture_output=True, text=True, check=True).stdout
        with open(out, "w") as f:
            f.write(txt)
    pat = os.path.join(CSRC, "gen_patterns.py")
    if _newer(pat, os.path.join(CSRC, "dedisp_patterns.cuh")):
        subprocess.run([sys.executable, pat], check=True)


def build(jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    gen_codelets()
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h", ".hpp"))]
    headers.append(os.path.join(REPO, "include", "vfrb.h"))
    srcs = [s for s in LIB_SOURCES] + [s for s in LIB_SOURCES_OPTIONAL if os.path.exists(os.path.join(CSRC, s))]
    jobs_list = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s + ".o")
        if _newer(src, obj, headers):
            cmd = [NVCC, *ARCH, *COMMON, "-Xptxas", "-v" if verbose else "-O3", "-c", src, "-o", obj]
            if s.endswith(".cpp"):
                cmd = [NVCC, *COMMON, "-x", "cu", "-c", src, "-o", obj, *ARCH]
            jobs_list.append(cmd)
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for out in ex.map(_run, jobs_list):
            logs.append(out)
    objs = [os.path.join(OBJ, s + ".o") for s in srcs]
    so = os.path.join(LIB, "libvfrb.so")
    if any(_newer(o, so) for o in objs):
        _run([NVCC, *ARCH, "-shared", "-o", so, *objs, "-lpthread"])
    # command-line tools (link against the shared library, rpath to lib/)
    for m in TOOL_MAINS:
        src = os.path.join(TOOLS, m)
        if not os.path.exists(src):
            continue
        exe = os.path.join(BIN, m[:-4])
        if _newer(src, exe, headers + [so] + [os.path.join(TOOLS, h) for h in os.listdir(TOOLS) if h.endswith(".h")]):
            _run([NVCC, *COMMON, "-x", "cu", src, "-o", exe, *ARCH, *psrdada_flags(m), "-L" + LIB, "-lvfrb",
                  "-Xlinker", "-rpath," + LIB, "-Xlinker", "-rpath,$ORIGIN/../lib"])
    return "\n".join(logs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true", help="print ptxas register/smem usage")
    a = ap.parse_args()
    if a.clean:
        for d in (OBJ, LIB, BIN):
            shutil.rmtree(d, ignore_errors=True)
    log = build(a.j, a.v)
    if a.v:
        print(log)
    print("built", os.path.join(LIB, "libvfrb.so"))


if __name__ == "__main__":
    main()
