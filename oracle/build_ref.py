#!/usr/bin/env python3
"""Compiles the reference's own sources (read from the reference checkout;
never copied into the repository) with the project-written stand-ins in ref_shim/ and
the harness ref_harness.cu into oracle/_ref/libref_{pipe,stats,ts}.so.

TEST INFRASTRUCTURE ONLY: the libraries pin the oracle (tests/test_ref_pin.py)
and, on the GPU, give the reference's own cuFFT/kernel chain as a baseline.
The reference's Makefile is not used (it needs psrdada, vdifio and dedisp at
fixed paths).  Changes needed to build it here:
  * main() renamed (-Dmain=...), so the harness drives the functions;
  * GCC 13 rejects the ordered comparisons of FILE* with 0 (`outflog<0`,
    PIPE:257,262,271,279,354; STATS:187,196; TS:266,567-570,583,713-716,728)
    even with -fpermissive, so each tool is compiled from a temporary copy
    under /tmp in which exactly those comparisons read `== NULL`; the copy is
    deleted after the build and never enters the repository;
  * -fpermissive for the remaining string-literal-as-char* conversions;
  * relocatable device code, so the harness can launch the tool's kernels.
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: $VFRB_REFERENCE_DIR, else "reference" beside this repository
REF = os.environ.get("VFRB_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
OUT = os.path.join(HERE, "_ref")
NVCC = "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
TOOLS = {"pipe": ("vdifFILE2dedisp_PIPELINE.cu", "REF_PIPE"),
         "stats": ("vdifDADA2stats.cu", "REF_STATS"),
         "ts": ("vdifDADA2timeseries.cu", "REF_TS")}


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(" ".join(cmd) + "\n" + r.stdout[-4000:] + r.stderr[-4000:])


def build():
    if not os.path.isdir(REF):
        print("reference checkout not present; oracle/_ref not rebuilt")
        return False
    os.makedirs(OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim")
    inc = ["-I" + shim, "-I" + REF]
    shim_o = os.path.join(OUT, "ref_shim.o")
    run(["gcc", "-O2", "-fPIC", "-c", os.path.join(shim, "ref_shim.c"), *inc, "-o", shim_o])
    for name, (src, flag) in TOOLS.items():
        so = os.path.join(OUT, f"libref_{name}.so")
        srcs = [os.path.join(REF, src), os.path.join(HERE, "ref_harness.cu"), os.path.join(shim, "ref_shim.c")]
        if os.path.exists(so) and all(os.path.getmtime(so) > os.path.getmtime(s) for s in srcs):
            continue
        tool_o = os.path.join(OUT, f"{name}.o")
        harn_o = os.path.join(OUT, f"harness_{name}.o")
        common = [NVCC, *ARCH, "-O2", "-rdc=true", "-w", "-Xcompiler", "-fPIC,-fpermissive", *inc]
        tmp = tempfile.mkdtemp(prefix="vfrb_refbuild_")
        try:
            txt = open(os.path.join(REF, src)).read()
            txt = re.sub(r"\b(outflog|outf1|outf2|outf3|ft)<0\)", r"\1==NULL)", txt)
            txt = re.sub(r'("wb"\)\))(\s*)<0\)', r"\1\2==NULL)", txt)
            tsrc = os.path.join(tmp, src)
            with open(tsrc, "w") as f:
                f.write(txt)
            run([*common, f"-Dmain=ref_main_{name}", "-c", tsrc, "-o", tool_o])
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
        run([*common, f"-D{flag}", "-c", os.path.join(HERE, "ref_harness.cu"), "-o", harn_o])
        run([NVCC, *ARCH, "-rdc=true", "-shared", tool_o, harn_o, shim_o, "-lcufft", "-o", so])
    return True


if __name__ == "__main__":
    ok = build()
    sys.exit(0 if ok or not os.path.isdir(REF) else 1)
