#!/usr/bin/env python3
"""Builds the oracle's C restatement (test infrastructure only):
oracle/_build/liboracle64.so (REAL=double, checker) and liboracle32.so
(REAL=float, timed CPU baseline), both with OpenMP."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")


def build():
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(HERE, "oracle.c")
    for bits, real in ((64, "double"), (32, "float")):
        so = os.path.join(OUT, f"liboracle{bits}.so")
        if os.path.exists(so) and os.path.getmtime(so) > os.path.getmtime(src):
            continue
        subprocess.run(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", f"-DREAL={real}",
                        "-o", so, src, "-lm"], check=True)
    ref = os.path.join(HERE, "build_ref.py")
    refdir = os.environ.get("VFRB_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
    if os.path.exists(ref) and os.path.isdir(refdir):
        subprocess.run([sys.executable, ref], check=False)


if __name__ == "__main__":
    build()
