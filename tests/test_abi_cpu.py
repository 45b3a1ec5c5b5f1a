"""The Python binding's ctypes mirrors of the C-ABI structs in include/vfrb.h
have the C layout: for every mirrored struct, the same size and, for every
field, the same offset as gcc gives when compiling against the header.  A
mismatch would hand the library shifted arguments without any error, so this
runs on the CPU (no GPU, nothing launched)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# ctypes class -> C type; ctypes field names that differ from the C ones
STRUCTS = {
    "Hdr": "vfrb_hdr",
    "Layout": "vfrb_layout",
    "ChanArgs": "vfrb_chan_args",
    "BpArgs": "vfrb_bp_args",
    "DdArgs": "vfrb_dd_args",
    "CsArgs": "vfrb_cs_args",
    "Params": "vfrb_params",
    "Cand": "vfrb_cand",
    "Result": "vfrb_result",
}
RENAMED = {("BpArgs", "inp"): "in"}


def _c_layout(tmp_path, vf):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vfrb.h"', "int main(void) {"]
    for py, cn in STRUCTS.items():
        lines.append(f'  printf("{py} size %zu\\n", sizeof({cn}));')
        for f, _ in getattr(vf, py)._fields_:
            cf = RENAMED.get((py, f), f)
            lines.append(f'  printf("{py} {f} %zu\\n", offsetof({cn}, {cf}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        py, f, v = ln.split()
        got[(py, f)] = int(v)
    return got


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirrors_match_the_header(tmp_path, vf):
    got = _c_layout(tmp_path, vf)
    for py in STRUCTS:
        cls = getattr(vf, py)
        assert C.sizeof(cls) == got[(py, "size")], (py, C.sizeof(cls), got[(py, "size")])
        for f, _ in cls._fields_:
            assert getattr(cls, f).offset == got[(py, f)], (py, f, getattr(cls, f).offset, got[(py, f)])
