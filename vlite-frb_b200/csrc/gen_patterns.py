#!/usr/bin/env python3
"""Writes dedisp_patterns.cuh: the in-group delay patterns the pattern-run
dedispersion kernel has straight-line code for.

For D adjacent trials of an equally spaced DM list, the delay of trial j in
channel c is floor(x_c + j*y_c) for the channel's x_c = k_c*DM_first and
y_c = k_c*dDM (the delay table truncates, TS:454-464), so the differences to
the first trial are Delta_j = floor(phi + j*y) with phi = frac(x_c).  The
patterns (0, Delta_1, ..., Delta_{D-1}) with Delta_{D-1} <= SMAX are the
"digital straight lines" through the origin; this script lists all of them
by sampling (phi, y) densely and keeping the distinct tuples.  Delay tables
whose groups fall outside the list (unequal DM spacing) are still handled,
by the kernel's generic path.

Usage: python gen_patterns.py  (rewrites dedisp_patterns.cuh next to it)
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GROUPS = {4: 20, 2: 16}  # D -> largest in-group delay difference (SMAX)


def patterns(D: int, smax: int, steps: int = 4000):
    ys = np.arange(0.0, smax / (D - 1) + 1.0, 1.0 / steps)
    out = set()
    for y in ys:
        ph = np.arange(0.0, 1.0, 1.0 / 512)
        t = np.stack([np.floor(ph + j * y) for j in range(1, D)], -1).astype(int)
        t = t[t.max(1) <= smax]
        out.update(map(tuple, t))
    return sorted(out, key=lambda p: (p[-1], p))


def main():
    lines = ["// Generated by gen_patterns.py -- do not edit.",
             "// In-group delay patterns (0, Delta_1, ..., Delta_{D-1}) of D adjacent,",
             "// equally spaced DM trials: Delta_j = floor(phi + j*y) (see gen_patterns.py).",
             "#pragma once", ""]
    for D, smax in GROUPS.items():
        ps = patterns(D, smax)
        assert len(ps) < 255
        lines.append(f"#define VFRB_PAT{D}_SMAX {smax}")
        lines.append(f"#define VFRB_PAT{D}_N {len(ps)}")
        lines.append(f"// X(id, Delta_1, ..., Delta_{D - 1})")
        body = [f"X({i}, {', '.join(map(str, p))})" for i, p in enumerate(ps)]
        rows = []
        for k in range(0, len(body), 6):
            rows.append("  " + " ".join(body[k:k + 6]))
        lines.append(f"#define VFRB_PAT{D}_LIST(X) \\")
        lines.append(" \\\n".join(rows))
        lines.append("")
    with open(os.path.join(HERE, "dedisp_patterns.cuh"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
