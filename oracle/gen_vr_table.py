"""Generate the Vioreanu-Rokhlin node/weight table header from the reference's
tabulated data.

The Vioreanu-Rokhlin interpolation nodes and quadrature weights on the simplex
(0,0),(1,0),(0,1) are published numeric tables.  The reference ships them as
the MATLAB function ``utils/get_vioreanu_nodes.m`` (degrees 0..20); the Fortran
routines ``get_vioreanu_nodes`` / ``get_vioreanu_wts`` that the hot path calls
(``src/patch_refine_mod.f90:132-133``) return the same table.  This script
parses that file and writes a C header holding the same numbers, so the
library and the oracle read identical nodes.

Usage:  python gen_vr_table.py <path-to-get_vioreanu_nodes.m> <out.h> [guard]
"""
import re
import sys


def parse(path):
    text = open(path).read()
    # the file has two sections: uvs(...) assignments then wts(...) assignments,
    # each grouped in "if(norder== k)" blocks.
    uvs, wts = {}, {}
    cur = None
    section = None
    for line in text.splitlines():
        m = re.match(r"\s*if\s*\(\s*norder\s*==\s*(\d+)\s*\)", line)
        if m:
            cur = int(m.group(1))
            continue
        m = re.match(r"\s*uvs\(\s*(\d)\s*,\s*(\d+)\s*\)\s*=\s*([-+0-9.eEdD]+)\s*;", line)
        if m:
            section = "uv"
            i, j, v = int(m.group(1)), int(m.group(2)), float(m.group(3).replace("D", "e").replace("d", "e"))
            uvs.setdefault(cur, {})[(i, j)] = v
            continue
        m = re.match(r"\s*wts\(\s*(\d+)\s*\)\s*=\s*([-+0-9.eEdD]+)\s*;", line)
        if m:
            section = "w"
            j, v = int(m.group(1)), float(m.group(2).replace("D", "e").replace("d", "e"))
            wts.setdefault(cur, {})[j] = v
    return uvs, wts


def main():
    src, out = sys.argv[1], sys.argv[2]
    guard = sys.argv[3] if len(sys.argv) > 3 else "QOL_VR_TABLE_H"
    uvs, wts = parse(src)
    degs = sorted(uvs)
    assert degs == list(range(0, 21)), degs
    lines = [
        "/* Vioreanu-Rokhlin nodes and weights on the simplex (0,0),(1,0),(0,1),",
        " * degrees 0..20, npts = (d+1)(d+2)/2.  Generated by gen_vr_table.py from",
        " * the reference's published table (utils/get_vioreanu_nodes.m). */",
        f"#ifndef {guard}",
        f"#define {guard}",
        "#define QOL_VR_MAXDEG 20",
        "static const int qol_vr_offset[22] = {",
    ]
    off = [0]
    for d in degs:
        n = (d + 1) * (d + 2) // 2
        assert len(wts[d]) == n and len(uvs[d]) == 2 * n, (d, len(wts[d]), len(uvs[d]))
        off.append(off[-1] + n)
    lines.append("  " + ", ".join(str(o) for o in off) + "};")
    lines.append(f"static const double qol_vr_uv[{2 * off[-1]}] = {{")
    for d in degs:
        n = (d + 1) * (d + 2) // 2
        vals = []
        for j in range(1, n + 1):
            vals += [uvs[d][(1, j)], uvs[d][(2, j)]]
        lines.append("  " + ", ".join(repr(v) for v in vals) + ",")
    lines.append("};")
    lines.append(f"static const double qol_vr_w[{off[-1]}] = {{")
    for d in degs:
        n = (d + 1) * (d + 2) // 2
        lines.append("  " + ", ".join(repr(wts[d][j]) for j in range(1, n + 1)) + ",")
    lines.append("};")
    lines.append("#endif")
    open(out, "w").write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
