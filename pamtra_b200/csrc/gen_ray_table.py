"""Writes the optical constants of liquid water for 0.2-1000 um that the Ray
water model interpolates below 1 mm wavelength (src/eps_water.f90:269-502:
Hale and Querry 1973 for 0.2-0.69 um, Palmer and Williams 1974 for
0.69-2 um, Downing and Williams 1975 for 2-1000 um; 518 wavelengths with
the real and imaginary refractive index at each).

The numbers are published measurements and must be the reference's to the
bit, so they are read from its source rather than typed: the reference
declares them as default-REAL literals in a REAL(8) parameter array, which
rounds each to single precision first, and both generated files keep them
as single-precision literals for the same reason.

Usage: python pamtra_b200/csrc/gen_ray_table.py <reference>/src/eps_water.f90
Writes pamtra_b200/csrc/ray_table.cuh (device tables) and
oracle/ray_table.inc (host tables for the CPU restatement).
"""
import os
import re
import sys

NAMES = ("wltabw", "rntabw", "cntabw")


def parse(path):
    text = open(path).read()
    out = {}
    for name in NAMES:
        m = re.search(r"dimension\((\d+)\),\s*parameter\s*::\s*%s\s*=\s*\(/(.*?)/\)" % name, text, re.S)
        if m is None:
            raise SystemExit("table %s not found in %s" % (name, path))
        vals = [v for v in re.split(r"[\s,&]+", m.group(2)) if v]
        if len(vals) != int(m.group(1)):
            raise SystemExit("table %s: %d values, expected %s" % (name, len(vals), m.group(1)))
        for v in vals:
            float(v)
        out[name] = vals
    return out


def _body(vals):
    lines, row = [], []
    for v in vals:
        row.append(v + "f")
        if len(row) == 8:
            lines.append("    " + ", ".join(row) + ",")
            row = []
    if row:
        lines.append("    " + ", ".join(row) + ",")
    return "\n".join(lines)


def emit(tabs, qual, guard):
    n = len(tabs["wltabw"])
    doc = ("// Generated by pamtra_b200/csrc/gen_ray_table.py from src/eps_water.f90:269-502:\n"
           "// wavelength [um], real and imaginary refractive index of liquid water,\n"
           "// single-precision literals as the reference declares them.\n")
    s = [doc, "#ifndef %s\n#define %s\n" % (guard, guard), "#define RAY_NUMWAT %d\n" % n]
    for name, cname in zip(NAMES, ("ray_wl", "ray_rn", "ray_cn")):
        s.append("%s float %s[RAY_NUMWAT] = {\n%s\n};\n" % (qual, cname, _body(tabs[name])))
    s.append("#endif\n")
    return "\n".join(s)


def main(argv):
    if len(argv) != 2:
        raise SystemExit(__doc__)
    tabs = parse(argv[1])
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(os.path.dirname(here))
    with open(os.path.join(here, "ray_table.cuh"), "w") as f:
        f.write(emit(tabs, "__device__ const", "PAMTRA_B200_RAY_TABLE_CUH"))
    with open(os.path.join(root, "oracle", "ray_table.inc"), "w") as f:
        f.write(emit(tabs, "static const", "PAMTRA_ORACLE_RAY_TABLE_INC"))


if __name__ == "__main__":
    main(sys.argv)
