"""Regenerates tests/golden/poly3tab.json from the reference source text.

The reference ships no test fixtures.  Its one table of known answers is the
poly3tab basis: W = S^{-1/2} and S for alpha = 1..11, written out as Fortran
literals in get_orthonormalization_matrix_poly3_tabulated
(src/soap_turbo_radial.f90:1235-1535).  This script reads that file as text
(nothing is compiled or run) and stores the numbers column-major, as the
reference's reshape(..., shape(W)) lays them out.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import re
import sys


def main(ref_root):
    src = open(os.path.join(ref_root, "src", "soap_turbo_radial.f90")).read()
    start = src.index("subroutine get_orthonormalization_matrix_poly3_tabulated")
    end = src.index("end subroutine", start)
    body = src[start:end]
    cases = re.split(r"\n\s*case\((\d+)\)", body)
    out = {}
    for i in range(1, len(cases), 2):
        a = int(cases[i])
        text = cases[i + 1]
        mats = {}
        for name in ("W", "S"):
            m = re.search(name + r"\s*=\s*reshape\(\[(.*?)\],\s*shape\(" + name + r"\)\)", text, re.S)
            nums = re.findall(r"[-+]?\d+\.\d+(?:[dDeE][-+]?\d+)?", m.group(1).replace("&", " "))
            vals = [float(x.replace("d", "e").replace("D", "e")) for x in nums]
            assert len(vals) == a * a, (a, name, len(vals))
            mats[name] = vals
        out[str(a)] = mats
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "poly3tab.json")
    with open(path, "w") as f:
        json.dump({"source": "src/soap_turbo_radial.f90:1235-1535 (column-major)", "tables": out}, f,
                  indent=0)
    print("wrote", path, sorted(int(k) for k in out))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
