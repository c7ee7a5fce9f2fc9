"""Writes sobol_dirnums.inc: the Joe-Kuo Sobol direction numbers (new-joe-kuo-6.21201,
S. Joe and F. Y. Kuo, "Constructing Sobol sequences with better two-dimensional
projections", SIAM J. Sci. Comput. 30, 2008) for dimensions 1-1023, the table pine's
1024-dimension SobolSampler is built from (util/sobolmetrices.h:10-12).

The numbers are read from the copy SciPy ships for scipy.stats.qmc.Sobol
(scipy/stats/_sobol_direction_numbers.npz: `poly`, the primitive polynomial with its
leading and trailing ones, and `vinit`, the initial direction integers m_1..m_s).  Each
dimension is written as: poly, then its s = degree initial m values.  Dimension 0 (van der
Corput) has no entry.

Run once to regenerate: python pine_b200/csrc/gen_sobol_dirnums.py
"""

import os

import numpy as np
import scipy

DIMS = 1024


def main():
    d = np.load(os.path.join(os.path.dirname(scipy.__file__), "stats",
                             "_sobol_direction_numbers.npz"))
    poly, vinit = d["poly"], d["vinit"]
    vals = []
    for dim in range(1, DIMS):
        p = int(poly[dim])
        s = p.bit_length() - 1
        vals.append(p)
        vals.extend(int(v) for v in vinit[dim, :s])
    assert max(vals) < 1 << 16
    lines = ["// Generated by gen_sobol_dirnums.py from the Joe-Kuo direction numbers",
             "// (new-joe-kuo-6.21201) for Sobol dimensions 1-1023: per dimension its primitive",
             "// polynomial (with leading and trailing ones), then one initial direction integer",
             "// m_k per degree.",
             f"static const uint16_t kSobolDirNums[{len(vals)}] = {{"]
    for i in range(0, len(vals), 16):
        lines.append("    " + ", ".join(str(v) for v in vals[i:i + 16]) + ",")
    lines.append("};")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sobol_dirnums.inc")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(out, len(vals), "values")


if __name__ == "__main__":
    main()
