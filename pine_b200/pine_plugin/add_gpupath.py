"""Writes pine's integrator.cpp with the GpuPath integrator registered: the one line a
maintainer adds to CreateIntegrator (src/core/integrator.cpp:20-37), plus its #include.

Usage:  python add_gpupath.py <pine src root> <output file>
Every other pine source is compiled unmodified (see Makefile).
"""

import os
import sys


def patch(src_root: str, out: str) -> None:
    with open(os.path.join(src_root, "core", "integrator.cpp")) as f:
        text = f.read()
    include = "#include <impl/integrator/path.h>\n"
    case = '        CASE("Path") return new PathIntegrator(params, scene);\n'
    if text.count(include) != 1 or text.count(case) != 1:
        raise SystemExit("integrator.cpp: the Path integrator's include or case was not found once")
    text = text.replace(include, include + "#include <gpupath.h>\n")
    text = text.replace(case, case + '        CASE("GpuPath") return new GpuPathIntegrator(params, scene);\n')
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out + ".tmp", "w") as f:
        f.write(text)
    os.replace(out + ".tmp", out)


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    patch(sys.argv[1], sys.argv[2])
