"""Builds libpinegpu.so (the CUDA library behind include/pine_gpu.h) in-tree for sm_100a,
the pine-gpu command line and the pine-scenegen scene-input generator.

The shared library links the CUDA runtime statically, so loading it needs only the
driver; on a machine without a GPU it still loads and exports its symbols, and every
entry point that touches the device returns PG_ERR_CUDA.  pine-scenegen is plain C++
(no CUDA, no link to the library): generating a benchmark scene loads none of the renderer.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libpinegpu.so")
CLI = os.path.join(HERE, "pine-gpu")
SCENEGEN = os.path.join(HERE, "pine-scenegen")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["pine_gpu.cu", "pg_kernels_pine.cu", "pg_kernels_fast.cu", "guide_mlp.cu",
           "scene_load.cpp", "bvh_build.cpp", "bvh_gpu.cu"]
HEADERS = ["pg_math.h", "pg_device.cuh", "pg_shade.cuh", "pg_kernels.cuh", "scene_load.h",
           "bvh_build.h", "guide_net.cuh", "guide_mlp.h", "pg_nodes.h", "pg_sampler.h",
           "pg_launch.cuh", "pg_error.h", "sobol_dirnums.inc"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, defines=(), out: str = None) -> str:
    """Builds libpinegpu.so (or `out`, with extra -D `defines`) when a source changed."""
    lib_path = out or LIB
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "pine_gpu.h"),
                                                            __file__]
    if force or _stale(lib_path, deps):
        objdir = os.path.join(HERE, "_build", os.path.basename(lib_path))
        os.makedirs(objdir, exist_ok=True)
        objs = []
        procs = []
        for src in srcs:
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            objs.append(obj)
            cmd = [_nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-pthread", "-I", INCLUDE, "-I", CSRC,
                   *[f"-D{d}" for d in defines], "-c", src, "-o", obj]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT, text=True)))
        failed = []
        for cmd, p in procs:
            out, _ = p.communicate()
            if verbose and out:
                sys.stdout.write(out)
            if p.returncode != 0:
                failed.append((cmd, out))
        if failed:
            msg = "\n".join(" ".join(c) + "\n" + o for c, o in failed)
            raise RuntimeError("libpinegpu build failed:\n" + msg)
        tmp = lib_path + ".tmp"
        subprocess.run([_nvcc(), "-shared", *ARCH, "-o", tmp, *objs, "-Xcompiler", "-pthread"],
                       check=True)
        os.replace(tmp, lib_path)
    if out:
        return lib_path
    build_scenegen(force)
    cli_src = os.path.join(CSRC, "pine_cli.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB])):
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", INCLUDE, cli_src, "-o", CLI,
                        "-L", HERE, "-lpinegpu", "-Wl,-rpath,$ORIGIN", "-pthread"], check=True)
    return LIB


def build_scenegen(force: bool = False) -> str:
    """Builds pine-scenegen (seeded cloud grids and icospheres; see csrc/scenegen.cpp)."""
    src = os.path.join(CSRC, "scenegen.cpp")
    if force or _stale(SCENEGEN, [src, __file__]):
        tmp = SCENEGEN + ".tmp"
        subprocess.run(["g++", "-std=c++17", "-O2", src, "-o", tmp, "-pthread"], check=True)
        os.replace(tmp, SCENEGEN)
    return SCENEGEN


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
