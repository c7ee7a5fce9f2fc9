"""Test infrastructure, not product code: ctypes access to the oracle.

* ``Restatement`` -- the plain-C restatement of pine's hot path (oracle/pine_oracle.c),
  built into oracle/_build/libpine_oracle.so by oracle/Makefile.
* ``REF_BIN`` -- pine itself, built from the reference sources into oracle/_ref/pine_ref
  (present only where the reference sources were available at build time);
  ``REF_BIN_CONST`` the same with the added `Constant` environment light
  (oracle/constant_env.py).
* ``REFERENCE_SRC`` -- where the pine sources are ($PINE_REFERENCE, else the Makefile's
  default), for the scripts that read them at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libpine_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "pine_ref")
REF_BIN_CONST = os.path.join(HERE, "_ref", "pine_ref_const")


def _reference_src() -> str:
    """The pine source tree: $PINE_REFERENCE, else the default of oracle/Makefile's REF."""
    env = os.environ.get("PINE_REFERENCE")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as f:
        for line in f:
            if line.startswith("REF") and "?=" in line:
                return line.split("?=", 1)[1].strip()
    return ""


# Only present where the pine sources are (the build machine); nothing run on the GPU
# machine reads it.
REFERENCE_SRC = _reference_src()
MATH_NAMES = ["sqrt", "log2", "log", "exp", "cos", "sin", "tan", "acos", "asin", "atan",
              "atan2", "pow"]

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        F, I32, U32 = (ctypes.POINTER(t) for t in (ctypes.c_float, ctypes.c_int32, ctypes.c_uint32))
        D = ctypes.POINTER(ctypes.c_double)
        L.po_math.restype = ctypes.c_float
        L.po_math.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float]
        L.po_stof.restype = ctypes.c_float
        L.po_stof.argtypes = [ctypes.c_char_p, ctypes.c_int64]
        L.po_stofs.argtypes = [ctypes.c_char_p, ctypes.c_int64, F]
        L.po_bsdf.argtypes = [F, F]
        L.po_scene_new.restype = ctypes.c_void_p
        L.po_scene_new.argtypes = [ctypes.c_void_p]
        L.po_scene_free.argtypes = [ctypes.c_void_p]
        L.po_intersect.argtypes = [ctypes.c_void_p, F, ctypes.c_int64, I32, I32, F, I32, ctypes.c_int]
        L.po_camera_ray.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, F]
        L.po_density.restype = ctypes.c_float
        L.po_density.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_float]
        L.po_render.restype = ctypes.c_int64
        L.po_render.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, D, D,
                                U32, ctypes.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def math(fn: str, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    L = lib()
    k = MATH_NAMES.index(fn)
    return np.array([L.po_math(k, float(x), float(y)) for x, y in zip(a, b)], np.float32)


def stof(s: str) -> float:
    b = s.encode()
    return lib().po_stof(b, len(b))


def stofs(s: str) -> np.ndarray:
    b = s.encode()
    out = np.zeros(3, np.float32)
    lib().po_stofs(b, len(b), _p(out, ctypes.c_float))
    return out


def bsdf(rows: np.ndarray) -> np.ndarray:
    rows = np.ascontiguousarray(rows, np.float32)
    out = np.zeros((rows.shape[0], 16), np.float32)
    L = lib()
    for i in range(rows.shape[0]):
        L.po_bsdf(_p(rows[i], ctypes.c_float), _p(out[i], ctypes.c_float))
    return out


class Restatement:
    """The C restatement over a scene flattened by pg_parse_scene_file."""

    def __init__(self, scene_path: str):
        import pine_b200
        self._parsed = pine_b200.ParsedScene(scene_path)
        self.desc = self._parsed.desc
        self._s = lib().po_scene_new(ctypes.byref(self.desc))
        if not self._s:
            self._parsed.close()
            raise ValueError("the restatement covers constant-valued materials only")
        self.width, self.height = self.desc.camera.width, self.desc.camera.height

    def close(self):
        if self._s:
            lib().po_scene_free(self._s)
            self._s = None
        self._parsed.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def intersect(self, rays: np.ndarray, threads: int = os.cpu_count() or 1):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        shape = np.empty(n, np.int32)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        amb = np.empty(n, np.int32)
        lib().po_intersect(self._s, _p(rays, ctypes.c_float), n, _p(shape, ctypes.c_int32),
                           _p(prim, ctypes.c_int32), _p(t, ctypes.c_float),
                           _p(amb, ctypes.c_int32), int(threads))
        return shape, prim, t, amb.astype(bool)

    def camera_ray(self, fx, fy, l0, l1):
        out = np.zeros(6, np.float32)
        lib().po_camera_ray(self._s, fx, fy, l0, l1, _p(out, ctypes.c_float))
        return out

    def density(self, medium: int, pts: np.ndarray) -> np.ndarray:
        L = lib()
        return np.array([L.po_density(self._s, medium, *map(float, p)) for p in pts], np.float32)

    def render(self, spp: int, max_depth: int = 0, seed: int = 0,
               threads: int = os.cpu_count() or 1):
        w, h = self.width, self.height
        mean = np.zeros((h, w, 3), np.float64)
        var = np.zeros((h, w, 3), np.float64)
        cnt = np.zeros((h, w), np.uint32)
        md = max_depth if max_depth > 0 else self.desc.max_depth
        dropped = lib().po_render(self._s, int(spp), int(md), int(seed),
                                  _p(mean, ctypes.c_double), _p(var, ctypes.c_double),
                                  _p(cnt, ctypes.c_uint32), int(threads))
        return {"mean": mean, "var": var, "count": cnt, "dropped": dropped}
