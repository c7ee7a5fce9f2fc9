"""pine_b200: a B200 (sm_100a) wavefront path tracer behind pine's integrator surface.

This module is a thin ctypes binding of the C ABI in ``include/pine_gpu.h``
(``libpinegpu.so``, built in-tree by :mod:`pine_b200.build`).  All rendering runs in
the CUDA library; there is no CPU fallback, and every call fails with
:class:`PgError` when the library or a GPU is missing.
"""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libpinegpu.so")
HEADER = os.path.join(ROOT, "include", "pine_gpu.h")

PG_OK = 0
STATUS_NAMES = {0: "PG_OK", 1: "PG_ERR_INVALID_ARG", 2: "PG_ERR_OOM", 3: "PG_ERR_CUDA",
                4: "PG_ERR_DEVICE_LIMIT", 5: "PG_ERR_UNSUPPORTED", 6: "PG_ERR_IO",
                7: "PG_ERR_PARSE"}
MATH_MODES = {"pine": 0, "fast": 1}


class PgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class RenderDesc(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_int32), ("max_depth", ctypes.c_int32),
                ("seed", ctypes.c_uint64), ("sample_offset", ctypes.c_int32),
                ("math_mode", ctypes.c_int32), ("guiding", ctypes.c_int32),
                ("accumulate", ctypes.c_int32), ("profile", ctypes.c_int32)]


KERNELS = ["regen", "trace", "shade", "shadow", "guide", "train", "track", "transmit", "sort"]


class KernelStats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("seconds", ctypes.c_double),
                ("items", ctypes.c_int64), ("volume_steps", ctypes.c_int64),
                ("bricks", ctypes.c_int64)]


class RenderStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("paths", ctypes.c_int64),
                ("rays", ctypes.c_int64), ("volume_steps", ctypes.c_int64),
                ("dropped", ctypes.c_int64), ("launches", ctypes.c_int64),
                ("kernels", KernelStats * len(KERNELS))]

    def to_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "kernels"}
        d["kernels"] = {name: {k: getattr(self.kernels[i], k) for k, _ in KernelStats._fields_}
                        for i, name in enumerate(KERNELS)}
        return d


# Flattened scene description (pg_scene_desc and the records it points to).
class Shape(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("material", ctypes.c_int32),
                ("medium_inside", ctypes.c_int32), ("medium_outside", ctypes.c_int32),
                ("mesh_first_triangle", ctypes.c_int64), ("mesh_num_triangles", ctypes.c_int64),
                ("p", ctypes.c_float * 12)]


class NodeOp(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("arg", ctypes.c_int32), ("c", ctypes.c_float * 3)]


class Bsdf(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("albedo", ctypes.c_float * 3),
                ("roughness", ctypes.c_float), ("eta", ctypes.c_float),
                ("albedo_node", ctypes.c_int32), ("roughness_node", ctypes.c_int32),
                ("eta_node", ctypes.c_int32)]


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("num_layers", ctypes.c_int32),
                ("layers", Bsdf * 4), ("emission", ctypes.c_float * 3),
                ("bump_node", ctypes.c_int32)]


class Light(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("p", ctypes.c_float * 12)]


class Medium(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("sigma_a", ctypes.c_float * 3),
                ("sigma_s", ctypes.c_float * 3), ("g", ctypes.c_float),
                ("size", ctypes.c_int32 * 3), ("position", ctypes.c_float * 3),
                ("scale", ctypes.c_float), ("interpolate", ctypes.c_int32),
                ("density", ctypes.POINTER(ctypes.c_float))]


class Camera(ctypes.Structure):
    _fields_ = [("from_", ctypes.c_float * 3), ("to", ctypes.c_float * 3),
                ("fov", ctypes.c_float), ("lens_radius", ctypes.c_float),
                ("focus_distance", ctypes.c_float), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("medium", ctypes.c_int32)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("num_shapes", ctypes.c_int32), ("shapes", ctypes.POINTER(Shape)),
                ("num_vertices", ctypes.c_int64), ("vertices", ctypes.POINTER(ctypes.c_float)),
                ("num_triangles", ctypes.c_int64), ("indices", ctypes.POINTER(ctypes.c_uint32)),
                ("num_materials", ctypes.c_int32), ("materials", ctypes.POINTER(Material)),
                ("num_media", ctypes.c_int32), ("media", ctypes.POINTER(Medium)),
                ("num_lights", ctypes.c_int32), ("lights", ctypes.POINTER(Light)),
                ("camera", Camera), ("light_sampler", ctypes.c_int32),
                ("max_depth", ctypes.c_int32), ("samples_per_pixel", ctypes.c_int32),
                ("num_node_ops", ctypes.c_int32), ("node_ops", ctypes.POINTER(NodeOp)),
                ("sampler", ctypes.c_int32), ("sampler_scramble", ctypes.c_int32),
                ("filter", ctypes.c_int32), ("filter_radius", ctypes.c_float * 2),
                ("filter_params", ctypes.c_float * 2), ("integrator", ctypes.c_int32)]


SAMPLER_INDEPENDENT, SAMPLER_HALTON, SAMPLER_SOBOL = 0, 1, 2
FILTERS = {"Box": 0, "Triangle": 1, "Gaussian": 2, "Mitchell": 3, "LanczosSinc": 4}


SHAPE_SPHERE, SHAPE_PLANE, SHAPE_TRIANGLE, SHAPE_RECT, SHAPE_MESH = range(5)


class Tuning(ctypes.Structure):
    _fields_ = [("queue_capacity", ctypes.c_int32), ("block_size", ctypes.c_int32),
                ("split_shadow", ctypes.c_int32), ("majorant_brick", ctypes.c_int32),
                ("sort_queue", ctypes.c_int32), ("group_kinds", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("scene_id", ctypes.c_int32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("spp", ctypes.c_int32),
                ("max_depth", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("out_mean", ctypes.POINTER(ctypes.c_float))]


class BatchResult(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("paths", ctypes.c_int64),
                ("request_seconds", ctypes.POINTER(ctypes.c_double))]


_lib = None
_P = ctypes.POINTER
_F = _P(ctypes.c_float)
_I32 = _P(ctypes.c_int32)
_U32 = _P(ctypes.c_uint32)


def declared_functions(header: str = HEADER):
    """Names of the functions include/pine_gpu.h declares."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:pg_status|void|const char\s*\*|float)\s+(pg_\w+)\s*\(",
                                 text, flags=re.M)))


def lib():
    """Loads libpinegpu.so (raising if it was not built) and declares its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PgError(3, f"{LIB_PATH} is not built; run pine_b200.build.build()")
    L = ctypes.CDLL(LIB_PATH)
    st = ctypes.c_int
    sig = {
        "pg_create": (st, [_P(ctypes.c_void_p), ctypes.c_int]),
        "pg_destroy": (None, [ctypes.c_void_p]),
        "pg_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
        "pg_upload_scene": (st, [ctypes.c_void_p, ctypes.c_void_p, _I32]),
        "pg_load_scene_file": (st, [ctypes.c_void_p, ctypes.c_char_p, _I32]),
        "pg_release_scene": (st, [ctypes.c_void_p, ctypes.c_int32]),
        "pg_scene_info": (st, [ctypes.c_void_p, ctypes.c_int32, _I32, _I32, _I32, _I32]),
        "pg_render": (st, [ctypes.c_void_p, ctypes.c_int32, _P(RenderDesc), _F, _F, _U32,
                           _P(RenderStats)]),
        "pg_render_noalloc": (st, [ctypes.c_void_p, ctypes.c_int32, _P(RenderDesc),
                                   ctypes.c_void_p, _P(RenderStats)]),
        "pg_intersect": (st, [ctypes.c_void_p, ctypes.c_int32, _F, ctypes.c_int64, _I32, _I32,
                              _F, _F]),
        "pg_intersect_device": (st, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                     ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p]),
        "pg_set_tuning": (st, [ctypes.c_void_p, _P(Tuning)]),
        "pg_get_tuning": (st, [ctypes.c_void_p, _P(Tuning)]),
        "pg_pstd_stof": (ctypes.c_float, [ctypes.c_char_p, ctypes.c_int64]),
        "pg_pstd_math_device": (st, [_F, ctypes.c_int64, _F]),
        "pg_parse_scene_file": (st, [ctypes.c_char_p, _P(SceneDesc), _P(ctypes.c_void_p)]),
        "pg_free_parsed_scene": (None, [ctypes.c_void_p]),
        "pg_guide_reset": (st, [ctypes.c_void_p, ctypes.c_uint64]),
        "pg_guide_config": (st, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
        "pg_guide_get_weights": (st, [ctypes.c_void_p, _F]),
        "pg_guide_set_weights": (st, [ctypes.c_void_p, _F]),
        "pg_guide_forward": (st, [ctypes.c_void_p, _F, ctypes.c_int64, _F]),
        "pg_guide_gradient": (st, [ctypes.c_void_p, _F, _F, ctypes.c_int64, _F,
                                   _P(ctypes.c_double)]),
        "pg_guide_train_step": (st, [ctypes.c_void_p, _F, _F, ctypes.c_int64, ctypes.c_float,
                                     _P(ctypes.c_double)]),
        "pg_guide_encode": (None, [_F, _F, _F, ctypes.c_int64, _F]),
        "pg_guide_mixture": (None, [_F, ctypes.c_int64, _F]),
        "pg_guide_pdf": (None, [_F, _F, ctypes.c_int64, _F]),
        "pg_guide_sample": (None, [_F, _F, ctypes.c_int64, _F]),
        "pg_guide_loss_grad": (None, [_F, _F, ctypes.c_int64, _F, _F]),
        "pg_set_bvh_builder": (st, [ctypes.c_void_p, ctypes.c_int32]),
        "pg_scene_bvh_info": (st, [ctypes.c_void_p, ctypes.c_int32, _P(ctypes.c_double),
                                   _P(ctypes.c_int32), _P(ctypes.c_int64)]),
        "pg_halton_sample": (st, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                  _P(ctypes.c_int64), ctypes.c_int64, _F]),
        "pg_sobol_sample": (st, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                 _P(ctypes.c_int64), ctypes.c_int64, _F]),
        "pg_filter_table": (st, [ctypes.c_int32, _F, _F, _F]),
        "pg_eval_nodes": (st, [_P(NodeOp), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                               _F, ctypes.c_int64, _F]),
        "pg_bump_normal": (st, [_P(NodeOp), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                _F, ctypes.c_int64, _F]),
    }
    for name, (res, args) in sig.items():
        if hasattr(L, name):
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
    if hasattr(L, "pg_render_batch"):
        L.pg_render_batch.restype = st
        L.pg_render_batch.argtypes = [ctypes.c_void_p, _P(Request), ctypes.c_int32,
                                      _P(BatchResult)]
        L.pg_autotune.restype = st
        L.pg_autotune.argtypes = [ctypes.c_void_p, _P(Request), ctypes.c_int32, _P(Tuning)]
    _lib = L
    return L


def _fptr(a):
    return None if a is None else a.ctypes.data_as(_F)


GUIDE_WEIGHTS = 6 * 64 * 64
GUIDE_FEATURES = 32
GUIDE_OUTPUTS = 40


def _f32(a, cols):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, cols)


def guide_encode(pos_unit, normal, wo):
    """Features (n x 32) of path vertices; a NaN normal marks a medium vertex."""
    p, nn, w = _f32(pos_unit, 3), _f32(normal, 3), _f32(wo, 3)
    out = np.empty((p.shape[0], GUIDE_FEATURES), np.float32)
    lib().pg_guide_encode(_fptr(p), _fptr(nn), _fptr(w), p.shape[0], _fptr(out))
    return out


def guide_mixture(raw):
    """Lobes (n x 8 x 5: axis xyz, kappa, weight) of raw network outputs (n x 40)."""
    r = _f32(raw, GUIDE_OUTPUTS)
    out = np.empty((r.shape[0], 8, 5), np.float32)
    lib().pg_guide_mixture(_fptr(r), r.shape[0], _fptr(out))
    return out


def guide_pdf(raw, dirs):
    r, d = _f32(raw, GUIDE_OUTPUTS), _f32(dirs, 3)
    out = np.empty(r.shape[0], np.float32)
    lib().pg_guide_pdf(_fptr(r), _fptr(d), r.shape[0], _fptr(out))
    return out


def guide_sample(raw, u):
    r, uu = _f32(raw, GUIDE_OUTPUTS), _f32(u, 3)
    out = np.empty((r.shape[0], 3), np.float32)
    lib().pg_guide_sample(_fptr(r), _fptr(uu), r.shape[0], _fptr(out))
    return out


def guide_loss_grad(raw, dir_weight):
    """Per-sample loss -w log q(d) and its gradient with respect to the raw outputs."""
    r, dw = _f32(raw, GUIDE_OUTPUTS), _f32(dir_weight, 4)
    g = np.empty_like(r)
    loss = np.empty(r.shape[0], np.float32)
    lib().pg_guide_loss_grad(_fptr(r), _fptr(dw), r.shape[0], _fptr(g), _fptr(loss))
    return loss, g


def _node_call(name, desc, ref, math_mode, inputs, cols):
    x = _f32(inputs, cols)
    out = np.empty((x.shape[0], 3), np.float32)
    st = getattr(lib(), name)(desc.node_ops, desc.num_node_ops, int(ref), MATH_MODES[math_mode],
                              _fptr(x), x.shape[0], _fptr(out))
    if st != PG_OK:
        raise PgError(st, (lib().pg_last_error(None) or b"").decode(errors="replace"))
    return out


def pstd_math_device(ab):
    """pine's pstd math as the kernels run it in pine mode, evaluated on the GPU: rows
    (a, b) -> 12 columns (sqrt, log2, log, exp, cos, sin, tan, acos, asin, atan of a,
    atan2(a, b), pow(a, b))."""
    ab = np.ascontiguousarray(ab, np.float32).reshape(-1, 2)
    out = np.empty((ab.shape[0], 12), np.float32)
    st = lib().pg_pstd_math_device(_fptr(ab), ab.shape[0], _fptr(out))
    if st != PG_OK:
        raise PgError(st, (lib().pg_last_error(None) or b"").decode(errors="replace"))
    return out


def halton_sample(width, height, rows, scramble=True):
    """pine's Halton samples for a width x height film at rows (n x 4: pixel x, pixel y,
    sample index, dimension); n floats."""
    r = np.ascontiguousarray(rows, dtype=np.int64).reshape(-1, 4)
    out = np.empty(r.shape[0], np.float32)
    st = lib().pg_halton_sample(int(width), int(height), int(bool(scramble)),
                                r.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), r.shape[0],
                                _fptr(out))
    if st != PG_OK:
        raise PgError(st, (lib().pg_last_error(None) or b"").decode(errors="replace"))
    return out


SOBOL_RANDOMIZERS = {"none": 0, "binaryPermutate": 1, "fastOwen": 2, "Owen": 3}


def sobol_sample(width, height, rows, randomize="fastOwen"):
    """pine's Sobol samples for a width x height film at rows (n x 4: pixel x, pixel y,
    sample index, dimension) under a randomizeStrategy name; n floats."""
    r = np.ascontiguousarray(rows, dtype=np.int64).reshape(-1, 4)
    out = np.empty(r.shape[0], np.float32)
    st = lib().pg_sobol_sample(int(width), int(height), SOBOL_RANDOMIZERS[randomize],
                               r.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), r.shape[0],
                               _fptr(out))
    if st != PG_OK:
        raise PgError(st, (lib().pg_last_error(None) or b"").decode(errors="replace"))
    return out


def filter_table(kind, radius=(0.5, 0.5), params=(0.0, 0.0)):
    """The film's 16 x 16 table of filter `kind` (a FILTERS name)."""
    rad = np.asarray(radius, np.float32)
    prm = np.asarray(params, np.float32)
    out = np.empty((16, 16), np.float32)
    st = lib().pg_filter_table(FILTERS[kind], _fptr(rad), _fptr(prm), _fptr(out))
    if st != PG_OK:
        raise PgError(st, (lib().pg_last_error(None) or b"").decode(errors="replace"))
    return out


def eval_nodes(desc, ref, inputs, math_mode="pine"):
    """Node program `ref` (1-based, from a Bsdf or Material of the SceneDesc) evaluated at
    inputs (n x 8: p, n, u, v) on the host; n x 3."""
    return _node_call("pg_eval_nodes", desc, ref, math_mode, inputs, 8)


def bump_normal(desc, ref, inputs, math_mode="pine"):
    """Shading normal of bump program `ref` at inputs (n x 14: p, n, u, v, dpdu, dpdv)."""
    return _node_call("pg_bump_normal", desc, ref, math_mode, inputs, 14)


class ParsedScene:
    """A pine scene file parsed into a flattened SceneDesc (host memory owned by the
    library until close())."""

    def __init__(self, path: str):
        self._lib = lib()
        self.desc = SceneDesc()
        self._h = ctypes.c_void_p()
        st = self._lib.pg_parse_scene_file(os.path.abspath(path).encode(),
                                          ctypes.byref(self.desc), ctypes.byref(self._h))
        if st != PG_OK:
            raise PgError(st, (self._lib.pg_last_error(None) or b"").decode(errors="replace"))

    def close(self):
        if self._h:
            self._lib.pg_free_parsed_scene(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device context of libpinegpu (not thread-safe, like pg_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        self._ctx = ctypes.c_void_p()
        self._check(self._lib.pg_create(ctypes.byref(self._ctx), int(device)), global_err=True)

    def _check(self, status: int, global_err: bool = False):
        if status != PG_OK:
            msg = self._lib.pg_last_error(None if global_err else self._ctx)
            raise PgError(status, (msg or b"").decode(errors="replace"))

    def close(self):
        if self._ctx:
            self._lib.pg_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- scenes
    def upload_scene(self, desc: "SceneDesc") -> int:
        sid = ctypes.c_int32(-1)
        self._check(self._lib.pg_upload_scene(self._ctx, ctypes.byref(desc), ctypes.byref(sid)))
        return sid.value

    def load_scene(self, path: str) -> int:
        sid = ctypes.c_int32(-1)
        self._check(self._lib.pg_load_scene_file(self._ctx, os.path.abspath(path).encode(),
                                                 ctypes.byref(sid)))
        return sid.value

    def release_scene(self, scene: int):
        self._check(self._lib.pg_release_scene(self._ctx, int(scene)))

    def scene_info(self, scene: int):
        w, h, s, d = (ctypes.c_int32() for _ in range(4))
        self._check(self._lib.pg_scene_info(self._ctx, int(scene), ctypes.byref(w),
                                            ctypes.byref(h), ctypes.byref(s), ctypes.byref(d)))
        return {"width": w.value, "height": h.value, "spp": s.value, "max_depth": d.value}

    def set_bvh_builder(self, builder: str):
        """"host" (binned SAH on the host threads), "gpu" (linear BVH on the GPU) or
        "gpu_sah" (the host's binned SAH tree, built on the GPU) for later load_scene calls."""
        self._check(self._lib.pg_set_bvh_builder(self._ctx, {"host": 0, "gpu": 1, "gpu_sah": 2}[builder]))

    def bvh_info(self, scene: int):
        sec, depth, nodes = ctypes.c_double(), ctypes.c_int32(), ctypes.c_int64()
        self._check(self._lib.pg_scene_bvh_info(self._ctx, int(scene), ctypes.byref(sec),
                                                ctypes.byref(depth), ctypes.byref(nodes)))
        return {"build_seconds": sec.value, "depth": depth.value, "nodes": nodes.value}

    # ---- rendering
    def render(self, scene: int, spp: int = 0, max_depth: int = 0, seed: int = 0,
               math_mode: str = "pine", sample_offset: int = 0, accumulate: bool = False,
               guiding: bool = False, outputs: bool = True, profile: bool = False, into=None):
        """Renders one image.  ``into`` may give preallocated (mean, var, count) arrays
        (e.g. pinned host memory) to fill instead of new ones."""
        info = self.scene_info(scene)
        w, h = info["width"], info["height"]
        desc = RenderDesc(int(spp), int(max_depth), int(seed), int(sample_offset),
                          MATH_MODES[math_mode], int(bool(guiding)), int(bool(accumulate)),
                          int(bool(profile)))
        stats = RenderStats()
        mean = var = count = None
        if into is not None:
            mean, var, count = into
        elif outputs:
            mean = np.zeros((h, w, 3), np.float32)
            var = np.zeros((h, w, 3), np.float32)
            count = np.zeros((h, w), np.uint32)
        self._check(self._lib.pg_render(self._ctx, int(scene), ctypes.byref(desc), _fptr(mean),
                                        _fptr(var),
                                        None if count is None else count.ctypes.data_as(_U32),
                                        ctypes.byref(stats)))
        return {"mean": mean, "var": var, "count": count, "stats": stats.to_dict()}

    def intersect(self, scene: int, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        sid = np.empty(n, np.int32)
        pid = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        uv = np.empty((n, 2), np.float32)
        self._check(self._lib.pg_intersect(self._ctx, int(scene), _fptr(rays), n,
                                           sid.ctypes.data_as(_I32), pid.ctypes.data_as(_I32),
                                           _fptr(t), _fptr(uv)))
        return sid, pid, t, uv

    # ---- guiding network
    def guide_reset(self, seed: int = 0):
        self._check(self._lib.pg_guide_reset(self._ctx, int(seed)))

    def guide_config(self, max_guided_depth: int = 0, step_budget: int = 0):
        """Guided renders: network sampling at bounce depths below max_guided_depth, and
        at most step_budget Adam steps per network (<= 0 keeps a setting)."""
        self._check(self._lib.pg_guide_config(self._ctx, int(max_guided_depth), int(step_budget)))

    def guide_weights(self) -> np.ndarray:
        w = np.empty((6, 64, 64), np.float32)
        self._check(self._lib.pg_guide_get_weights(self._ctx, _fptr(w)))
        return w

    def set_guide_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32).reshape(6, 64, 64)
        self._check(self._lib.pg_guide_set_weights(self._ctx, _fptr(w)))

    def guide_forward(self, features) -> np.ndarray:
        f = _f32(features, GUIDE_FEATURES)
        out = np.empty((f.shape[0], GUIDE_OUTPUTS), np.float32)
        self._check(self._lib.pg_guide_forward(self._ctx, _fptr(f), f.shape[0], _fptr(out)))
        return out

    def guide_gradient(self, features, dir_weight):
        f, dw = _f32(features, GUIDE_FEATURES), _f32(dir_weight, 4)
        g = np.empty((6, 64, 64), np.float32)
        loss = ctypes.c_double()
        self._check(self._lib.pg_guide_gradient(self._ctx, _fptr(f), _fptr(dw), f.shape[0],
                                                _fptr(g), ctypes.byref(loss)))
        return g, loss.value

    def guide_train_step(self, features, dir_weight, lr: float = 1e-2) -> float:
        f, dw = _f32(features, GUIDE_FEATURES), _f32(dir_weight, 4)
        loss = ctypes.c_double()
        self._check(self._lib.pg_guide_train_step(self._ctx, _fptr(f), _fptr(dw), f.shape[0],
                                                  float(lr), ctypes.byref(loss)))
        return loss.value

    # ---- tuning and batches
    def tuning(self) -> dict:
        t = Tuning()
        self._check(self._lib.pg_get_tuning(self._ctx, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def set_tuning(self, queue_capacity: int = 1 << 23, block_size: int = 128,
                   split_shadow: int = 1, majorant_brick: int = 64, sort_queue: int = 2,
                   group_kinds: int = 2):
        t = Tuning(int(queue_capacity), int(block_size), int(split_shadow), int(majorant_brick),
                   int(sort_queue), int(group_kinds))
        self._check(self._lib.pg_set_tuning(self._ctx, ctypes.byref(t)))

    @staticmethod
    def _requests(reqs, outputs):
        arr = (Request * len(reqs))()
        outs = []
        for i, r in enumerate(reqs):
            arr[i].scene_id = int(r["scene"])
            arr[i].width = int(r.get("width", 0))
            arr[i].height = int(r.get("height", 0))
            arr[i].spp = int(r["spp"])
            arr[i].max_depth = int(r.get("max_depth", 0))
            arr[i].seed = int(r.get("seed", i))
            out = None
            if outputs:
                out = np.zeros((int(r["out_height"]), int(r["out_width"]), 3), np.float32)
                arr[i].out_mean = out.ctypes.data_as(_F)
            outs.append(out)
        return arr, outs

    def render_batch(self, reqs, outputs: bool = True):
        """Renders many requests (dicts: scene, spp, width, height, max_depth, seed) in
        graph-captured wavefronts (one wave per scene with the default tuning).  Returns per-request means, per-request completion times
        (seconds from the batch start) and the batch's device time."""
        sizes = []
        for r in reqs:
            info = self.scene_info(int(r["scene"]))
            w = int(r.get("width", 0)) or info["width"]
            h = int(r.get("height", 0)) or info["height"]
            sizes.append((w, h))
        full = [dict(r, out_width=w, out_height=h) for r, (w, h) in zip(reqs, sizes)]
        arr, outs = self._requests(full, outputs)
        times = (ctypes.c_double * len(reqs))()
        res = BatchResult(0.0, 0, ctypes.cast(times, _P(ctypes.c_double)))
        self._check(self._lib.pg_render_batch(self._ctx, arr, len(reqs), ctypes.byref(res)))
        return {"means": outs, "request_seconds": list(times), "seconds": res.seconds,
                "paths": res.paths}

    def autotune(self, reqs) -> dict:
        arr, _ = self._requests(reqs, False)
        t = Tuning()
        self._check(self._lib.pg_autotune(self._ctx, arr, len(reqs), ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}
