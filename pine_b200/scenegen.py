"""Seeded synthetic scenes written in pine's scene-file format.

Every number is written as a plain decimal: pine's parser reads numbers with
``pstd::stof`` (src/pstd/string.cpp:50-68), which has no exponent support, and the
OBJ loader uses the same routine (src/util/objloader.cpp:31).

Scenes (sizes are the defaults; tests shrink them):

* ``spheres``: 64 seeded spheres (centres U([-5,5]x[0,3]x[-5,5]), radius U(0.2, 1)),
  materials split into thirds Lambertian / GGX conductor / dielectric (IOR 1.5), a
  diffuse ground plane, one rectangular area light (radiance 10) and an environment.
* ``mesh``: a noise-displaced icosphere (20*4^subdiv triangles) inside a 12-triangle
  Cornell-style box with a ceiling area light; diffuse and GGX conductor materials.
* ``volume``: an n^3 fractal-noise cloud (about 30% of voxels non-zero, max density 1,
  sigma_a 0.2 + sigma_s 19.8 = sigma_t 20), HG g = 0.8, lit by a directional sun
  (irradiance 5) plus an environment; the camera is attached to the medium as in pine's
  cloud scene and frames the cloud (about 80% of the pixels see non-zero density).

The environment is ``constant`` (uniform radiance, ``Environment{ environment:
Constant{ color } }``), ``sky`` (pine's ``Sky``) or ``none``.

The grids and meshes come from the ``pine-scenegen`` tool (csrc/scenegen.cpp, built by
:func:`pine_b200.build.build`), a separate executable, so generating a scene loads no part
of the renderer library.
"""

from __future__ import annotations

import json
import os
import subprocess

import numpy as np

from . import build as _build


def _scenegen(*args) -> dict:
    exe = _build.SCENEGEN
    if not os.path.exists(exe):
        exe = _build.build_scenegen()
    p = subprocess.run([exe, *[str(a) for a in args]], capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"pine-scenegen {args[0]} failed: {p.stderr.strip()}")
    return json.loads(p.stdout.strip().splitlines()[-1])


def gen_cloud_volume(path: str, n: int, seed: int = 0, nonzero_fraction: float = 0.3) -> str:
    """Writes the seeded n^3 fractal-noise cloud (pine's .vol format) to `path`."""
    _scenegen("cloud", int(n), int(seed), repr(float(nonzero_fraction)), path)
    return path


def gen_icosphere_obj(path: str, subdiv: int, radius=1.2, center=(0.0, 1.6, 0.5),
                      amplitude=0.1, seed: int = 0) -> int:
    """Writes the seeded noise-displaced icosphere as OBJ; returns its triangle count."""
    r = _scenegen("icosphere", int(subdiv), repr(float(radius)), *[repr(float(c)) for c in center],
                  repr(float(amplitude)), int(seed), path)
    return int(r["triangles"])


def _f(x: float) -> str:
    s = "%.6f" % float(x)
    if s.startswith("-") and float(s) == 0.0:
        s = s[1:]
    return s


def _v(*xs) -> str:
    return " ".join(_f(x) for x in xs)


def _env_block(env: str, radiance: float, sun_dir=(-0.4, 0.8, 0.45)) -> str:
    if env == "constant":
        return ("Light: Environment{\n    environment: Constant{\n"
                f"        color: {_f(radiance)}\n    }}\n}}\n")
    if env == "sky":
        # pine's Sky: gradient sky scaled by sunColor plus a delta sun (light.cpp:65-79).
        return ("Light: Environment{\n    environment: Sky{\n"
                f"        sunDirection: {_v(*sun_dir)}\n        sunColor: {_f(radiance)}\n"
                "    }\n}\n")
    if env == "none":
        return ""
    raise ValueError(f"unknown environment {env!r}")


def _header(max_depth: int, spp: int, sampler: str, width: int, height: int,
            cam_from, cam_to, fov: float, camera_medium: str | None = None) -> str:
    med = f"    medium: {camera_medium}\n" if camera_medium else ""
    return (
        "Integrator: Path{\n"
        f"    maxDepth: {int(max_depth)}\n"
        f"    sampler: {sampler}{{\n        samplesPerPixel: {int(spp)}\n    }}\n"
        "}\n\n"
        "Camera: ThinLen{\n"
        "    film{\n"
        f"        size: {int(width)} {int(height)}\n"
        "        filter: Box{\n            radius: 0.5\n        }\n"
        "        outputFileName: image.bmp\n"
        "    }\n"
        f"    from: {_v(*cam_from)}\n"
        f"    to: {_v(*cam_to)}\n"
        f"    fov: {_f(fov)}\n"
        f"{med}"
        "}\n\n")


def spheres_scene(path: str, *, width=640, height=360, spp=64, max_depth=8, seed=0,
                  n_spheres=64, env="constant", env_radiance=0.2, light_radiance=10.0,
                  sampler="Halton") -> str:
    rng = np.random.default_rng(seed)
    out = [_header(max_depth, spp, sampler, width, height, (0.0, 6.0, -15.0),
                   (0.0, 1.0, 0.0), 0.785398)]
    out.append("Shape: Plane{\n    position: 0 0 0\n    normal: 0 1 0\n"
               "    material: ground\n}\n")
    out.append("Shape: Rect{\n    position: 0 9 0\n    ex: 5 0 0\n    ey: 0 0 5\n"
               "    material: light\n}\n")
    mats = ["Material ground: Layered{\n    layer0: Diffuse{\n        albedo: 0.5\n    }\n}\n",
            f"Material light: Emissive{{\n    color: {_f(light_radiance)}\n}}\n"]
    for i in range(n_spheres):
        c = rng.uniform([-5.0, 0.0, -5.0], [5.0, 3.0, 5.0])
        r = rng.uniform(0.2, 1.0)
        kind = i % 3
        if kind == 0:
            a = rng.uniform(0.1, 0.9, 3)
            body = f"    layer0: Diffuse{{\n        albedo: {_v(*a)}\n    }}\n"
        elif kind == 1:
            rough = rng.uniform(0.05, 0.5)
            body = ("    layer0: Conductor{\n        albedo: 0.9\n"
                    f"        roughness: {_f(rough)}\n    }}\n")
        else:
            body = ("    layer0: Dielectric{\n        roughness: 0.0\n"
                    "        eta: 1.5\n    }\n")
        mats.append(f"Material m{i}: Layered{{\n{body}}}\n")
        out.append(f"Shape: Sphere{{\n    position: {_v(*c)}\n    radius: {_f(r)}\n"
                   f"    material: m{i}\n}}\n")
    out.extend(mats)
    out.append(_env_block(env, env_radiance))
    text = "\n".join(out)
    with open(path, "w") as f:
        f.write(text)
    return path


def cornell_box_obj(path: str, half=3.0, height=6.0) -> str:
    """Five walls (floor, ceiling, back, left, right) plus a lintel strip across the
    open front, two triangles each: 12 triangles."""
    h, y = half, height
    v = [(-h, 0, -h), (h, 0, -h), (h, 0, h), (-h, 0, h),          # floor 1..4
         (-h, y, -h), (h, y, -h), (h, y, h), (-h, y, h),          # ceiling 5..8
         (-h, y - 0.6, -h), (h, y - 0.6, -h)]                     # lintel bottom 9..10
    f = [(1, 2, 3), (1, 3, 4),        # floor (z = +h is the back)
         (5, 7, 6), (5, 8, 7),        # ceiling
         (4, 3, 7), (4, 7, 8),        # back wall z = +h
         (1, 4, 8), (1, 8, 5),        # left wall x = -h
         (2, 6, 7), (2, 7, 3),        # right wall x = +h
         (9, 10, 6), (9, 6, 5)]       # lintel at the open front z = -h
    with open(path, "w") as fh:
        for p in v:
            fh.write("v " + _v(*p) + "\n")
        for t in f:
            fh.write("f %d %d %d\n" % t)
    return path


def mesh_scene(path: str, *, subdiv=8, width=1920, height=1080, spp=256, max_depth=16,
               seed=0, env="none", env_radiance=0.2, sampler="Halton",
               obj_name=None) -> str:
    d = os.path.dirname(os.path.abspath(path))
    obj = obj_name or f"ico{subdiv}_s{seed}.obj"
    obj_path = os.path.join(d, obj)
    if not os.path.exists(obj_path):
        gen_icosphere_obj(obj_path + ".tmp", subdiv, seed=seed)
        os.replace(obj_path + ".tmp", obj_path)
    cornell_box_obj(os.path.join(d, "cornell.obj"))
    rng = np.random.default_rng(seed + 1)
    rough_obj = rng.uniform(0.1, 0.6)
    out = [_header(max_depth, spp, sampler, width, height, (0.0, 3.0, -11.0),
                   (0.0, 2.6, 0.0), 0.6)]
    out.append(f"Shape: TriangleMesh{{\n    file: {obj}\n    material: metal\n}}\n")
    out.append("Shape: TriangleMesh{\n    file: cornell.obj\n    material: walls\n}\n")
    out.append("Shape: Rect{\n    position: 0 5.99 0.5\n    ex: 2 0 0\n    ey: 0 0 2\n"
               "    material: light\n}\n")
    out.append("Material walls: Layered{\n    layer0: Diffuse{\n        albedo: 0.7 0.65 0.6\n"
               "    }\n}\n")
    out.append("Material metal: Layered{\n    layer0: Conductor{\n        albedo: 0.95 0.7 0.4\n"
               f"        roughness: {_f(rough_obj)}\n    }}\n}}\n")
    out.append("Material light: Emissive{\n    color: 12\n}\n")
    out.append(_env_block(env, env_radiance))
    with open(path, "w") as f:
        f.write("\n".join(out))
    return path


def volume_scene(path: str, *, n=512, width=1280, height=720, spp=256, max_depth=128,
                 seed=0, env="constant", env_radiance=0.3, sun_irradiance=5.0,
                 sampler="Uniform", vol_name=None, sigma_a=0.2, sigma_s=19.8, g=0.8) -> str:
    d = os.path.dirname(os.path.abspath(path))
    vol = vol_name or f"cloud{n}_s{seed}.vol"
    vol_path = os.path.join(d, vol)
    if not os.path.exists(vol_path):
        gen_cloud_volume(vol_path + ".tmp", n, seed)
        os.replace(vol_path + ".tmp", vol_path)
    sun = (-0.4, 0.8, 0.45)
    # The camera sits just outside the grid's box and frames the cloud: about 80% of the
    # pixels of a 16:9 film look through non-zero density.
    out = [_header(max_depth, spp, sampler, width, height, (0.0, 0.05, -0.8),
                   (0.0, 0.0, 0.0), 0.75, camera_medium="cloud")]
    out.append("Medium cloud: Grid{\n"
               f"    file: {vol}\n    sigma_a: {_f(sigma_a)}\n    sigma_s: {_f(sigma_s)}\n"
               f"    g: {_f(g)}\n    position: 0 0 0\n    scale: 1\n}}\n")
    out.append(f"Light: Directional{{\n    direction: {_v(*sun)}\n"
               f"    color: {_f(sun_irradiance)}\n}}\n")
    out.append(_env_block(env, env_radiance, sun_dir=sun))
    with open(path, "w") as f:
        f.write("\n".join(out))
    return path
