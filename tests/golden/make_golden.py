"""Regenerates the golden fixtures in tests/golden/ by running the reference renderer.

The reference is pine built from its own sources by oracle/Makefile (oracle/_ref/pine_ref,
a harness that calls pine's functions; see oracle/ref_harness.cpp).  Scene inputs come
from the seeded generators in pine_b200.scenegen; everything a test needs to replay a case
(scene text, OBJ/volume assets, rays, outputs) is stored in the .npz so that the tests do
not depend on the generators or on the reference being present.

    python tests/golden/make_golden.py           # needs oracle/_ref/pine_ref
    python tests/golden/make_golden.py nodes pine_spheres sampler filtered randomwalk
    python tests/golden/make_golden.py volume512 mesh_full spheres_c0   # benchmark scenes
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.path.join(ROOT, "oracle", "_ref", "pine_ref")
REF_CONST = os.path.join(ROOT, "oracle", "_ref", "pine_ref_const")
from oracle import REFERENCE_SRC  # noqa: E402

HIT_DTYPE = np.dtype([("shape", "<i4"), ("tri", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])


def run(*args, cwd=None):
    p = subprocess.run([REF, *args], capture_output=True, text=True, cwd=cwd)
    if p.returncode != 0:
        raise RuntimeError(f"pine_ref {args[0]} failed: {p.stderr[-2000:]}")
    return p.stdout


def math_kat(tmp, rng):
    a = np.concatenate([
        np.exp(rng.uniform(-30, 30, 1024)),            # sqrt / log domain, many magnitudes
        rng.uniform(1e-4, 4.0, 512),
        rng.uniform(-20, 20, 1024),                     # cos / sin / tan / atan
        rng.uniform(-1, 1, 512),                        # acos / asin
        np.array([0.0, 1.0, -1.0, 0.5, 2.0, 1e-20, 1e20, 3.14159265, 1.5707963]),
    ]).astype(np.float32)
    b = rng.uniform(-5, 5, a.size).astype(np.float32)
    b[-9:] = [1, 1, 2, 0.5, 5, 1, 1, -1, 3]
    inp = np.stack([a, b], 1).astype(np.float32)
    inp.tofile(f"{tmp}/m.in")
    run("math", f"{tmp}/m.in", f"{tmp}/m.out")
    out = np.fromfile(f"{tmp}/m.out", np.float32).reshape(-1, 12)
    names = np.array(["sqrt", "log2", "log", "exp", "cos", "sin", "tan", "acos", "asin", "atan",
                      "atan2", "pow"])
    np.savez_compressed(f"{HERE}/pstd_math.npz", inputs=inp, outputs=out, names=names)


def stof_kat(tmp, rng):
    strs = ["0", "1", "-1", "0.5", "-0.5", "0.785398", "3.14159265", "10", "255", "1000000",
            "123456789", "0.1", "0.2", "0.3", "19.8", "0.000001", "-0.000001", ".5", "-.25",
            "1.", "5 0 0", "0 0 5", "-0.4 0.8 0.45", "1 2", "1e-5", "2.5e3", "", "  7", "abc",
            "1.5.2", "-", "12 -3.5 .75 9", "0.123456789012", "99999.999999"]
    for _ in range(600):
        x = rng.uniform(-1000, 1000) * 10.0 ** int(rng.integers(-4, 2))
        strs.append("%.*f" % (int(rng.integers(0, 8)), x))
    for _ in range(200):
        v = rng.uniform(-10, 10, 3)
        strs.append(" ".join("%.6f" % t for t in v))
    with open(f"{tmp}/s.in", "w") as f:
        f.write("\n".join(strs) + "\n")
    run("stof", f"{tmp}/s.in", f"{tmp}/s.out")
    out = np.fromfile(f"{tmp}/s.out", np.float32).reshape(-1, 4)
    np.savez_compressed(f"{HERE}/pstd_stof.npz", strings=np.array(strs, dtype=object),
                        outputs=out, allow_pickle=True)


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def bsdf_kat(tmp, rng):
    rows = []
    for i in range(3000):
        typ = i % 4
        albedo = rng.uniform(0.05, 1.0, 3)
        rough = rng.choice([0.0, 0.05, 0.2, 0.5, 0.9, 1.0]) if typ != 0 else 0.5
        eta = rng.choice([1.33, 1.5, 2.4]) if typ == 2 else (rng.uniform(-0.9, 0.9) if typ == 3 else 1.5)
        wi = unit(rng.normal(size=3))
        if typ in (1, 2) and rng.uniform() < 0.7:
            wi[2] = abs(wi[2])
        wo = unit(rng.normal(size=3))
        if rng.uniform() < 0.5:
            wo[2] = np.sign(wi[2]) * abs(wo[2])
        u1 = rng.uniform()
        u2 = rng.uniform(size=2)
        rows.append([typ, *albedo, rough, eta, *wi, *wo, u1, *u2, 0, 0, 0])
    inp = np.array(rows, np.float32)
    inp.tofile(f"{tmp}/b.in")
    run("bsdf", f"{tmp}/b.in", f"{tmp}/b.out")
    out = np.fromfile(f"{tmp}/b.out", np.float32).reshape(-1, 16)
    np.savez_compressed(f"{HERE}/bsdf.npz", inputs=inp, outputs=out)


def read_assets(paths):
    return {os.path.basename(p): open(p, "rb").read() for p in paths}


def pack_scene(scene_path, extra_assets=()):
    d = os.path.dirname(scene_path)
    assets = read_assets([os.path.join(d, a) for a in extra_assets])
    return {"scene_text": np.array(open(scene_path).read()),
            "asset_names": np.array(list(assets.keys()), dtype=object),
            "asset_blobs": np.array([np.frombuffer(v, np.uint8) for v in assets.values()],
                                    dtype=object)}


def rays_for(rng, n, lo, hi):
    o = rng.uniform(lo, hi, (n, 3))
    d = unit(rng.normal(size=(n, 3)))
    r = np.concatenate([o, d, np.zeros((n, 1)), np.full((n, 1), 3.4e38)], 1).astype(np.float32)
    return r


def hits_case(tmp, name, scene, assets, rays):
    rays.tofile(f"{tmp}/{name}.rays")
    run("hits", scene, f"{tmp}/{name}.rays", f"{tmp}/{name}.hits")
    rec = np.fromfile(f"{tmp}/{name}.hits", HIT_DTYPE)
    np.savez_compressed(f"{HERE}/hits_{name}.npz", rays=rays, hits=rec,
                        **pack_scene(scene, assets), allow_pickle=True)
    return rec


def camera_rays(rng, scene):
    n = 2048
    inp = rng.uniform(0, 1, (n, 4)).astype(np.float32)
    inp[:8, :2] = [[0, 0], [1, 1], [0.5, 0.5], [0, 1], [1, 0], [0.25, 0.75], [0.999, 0.001], [0.5, 0]]
    d = os.path.dirname(scene)
    inp.tofile(f"{d}/cam.in")
    run("camera", scene, f"{d}/cam.in", f"{d}/cam.out")
    out = np.fromfile(f"{d}/cam.out", np.float32).reshape(-1, 6)
    return inp, out


def image_case(name, scene, assets):
    d = os.path.dirname(scene)
    info = json.loads(run("render", scene, f"{d}/{name}").strip().splitlines()[-1])
    h, w = info["height"], info["width"]
    mean = np.fromfile(f"{d}/{name}_mean.f64").reshape(h, w, 3)
    var = np.fromfile(f"{d}/{name}_var.f64").reshape(h, w, 3)
    cnt = np.fromfile(f"{d}/{name}_count.i64", np.int64).reshape(h, w)
    np.savez_compressed(f"{HERE}/image_{name}.npz", mean=mean.astype(np.float32),
                        var=var.astype(np.float32), count=cnt.astype(np.int32),
                        info=np.array(json.dumps(info)), **pack_scene(scene, assets),
                        allow_pickle=True)


# Shader-node graphs in pine's syntax: every node type of CreateNode (node.cpp:33-98)
# except Texture (image files), in both evaluation modes.
NODE_GRAPHS = [
    "Checkerboard{\n input: TexCoord\n frequency: 4.0\n}",
    "MultiplyAdd{\n input: Checkerboard{\n input: Position\n frequency: 2.5\n }\n"
    " mulFactor: 0.95\n addFactor: 0.05\n}",
    "Noise{\n input: Position\n frequency: 20\n octaves: 4.0\n}",
    "Noise3D{\n input: Position\n frequency: 10\n octaves: 4\n}",
    "Multiply{\n input: Noise{\n input: Position\n frequency: 20\n octaves: 4.0\n }\n"
    " factor: 0.05\n}",
    "Decompose{\n input: Normal\n dimension: 1\n}",
    "Composite{\n inputX: Sin{\n input: Decompose{\n input: Position\n dimension: 0\n }\n }\n"
    " inputY: Cos{\n input: Decompose{\n input: Position\n dimension: 2\n }\n }\n"
    " inputZ: Tan{\n input: 0.3\n }\n}",
    "Length{\n input: Position\n}",
    "Sqrt{\n input: Add{\n input: Sqr{\n input: Position\n }\n factor: 1.0\n }\n}",
    "Pow{\n input: Fract{\n input: Position\n }\n exp: 2.2\n}",
    "Divide{\n input: Substract{\n input: TexCoord\n factor: 0.25\n }\n factor: 3.0\n}",
    "Invert{\n input: Constant{\n float: 0.25\n vec3: 0.1 0.2 0.3\n }\n}",
    "Add{\n input: Position\n factor: Normal\n}",
    "Noise3D{\n input: Multiply{\n input: TexCoord\n factor: 3.0\n }\n frequency: 2.7\n"
    " octaves: 2.9\n}",
]
BUMP_GRAPH = ("Multiply{\n input: Noise{\n input: Position\n frequency: 20\n octaves: 4.0\n }\n"
              " factor: 0.05\n}")


def nodes_kat(tmp):
    rng = np.random.default_rng(777)
    n = 512
    p = np.concatenate([rng.uniform(-3, 3, (n // 2, 3)), rng.uniform(-0.2, 1.2, (n // 2, 3))])
    nn = unit(rng.normal(size=(n, 3)))
    uv = rng.uniform(-0.5, 1.5, (n, 2))
    inp = np.concatenate([p, nn, uv], axis=1).astype(np.float32)
    inp.tofile(f"{tmp}/n.in")
    with open(f"{tmp}/graphs.txt", "w") as f:
        for k, g in enumerate(NODE_GRAPHS):
            f.write(f"g{k}: {g}\n")
    run("nodes", f"{tmp}/graphs.txt", f"{tmp}/n.in", f"{tmp}/n.out")
    out = np.fromfile(f"{tmp}/n.out", np.float32).reshape(len(NODE_GRAPHS), n, 4)
    # Bump normals at random tangent frames.
    du = rng.normal(size=(n, 3))
    dv = rng.normal(size=(n, 3))
    binp = np.concatenate([p, nn, uv, du, dv], axis=1).astype(np.float32)
    binp.tofile(f"{tmp}/b.in")
    with open(f"{tmp}/bump.txt", "w") as f:
        f.write(f"g0: {BUMP_GRAPH}\n")
    run("bump", f"{tmp}/bump.txt", f"{tmp}/b.in", f"{tmp}/b.out")
    bout = np.fromfile(f"{tmp}/b.out", np.float32).reshape(n, 3)
    np.savez_compressed(f"{HERE}/nodes.npz", graphs=np.array(NODE_GRAPHS, dtype=object),
                        inputs=inp, float_out=out[:, :, 0], vec3_out=out[:, :, 1:],
                        bump_graph=np.array(BUMP_GRAPH), bump_inputs=binp, bump_out=bout,
                        allow_pickle=True)


HALTON_FILMS = [(48, 27), (128, 36), (1280, 360), (7, 5), (1, 1), (300, 200)]
FILTER_BLOCKS = [
    "",  # no filter block: pine's default LanczosSinc of radius 0.5
    "filter: Box{\n radius: 0.5\n}",
    "filter: Box{\n radius: 1.5 0.75\n}",
    "filter: Triangle{\n radius: 1 0.7\n}",
    "filter: Gaussian{\n radius: 1.5\n alpha: 2\n}",
    "filter: Mitchell{\n radius: 2\n}",
    "filter: Mitchell{\n radius: 1.5 1.25\n B: 0\n C: 0.5\n}",
    "filter: LanczosSinc{\n radius: 0.5\n}",
    "filter: LanczosSinc{\n radius: 2 1.5\n tau: 2\n}",
]


def sampler_filter_kat(tmp):
    """pine's HaltonSampler values at random (pixel, sample, dimension) rows for several
    film sizes and both randomize strategies, and the film's filter tables."""
    rng = np.random.default_rng(4242)
    rows_all, vals_all, meta = [], [], []
    for (w, h) in HALTON_FILMS:
        for strat in ("permutateDigits", "none"):
            n = 768
            rows = np.stack([rng.integers(0, w, n), rng.integers(0, h, n),
                             rng.integers(0, 4096, n), rng.integers(2, 1000, n)], 1)
            rows[:64, 3] = np.arange(2, 66)
            rows[64:80, 2] = rng.integers(150000, 300000, 16)  # indices above 2^32
            rows[80:84, 3] = 999
            rows = rows.astype(np.int64)
            rows.tofile(f"{tmp}/h.in")
            run("halton", str(w), str(h), strat, f"{tmp}/h.in", f"{tmp}/h.out")
            rows_all.append(rows)
            vals_all.append(np.fromfile(f"{tmp}/h.out", np.float32))
            meta.append((w, h, 1 if strat == "permutateDigits" else 0))
    tables = []
    for block in FILTER_BLOCKS:
        with open(f"{tmp}/f.txt", "w") as f:
            f.write("Camera: ThinLen{\n film{\n size: 8 8\n " + block + "\n }\n}\n")
        run("filter", f"{tmp}/f.txt", f"{tmp}/f.out")
        tables.append(np.fromfile(f"{tmp}/f.out", np.float32))
    np.savez_compressed(f"{HERE}/sampler_filter.npz", halton_meta=np.array(meta, np.int32),
                        halton_rows=np.stack(rows_all), halton_values=np.stack(vals_all),
                        filter_blocks=np.array(FILTER_BLOCKS, dtype=object),
                        filter_tables=np.stack(tables), allow_pickle=True)


SOBOL_FILMS = [(48, 27), (128, 36), (1280, 720), (7, 5), (1, 1), (1920, 1080)]
SOBOL_STRATEGIES = ["none", "binaryPermutate", "fastOwen", "Owen"]


def sobol_kat(tmp):
    """pine's SobolSampler values at random (pixel, sample, dimension) rows for several film
    sizes and every randomize strategy (sobol.npz)."""
    rng = np.random.default_rng(5151)
    rows_all, vals_all, meta = [], [], []
    for (w, h) in SOBOL_FILMS:
        for k, strat in enumerate(SOBOL_STRATEGIES):
            n = 512
            rows = np.stack([rng.integers(0, w, n), rng.integers(0, h, n),
                             rng.integers(0, 4096, n), rng.integers(2, 1024, n)], 1)
            rows[:64, 3] = np.arange(2, 66)
            rows[64:80, 2] = rng.integers(1 << 16, 1 << 20, 16)  # many samples per pixel
            rows[80:84, 3] = 1023
            rows[84:88, 2] = 0
            if w * h > 4096:  # keep the frame within the resolution's table row
                rows[64:80, 2] = rng.integers(4096, 1 << 14, 16)
            rows = rows.astype(np.int64)
            rows.tofile(f"{tmp}/s.in")
            run("sobol", str(w), str(h), strat, f"{tmp}/s.in", f"{tmp}/s.out")
            rows_all.append(rows)
            vals_all.append(np.fromfile(f"{tmp}/s.out", np.float32))
            meta.append((w, h, k))
    np.savez_compressed(f"{HERE}/sobol.npz", meta=np.array(meta, np.int32),
                        strategies=np.array(SOBOL_STRATEGIES), rows=np.stack(rows_all),
                        values=np.stack(vals_all))


def sobol_case(tmp):
    """The spheres fixture's scene with pine's Sobol sampler (fastOwen, the default) at 1024
    spp: the GPU draws pine's sequence in pine's order, so its image follows pine's sample
    by sample."""
    z = np.load(f"{HERE}/image_spheres.npz", allow_pickle=True)
    text = str(z["scene_text"])
    assert "sampler: Halton{" in text
    text = text.replace("sampler: Halton{", "sampler: Sobol{", 1)
    path = f"{tmp}/sobol.txt"
    with open(path, "w") as f:
        f.write(text)
    image_case("sobol", path, [])


def filtered_case(tmp):
    """The spheres fixture's scene with a wide Gaussian filter (samples reach up to four
    pixels) at 256 spp."""
    z = np.load(f"{HERE}/image_spheres.npz", allow_pickle=True)
    text = str(z["scene_text"])
    old = "filter: Box{\n            radius: 0.5\n        }"
    assert old in text
    text = text.replace(old, "filter: Gaussian{\n            radius: 1.5\n            alpha: 2\n        }")
    text = text.replace("samplesPerPixel: 1024", "samplesPerPixel: 256")
    assert "samplesPerPixel: 256" in text
    path = f"{tmp}/filtered.txt"
    with open(path, "w") as f:
        f.write(text)
    image_case("filtered", path, [])


def randomwalk_case(tmp):
    """The spheres fixture's scene rendered by pine's RandomWalk integrator at 512 spp."""
    z = np.load(f"{HERE}/image_spheres.npz", allow_pickle=True)
    text = str(z["scene_text"])
    assert text.startswith("Integrator: Path{")
    text = text.replace("Integrator: Path{", "Integrator: RandomWalk{", 1)
    text = text.replace("samplesPerPixel: 1024", "samplesPerPixel: 512")
    assert "samplesPerPixel: 512" in text
    path = f"{tmp}/randomwalk.txt"
    with open(path, "w") as f:
        f.write(text)
    image_case("randomwalk", path, [])


def shipped_spheres_case(tmp):
    """pine's own scenes/spheres.txt (textures, noise, bump map, two-layer plastic) at a
    tenth of its film size and 512 spp."""
    src = os.path.join(REFERENCE_SRC, "scenes", "spheres.txt")
    text = open(src).read()
    text = text.replace("size: 1280 360", "size: 128 36").replace("samplesPerPixel: 32",
                                                                 "samplesPerPixel: 512")
    assert "size: 128 36" in text and "samplesPerPixel: 512" in text
    path = f"{tmp}/pine_spheres.txt"
    with open(path, "w") as f:
        f.write(text)
    image_case("pine_spheres", path, [])


def sha256(path):
    import hashlib
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 22), b""):
            h.update(chunk)
    return h.hexdigest()


def image_case_generated(name, scene, assets, generated, binary=REF):
    """image_case for scenes whose large assets are too big to store: the fixture keeps the
    generator's arguments and each file's SHA-256 (`generated`: {file: [args...]}), and
    tests/conftest.py regenerates and checks them."""
    d = os.path.dirname(scene)
    p = subprocess.run([binary, "render", scene, f"{d}/{name}"], capture_output=True, text=True,
                       cwd=d)
    if p.returncode != 0:
        raise RuntimeError(f"{os.path.basename(binary)} render failed: {p.stderr[-2000:]}")
    info = json.loads(p.stdout.strip().splitlines()[-1])
    h, w = info["height"], info["width"]
    mean = np.fromfile(f"{d}/{name}_mean.f64").reshape(h, w, 3)
    var = np.fromfile(f"{d}/{name}_var.f64").reshape(h, w, 3)
    cnt = np.fromfile(f"{d}/{name}_count.i64", np.int64).reshape(h, w)
    gen = {f: {"args": a, "sha256": sha256(os.path.join(d, f))} for f, a in generated.items()}
    info["reference_binary"] = os.path.basename(binary)
    np.savez_compressed(f"{HERE}/image_{name}.npz", mean=mean.astype(np.float32),
                        var=var.astype(np.float32), count=cnt.astype(np.int32),
                        info=np.array(json.dumps(info)), generated=np.array(json.dumps(gen)),
                        **pack_scene(scene, assets), allow_pickle=True)


def volume512_case(tmp):
    """The volume benchmark scene itself (512^3 cloud, constant sky 0.3, sun 5, max 128
    events) at 128 x 72 and 1024 spp, rendered by pine with the added Constant environment
    (oracle/_ref/pine_ref_const).  The 512 MiB grid is stored as its generator arguments
    and hash."""
    from pine_b200 import scenegen
    vs = scenegen.volume_scene(f"{tmp}/volume512.txt", n=512, width=128, height=72, spp=1024,
                               env="constant", env_radiance=0.3)
    image_case_generated("volume512", vs, [], {"cloud512_s0.vol": ["cloud", 512, 0, "0.3"]},
                         binary=REF_CONST)


def mesh_full_case(tmp, spp=16384):
    """The mesh benchmark scene itself (1,310,720-triangle displaced icosphere in the
    12-triangle box, max depth 16, independent sampler) at 48 x 27, rendered by pine (its
    full-sweep SAH build of this mesh takes about 13 minutes on one host thread).  16384 spp
    bring the Monte Carlo error of the image to about 0.6% (relative L2).  The OBJ is
    stored as its generator arguments and hash."""
    from pine_b200 import scenegen
    ms = scenegen.mesh_scene(f"{tmp}/mesh_full.txt", subdiv=8, width=48, height=27, spp=spp,
                             max_depth=16, sampler="Uniform")
    image_case_generated("mesh_full", ms, ["cornell.obj"],
                         {"ico8_s0.obj": ["icosphere", 8, "1.2", "0.0", "1.6", "0.5", "0.1", 0,
                                          ]})


def spheres_c0_case(tmp, spp=131072):
    """The spheres benchmark scene itself (64 seeded spheres, plane, rect light, constant
    environment 0.2, max depth 8, independent sampler) at 48 x 27, rendered by pine with the
    added Constant environment.  The dielectric spheres' caustics make the image noisy:
    131072 spp bring its Monte Carlo error to about 0.7% (relative L2)."""
    from pine_b200 import scenegen
    sp = scenegen.spheres_scene(f"{tmp}/spheres_c0.txt", width=48, height=27, spp=spp,
                                max_depth=8, env="constant", env_radiance=0.2,
                                sampler="Uniform")
    image_case_generated("spheres_c0", sp, [], {}, binary=REF_CONST)


def main():
    if not os.path.exists(REF):
        sys.exit("oracle/_ref/pine_ref is missing: run `make -C oracle ref` first")
    only = set(sys.argv[1:])
    if only:
        with tempfile.TemporaryDirectory() as tmp:
            if "nodes" in only:
                nodes_kat(tmp)
            if "sampler" in only:
                sampler_filter_kat(tmp)
            if "filtered" in only:
                filtered_case(tmp)
            if "sobol" in only:
                sobol_kat(tmp)
                sobol_case(tmp)
            if "randomwalk" in only:
                randomwalk_case(tmp)
            if "pine_spheres" in only:
                shipped_spheres_case(tmp)
            if "volume512" in only:
                volume512_case(tmp)
            if "mesh_full" in only:
                mesh_full_case(tmp)
            if "spheres_c0" in only:
                spheres_c0_case(tmp)
        print("fixtures written to", HERE)
        return
    from pine_b200 import scenegen
    rng = np.random.default_rng(20261203)
    with tempfile.TemporaryDirectory() as tmp:
        math_kat(tmp, rng)
        stof_kat(tmp, rng)
        bsdf_kat(tmp, rng)

        # Spheres (pine Sky in place of the constant environment pine lacks).
        sp = scenegen.spheres_scene(f"{tmp}/spheres.txt", width=48, height=27, spp=1024,
                                    env="sky", env_radiance=0.5)
        hits_case(tmp, "spheres", sp, [], rays_for(rng, 8000, [-6, 0.5, -6], [6, 5, 6]))
        cam_in, cam_out = camera_rays(rng, sp)
        np.savez_compressed(f"{HERE}/camera.npz", inputs=cam_in, outputs=cam_out,
                            **pack_scene(sp), allow_pickle=True)
        image_case("spheres", sp, [])

        # Mesh: 5120-triangle displaced icosphere in the 12-triangle box.
        ms = scenegen.mesh_scene(f"{tmp}/mesh.txt", subdiv=4, width=48, height=27,
                                 spp=512, max_depth=16)
        mesh_assets = ["ico4_s0.obj", "cornell.obj"]
        # Rays from inside the box toward the sphere and walls, and from the camera side.
        r1 = rays_for(rng, 6000, [-2.8, 0.2, -2.8], [2.8, 5.8, 2.8])
        r2 = rays_for(rng, 2000, [-6, 1, -12], [6, 5, -6])
        hits_case(tmp, "mesh", ms, mesh_assets, np.concatenate([r1, r2]))
        image_case("mesh", ms, mesh_assets)

        # Volume: 32^3 cloud for density lookups, 64^3 for the image.
        vs = scenegen.volume_scene(f"{tmp}/vol32.txt", n=32, width=16, height=9, spp=1,
                                   env="sky", env_radiance=1.0)
        pts = np.concatenate([rng.uniform(-0.05, 1.05, (3000, 3)),
                              rng.integers(0, 33, (200, 3)) / 32.0]).astype(np.float32)
        pts.tofile(f"{tmp}/p.in")
        run("density", vs, f"{tmp}/p.in", f"{tmp}/p.out")
        dens = np.fromfile(f"{tmp}/p.out", np.float32)
        np.savez_compressed(f"{HERE}/density.npz", points=pts, density=dens,
                            **pack_scene(vs, ["cloud32_s0.vol"]), allow_pickle=True)
        vi = scenegen.volume_scene(f"{tmp}/volume.txt", n=64, width=48, height=27,
                                   spp=1024, env="sky", env_radiance=1.0)
        image_case("volume", vi, ["cloud64_s0.vol"])
        nodes_kat(tmp)
        shipped_spheres_case(tmp)
        sampler_filter_kat(tmp)
        filtered_case(tmp)
        randomwalk_case(tmp)
        sobol_kat(tmp)
        sobol_case(tmp)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
