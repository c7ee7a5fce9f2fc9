"""Image parity of the CUDA path tracer with pine at equal spp, and properties of
full-size renders.

Equal-spp agreement (the acceptance test): per-pixel z-scores of the GPU image against
pine's render, each side with its own per-pixel sample variance, pass |z| < 2.576 (the
99% two-sided bound) for >= 98% of pixels; relative L2 of the difference must be within
Monte Carlo error (<= 1.25x what the two variances predict).

The three benchmark scenes are fixtures themselves, at a reduced film with everything
else as benchmarked: `volume512` (the 512^3 cloud with the constant sky, 1024 spp),
`mesh_full` (the 1.31M-triangle icosphere, 16384 spp) and `spheres_c0` (64 spheres with
the constant environment, 131072 spp).  At those sample counts the Monte Carlo error of
the first two is below 0.7%, and the GPU image must agree with pine's to relative L2 < 1%;
so must the 64^3 `volume` fixture at 1024 spp.  In the spheres scene pine's near-specular
dielectrics (roughness 0, so GGX alpha 0.001) give rare samples of 1e9-1e11, and NaN/Inf
ones that pine drops (32 of its 170M): the pixels such a sample lands in do not converge
like 1/sqrt(spp), in pine's image or the GPU's.  `spheres_c0` is held to relative
L2 < 1% over the pixels that no single sample dominates (relative standard error below 5%
in both images; 3 of pine's 1296 pixels are out, and about 1.4% of the pixels of a GPU
render in pine's numerics).  The other fixtures' noise at their
sample counts is 2-24% (dielectric caustics, random walks), so they are held to the
z-score and MC-error bounds only.  `pine_spheres` is the reference's own scenes/spheres.txt
(checkerboard, noise and 3-D noise textures, a noise bump map, a two-layer plastic) at
128 x 36 and 512 spp, rendered by pine with its Halton sampler."""

import json
import os

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

import oracle
import pine_b200 as pb

pytestmark = pytest.mark.gpu


def zfrac(a_mean, a_var, a_n, b_mean, b_var, b_n):
    se = np.sqrt(a_var / a_n[..., None] + b_var / b_n[..., None])
    v = se > 0
    z = np.where(v, (a_mean - b_mean) / np.where(v, se, 1), 0)
    return np.mean(np.abs(z[v]) < 2.576), z[v]


def _spp(z):
    return json.loads(str(z["info"]))["spp"]


# Fixtures whose Monte Carlo error is below 1% (relative L2 of the image).
CONVERGED = {"volume", "volume512", "mesh_full"}
# Fixtures with rare samples so large that a few pixels never converge (see above).
HEAVY_TAILED = {"spheres_c0"}
# Independent sampler with a box filter of radius 0.5: every sample lands in its own pixel.
ONE_PIXEL = {"volume", "volume512", "spheres_c0", "mesh_full"}


@pytest.mark.parametrize("name", ["spheres", "mesh", "volume", "pine_spheres", "filtered",
                                  "randomwalk", "sobol", "volume512", "spheres_c0", "mesh_full"])
@pytest.mark.parametrize("math_mode", ["pine", "fast"])
def test_equal_spp_against_reference(ctx, tmp_path, name, math_mode):
    z = golden(f"image_{name}.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    spp = _spp(z)
    r = ctx.render(sid, spp=spp, seed=17, math_mode=math_mode)
    dropped = r["stats"]["dropped"]
    total = spp * r["count"].size
    # NaN/Inf samples are dropped and not counted (integrator.cpp:156-157), as pine does.
    assert dropped <= (1e-6 * total if name in HEAVY_TAILED else 0)
    if name in ONE_PIXEL:
        assert (r["count"] <= spp).all() and r["count"].sum() == total - dropped
    else:  # Film::AddSample moves a sample that rounding puts on a pixel edge
        assert abs(r["count"].sum() / z["count"].sum() - 1) < 2e-3
    g, gv = r["mean"].astype(np.float64), r["var"].astype(np.float64)
    rm, rv = z["mean"].astype(np.float64), z["var"].astype(np.float64)
    frac, zs = zfrac(g, gv, r["count"].astype(float), rm, rv, z["count"].astype(float))
    assert frac >= 0.98, f"{frac:.4f} of pixels within 99% bounds"
    assert abs(zs.mean()) < 0.1
    rel = np.linalg.norm(g - rm) / np.linalg.norm(rm)
    expected = np.sqrt(np.sum(gv / spp + rv / z["count"][..., None])) / np.linalg.norm(rm)
    assert rel <= 1.25 * expected, (rel, expected)
    if name in CONVERGED:
        assert expected < 0.01 and rel < 0.01, (rel, expected)
    if name in HEAVY_TAILED:
        rse_g = np.sqrt(gv / r["count"][..., None]) / np.maximum(np.abs(g), 1e-30)
        rse_r = np.sqrt(rv / z["count"][..., None]) / np.maximum(np.abs(rm), 1e-30)
        ok = np.all((rse_g < 0.05) & (rse_r < 0.05), axis=-1)
        assert ok.mean() > 0.97, ok.mean()
        d, ref = (g - rm)[ok], rm[ok]
        rel_ok = np.linalg.norm(d) / np.linalg.norm(ref)
        exp_ok = np.sqrt(np.sum((gv / r["count"][..., None] + rv / z["count"][..., None])[ok])) / \
            np.linalg.norm(ref)
        assert exp_ok < 0.01 and rel_ok < 0.01, (rel_ok, exp_ok, ok.mean())
    ctx.release_scene(sid)


@pytest.mark.parametrize("name", ["spheres", "mesh", "pine_spheres", "filtered", "randomwalk",
                                  "sobol"])
def test_halton_renders_follow_pine_sample_by_sample(ctx, tmp_path, name):
    """Seed 0 draws pine's own Halton (or, for `sobol`, Sobol) sequence in the order pine's
    PathIntegrator::Li draws it, so with pine's numerics the GPU traces pine's paths: pixels
    agree far inside Monte Carlo error, and filtered samples reach the same pixels."""
    z = golden(f"image_{name}.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    r = ctx.render(sid, spp=_spp(z), seed=0, math_mode="pine")
    g, ref = r["mean"].astype(np.float64), z["mean"].astype(np.float64)
    se = np.sqrt(z["var"].astype(np.float64) / z["count"][..., None])
    close = np.abs(g - ref) <= 1e-4 * np.abs(ref) + 1e-6
    tiny = np.abs(g - ref) <= 0.05 * se + 1e-6
    same_count = np.mean(r["count"] == z["count"])
    print(f"{name}: close {close.mean():.4f} within 0.05 se {tiny.mean():.4f} "
          f"same count {same_count:.4f} max |d|/se {np.max(np.abs(g - ref) / (se + 1e-9)):.3g}")
    assert same_count >= 0.99
    # The shipped scene's noise textures and bump map go through pine's float functions in
    # a different order on the device; paths that meet them drift apart within MC error.
    assert tiny.mean() >= (0.8 if name == "pine_spheres" else 0.95)
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    assert rel < 0.01
    ctx.release_scene(sid)


def test_against_restatement_other_seeds(ctx, tmp_path):
    """The C restatement at 256 spp vs the GPU on the spheres scene, new seeds."""
    z = golden("image_spheres.npz")
    path = write_fixture_scene(z, str(tmp_path))
    ref = oracle.Restatement(path)
    o = ref.render(spp=256, seed=99)
    ref.close()
    sid = ctx.load_scene(path)
    r = ctx.render(sid, spp=1024, seed=5)
    frac, _ = zfrac(r["mean"].astype(float), r["var"].astype(float), r["count"].astype(float),
                    o["mean"], o["var"], o["count"].astype(float))
    assert frac >= 0.98


def test_determinism_and_progressive_passes(ctx, tmp_path):
    z = golden("image_volume.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    a = ctx.render(sid, spp=64, seed=3)
    b = ctx.render(sid, spp=64, seed=3)
    assert np.array_equal(a["count"], b["count"])
    np.testing.assert_allclose(a["mean"], b["mean"], rtol=1e-5, atol=1e-7)
    c = ctx.render(sid, spp=64, seed=4)
    assert not np.allclose(a["mean"], c["mean"])
    # Two progressive passes of 32 spp (sample_offset) equal one pass of 64 spp.
    ctx.render(sid, spp=32, seed=3, outputs=False)
    p = ctx.render(sid, spp=32, seed=3, sample_offset=32, accumulate=True)
    assert (p["count"] == 64).all()
    np.testing.assert_allclose(p["mean"], a["mean"], rtol=1e-4, atol=1e-6)
    ctx.release_scene(sid)


def test_full_size_volume_properties(ctx, tmp_path):
    """The benchmark scene itself (512^3 grid, 1280x720), 4 spp: every pixel gets every
    sample, no NaN/Inf, radiance bounded by the brightest light path, and two seeds agree
    within their variance."""
    from pine_b200 import scenegen
    path = scenegen.volume_scene(str(tmp_path / "v.txt"), n=512, spp=4)
    sid = ctx.load_scene(path)
    a = ctx.render(sid, seed=1)
    b = ctx.render(sid, seed=2)
    assert (a["count"] == 4).all() and a["stats"]["dropped"] == 0
    assert a["stats"]["paths"] == 1280 * 720 * 4
    assert a["stats"]["volume_steps"] > 0
    for r in (a, b):
        assert np.isfinite(r["mean"]).all() and (r["mean"] >= 0).all()
    ma, mb = a["mean"].mean(), b["mean"].mean()
    se = np.sqrt(a["var"].mean() / 4 / a["mean"][..., 0].size * 3)
    assert abs(ma - mb) < 6 * se + 1e-4
    ctx.release_scene(sid)


def test_full_size_spheres_counts(ctx, tmp_path):
    from pine_b200 import scenegen
    path = scenegen.spheres_scene(str(tmp_path / "s.txt"), spp=8)
    sid = ctx.load_scene(path)
    r = ctx.render(sid)
    # A Halton scene: a sample reaches its own pixel, or also or instead a neighbour in the
    # rare case that rounding puts it on the pixel's edge (Film::AddSample, film.h:26-45).
    assert r["stats"]["dropped"] == 0
    assert abs(int(r["count"].sum()) - 640 * 360 * 8) < 640 * 360 * 8 * 1e-3
    assert r["stats"]["paths"] == 640 * 360 * 8
    ctx.release_scene(sid)


def test_compressed_volume_renders_like_its_float_grid(ctx, tmp_path):
    """A `.compressed` grid and the float grid it decodes to give the same image."""
    import struct
    from test_compressed_volume import _scene, write_compressed
    rng = np.random.default_rng(8)
    size = (24, 16, 20)
    dens = np.where(rng.uniform(size=size[::-1]) < 0.5, 0.0,
                    rng.gamma(2.0, 2.0, size[::-1])).astype(np.float32)
    grid = write_compressed(tmp_path / "v.compressed", dens, size)
    with open(tmp_path / "v.vol", "wb") as f:
        f.write(struct.pack("<3i", *size) + grid.astype(np.float32).tobytes())
    images = []
    for name in ("v.compressed", "v.vol"):
        d = tmp_path / name.replace(".", "_")
        d.mkdir()
        os.symlink(tmp_path / name, d / name)
        sid = ctx.load_scene(_scene(d, name))
        images.append(ctx.render(sid, spp=64, seed=3, math_mode="fast")["mean"])
        ctx.release_scene(sid)
    assert np.abs(images[0]).sum() > 0
    np.testing.assert_allclose(images[0], images[1], rtol=1e-5, atol=1e-7)
