"""Image parity of the CUDA path tracer with pine at equal spp, and properties of
full-size renders.

Equal-spp agreement (the acceptance test): per-pixel z-scores of the GPU image against
pine's render, each side with its own per-pixel sample variance, pass |z| < 2.576 (the
99% two-sided bound) for >= 98% of pixels; relative L2 of the difference must be within
Monte Carlo error (<= 1.25x what the two variances predict), and below 1% for the volume
scene at 1024 spp.  `pine_spheres` is the reference's own scenes/spheres.txt (checkerboard,
noise and 3-D noise textures, a noise bump map, a two-layer plastic) at 128 x 36 and 512
spp, rendered by pine with its Halton sampler."""

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


@pytest.mark.parametrize("name", ["spheres", "mesh", "volume", "pine_spheres", "filtered",
                                  "randomwalk"])
@pytest.mark.parametrize("math_mode", ["pine", "fast"])
def test_equal_spp_against_reference(ctx, tmp_path, name, math_mode):
    z = golden(f"image_{name}.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    spp = _spp(z)
    r = ctx.render(sid, spp=spp, seed=17, math_mode=math_mode)
    assert r["stats"]["dropped"] == 0
    if name == "volume":  # independent stream, box filter of radius 0.5: one pixel a sample
        assert (r["count"] == spp).all()
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
    if name == "volume":
        assert rel < 0.01
    ctx.release_scene(sid)


@pytest.mark.parametrize("name", ["spheres", "mesh", "pine_spheres", "filtered", "randomwalk"])
def test_halton_renders_follow_pine_sample_by_sample(ctx, tmp_path, name):
    """Seed 0 draws pine's own Halton sequence in the order pine's PathIntegrator::Li
    draws it, so with pine's numerics the GPU traces pine's paths: pixels agree far inside
    Monte Carlo error, and filtered samples reach the same pixels."""
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
    path = scenegen.volume_scene(str(tmp_path / "v.txt"), pb.lib(), n=512, spp=4)
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
