"""Pins the C restatement (oracle/pine_oracle.c) to the reference: every golden fixture
here was produced by running pine itself (tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

import oracle

BITEXACT = ["sqrt", "log2", "log", "pow"]


def test_pstd_math_against_reference():
    z = golden("pstd_math.npz")
    inp, out = z["inputs"], z["outputs"]
    a, b = inp[:, 0], inp[:, 1]
    for k, name in enumerate(oracle.MATH_NAMES):
        r = oracle.math(name, a, b)
        ref = out[:, k]
        if name in BITEXACT:
            same = (r.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(r) & np.isnan(ref))
            assert same.all(), f"pstd::{name} differs on {np.count_nonzero(~same)} inputs"
            continue
        # pine's -ffast-math build multiplies by reciprocals of the Taylor constants, so
        # the restatement (strict IEEE) agrees to ~1 ulp in each function's well
        # conditioned domain.
        if name in ("cos", "sin", "exp"):
            dom = np.abs(a) <= 20
        elif name == "tan":
            dom = (np.abs(a) <= 20) & (np.abs(np.cos(a)) > 0.1)
        elif name in ("acos", "asin"):
            dom = np.abs(a) <= 1
        elif name == "atan":
            dom = np.abs(a) <= 4
        else:
            dom = (np.abs(a) <= 4) & (np.abs(b) > 0.25)
        d = np.abs(r.astype(np.float64) - ref) / np.maximum(1.0, np.abs(ref))
        assert np.nanmax(d[dom]) < (1e-5 if name == "tan" else 2e-6), name


def test_stof_against_reference():
    z = golden("pstd_stof.npz")
    for s, o in zip(z["strings"], z["outputs"]):
        v = np.float32(oracle.stof(str(s)))
        assert v.view(np.uint32) == o[0].view(np.uint32), repr(s)
        assert np.array_equal(oracle.stofs(str(s)).view(np.uint32), o[1:4].view(np.uint32)), repr(s)


def test_bsdf_and_phase_against_reference():
    z = golden("bsdf.npz")
    inp, ref = z["inputs"], z["outputs"]
    out = oracle.bsdf(inp)
    # Evaluation (F, PDF): relative 1e-4 (fast-math reassociation in pine's build).
    scale = np.maximum(np.abs(ref[:, :4]), 1e-3)
    assert np.all(np.abs(out[:, :4] - ref[:, :4]) / scale < 1e-3)
    both = (out[:, 4] == 1) & (ref[:, 4] == 1)
    # The sampled/rejected decision matches except for borderline cases.
    assert np.mean(out[:, 4] == ref[:, 4]) > 0.995
    assert np.all(np.abs(out[both, 5:8] - ref[both, 5:8]) < 1e-4)
    # Sampled f and pdf: for near-specular lobes (roughness < 0.1, alpha down to 0.001)
    # both swing with the last ulp of the half vector, so compare their ratio, the sample
    # weight the estimator uses; otherwise compare each.
    rough = inp[both, 4] >= 0.1
    f, pdf, rf, rpdf = out[both, 8:11], out[both, 11:12], ref[both, 8:11], ref[both, 11:12]
    fs = np.maximum(np.abs(ref[both, 8:12]), 1e-2)
    close = np.all(np.abs(out[both, 8:12] - ref[both, 8:12]) / fs < 1e-3, axis=1)
    assert np.mean(close[rough]) > 0.99
    w, rw = f / pdf, rf / rpdf
    assert np.all(np.abs(w - rw) <= 1e-3 * np.maximum(np.abs(rw), 1e-2))


def test_camera_and_density_against_reference(tmp_path):
    z = golden("camera.npz")
    s = oracle.Restatement(write_fixture_scene(z, str(tmp_path / "cam")))
    for (fx, fy, l0, l1), ref in zip(z["inputs"], z["outputs"]):
        np.testing.assert_allclose(s.camera_ray(fx, fy, l0, l1), ref, atol=2e-6)
    s.close()
    z = golden("density.npz")
    s = oracle.Restatement(write_fixture_scene(z, str(tmp_path / "vol")))
    d = s.density(0, z["points"])
    np.testing.assert_allclose(d, z["density"], atol=2e-6)
    s.close()


@pytest.mark.parametrize("name", ["spheres", "mesh"])
def test_nearest_hits_against_reference(tmp_path, name):
    z = golden(f"hits_{name}.npz")
    s = oracle.Restatement(write_fixture_scene(z, str(tmp_path)))
    shape, prim, t, amb = s.intersect(z["rays"])
    h = z["hits"]
    ok = amb | ((shape == h["shape"]) & (prim == h["tri"]))
    assert ok.all(), f"{np.count_nonzero(~ok)} rays disagree with pine's BVH"
    hit = (h["shape"] >= 0) & ~amb
    assert hit.sum() > 1000
    # Hit distances: bit-exact (the restatement evaluates pine's compiled order).
    assert np.array_equal(t[hit].view(np.uint32), h["t"][hit].view(np.uint32))
    s.close()


def block_stats(mean, var, n, b):
    """Per-block mean and variance-of-the-mean over b x b pixel blocks."""
    h, w = mean.shape[0] // b * b, mean.shape[1] // b * b
    m = mean[:h, :w].reshape(h // b, b, w // b, b, 3).mean(axis=(1, 3))
    v = (var[:h, :w] / n[:h, :w, None]).reshape(h // b, b, w // b, b, 3).sum(axis=(1, 3)) / (b * b) ** 2
    return m, v


def zscore_check(mean, var, n, ref_mean, ref_var, ref_n, frac_min=0.98, block=1):
    """Fraction of pixels (or b x b blocks) whose difference from the reference is within
    2.576 standard errors, using both sides' per-pixel sample variances."""
    m, v = block_stats(mean, var, n, block)
    rm, rv = block_stats(ref_mean, ref_var, ref_n, block)
    se = np.sqrt(v + rv)
    valid = se > 0
    z = np.where(valid, (m - rm) / np.where(valid, se, 1), 0.0)
    frac = np.mean(np.abs(z[valid]) < 2.576) if valid.any() else 1.0
    # Pixels with zero variance on both sides are deterministic and must match.
    assert np.allclose(m[~valid], rm[~valid], atol=1e-5)
    assert frac >= frac_min, f"only {frac:.4f} of pixels pass |z| < 2.576"
    return frac


@pytest.mark.parametrize("name,spp,block", [("spheres", 256, 1), ("volume", 256, 1),
                                             ("mesh", 64, 3)])
def test_render_against_reference(tmp_path, name, spp, block):
    z = golden(f"image_{name}.npz")
    s = oracle.Restatement(write_fixture_scene(z, str(tmp_path)))
    r = s.render(spp=spp, seed=11)
    assert r["dropped"] == 0
    zscore_check(r["mean"], r["var"], r["count"].astype(np.float64), z["mean"], z["var"],
                 z["count"].astype(np.float64), frac_min=0.98 if block == 1 else 0.95,
                 block=block)
    s.close()
