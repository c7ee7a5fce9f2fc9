"""The drop-in surfaces run end to end:

* pine's own command line (src/cli/main.cpp) built with the GpuPath integrator registered
  (pine_b200/pine_plugin: gpupath.h/.cpp plus the one-line CASE("GpuPath") in
  CreateIntegrator, src/core/integrator.cpp:20-37), run as `pine scene.txt` on fixture
  scenes whose integrator line reads `Integrator: GpuPath{`: its film agrees with pine's
  own Path render of the same scene within Monte Carlo error, and pine writes its image;
* pine-gpu, this library's command line (`pine-gpu scene.txt`, pine's main.cpp:6-29 with
  the GPU integrator), writing the linear film as PFM.

The pine build exists only where pine's sources were present when __graft_entry__.build()
ran; without it the first test is skipped."""

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden, write_fixture_scene

pytestmark = pytest.mark.gpu

PINE_GPUPATH = os.path.join(ROOT, "pine_b200", "_build", "pine_gpupath", "pine")
PINE_GPU_CLI = os.path.join(ROOT, "pine_b200", "pine-gpu")


def _spp(z):
    return json.loads(str(z["info"]))["spp"]


def _agree(g, gv, gn, z):
    rm, rv, rn = (z["mean"].astype(np.float64), z["var"].astype(np.float64),
                  z["count"].astype(np.float64))
    se = np.sqrt(gv / gn[..., None] + rv / rn[..., None])
    v = se > 0
    zz = (g - rm)[v] / se[v]
    frac = np.mean(np.abs(zz) < 2.576)
    rel = np.linalg.norm(g - rm) / np.linalg.norm(rm)
    expected = np.sqrt(np.sum(gv / gn[..., None] + rv / rn[..., None])) / np.linalg.norm(rm)
    return frac, abs(zz.mean()), rel, expected


@pytest.mark.skipif(not os.path.exists(PINE_GPUPATH),
                    reason="pine with the GpuPath integrator was not built (no pine sources)")
@pytest.mark.parametrize("name,math", [("mesh", "pine"), ("spheres", "fast"), ("volume", "fast")])
def test_pine_renders_with_the_gpupath_integrator(pglib, tmp_path, name, math):
    z = golden(f"image_{name}.npz")
    path = write_fixture_scene(z, str(tmp_path))
    text = open(path).read()
    assert text.startswith("Integrator: Path{")
    text = text.replace("Integrator: Path{",
                        f"Integrator: GpuPath{{\n    linearFile: gpu.lin\n    mathMode: {math}\n"
                        "    seed: 5\n", 1)
    with open(path, "w") as f:
        f.write(text)
    p = subprocess.run([PINE_GPUPATH, "./scene.txt"], cwd=str(tmp_path), capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert "[GpuPath]" in p.stdout
    # pine's Film wrote its image (tonemapped BMP) as it does for its own integrators.
    assert os.path.getsize(tmp_path / "image.bmp") > 54
    raw = open(tmp_path / "gpu.lin", "rb").read()
    w, h = np.frombuffer(raw[:8], np.int32)
    npx = int(w) * int(h)
    body = np.frombuffer(raw[8:], np.float32)
    mean = body[:3 * npx].reshape(h, w, 3).astype(np.float64)
    var = body[3 * npx:6 * npx].reshape(h, w, 3).astype(np.float64)
    cnt = body[6 * npx:].view(np.uint32).reshape(h, w).astype(np.float64)
    assert (h, w) == z["mean"].shape[:2]
    assert abs(cnt.sum() / (npx * _spp(z)) - 1) < 2e-3
    frac, mz, rel, expected = _agree(mean, var, cnt, z)
    assert frac >= 0.98 and mz < 0.1, (frac, mz)
    assert rel <= 1.25 * expected, (rel, expected)


def test_pine_gpu_command_line(pglib, tmp_path):
    z = golden("image_volume.npz")
    path = write_fixture_scene(z, str(tmp_path))
    spp = _spp(z)
    p = subprocess.run([PINE_GPU_CLI, "--seed", "9", "--out", str(tmp_path / "v.pfm"), path],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "[pine-gpu]" in p.stdout
    raw = open(tmp_path / "v.pfm", "rb").read()
    header, rest = raw.split(b"\n", 3)[:3], raw.split(b"\n", 3)[3]
    assert header[0] == b"PF" and header[2] == b"-1.0"
    w, h = map(int, header[1].split())
    img = np.frombuffer(rest, np.float32).reshape(h, w, 3).astype(np.float64)
    # The PFM holds the mean only: the GPU film's variance is taken as pine's.
    rv = z["var"].astype(np.float64)
    cnt = np.full((h, w), float(spp))
    frac, mz, rel, expected = _agree(img, rv, cnt, z)
    assert frac >= 0.98 and mz < 0.1, (frac, mz)
    assert rel <= 1.25 * expected, (rel, expected)
