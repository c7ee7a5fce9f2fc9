import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=True)


GENERATED_CACHE = os.path.join(tempfile.gettempdir(), "pine_b200_fixture_assets")
_verified = {}


def _sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 22), b""):
            h.update(chunk)
    return h.hexdigest()


def generated_asset(name, args, digest):
    """A fixture asset too large to store (the benchmark scenes' 512^3 grid and 1.31M-triangle
    mesh): regenerated by pine-scenegen from the arguments the fixture recorded, once per
    machine, and checked against the recorded SHA-256."""
    from pine_b200 import build
    os.makedirs(GENERATED_CACHE, exist_ok=True)
    path = os.path.join(GENERATED_CACHE, f"{digest[:16]}_{name}")
    if path in _verified:
        return path
    if not os.path.exists(path):
        exe = build.SCENEGEN if os.path.exists(build.SCENEGEN) else build.build_scenegen()
        subprocess.run([exe, *[str(a) for a in args], path + ".tmp"], check=True,
                       stdout=subprocess.DEVNULL)
        os.replace(path + ".tmp", path)
    got = _sha256(path)
    assert got == digest, f"regenerated {name} differs from the fixture's ({got} != {digest})"
    _verified[path] = True
    return path


def write_fixture_scene(npz, directory, name="scene.txt"):
    """Writes a fixture's scene text and its OBJ/volume assets into `directory`
    (regenerated assets are linked from the per-machine cache)."""
    os.makedirs(directory, exist_ok=True)
    for n, blob in zip(npz["asset_names"], npz["asset_blobs"]):
        with open(os.path.join(directory, str(n)), "wb") as f:
            f.write(np.asarray(blob, np.uint8).tobytes())
    if "generated" in npz.files:
        for n, g in json.loads(str(npz["generated"])).items():
            src = generated_asset(n, g["args"], g["sha256"])
            dst = os.path.join(directory, n)
            if not os.path.exists(dst):
                os.symlink(src, dst)
    path = os.path.join(directory, name)
    with open(path, "w") as f:
        f.write(str(npz["scene_text"]))
    return path


@pytest.fixture(scope="session")
def pglib():
    import pine_b200
    from pine_b200 import build
    build.build()
    return pine_b200.lib()


@pytest.fixture(scope="session")
def ctx(pglib):
    import pine_b200
    c = pine_b200.Context(0)
    yield c
    c.close()
