import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=True)


def write_fixture_scene(npz, directory, name="scene.txt"):
    """Writes a fixture's scene text and its OBJ/volume assets into `directory`."""
    os.makedirs(directory, exist_ok=True)
    for n, blob in zip(npz["asset_names"], npz["asset_blobs"]):
        with open(os.path.join(directory, str(n)), "wb") as f:
            f.write(np.asarray(blob, np.uint8).tobytes())
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
