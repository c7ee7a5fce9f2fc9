"""Host-side checks of libpinegpu that need no GPU: the C ABI exports, pine's number
parser and scene grammar, error statuses, and the synthetic scene generators."""

import ctypes
import os

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

import pine_b200 as pb


def test_library_exports_every_declared_symbol(pglib):
    names = pb.declared_functions()
    assert "pg_render" in names and "pg_intersect" in names
    missing = [n for n in names if not hasattr(pglib, n)]
    assert not missing, f"declared in include/pine_gpu.h but not exported: {missing}"


def test_stof_is_bit_exact_with_pine(pglib):
    z = golden("pstd_stof.npz")
    for s, o in zip(z["strings"], z["outputs"]):
        b = str(s).encode()
        v = np.float32(pglib.pg_pstd_stof(b, len(b)))
        assert v.view(np.uint32) == o[0].view(np.uint32), repr(s)


def test_parse_fixture_scenes(pglib, tmp_path):
    z = golden("image_spheres.npz")
    ps = pb.ParsedScene(write_fixture_scene(z, str(tmp_path / "s")))
    d = ps.desc
    assert d.num_shapes == 66 and d.num_materials == 66
    assert (d.camera.width, d.camera.height) == (48, 27)
    assert d.max_depth == 8 and d.samples_per_pixel == 1024
    assert d.shapes[0].type == pb.SHAPE_PLANE and d.shapes[1].type == pb.SHAPE_RECT
    assert d.lights[0].type == 2  # Sky
    ps.close()
    z = golden("image_mesh.npz")
    ps = pb.ParsedScene(write_fixture_scene(z, str(tmp_path / "m")))
    d = ps.desc
    assert d.num_triangles == 5120 + 12
    assert d.shapes[0].type == pb.SHAPE_MESH and d.shapes[0].mesh_num_triangles == 5120
    ps.close()
    z = golden("image_volume.npz")
    ps = pb.ParsedScene(write_fixture_scene(z, str(tmp_path / "v")))
    d = ps.desc
    m = d.media[0]
    assert m.type == 1 and list(m.size) == [64, 64, 64] and d.camera.medium == 0
    assert abs(m.sigma_a[0] + m.sigma_s[0] - 20.0) < 1e-5
    ps.close()


def _scene(tmp_path, body):
    p = tmp_path / "bad.txt"
    p.write_text("Integrator: Path{\n    maxDepth: 4\n    sampler: Uniform{\n"
                 "        samplesPerPixel: 1\n    }\n}\nCamera: ThinLen{\n    film{\n"
                 "        size: 8 8\n    }\n    from: 0 0 -5\n    to: 0 0 0\n    fov: 0.7\n}\n"
                 + body)
    return str(p)


@pytest.mark.parametrize("body,status", [
    ("Shape: Sphere{\n    position: 0 0 0\n    radius: 1\n    material: nope\n}\n", 7),
    ("Material m: Layered{\n    layer0: Diffuse{\n        albedo: Texture{\n"
     "            filename: wood.png\n        }\n    }\n}\n", 5),
    ("Shape: Disk{\n    position: 0 0 0\n    normal: 0 1 0\n    radius: 1\n}\n", 5),
    ("Shape: TriangleMesh{\n    file: missing.obj\n}\n", 6),
    ("Medium m: Grid{\n    file: missing.vol\n    sigma_a: 1\n    sigma_s: 1\n"
     "    position: 0 0 0\n}\n", 6),
    ("Light: Environment{\n    environment: Atmosphere{\n    }\n}\n", 5),
])
def test_loader_errors_follow_pine(pglib, tmp_path, body, status):
    with pytest.raises(pb.PgError) as e:
        pb.ParsedScene(_scene(tmp_path, body))
    assert e.value.status == status


def test_parser_comments_and_typed_blocks(pglib, tmp_path):
    path = _scene(tmp_path, "// a comment line\nMaterial shiny: Layered{\n"
                            "    layer1: Dielectric{\n        roughness: 0\n        eta: 1.45\n    }\n"
                            "    layer0: Diffuse{\n        albedo: 0.98 0.55 0.02\n    }\n}\n"
                            "Shape: Sphere{\n    position: 0 0 0\n    radius: 1\n"
                            "    material: shiny\n}\n")
    ps = pb.ParsedScene(path)
    m = ps.desc.materials[0]
    # Layers ordered by index, highest (top) first (material.cpp:33-43).
    assert m.num_layers == 2 and m.layers[0].type == 2 and m.layers[1].type == 0
    assert abs(m.layers[0].eta - 1.45) < 1e-6
    assert np.allclose(list(m.layers[1].albedo), [0.98, 0.55, 0.02])
    assert list(m.layers[0].albedo) == [1.0, 1.0, 1.0]  # Dielectric default (bxdf.cpp:176-181)
    ps.close()


def test_context_without_gpu_reports_cuda_error(pglib):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(pb.PgError) as e:
        pb.Context(0)
    assert e.value.status == 3


def test_cloud_generator(tmp_path):
    """pine-scenegen's cloud: ~30% of voxels non-zero, max exactly 1, and the same file for
    the same seed (the benchmark fixtures identify grids by their hash)."""
    from pine_b200 import scenegen
    n = 48
    a, b, c = (str(tmp_path / f"{k}.vol") for k in "abc")
    scenegen.gen_cloud_volume(a, n, seed=7)
    scenegen.gen_cloud_volume(b, n, seed=7)
    scenegen.gen_cloud_volume(c, n, seed=8)
    hdr = np.fromfile(a, np.int32, 3)
    assert list(hdr) == [n, n, n]
    d = np.fromfile(a, np.float32)[3:]
    assert d.size == n ** 3
    assert abs((d > 0).mean() - 0.3) < 0.02 and d.max() == 1.0 and d.min() == 0.0
    assert open(a, "rb").read() == open(b, "rb").read()
    assert open(a, "rb").read() != open(c, "rb").read()


def test_scenegen_rejects_bad_arguments(tmp_path):
    from pine_b200 import scenegen
    with pytest.raises(RuntimeError):
        scenegen.gen_cloud_volume(str(tmp_path / "x.vol"), 1)
    with pytest.raises(RuntimeError):
        scenegen.gen_icosphere_obj(str(tmp_path / "x.obj"), 12)
    with pytest.raises(RuntimeError):
        scenegen.gen_cloud_volume(str(tmp_path / "no" / "such" / "dir.vol"), 8)


def test_icosphere_generator(tmp_path):
    from pine_b200 import scenegen
    p = str(tmp_path / "ico.obj")
    nt = scenegen.gen_icosphere_obj(p, 3, radius=1.0, center=(0.0, 0.0, 0.0), amplitude=0.1)
    assert nt == 20 * 4 ** 3
    text = open(p).read()
    assert "e" not in text.replace("\n", " ").split("f ")[0]  # no exponents anywhere
