"""Error statuses and resource handling of the C ABI on a GPU."""

import ctypes

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

import pine_b200 as pb

pytestmark = pytest.mark.gpu


def test_invalid_arguments(ctx, tmp_path):
    with pytest.raises(pb.PgError) as e:
        ctx.render(12345)
    assert e.value.status == 1
    z = golden("image_spheres.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    with pytest.raises(pb.PgError) as e:
        ctx.render(sid, math_mode="pine", spp=1, seed=0, sample_offset=-1)
    assert e.value.status == 1
    with pytest.raises(pb.PgError) as e:
        ctx.set_tuning(queue_capacity=10)
    assert e.value.status == 1
    with pytest.raises(pb.PgError) as e:
        pb.Context(999)
    assert e.value.status == 1
    L = pb.lib()
    assert L.pg_upload_scene(ctx._ctx, None, None) == 1
    assert L.pg_render(None, 0, None, None, None, None, None) == 1
    ctx.release_scene(sid)
    with pytest.raises(pb.PgError):
        ctx.release_scene(sid)


def test_scene_ids_are_reused_and_independent(ctx, tmp_path):
    za, zb = golden("image_spheres.npz"), golden("image_volume.npz")
    a = ctx.load_scene(write_fixture_scene(za, str(tmp_path / "a")))
    b = ctx.load_scene(write_fixture_scene(zb, str(tmp_path / "b")))
    ra = ctx.render(a, spp=16, seed=1)
    ctx.release_scene(a)
    c = ctx.load_scene(write_fixture_scene(za, str(tmp_path / "c")))
    assert c == a
    rc = ctx.render(c, spp=16, seed=1)
    np.testing.assert_allclose(ra["mean"], rc["mean"], rtol=1e-5, atol=1e-7)
    rb = ctx.render(b, spp=4, seed=1)
    assert rb["mean"].shape == (27, 48, 3)
    ctx.release_scene(b)
    ctx.release_scene(c)


def test_upload_from_flattened_description(ctx, tmp_path):
    """pg_upload_scene with a caller-built description (the drop-in path an integrator
    inside pine would use) renders the same image as loading the file."""
    z = golden("image_spheres.npz")
    path = write_fixture_scene(z, str(tmp_path))
    ps = pb.ParsedScene(path)
    s1 = ctx.upload_scene(ps.desc)
    ps.close()
    s2 = ctx.load_scene(path)
    r1 = ctx.render(s1, spp=32, seed=8)
    r2 = ctx.render(s2, spp=32, seed=8)
    np.testing.assert_allclose(r1["mean"], r2["mean"], rtol=1e-5, atol=1e-7)
    ctx.release_scene(s1)
    ctx.release_scene(s2)
