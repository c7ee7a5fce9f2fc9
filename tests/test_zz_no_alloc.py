"""pg_render_noalloc, the render entry point that allocates no device memory, called
through the C ABI and compared with pg_render on the same scene, seed and sample count.

The file name puts it last in collection, so it runs after the other GPU tests have used
the library on this GPU; it also passes alone in a fresh process.  Every path draws its
random numbers from its sample id alone, so both entry points trace the same paths and
the images differ only by the order of float additions into each pixel."""
import ctypes

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

pytestmark = pytest.mark.gpu

PG_ERR_INVALID_ARG = 1


def _noalloc(ctx, sid, out, spp, seed, math, accumulate=0):
    import pine_b200 as pb
    desc = pb.RenderDesc(spp, 0, seed, 0, pb.MATH_MODES[math], 0, accumulate, 0)
    stats = pb.RenderStats()
    status = pb.lib().pg_render_noalloc(ctx._ctx, sid, ctypes.byref(desc),
                                        ctypes.c_void_p(out.data_ptr()), ctypes.byref(stats))
    return status, stats


@pytest.mark.parametrize("name,math,spp", [("spheres", "pine", 64), ("volume", "fast", 32)])
def test_noalloc_matches_pg_render(pglib, tmp_path, name, math, spp):
    import torch
    import pine_b200 as pb
    with pb.Context(0) as ctx:
        sid = ctx.load_scene(write_fixture_scene(golden(f"image_{name}.npz"), str(tmp_path)))
        info = ctx.scene_info(sid)
        h, w = info["height"], info["width"]
        ref = ctx.render(sid, spp=spp, seed=11, math_mode=math)["mean"]
        out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda:0")
        scale = float(np.abs(ref).max())
        for call in range(2):  # two calls in a row reuse the same scratch array
            out.fill_(-1.0)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info(0)[0]
            status, stats = _noalloc(ctx, sid, out, spp, 11, math)
            assert status == 0, ctx._lib.pg_last_error(ctx._ctx)
            torch.cuda.synchronize()
            if call == 1:  # after the first call: no device memory taken or given back
                assert torch.cuda.mem_get_info(0)[0] == free_before
            got = out.cpu().numpy()
            assert stats.paths == h * w * spp
            np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-6 * scale,
                                       err_msg=f"call {call}")


def test_noalloc_rejects_what_it_cannot_hold(pglib, tmp_path):
    import torch
    import pine_b200 as pb
    z = golden("image_spheres.npz")
    text = str(z["scene_text"]).replace("size: 48 27", "size: 1024 1024")
    assert "1024 1024" in text
    path = write_fixture_scene(z, str(tmp_path))
    with open(path, "w") as f:
        f.write(text)
    with pb.Context(0) as ctx:
        big = ctx.load_scene(path)
        out = torch.empty(16, dtype=torch.float32, device="cuda:0")
        status, _ = _noalloc(ctx, big, out, 1, 0, "fast")
        assert status == PG_ERR_INVALID_ARG
        assert b"524288" in ctx._lib.pg_last_error(ctx._ctx)
        small = ctx.load_scene(write_fixture_scene(z, str(tmp_path / "small")))
        out = torch.empty(48 * 27 * 3, dtype=torch.float32, device="cuda:0")
        status, _ = _noalloc(ctx, small, out, 1, 0, "fast", accumulate=1)
        assert status == PG_ERR_INVALID_ARG
