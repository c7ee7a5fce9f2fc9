"""Guided rendering (pg_render with guiding = 1) on the GPU: the guided estimator agrees
with the plain path tracer within Monte Carlo error, and on a scene lit indirectly it has
a lower error at equal samples per pixel than the method without the network."""
import numpy as np
import pytest

from conftest import golden, write_fixture_scene

pytestmark = pytest.mark.gpu

# A closed box whose only light is a small panel just under the ceiling, emitting upwards:
# everything the camera sees is lit by the bright patch the panel makes on the ceiling,
# which next-event estimation cannot reach and BSDF sampling rarely finds.
INDIRECT_BOX = """Integrator: Path{
    maxDepth: 8
    sampler: Uniform{
        samplesPerPixel: 64
    }
}

Camera: ThinLen{
    film{
        size: 96 72
        filter: Box{
            radius: 0.5
        }
        outputFileName: image.bmp
    }
    from: 0 1 -1.9
    to: 0 1 0
    fov: 1.2
}

Shape: Rect{
    position: 0 0 0
    ex: 4 0 0
    ey: 0 0 4
    material: wall
}

Shape: Rect{
    position: 0 2 0
    ex: 4 0 0
    ey: 0 0 4
    material: wall
}

Shape: Rect{
    position: -2 1 0
    ex: 0 2 0
    ey: 0 0 4
    material: red
}

Shape: Rect{
    position: 2 1 0
    ex: 0 2 0
    ey: 0 0 4
    material: green
}

Shape: Rect{
    position: 0 1 2
    ex: 4 0 0
    ey: 0 2 0
    material: wall
}

Shape: Rect{
    position: 0 1 -2
    ex: 4 0 0
    ey: 0 2 0
    material: wall
}

Shape: Rect{
    position: 0.6 1.85 0.8
    ex: 0 0 0.3
    ey: 0.3 0 0
    material: light
}

Material wall: Layered{
    layer0: Diffuse{
        albedo: 0.75
    }
}

Material red: Layered{
    layer0: Diffuse{
        albedo: 0.7 0.15 0.1
    }
}

Material green: Layered{
    layer0: Diffuse{
        albedo: 0.15 0.7 0.1
    }
}

Material light: Emissive{
    color: 60
}
"""


def _zfrac(a, b):
    va = a["var"] / a["count"][..., None]
    vb = b["var"] / b["count"][..., None]
    z = (a["mean"] - b["mean"]) / np.sqrt(np.maximum(va + vb, 1e-20))
    return np.mean(np.abs(z) < 2.576), z


@pytest.mark.parametrize("name,spp,depth", [("spheres", 256, 0), ("volume", 128, 0),
                                           ("spheres", 256, 1), ("volume", 128, 2)])
def test_guided_matches_plain_within_mc_error(ctx, tmp_path, name, spp, depth):
    """Guided renders have the plain tracer's expectation, with every eligible vertex
    guided (depth 0: the default) or only those below a bounce depth (pg_guide_config)."""
    sid = ctx.load_scene(write_fixture_scene(golden(f"image_{name}.npz"), str(tmp_path)))
    plain = ctx.render(sid, spp=spp, seed=1, math_mode="fast")
    ctx.guide_config(max_guided_depth=depth if depth else 1 << 30)
    ctx.guide_reset(seed=0)
    guided = ctx.render(sid, spp=spp, seed=2, math_mode="fast", guiding=True)
    ctx.guide_config(max_guided_depth=1 << 30)
    st = guided["stats"]
    assert st["kernels"]["guide"]["items"] > 0 and st["kernels"]["train"]["items"] > 0
    assert st["dropped"] == 0 and st["paths"] == plain["stats"]["paths"]
    # Samples on a pixel edge may reach a neighbour (Halton scene, pine's film splat).
    assert abs(int(guided["count"].sum()) - guided["count"].size * spp) <= guided["count"].size
    frac, z = _zfrac(guided, plain)
    assert frac >= 0.97, (frac, np.abs(z).max())
    # Whole-image mean within four standard errors.
    d = guided["mean"].mean() - plain["mean"].mean()
    se = np.sqrt((guided["var"].sum() + plain["var"].sum()) / spp) / guided["mean"].size
    assert abs(d) <= 4 * se + 1e-6, (d, se)


def test_trained_network_lowers_variance_on_indirect_box(ctx, tmp_path):
    """What the trained network gains: after a guided warm-up render has trained it, a
    guided render's per-sample variance (the film's per-pixel sample variance) and its
    error against a high-spp reference are both clearly below the plain path tracer's at
    equal samples per pixel."""
    # The default tuning: an autotuned context (tests/test_gpu_batch.py shares it) sizes
    # the training passes differently, and the gain measured here is for the defaults.
    ctx.set_tuning()
    path = tmp_path / "box.txt"
    path.write_text(INDIRECT_BOX)
    sid = ctx.load_scene(str(path))
    ref = ctx.render(sid, spp=16384, seed=9, math_mode="fast")["mean"]
    plain = ctx.render(sid, spp=256, seed=1, math_mode="fast")
    ctx.guide_reset(seed=0)
    ctx.render(sid, spp=1024, seed=3, math_mode="fast", guiding=True)  # warm-up: trains
    guided = ctx.render(sid, spp=256, seed=2, math_mode="fast", guiding=True)
    var_plain = float(plain["var"].mean())
    var_guided = float(guided["var"].mean())
    mse_plain = float(np.mean((plain["mean"] - ref) ** 2))
    mse_guided = float(np.mean((guided["mean"] - ref) ** 2))
    print(f"indirect box, 256 spp: sample variance plain {var_plain:.4g} guided {var_guided:.4g}; "
          f"MSE plain {mse_plain:.4g} guided {mse_guided:.4g}")
    assert var_guided < 0.7 * var_plain, (var_guided, var_plain)
    assert mse_guided < 0.85 * mse_plain, (mse_guided, mse_plain)


def test_guided_matches_reference_on_indirect_box_at_high_spp(ctx, tmp_path):
    """The indirect box's samples are heavy-tailed (rare paths find the bright patch), so
    its agreement test runs at high spp, on 4 x 4 pixel blocks, against a plain reference."""
    path = tmp_path / "box.txt"
    path.write_text(INDIRECT_BOX)
    sid = ctx.load_scene(str(path))
    ref = ctx.render(sid, spp=32768, seed=9, math_mode="fast")
    ctx.guide_reset(seed=0)
    guided = ctx.render(sid, spp=4096, seed=2, math_mode="fast", guiding=True)
    h, w = ref["mean"].shape[:2]
    blk = lambda a: a.reshape(h // 4, 4, w // 4, 4, -1).mean(axis=(1, 3))
    var = blk(guided["var"] / 4096 + ref["var"] / 32768) / 16
    z = (blk(guided["mean"]) - blk(ref["mean"])) / np.sqrt(var)
    assert np.mean(np.abs(z) < 2.576) >= 0.97, np.mean(np.abs(z) < 2.576)
    d = guided["mean"].mean() - ref["mean"].mean()
    se = np.sqrt(guided["var"].sum() / 4096 + ref["var"].sum() / 32768) / guided["mean"].size
    assert abs(d) <= 4 * se, (d, se)
