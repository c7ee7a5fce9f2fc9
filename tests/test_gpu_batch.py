"""Batched requests in graph-captured persistent wavefronts (pg_render_batch) and the
autotuner (pg_autotune)."""

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

pytestmark = pytest.mark.gpu


def test_batch_matches_individual_renders(ctx, tmp_path):
    names = ["spheres", "volume", "mesh"]
    ids = [ctx.load_scene(write_fixture_scene(golden(f"image_{n}.npz"), str(tmp_path / n)))
           for n in names]
    reqs = [dict(scene=ids[0], spp=256, seed=1),
            dict(scene=ids[1], spp=256, seed=2),
            dict(scene=ids[2], spp=128, seed=3),
            dict(scene=ids[1], spp=64, width=40, height=30, seed=4),
            dict(scene=ids[0], spp=32, width=17, height=9, seed=5)]
    out = ctx.render_batch(reqs)
    assert out["paths"] == sum(r["spp"] * (r.get("width", 48) * r.get("height", 27)) for r in reqs)
    t = np.array(out["request_seconds"])
    assert (t > 0).all() and (t <= out["seconds"] * 1.01 + 1e-3).all()
    for r, mean in zip(reqs[:3], out["means"][:3]):
        single = ctx.render(r["scene"], spp=r["spp"], seed=100 + r["seed"])
        se = np.sqrt(single["var"].astype(float) / r["spp"] * 2)
        v = se > 0
        z = np.abs(mean - single["mean"])[v] / se[v]
        # Different random streams: agreement within Monte Carlo error (the 128-spp mesh
        # request has heavy-tailed pixels, hence 95% rather than 99%).
        assert np.mean(z < 2.576) > 0.95
        assert abs(mean.mean() - single["mean"].mean()) < 0.03 * single["mean"].mean() + 1e-3
    # A request with its own film size renders that size.
    assert out["means"][3].shape == (30, 40, 3) and out["means"][4].shape == (9, 17, 3)
    assert np.isfinite(out["means"][3]).all() and out["means"][3].mean() > 0
    for i in ids:
        ctx.release_scene(i)


@pytest.mark.parametrize("group", [1, 2])
def test_grouped_batch_matches_one_launch(ctx, tmp_path, group):
    """Splitting a mixed batch into waves (one per scene kind or one per scene, each
    launching only its scenes' kernels) keeps every request's random streams, so its images
    match those of the one-wave batch up to float rounding; latencies stay within the
    batch's time, which spans all the waves."""
    names = ["spheres", "volume", "mesh"]
    ids = [ctx.load_scene(write_fixture_scene(golden(f"image_{n}.npz"), str(tmp_path / n)))
           for n in names]
    reqs = [dict(scene=ids[1], spp=128, seed=1),
            dict(scene=ids[0], spp=64, seed=2),
            dict(scene=ids[2], spp=64, seed=3),
            dict(scene=ids[0], spp=16, width=17, height=9, seed=4),
            dict(scene=ids[1], spp=32, width=40, height=30, seed=5)]
    before = ctx.tuning()
    outs = []
    for g in (0, group):
        ctx.set_tuning(**dict(before, group_kinds=g))
        outs.append(ctx.render_batch(reqs))
    ctx.set_tuning(**before)
    assert outs[0]["paths"] == outs[1]["paths"]
    for o in outs:
        t = np.array(o["request_seconds"])
        assert (t > 0).all() and (t <= o["seconds"] * 1.01 + 1e-3).all()
    for a, b in zip(outs[0]["means"], outs[1]["means"]):
        assert a.shape == b.shape and np.isfinite(b).all()
        scale = max(float(a.mean()), 1e-6)
        close = np.abs(a - b) <= 1e-4 * np.abs(a) + 1e-5 * scale
        assert close.mean() >= 0.99
        assert abs(float(a.mean()) - float(b.mean())) <= 1e-3 * scale
    for i in ids:
        ctx.release_scene(i)


def test_autotune_returns_a_valid_tuning(ctx, tmp_path):
    ids = [ctx.load_scene(write_fixture_scene(golden(f"image_{n}.npz"), str(tmp_path / n)))
           for n in ["volume", "spheres"]]
    before = ctx.tuning()
    t = ctx.autotune([dict(scene=ids[0], spp=64), dict(scene=ids[1], spp=64)])
    assert t["majorant_brick"] in (8, 16, 32, 64) and t["split_shadow"] in (0, 1)
    assert t["block_size"] in (32, 64, 128) and 1 << 20 <= t["queue_capacity"] <= 1 << 23
    assert t["sort_queue"] in (0, 1, 2) and t["group_kinds"] in (0, 1, 2)
    assert ctx.tuning() == t
    # Whatever was chosen renders the same image statistically.
    r = ctx.render(ids[1], spp=256, seed=9)
    ctx.set_tuning(**before)
    q = ctx.render(ids[1], spp=256, seed=10)
    se = np.sqrt((r["var"] + q["var"]).astype(float) / 256)
    v = se > 0
    assert np.mean(np.abs(r["mean"] - q["mean"])[v] / se[v] < 2.576) > 0.97
    for i in ids:
        ctx.release_scene(i)


@pytest.mark.parametrize("split,brick,sort", [(0, 8, 0), (1, 32, 1), (0, 16, 1), (1, 64, 1)])
def test_tunings_agree(ctx, tmp_path, split, brick, sort):
    """Every shadow split, majorant brick size and queue order renders the same image
    statistically."""
    z = golden("image_volume.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    before = ctx.tuning()
    ctx.set_tuning(queue_capacity=1 << 20, block_size=128, split_shadow=split,
                   majorant_brick=brick, sort_queue=sort)
    r = ctx.render(sid, spp=1024, seed=31)
    ctx.set_tuning(**before)
    se = np.sqrt(r["var"].astype(float) / 1024 + z["var"] / z["count"][..., None])
    v = se > 0
    assert np.mean(np.abs(r["mean"] - z["mean"])[v] / se[v] < 2.576) >= 0.98
    ctx.release_scene(sid)


@pytest.mark.parametrize("split", [0, 1])
def test_queue_sorting_changes_no_path(ctx, tmp_path, split):
    """Ordering the active list by medium cell changes which lanes take which paths, not
    the paths: a path's random streams follow its sample, and the film is summed per
    sample, so the image is the same bit for bit with and without sorting."""
    z = golden("image_volume.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    before = ctx.tuning()
    out = []
    for sort in (0, 1):
        ctx.set_tuning(**dict(before, queue_capacity=1 << 20, split_shadow=split, sort_queue=sort))
        out.append(ctx.render(sid, spp=256, seed=7, math_mode="fast"))
    ctx.set_tuning(**before)
    assert out[0]["stats"]["kernels"]["sort"]["launches"] == 0
    assert out[1]["stats"]["kernels"]["sort"]["launches"] > 0
    assert out[1]["stats"]["kernels"]["sort"]["items"] > 0
    np.testing.assert_array_equal(out[0]["count"], out[1]["count"])
    np.testing.assert_array_equal(out[0]["mean"], out[1]["mean"])
    np.testing.assert_array_equal(out[0]["var"], out[1]["var"])
    ctx.release_scene(sid)


def test_slot_order_changes_no_path(ctx, tmp_path):
    """Rebuilding the active list in slot order (the default in scenes with surfaces) only
    changes which lanes take which paths: the spheres scene with the counter-based stream
    and a box film renders the same image bit for bit in queue order and in slot order."""
    z = golden("image_spheres_c0.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    before = ctx.tuning()
    out = []
    for sort in (0, 2):
        ctx.set_tuning(**dict(before, queue_capacity=1 << 20, sort_queue=sort))
        out.append(ctx.render(sid, spp=256, seed=5, math_mode="fast"))
    ctx.set_tuning(**before)
    assert out[0]["stats"]["kernels"]["sort"]["launches"] == 0
    assert out[1]["stats"]["kernels"]["sort"]["launches"] > 0
    np.testing.assert_array_equal(out[0]["count"], out[1]["count"])
    np.testing.assert_array_equal(out[0]["mean"], out[1]["mean"])
    np.testing.assert_array_equal(out[0]["var"], out[1]["var"])
    ctx.release_scene(sid)
