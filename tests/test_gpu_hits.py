"""Nearest-hit parity of the CUDA traversal (pg_intersect) with pine's BVH.

Golden records come from pine itself (tests/golden/make_golden.py); at the full 1.3M
triangle mesh size the oracle is the C restatement's exhaustive search (the closest hit
does not depend on the acceleration structure)."""

import os

import numpy as np
import pytest

from conftest import golden, write_fixture_scene

import oracle
import pine_b200 as pb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["spheres", "mesh"])
def test_hits_match_reference(ctx, tmp_path, name):
    z = golden(f"hits_{name}.npz")
    path = write_fixture_scene(z, str(tmp_path))
    sid = ctx.load_scene(path)
    shape, prim, t, uv = ctx.intersect(sid, z["rays"])
    h = z["hits"]
    ref = oracle.Restatement(path)
    _, _, _, amb = ref.intersect(z["rays"])
    ref.close()
    same = (shape == h["shape"]) & (prim == h["tri"])
    # Rays whose two nearest candidates lie within 1e-6 of each other are decided by
    # traversal order; everything else must match bit for bit.
    assert same[~amb].all(), f"{np.count_nonzero(~same & ~amb)} rays differ"
    hit = (h["shape"] >= 0) & same
    assert np.array_equal(t[hit].view(np.uint32), h["t"][hit].view(np.uint32))
    tri = hit & (h["tri"] >= 0)
    np.testing.assert_allclose(uv[tri, 0], h["u"][tri], atol=1e-6)
    np.testing.assert_allclose(uv[tri, 1], h["v"][tri], atol=1e-6)
    # Texture coordinates of spheres, planes and rects (Interaction::uv, which the shader
    # nodes read through TexCoord): sphere uv goes through pstd's acos and atan2.
    other = hit & (h["tri"] < 0)
    np.testing.assert_allclose(uv[other, 0], h["u"][other], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(uv[other, 1], h["v"][other], rtol=1e-5, atol=1e-5)
    ctx.release_scene(sid)


def test_empty_and_degenerate_rays(ctx, tmp_path):
    z = golden("hits_spheres.npz")
    sid = ctx.load_scene(write_fixture_scene(z, str(tmp_path)))
    s, p, t, uv = ctx.intersect(sid, np.zeros((0, 8), np.float32))
    assert s.size == 0
    rays = np.array([[0, 2, 0, 0, -1, 0, 0, 3.4e38],     # straight down onto the ground plane
                     [0, 20, 0, 0, 1, 0, 0, 0.5],         # up from above the light, tmax 0.5
                     [0, 2, 0, 1, 0, 0, 5, 4],            # tmin > tmax
                     [0, 50, 0, 0, 1, 0, 0, 3.4e38]],     # from above everything, going up
                    np.float32)
    s, p, t, uv = ctx.intersect(sid, rays)
    assert s[0] == 0 and abs(t[0] - 2.0) < 1e-6
    assert (s[1:] == -1).all() and (p == -1).all()
    ctx.release_scene(sid)


def test_full_size_mesh_hits(ctx, tmp_path):
    """1.31M-triangle displaced icosphere (20 * 4^8) in the Cornell box, 3000 seeded rays:
    GPU vs exhaustive search."""
    from pine_b200 import scenegen
    path = scenegen.mesh_scene(str(tmp_path / "mesh.txt"), subdiv=8, width=64,
                               height=36, spp=1)
    sid = ctx.load_scene(path)
    rng = np.random.default_rng(3)
    n = 3000
    o = np.concatenate([rng.uniform([-2.8, 0.2, -2.8], [2.8, 5.8, 2.8], (n // 2, 3)),
                        rng.uniform([-1, 1, -11], [1, 4, -9], (n - n // 2, 3))])
    target = rng.uniform([-1.3, 0.3, -0.8], [1.3, 2.9, 1.8], (n, 3))
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d, np.zeros((n, 1)), np.full((n, 1), 3.4e38)], 1).astype(np.float32)
    s, p, t, _ = ctx.intersect(sid, rays)
    ref = oracle.Restatement(path)
    rs, rp, rt, amb = ref.intersect(rays)
    ref.close()
    same = (s == rs) & (p == rp)
    assert same[~amb].all(), f"{np.count_nonzero(~same & ~amb)} rays differ"
    hit = (rs >= 0) & same
    assert hit.sum() > n * 0.9
    assert np.array_equal(t[hit].view(np.uint32), rt[hit].view(np.uint32))
    assert (rs == 0).sum() > n // 3  # most rays were aimed at the sphere


@pytest.mark.parametrize("builder", ["gpu", "gpu_sah"])
@pytest.mark.parametrize("name", ["spheres", "mesh"])
def test_gpu_built_bvh_gives_the_same_hits(pglib, tmp_path, name, builder):
    """The trees built on the GPU (linear BVH; binned SAH): closest hits do not depend on the
    tree, so they match pine's exactly, as the host-built tree's do."""
    z = golden(f"hits_{name}.npz")
    path = write_fixture_scene(z, str(tmp_path))
    with pb.Context(0) as ctx:
        ctx.set_bvh_builder(builder)
        sid = ctx.load_scene(path)
        info = ctx.bvh_info(sid)
        assert info["nodes"] > 0 and info["depth"] > 0
        shape, prim, t, uv = ctx.intersect(sid, z["rays"])
    h = z["hits"]
    ref = oracle.Restatement(path)
    _, _, _, amb = ref.intersect(z["rays"])
    ref.close()
    same = (shape == h["shape"]) & (prim == h["tri"])
    assert same[~amb].all(), f"{np.count_nonzero(~same & ~amb)} rays differ"
    hit = (h["shape"] >= 0) & same
    assert np.array_equal(t[hit].view(np.uint32), h["t"][hit].view(np.uint32))


def test_gpu_built_bvh_on_the_full_mesh(pglib, tmp_path):
    """The benchmark mesh (about 1.3M triangles): every builder's tree gives the same
    closest hits on 65536 random rays, the GPU builds are faster, and the GPU binned SAH
    build makes the host build's tree (the same 8-wide node count and depth)."""
    from pine_b200 import scenegen
    path = scenegen.mesh_scene(str(tmp_path / "m.txt"), width=64, height=36, spp=1,
                               sampler="Uniform")
    rng = np.random.default_rng(9)
    o = rng.uniform(-3, 3, (65536, 3))
    d = rng.normal(size=(65536, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d, np.zeros((65536, 1)), np.full((65536, 1), 3.4e38)], 1)
    out = {}
    with pb.Context(0) as ctx:
        for builder in ("host", "gpu", "gpu_sah"):
            ctx.set_bvh_builder(builder)
            sid = ctx.load_scene(path)
            out[builder] = ctx.intersect(sid, rays), ctx.bvh_info(sid)
            ctx.release_scene(sid)
    (hs, hp, ht, _), hi = out["host"]
    for builder in ("gpu", "gpu_sah"):
        (gs, gp, gt, _), gi = out[builder]
        same = (hs == gs) & (hp == gp)
        # Ties between two triangles at the same distance may go either way.
        assert same.mean() > 0.9999
        assert np.array_equal(ht[same].view(np.uint32), gt[same].view(np.uint32))
        print(f"{builder}: host build {hi['build_seconds']:.3f} s, GPU build "
              f"{gi['build_seconds']:.3f} s; depth {hi['depth']} / {gi['depth']}, nodes "
              f"{hi['nodes']} / {gi['nodes']}")
        assert gi["build_seconds"] < hi["build_seconds"]
    si = out["gpu_sah"][1]
    assert (si["nodes"], si["depth"]) == (hi["nodes"], hi["depth"])
