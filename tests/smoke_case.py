"""One tiny render and a few intersections on cuda:0, checked against the oracle."""

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def run():
    import oracle
    import pine_b200
    from pine_b200 import scenegen

    with tempfile.TemporaryDirectory() as d:
        path = scenegen.spheres_scene(os.path.join(d, "s.txt"), width=24, height=16, spp=64,
                                      n_spheres=12, env="sky", env_radiance=0.5)
        ref = oracle.Restatement(path)
        with pine_b200.Context(0) as ctx:
            sid = ctx.load_scene(path)
            rng = np.random.default_rng(5)
            o = rng.uniform([-6, 0.5, -6], [6, 5, 6], (256, 3))
            dd = rng.normal(size=(256, 3))
            dd /= np.linalg.norm(dd, axis=1, keepdims=True)
            rays = np.concatenate([o, dd, np.zeros((256, 1)), np.full((256, 1), 3.4e38)], 1)
            s, p, t, _ = ctx.intersect(sid, rays)
            rs, rp, rt, amb = ref.intersect(rays)
            ok = amb | ((s == rs) & (p == rp))
            assert ok.all(), f"hit ids differ on {np.count_nonzero(~ok)} rays"
            hit = (rs >= 0) & ~amb
            assert np.all(np.abs(t[hit] - rt[hit]) <= 1e-6 * np.abs(rt[hit]))
            r = ctx.render(sid, spp=64, seed=3)
            assert r["stats"]["paths"] == 24 * 16 * 64
            # Halton scene, box of radius 0.5: each sample reaches its own pixel, except
            # that rounding can put one exactly on a pixel edge (then a neighbour too).
            assert abs(int(r["count"].sum()) - 24 * 16 * 64) <= 16
            img = ref.render(spp=64, seed=3)
            g, o_ = r["mean"].astype(np.float64), img["mean"]
            se = np.sqrt(r["var"] / 64 + img["var"] / 64) + 1e-9
            frac = np.mean(np.abs(g - o_) / se < 4.0)
            assert frac > 0.97, f"only {frac:.3f} of pixels within 4 sigma of the oracle"
        ref.close()
    print("smoke ok")


if __name__ == "__main__":
    run()
