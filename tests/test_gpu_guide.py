"""Guiding network on the GPU (tcgen05 kernels) against the float64 oracle: forward
outputs, weight gradients, the Adam step, and learning on a synthetic target."""
import numpy as np
import pytest

from oracle import guide_oracle as go

pytestmark = pytest.mark.gpu


def _unit(rng, n):
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def _features(rng, n):
    nrm = _unit(rng, n)
    nrm[::5] = np.nan
    return go.encode(rng.uniform(size=(n, 3)), nrm, _unit(rng, n))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 40000])
def test_forward_matches_oracle(ctx, n):
    rng = np.random.default_rng(n)
    ctx.guide_reset(seed=n)
    w = ctx.guide_weights()
    assert np.all(w[0, :, 33:] == 0) and np.all(w[5, 40:, :] == 0)
    f = _features(rng, n)
    raw = ctx.guide_forward(f)
    ref, _ = go.forward(w, f)
    assert raw.shape == (n, 40)
    assert np.all(np.isfinite(raw))
    scale = np.abs(ref).max()
    assert np.abs(raw - ref).max() <= 2e-2 * scale
    assert _rel(raw, ref) < 5e-3


@pytest.mark.parametrize("n", [200, 4096, 65537])
def test_gradient_matches_oracle(ctx, n):
    rng = np.random.default_rng(100 + n)
    ctx.guide_reset(seed=7)
    w = ctx.guide_weights()
    f = _features(rng, n)
    dw = np.concatenate([_unit(rng, n), rng.uniform(0.0, 2.0, (n, 1))], axis=1)
    g, loss = ctx.guide_gradient(f, dw)
    ref, rloss = go.gradient(w, f, dw)
    assert abs(loss - rloss) <= 1e-3 * abs(rloss) + 1e-6
    for l in range(6):
        assert _rel(g[l], ref[l]) < 3e-2, (l, _rel(g[l], ref[l]))
    assert np.all(g[0, :, 33:] == 0) and np.all(g[5, 40:, :] == 0)


def test_train_step_matches_oracle_adam(ctx):
    rng = np.random.default_rng(5)
    n = 8192
    ctx.guide_reset(seed=3)
    w0 = ctx.guide_weights().astype(np.float64)
    f = _features(rng, n)
    dw = np.concatenate([_unit(rng, n), rng.uniform(0.0, 2.0, (n, 1))], axis=1)
    ctx.guide_train_step(f, dw, lr=1e-2)
    w1 = ctx.guide_weights()
    g, _ = go.gradient(w0, f, dw, weight_scale=dw[:, 3].mean())
    ref, _, _ = go.adam(w0, 0 * w0, 0 * w0, g, 1, 1e-2)
    # The first Adam step moves every weight with a clear gradient by about lr.
    moved = np.abs(g) > 1e-3 * np.abs(g).max()
    np.testing.assert_allclose(w1[moved], ref[moved], atol=2e-3)
    assert np.all(w1[0, :, 33:] == 0) and np.all(w1[5, 40:, :] == 0)


def test_training_learns_a_position_dependent_lobe(ctx):
    """Samples pointing along +x for x < 0.5 and along +z otherwise: the loss falls and
    the learned mixture puts its mass in the right direction on both halves."""
    rng = np.random.default_rng(9)
    ctx.guide_reset(seed=1)

    def batch(n):
        pos = rng.uniform(size=(n, 3))
        axis = np.where((pos[:, 0] < 0.5)[:, None], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0])
        d = axis + 0.15 * rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        nrm = np.full((n, 3), np.nan)
        f = go.encode(pos, nrm, _unit(rng, n))
        return pos, f, np.concatenate([d, np.ones((n, 1))], axis=1)

    losses = []
    for step in range(150):
        _, f, dw = batch(16384)
        losses.append(ctx.guide_train_step(f, dw, lr=1e-2))
    assert np.mean(losses[-10:]) < np.mean(losses[:3]) - 2.0
    pos, f, dw = batch(4096)
    raw = ctx.guide_forward(f)
    from pine_b200 import guide_pdf
    p_true = guide_pdf(raw, dw[:, :3])
    # Density at the sample's own direction versus uniform (1 / 4 pi).
    assert np.median(p_true) > 20 / (4 * np.pi)
