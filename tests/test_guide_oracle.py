"""Guiding network on the CPU: the float64 oracle checked by finite differences, and the
library's host restatements (the same functions the renderer's kernels run) checked
against the oracle."""
import numpy as np
import pytest

from oracle import guide_oracle as go


def _unit(rng, n):
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def _raw(rng, n):
    raw = rng.normal(size=(n, 40))
    raw.reshape(n, 8, 5)[:, :, 3] = rng.uniform(-2.5, 5.0, size=(n, 8))
    return raw


def test_oracle_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    raw = _raw(rng, 16)
    dw = np.concatenate([_unit(rng, 16), rng.uniform(0.1, 3.0, (16, 1))], axis=1)
    loss, g = go.loss_and_grad(raw, dw)
    eps = 1e-6
    num = np.zeros_like(raw)
    for j in range(40):
        rp, rm = raw.copy(), raw.copy()
        rp[:, j] += eps
        rm[:, j] -= eps
        num[:, j] = (go.loss_and_grad(rp, dw)[0] - go.loss_and_grad(rm, dw)[0]) / (2 * eps)
    np.testing.assert_allclose(g, num, rtol=1e-5, atol=1e-7)


def test_oracle_network_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    n = 12
    feats = go.encode(rng.uniform(size=(n, 3)), _unit(rng, n), _unit(rng, n))
    w = rng.normal(scale=0.3, size=(6, 64, 64))
    w[0, :, 33:] = 0
    w[5, 40:, :] = 0
    dw = np.concatenate([_unit(rng, n), rng.uniform(0.1, 2.0, (n, 1))], axis=1)
    grad, loss = go.gradient(w, feats, dw, fp16=False)

    def f(wt):
        raw, _ = go.forward(wt, feats, fp16=False)
        return go.loss_and_grad(raw, dw)[0].mean()

    assert abs(loss - f(w)) < 1e-12
    eps = 1e-6
    for l, o, i in [(0, 3, 5), (0, 10, 32), (2, 7, 9), (4, 60, 1), (5, 0, 12), (5, 39, 63)]:
        wp, wm = w.copy(), w.copy()
        wp[l, o, i] += eps
        wm[l, o, i] -= eps
        num = (f(wp) - f(wm)) / (2 * eps)
        assert abs(grad[l, o, i] - num) <= 1e-6 + 1e-4 * abs(num), (l, o, i)


def test_oracle_mixture_is_a_density_and_sampling_follows_it():
    rng = np.random.default_rng(3)
    raw = np.repeat(_raw(rng, 1), 200000, axis=0)
    d = go.sample(raw, rng.uniform(size=(200000, 3)))
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-9)
    p = go.pdf(raw, d)
    # E_q[1 / q] is the area of the sphere.
    assert abs(np.mean(1.0 / p) / (4 * np.pi) - 1.0) < 0.05
    # Uniform directions: E_uniform[q] * 4 pi = 1.
    u = _unit(rng, 200000)
    assert abs(np.mean(go.pdf(raw, u)) * 4 * np.pi - 1.0) < 0.05


def test_host_restatement_matches_oracle(pglib):
    import pine_b200 as pb
    rng = np.random.default_rng(4)
    n = 512
    pos = rng.uniform(-0.1, 1.1, size=(n, 3))
    nrm = _unit(rng, n)
    nrm[::7] = np.nan
    wo = _unit(rng, n)
    np.testing.assert_allclose(pb.guide_encode(pos, nrm, wo), go.encode(pos, nrm, wo), atol=2e-6)
    raw = _raw(rng, n)
    mu, kappa, w = go.mixture(raw)
    lobes = pb.guide_mixture(raw)
    np.testing.assert_allclose(lobes[:, :, :3], mu, atol=1e-6)
    np.testing.assert_allclose(lobes[:, :, 3], kappa, rtol=1e-5)
    np.testing.assert_allclose(lobes[:, :, 4], w, rtol=1e-5, atol=1e-7)
    dirs = _unit(rng, n)
    np.testing.assert_allclose(pb.guide_pdf(raw, dirs), go.pdf(raw, dirs), rtol=2e-4, atol=1e-7)
    u = rng.uniform(size=(n, 3))
    np.testing.assert_allclose(pb.guide_sample(raw, u), go.sample(raw, u), atol=2e-3)
    dw = np.concatenate([dirs, rng.uniform(0.1, 3.0, (n, 1))], axis=1)
    loss, g = pb.guide_loss_grad(raw, dw)
    oloss, og = go.loss_and_grad(raw, dw)
    np.testing.assert_allclose(loss, oloss, rtol=1e-4, atol=1e-5)
    scale = np.abs(og).max(axis=1, keepdims=True)
    assert np.all(np.abs(g - og) <= 1e-3 * scale + 1e-6)


@pytest.mark.parametrize("step", [1, 2, 10])
def test_oracle_adam_matches_formula(step):
    w, m, v = np.ones(4), np.zeros(4), np.zeros(4)
    g = np.array([1.0, -2.0, 0.0, 1e-3])
    w1, m1, v1 = go.adam(w, m, v, g, step, 1e-2)
    mh = (0.1 * g) / (1 - 0.9 ** step)
    vh = (0.01 * g * g) / (1 - 0.99 ** step)
    np.testing.assert_allclose(w1, w - 1e-2 * mh / (np.sqrt(vh) + 1e-8))
