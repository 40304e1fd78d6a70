"""CPU checks of the learned-preconditioner oracle (oracle/learned_oracle.py), which the
GPU tests use as their reference: BF16 rounding, the MLP gradient against finite
differences, the structure of the fixed multilevel operator (symmetric, positive
definite on mean-free fields, homogeneous) and the energy-norm loss gradient against
finite differences through the oracle's own metric product."""
import numpy as np
import pytest

import oracle
from oracle import learned_oracle as LO
from repulsor_b200 import meshes


def _theta(seed, out_scale=0.3):
    rng = np.random.default_rng(seed)
    th = np.zeros(LO.NPARAM)
    th[LO.OFF_W1:LO.OFF_B1] = rng.uniform(-0.5, 0.5, LO.NH * LO.NF)
    th[LO.OFF_B1:LO.OFF_W2] = rng.normal(0, 0.1, LO.NH)
    th[LO.OFF_W2:LO.OFF_B2] = rng.uniform(-0.2, 0.2, LO.NH * LO.NH)
    th[LO.OFF_B2:LO.OFF_W3] = rng.normal(0, 0.1, LO.NH)
    th[LO.OFF_W3:LO.OFF_B3] = rng.uniform(-out_scale, out_scale, LO.NO * LO.NH)
    th[LO.OFF_B3:] = rng.normal(0, 0.1, LO.NO)
    return th


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.140625], np.float32)
    r = LO.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1); 1 + 3*2^-8 -> 1 + 2^-6
    np.testing.assert_array_equal(r, [1.0, 1.0, 1.0 + 2.0 ** -6, 1.0, -2.5, 3.140625])


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    th = _theta(1)
    F = rng.normal(size=(7, LO.NF))
    dO = rng.normal(size=(7, LO.NO))
    O, cache = LO.mlp_forward(th, F, quantize=False)
    g = LO.mlp_backward(th, cache, dO, quantize=False)
    h = 1e-6
    for k in rng.choice(LO.NPARAM, 40, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = ((LO.mlp_forward(tp, F, False)[0] - LO.mlp_forward(tm, F, False)[0]) * dO).sum() / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


@pytest.fixture(scope="module")
def small_surface():
    V, S = meshes.icosphere_sh(level=2, seed=11)
    om = oracle.OracleMesh(2, V, S, threads=4)
    return V, S, om, LO.LearnedGeometry(V, S, om.tree())


def test_fixed_operator_is_symmetric_positive_definite(small_surface):
    V, S, om, G = small_surface
    th = np.zeros(LO.NPARAM)             # all outputs 0 -> all gains 1
    n = V.shape[0]
    cols = []
    for v in range(n):
        for c in range(3):
            X = np.zeros((n, 3))
            X[v, c] = 1.0
            X -= X.mean(0)
            cols.append(G.apply(th, X, quantize=False).ravel())
    B = np.array(cols).T
    assert np.allclose(B, B.T, atol=1e-12 * np.abs(B).max())
    # positive on the mean-free subspace
    rng = np.random.default_rng(0)
    for _ in range(5):
        r = rng.normal(size=(n, 3))
        r -= r.mean(0)
        assert (G.apply(th, r, quantize=False) * r).sum() > 0


def test_preconditioner_is_homogeneous_and_positive(small_surface):
    V, S, om, G = small_surface
    th = _theta(5, out_scale=1.0)
    rng = np.random.default_rng(1)
    r = rng.normal(size=(V.shape[0], 3))
    r -= r.mean(0)
    z = G.apply(th, r)
    np.testing.assert_allclose(G.apply(th, 7.5 * r), 7.5 * z, rtol=1e-12, atol=1e-12 * np.abs(z).max())
    assert (z * r).sum() > 0
    np.testing.assert_allclose(z.mean(0), 0.0, atol=1e-12 * np.abs(z).max())


def test_energy_loss_gradient_matches_finite_differences(small_surface):
    V, S, om, G = small_surface
    th = _theta(7)
    rng = np.random.default_rng(2)
    b = rng.normal(size=(V.shape[0], 3))
    b -= b.mean(0)
    A = lambda X: om.metric_multiply(X)
    x, _, _ = oracle.pcg(A, lambda r: r, b, tol=1e-10, max_iter=5000)
    loss, g = G.loss_and_grad(th, b, x, A, quantize=False)
    assert 0.0 <= loss <= 1.0
    h = 1e-5
    idx = np.concatenate([rng.choice(np.arange(LO.OFF_W3, LO.NPARAM), 10, replace=False),
                          rng.choice(LO.OFF_W3, 10, replace=False)])
    for k in idx:
        tp, tm = th.copy(), th.copy()
        tp[k] += h
        tm[k] -= h
        fd = (G.loss_and_grad(tp, b, x, A, quantize=False)[0] - G.loss_and_grad(tm, b, x, A, quantize=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-4 * np.abs(g).max() + 1e-6 * abs(fd), (k, fd, g[k])
