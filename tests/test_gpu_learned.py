"""Learned preconditioner on the GPU against the CPU oracle (oracle/learned_oracle.py):
the MLP forward/backward kernels, the preconditioner application, the training
gradient through the whole chain (including the metric product), and the gain of the
trained network in flexible CG over plain CG on the same mesh."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from oracle import learned_oracle as LO
from repulsor_b200 import meshes
from repulsor_b200.learned import LearnedPreconditioner, train, training_pairs

pytestmark = pytest.mark.gpu

# The device MLP runs on the tensor cores with BF16 layer inputs and FP32 accumulation; the
# oracle rounds the same activations in FP64 arithmetic, so an activation can round to the
# neighbouring BF16 value (relative step 2^-8) where the FP32 and FP64 sums straddle a tie.
O_TOL = 5e-3        # MLP outputs, relative to max |O|
G_TOL = 1e-2        # parameter gradients, relative in the 2-norm
Z_TOL = 2e-3        # preconditioner output, relative in the max norm
Q, P = 6.0, 12.0


def _theta(seed, out_scale=0.3):
    rng = np.random.default_rng(seed)
    th = np.zeros(LO.NPARAM, np.float32)
    th[LO.OFF_W1:LO.OFF_B1] = rng.uniform(-0.5, 0.5, LO.NH * LO.NF)
    th[LO.OFF_B1:LO.OFF_W2] = rng.normal(0, 0.1, LO.NH)
    th[LO.OFF_W2:LO.OFF_B2] = rng.uniform(-0.2, 0.2, LO.NH * LO.NH)
    th[LO.OFF_B2:LO.OFF_W3] = rng.normal(0, 0.1, LO.NH)
    th[LO.OFF_W3:LO.OFF_B3] = rng.uniform(-out_scale, out_scale, LO.NO * LO.NH)
    th[LO.OFF_B3:] = rng.normal(0, 0.1, LO.NO)
    return th


def test_param_count_and_roundtrip():
    net = LearnedPreconditioner(seed=1)
    assert net.param_count() == LO.NPARAM == 5443
    th = _theta(2)
    net.set_params(th)
    np.testing.assert_array_equal(net.get_params(), th)


@pytest.mark.parametrize("n", [1, 129, 5000])
def test_mlp_forward_backward_match_oracle(n):
    rng = np.random.default_rng(n)
    th = _theta(3)
    net = LearnedPreconditioner(params=th)
    F = rng.normal(size=(n, LO.NF)).astype(np.float32)
    dO = rng.normal(size=(n, LO.NO)).astype(np.float32)
    O, g = net.eval(F, dO)
    O_ref, cache = LO.mlp_forward(th, F)
    g_ref = LO.mlp_backward(th, cache, dO.astype(np.float64))
    assert np.abs(O - O_ref).max() <= O_TOL * np.abs(O_ref).max()
    assert np.linalg.norm(g - g_ref) <= G_TOL * np.linalg.norm(g_ref)


@pytest.fixture(scope="module")
def surface():
    V, S = meshes.icosphere_sh(level=3, seed=21)
    M = rpb.SimplicialMesh(V, S)
    om = oracle.OracleMesh(2, V, S, threads=8)
    G = LO.LearnedGeometry(V, S, M.tree())
    return V, S, M, om, G


def test_apply_matches_oracle(surface):
    V, S, M, om, G = surface
    th = _theta(4, out_scale=0.5)
    net = LearnedPreconditioner(params=th)
    rng = np.random.default_rng(0)
    for _ in range(2):
        r = rng.normal(size=V.shape)
        r -= r.mean(0)
        z = net.apply(M, r)
        z_ref = G.apply(th, r)
        assert np.abs(z - z_ref).max() <= Z_TOL * np.abs(z_ref).max()


def test_training_gradient_matches_oracle(surface):
    V, S, M, om, G = surface
    th = _theta(6)
    net = LearnedPreconditioner(params=th)
    tpm = rpb.TangentPointMetric0(Q, P)
    R, E = training_pairs(M, tpm, n_rhs=1, checkpoints=(0, 8), seed=5, exact_tol=1e-10)
    loss, g = net.train_step(M, tpm, R, E, lr=0.0, want_grad=True)
    A = lambda X: om.metric_multiply(X, q=Q, p=P)
    ref = [G.loss_and_grad(th, R[k], E[k], A) for k in range(R.shape[0])]
    loss_ref = np.mean([l for l, _ in ref])
    g_ref = np.mean([gg for _, gg in ref], axis=0)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.linalg.norm(g - g_ref) <= G_TOL * np.linalg.norm(g_ref)
    np.testing.assert_array_equal(net.get_params(), th)     # lr = 0: no step


def test_frozen_gain_application_matches_oracle(surface):
    """apply_pair: M(R) as apply gives it, and the application to Y with R's gains."""
    V, S, M, om, G = surface
    th = _theta(8, out_scale=0.5)
    net = LearnedPreconditioner(params=th)
    rng = np.random.default_rng(3)
    r, y = rng.normal(size=V.shape), rng.normal(size=V.shape)
    z, zy = net.apply_pair(M, r, y)
    z_ref, zy_ref = G.apply(th, r), G.apply_frozen(th, r, y)
    assert np.abs(z - z_ref).max() <= Z_TOL * np.abs(z_ref).max()
    assert np.abs(zy - zy_ref).max() <= Z_TOL * np.abs(zy_ref).max()
    # with Y = R it is the application itself
    _, zr = net.apply_pair(M, r, r)
    assert np.abs(zr - z).max() <= 1e-12 * np.abs(z).max()


def test_sensitivity_training_gradient_matches_oracle(surface):
    """train_step_sens: the gradient of sum_k G_k . M(R_k) (with the gain penalty) for given
    sensitivities, as the unrolled-solve training uses it."""
    V, S, M, om, G = surface
    th = _theta(9)
    net = LearnedPreconditioner(params=th)
    rng = np.random.default_rng(4)
    R = rng.normal(size=(3,) + V.shape)
    Gs = rng.normal(size=(3,) + V.shape)
    obj, g = net.train_step_sens(M, R, Gs, lr=0.0, reg=0.1, want_grad=True)
    ref = [G.grad_given(th, R[k], Gs[k], reg=0.1) for k in range(3)]
    obj_ref = sum(o for o, _ in ref)
    g_ref = np.sum([gg for _, gg in ref], axis=0)
    scale = sum(np.abs(Gs[k]).sum() * np.abs(G.apply(th, R[k])).max() for k in range(3))
    assert abs(obj - obj_ref) <= Z_TOL * scale
    assert np.linalg.norm(g - g_ref) <= G_TOL * np.linalg.norm(g_ref)
    np.testing.assert_array_equal(net.get_params(), th)     # lr = 0: no step


def test_trained_network_beats_plain_cg(surface):
    """Train on pairs from plain CG solves on the mesh, then solve a held-out right-hand
    side: flexible CG with the trained network needs far fewer iterations than plain CG
    to the same 1e-6 true residual (checked with the oracle's FP64 metric product). The
    untrained multilevel operator (all gains 1) is reported beside it; training may move
    the count by a few per cent either way, but must not lose the multilevel gain."""
    V, S, M, om, G = surface
    tpm = rpb.TangentPointMetric0(Q, P)
    R, E = training_pairs(M, tpm, n_rhs=4, checkpoints=(0, 4, 16, 48, 128), seed=100)
    b = meshes.random_rhs(V.shape[0], seed=7, project=True)

    tpm.Solve(M, 1.0, b, max_iter=20000, tolerance=1e-6, precond=rpb.PRECOND_NONE)
    it_plain = tpm.Solver_IterationCount()

    net = LearnedPreconditioner(seed=3)
    zero = net.get_params()
    zero[LO.OFF_W3:] = 0.0                          # untrained multilevel operator: gains 1
    net.set_params(zero)
    net.attach(M)
    tpm.Solve(M, 1.0, b, max_iter=20000, tolerance=1e-6, precond=rpb.PRECOND_LEARNED)
    it_prior = tpm.Solver_IterationCount()

    net = LearnedPreconditioner(seed=3)
    hist = train(net, tpm, [(M, R, E)], epochs=40, lr=1e-3, batch=4, seed=0)
    assert hist[-1] < hist[0]
    net.attach(M)
    X = tpm.Solve(M, 1.0, b, max_iter=20000, tolerance=1e-6, precond=rpb.PRECOND_LEARNED)
    it_learned = tpm.Solver_IterationCount()
    rel = np.linalg.norm(b - om.metric_multiply(X, q=Q, p=P), axis=0) / np.linalg.norm(b, axis=0)
    print(f"iterations: plain CG {it_plain}, untrained multilevel {it_prior}, learned FCG {it_learned}; "
          f"loss {hist[0]:.4f} -> {hist[-1]:.4f}")
    assert rel.max() <= 2e-6
    assert it_learned <= 0.6 * it_plain
    assert it_learned <= 1.2 * it_prior
