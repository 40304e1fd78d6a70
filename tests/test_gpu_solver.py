"""MultiplyPreconditioner and Solve on the B200 through the C ABI.

Preconditioner: H1^{-1} L_{2-s} H1^{-1} against the oracle (scipy factorization of the
oracle's H1 and the oracle pseudo-Laplacian), 1e-5 relative in max norm; the H1 factor's
numeric phase runs on the GPU (supernodal, one CTA per supernode of a level).
Solve: the true relative residual of the returned solution, measured with the FP64
oracle's metric operator, is at the requested 1e-6 (plus the 1e-5-level operator
difference times the solution's conditioning margin: bound 5e-6)."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes

pytestmark = pytest.mark.gpu
Q, P = 6.0, 12.0


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("cfg", [1, 2, 3])
def test_preconditioner_matches_oracle(cfg):
    dom, (V, S) = meshes.config_mesh(cfg, small=True)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    X = np.random.default_rng(cfg).standard_normal(V.shape)
    Y = tpm.MultiplyPreconditioner(M, 1.0, X)
    assert rel_max(Y, O.precondition(X, Q, P)) <= 1e-5
    assert tpm.SolveInfo(M)["factor_on_device"] == 1


@pytest.mark.parametrize("cfg", [2, 3])
def test_preconditioner_matches_oracle_full_size(cfg):
    """Full-size torus and icosphere level 6: deeper supernode schedules, whose upper levels
    run as split levels with up to 256 lanes per row (the small meshes use warp levels
    mostly)."""
    dom, (V, S) = meshes.config_mesh(cfg, small=False)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S, threads=8)
    tpm = rpb.TangentPointMetric0(Q, P)
    X = np.random.default_rng(10 + cfg).standard_normal(V.shape)
    Y = tpm.MultiplyPreconditioner(M, 1.0, X)
    assert rel_max(Y, O.precondition(X, Q, P)) <= 1e-5
    assert tpm.SolveInfo(M)["factor_on_device"] == 1


@pytest.mark.parametrize("cfg,precond", [(1, rpb.PRECOND_NONE), (2, rpb.PRECOND_NONE), (3, rpb.PRECOND_NONE),
                                         (2, rpb.PRECOND_REFERENCE), (3, rpb.PRECOND_REFERENCE)])
def test_solve_reaches_tolerance(cfg, precond):
    dom, (V, S) = meshes.config_mesh(cfg, small=True)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    B = meshes.random_rhs(V.shape[0], seed=cfg)
    X = tpm.Solve(M, 1.0, B, max_iter=20000, tolerance=1e-6, precond=precond)
    assert np.all(tpm.Solver_RelativeResiduals() <= 1e-6)
    R = B - O.metric_multiply(X, Q, P)
    rel = np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)
    assert np.all(rel <= 5e-6), rel


def test_solve_alpha_beta_semantics():
    dom, (V, S) = meshes.config_mesh(2, small=True)
    M = rpb.SimplicialMesh(V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    B = meshes.random_rhs(V.shape[0], seed=4)
    X1 = tpm.Solve(M, 1.0, B, precond=rpb.PRECOND_REFERENCE)
    X0 = np.random.default_rng(1).standard_normal(V.shape)
    X2 = tpm.Solve(M, 2.0, B, beta=-1.0, X=X0.copy(), precond=rpb.PRECOND_REFERENCE)
    assert np.max(np.abs(X2 - (2.0 * X1 - X0))) <= 1e-5 * np.max(np.abs(X2))


def test_solve_reports_non_convergence():
    dom, (V, S) = meshes.config_mesh(1, small=True)
    M = rpb.SimplicialMesh(V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    B = meshes.random_rhs(V.shape[0], seed=9)
    with pytest.raises(rpb.RepulsorError) as e:
        tpm.Solve(M, 1.0, B, max_iter=2, tolerance=1e-12, precond=rpb.PRECOND_NONE)
    assert "RPB_ENOTCONV" in str(e.value)


def test_hybrid_preconditioner_on_linked_tori():
    """RPB_PRECOND_HYBRID: flexible CG with z = P_ref r + w M(r), the reference
    preconditioner plus the attached network's multilevel output (untrained: every gain
    1), on two linked tori of 96 x 128 vertices each (49,152 triangles) with the energy's
    differential as right-hand side. It reaches the 1e-6 true residual (checked with the
    oracle's FP64 metric operator) in fewer iterations than CG with the reference
    preconditioner alone (measured 870-920 against 1,463; on 192 x 256 tori 1,280-1,506
    against 6,940)."""
    from repulsor_b200.learned import NPARAM_OUTPUT_OFFSET, LearnedPreconditioner

    V, S = meshes.linked_tori(n_major=96, n_minor=128)
    M = rpb.SimplicialMesh(V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    D = rpb.TangentPointEnergy0(Q, P).Differential(M)
    B = D - D.mean(0)
    net = LearnedPreconditioner(seed=1)
    th = net.get_params()
    th[NPARAM_OUTPUT_OFFSET:] = 0.0
    net.set_params(th)
    net.attach(M)
    tpm.Solve(M, 1.0, B, max_iter=6000, tolerance=1e-6, precond=rpb.PRECOND_REFERENCE)
    it_ref = tpm.Solver_IterationCount()
    X = tpm.Solve(M, 1.0, B, max_iter=6000, tolerance=1e-6, precond=rpb.PRECOND_HYBRID)
    it_hyb = tpm.Solver_IterationCount()
    assert tpm.SolveInfo(M)["fallback_iteration"] == -1
    O = oracle.OracleMesh(2, V, S, threads=8)
    rel = np.linalg.norm(B - O.metric_multiply(X, Q, P), axis=0) / np.linalg.norm(B, axis=0)
    print(f"linked tori 96 x 128: reference CG {it_ref} iterations, hybrid FCG {it_hyb}")
    assert rel.max() <= 5e-6
    assert it_hyb <= 0.8 * it_ref
