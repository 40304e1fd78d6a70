"""The FP64 oracle (oracle/tp0_oracle.cpp) against identities of the reference mathematics
and against its committed golden fixtures (tests/golden/make_golden.py).

The reference binary cannot be built here (its Tensors submodule is missing), so these
identities pin the restatement: translation invariance of the energy, Euler homogeneity
sum_v x_v . dE/dx_v = (2n + q - p) E (the tree and pair lists are scale-free), central
finite differences of Value vs Differential (exact for the fixed-list approximation),
symmetry and translation kernel of the metric, the chain rule in closed form vs
forward-mode differentiation, and convergence to the all-pairs sum as theta -> 0."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from repulsor_b200 import meshes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
Q, P = 6.0, 12.0


def small(cfg):
    return meshes.config_mesh(cfg, small=True)


@pytest.mark.parametrize("cfg", [1, 2, 3])
def test_translation_and_homogeneity(cfg):
    dom, (V, S) = small(cfg)
    O = oracle.OracleMesh(dom, V, S)
    E, D = O.differential(Q, P)
    assert np.all(np.abs(D.sum(axis=0)) <= 1e-10 * np.abs(D).sum())
    assert abs((V * D).sum() - (2 * dom + Q - P) * E) <= 1e-10 * abs(E)


@pytest.mark.parametrize("cfg", [1, 3])
def test_scaling_law(cfg):
    dom, (V, S) = small(cfg)
    lam = 1.7
    E1 = oracle.OracleMesh(dom, V, S).energy(Q, P)
    E2 = oracle.OracleMesh(dom, lam * V, S).energy(Q, P)
    assert E2 == pytest.approx(lam ** (2 * dom + Q - P) * E1, rel=1e-12)


@pytest.mark.parametrize("cfg", [1, 2])
def test_finite_differences(cfg):
    dom, (V, S) = small(cfg)
    O = oracle.OracleMesh(dom, V, S)
    _, D = O.differential(Q, P)
    rng = np.random.default_rng(3)
    def central(dV, h):
        O.semistatic_update(V + h * dV)
        Ep = O.energy(Q, P)
        O.semistatic_update(V - h * dV)
        Em = O.energy(Q, P)
        return (Ep - Em) / (2 * h)

    for _ in range(3):
        dV = rng.standard_normal(V.shape)
        h = 1e-5 * np.abs(V).max()
        fd = (4.0 * central(dV, 0.5 * h) - central(dV, h)) / 3.0   # Richardson: O(h^4)
        assert fd == pytest.approx((D * dV).sum(), rel=1e-7)
    O.semistatic_update(V)


def test_chain_rule_closed_form_matches_forward_mode():
    lib = oracle._load()
    lib.oracle_set_chain_rule.argtypes = [ctypes.c_int]
    for cfg in (1, 2, 3):
        dom, (V, S) = small(cfg)
        O = oracle.OracleMesh(dom, V, S)
        lib.oracle_set_chain_rule(1)
        _, D1 = O.differential(Q, P)
        lib.oracle_set_chain_rule(0)
        _, D0 = O.differential(Q, P)
        assert np.max(np.abs(D1 - D0)) <= 1e-12 * np.max(np.abs(D1))


def test_metric_symmetric_psd_and_translation_kernel():
    dom, (V, S) = small(3)
    O = oracle.OracleMesh(dom, V, S)
    rng = np.random.default_rng(1)
    X, Z = rng.standard_normal(V.shape), rng.standard_normal(V.shape)
    AX, AZ = O.metric_multiply(X), O.metric_multiply(Z)
    assert abs((Z * AX).sum() - (X * AZ).sum()) <= 1e-12 * np.sqrt((X * AX).sum() * (Z * AZ).sum())
    assert (X * AX).sum() > 0
    T = np.tile([[0.3, -1.0, 2.0]], (V.shape[0], 1))
    assert np.max(np.abs(O.metric_multiply(T))) <= 1e-12 * np.max(np.abs(AX))


def test_fmm_converges_to_all_pairs():
    V, S = meshes.torus_knot(n=300, seed=5)
    errs = []
    for theta in (0.5, 0.25, 0.125):
        O = oracle.OracleMesh(1, V, S, theta_far=theta)
        errs.append(abs(O.energy(Q, P) - O.allpairs_energy(Q, P)) / O.allpairs_energy(Q, P))
    assert errs[2] < errs[0]
    assert errs[2] < 1e-3


@pytest.mark.parametrize("name", ["knot400", "torus40x30", "icosphere3_sh"])
def test_golden_fixtures(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    dom = g["S"].shape[1] - 1
    O = oracle.OracleMesh(dom, g["V"], g["S"])
    assert np.array_equal(O.tree()["perm"], g["perm"])
    c = O.counts()
    assert c["near_nnz"] == int(g["near_nnz"]) and c["far_nnz"] == int(g["far_nnz"])
    assert O.energy(Q, P) == pytest.approx(float(g["energy"]), rel=1e-12)
    _, D = O.differential(Q, P)
    assert np.max(np.abs(D - g["differential"])) <= 1e-11 * np.max(np.abs(g["differential"]))
    assert np.max(np.abs(O.metric_multiply(g["X"]) - g["AX"])) <= 1e-11 * np.max(np.abs(g["AX"]))
    assert np.max(np.abs(O.precondition(g["X"]) - g["PX"])) <= 1e-9 * np.max(np.abs(g["PX"]))
    assert O.allpairs_energy(Q, P) == pytest.approx(float(g["allpairs_energy"]), rel=1e-12)


@pytest.mark.parametrize("cfg", [1, 2])
def test_oracle_densities_integrate_to_the_energy(cfg):
    """Sum over simplices of a_i * rho_i is the energy (every ordered pair once)."""
    dom, (V, S) = meshes.config_mesh(cfg, small=True)
    om = oracle.OracleMesh(dom, V, S, threads=8)
    en, rho = om.simplex_densities()
    Pn, _ = om.primitive_data()
    a = np.zeros(S.shape[0])
    a[om.tree()["perm"]] = Pn[:, 0]
    assert abs((a * rho).sum() - en) <= 1e-12 * abs(en)
    assert abs(en - om.energy()) <= 1e-12 * abs(en)
    ev, rv = om.vertex_densities()
    assert rv.shape == (V.shape[0],) and np.all(rv > 0)
