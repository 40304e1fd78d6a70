"""Host H1 metric + nested-dissection sparse Cholesky against scipy's sparse LU of the
oracle's H1 assembly (src/SimplicialMesh/H1Metric.hpp:36-257)."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes


@pytest.mark.parametrize("cfg", [1, 2, 3])
def test_h1_solve_matches_scipy(cfg):
    dom, (V, S) = meshes.config_mesh(cfg, small=True)
    T = rpb.HostTree(V, S)
    B = np.random.default_rng(cfg).standard_normal((V.shape[0], 3))
    X = T.h1_solve(V, S, B)
    O = oracle.OracleMesh(dom, V, S)
    X_ref = O.h1_solve(B)
    assert np.max(np.abs(X - X_ref)) <= 1e-10 * np.max(np.abs(X_ref))
    H = O.h1_matrix()
    assert np.max(np.abs(H @ X - B)) <= 1e-10 * np.max(np.abs(B))
