"""TangentPointMetric0 MultiplyMetric on the B200 through the C ABI, against the FP64
oracle (1e-5 relative in max norm)."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes

pytestmark = pytest.mark.gpu
M_TOL = 1e-5
Q, P = 6.0, 12.0


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("cfg", [1, 2, 3])
@pytest.mark.parametrize("small", [True, False])
def test_metric_multiply_matches_oracle(cfg, small):
    dom, (V, S) = meshes.config_mesh(cfg, small=small)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S, threads=8)
    tpm = rpb.TangentPointMetric0(Q, P)
    rng = np.random.default_rng(cfg)
    for X in (rng.standard_normal(V.shape), np.ascontiguousarray(V), np.sin(3 * V)):
        Y = tpm.MultiplyMetric(M, 1.0, X)
        Y_ref = O.metric_multiply(X, Q, P)
        assert rel_max(Y, Y_ref) <= M_TOL, rel_max(Y, Y_ref)


def test_metric_flags_alpha_beta():
    dom, (V, S) = meshes.config_mesh(2, small=True)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    rng = np.random.default_rng(3)
    X = rng.standard_normal(V.shape)
    for flags in (2, 4, 6):
        Y = tpm.MultiplyMetric(M, 1.0, X, NF_flag=bool(flags & 2), FF_flag=bool(flags & 4))
        Y_ref = O.metric_multiply(X, Q, P, flags=flags)
        assert rel_max(Y, Y_ref) <= M_TOL
    Y0 = rng.standard_normal(V.shape)
    Y = tpm.MultiplyMetric(M, -2.0, X, 0.5, Y0.copy())
    assert rel_max(Y, -2.0 * O.metric_multiply(X, Q, P) + 0.5 * Y0) <= M_TOL


def test_metric_symmetric_and_kills_translations():
    dom, (V, S) = meshes.config_mesh(3, small=True)
    M = rpb.SimplicialMesh(V, S)
    tpm = rpb.TangentPointMetric0(Q, P)
    rng = np.random.default_rng(5)
    X, Z = rng.standard_normal(V.shape), rng.standard_normal(V.shape)
    AX, AZ = tpm.MultiplyMetric(M, 1.0, X), tpm.MultiplyMetric(M, 1.0, Z)
    assert abs((Z * AX).sum() - (X * AZ).sum()) <= 1e-5 * np.sqrt((X * AX).sum() * (Z * AZ).sum())
    T = np.tile([[1.0, -2.0, 0.5]], (V.shape[0], 1))
    assert np.max(np.abs(tpm.MultiplyMetric(M, 1.0, T))) <= 1e-5 * np.max(np.abs(AX))


def test_metric_rejects_wrong_nrhs():
    dom, (V, S) = meshes.config_mesh(1, small=True)
    M = rpb.SimplicialMesh(V, S)
    with pytest.raises(rpb.RepulsorError):
        rpb.TangentPointMetric0(Q, P).MultiplyMetric(M, 1.0, np.zeros((V.shape[0], 2)))
