"""Edge cases of TangentPointEnergy0 / TangentPointMetric0 on the B200 through the C ABI:
meshes with one simplex, two far-apart simplices, an unreferenced vertex, a three-edge
polygon, and a simplex index out of range (rejected on the host before any GPU work).
Tolerances as in test_gpu_energy.py: energy 1e-6 relative, differential 1e-5 relative
in max norm (absolute where the oracle's value is zero)."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb

pytestmark = pytest.mark.gpu
Q, P = 6.0, 12.0


def check_against_oracle(dom, V, S):
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S, threads=2)
    tpe = rpb.TangentPointEnergy0(Q, P)
    D = np.zeros((V.shape[0], 3))
    E = tpe.Differential(M, 1.0, 0.0, D)
    E_ref, D_ref = O.differential(Q, P)
    scale_e = max(abs(E_ref), 1e-300)
    assert abs(E - E_ref) <= 1e-6 * scale_e, (E, E_ref)
    scale_d = float(np.max(np.abs(D_ref)))
    if scale_d == 0.0:
        assert np.all(D == 0.0)
    else:
        assert float(np.max(np.abs(D - D_ref))) <= 1e-5 * scale_d
    return E, D


def triangle(offset=(0.0, 0.0, 0.0)):
    V = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.2, 0.9, 0.1]]) + np.asarray(offset)
    return V


def test_single_triangle_has_no_pairs():
    V = triangle()
    S = np.array([[0, 1, 2]], dtype=np.int32)
    E, D = check_against_oracle(2, V, S)
    assert E == 0.0 and np.all(D == 0.0)


@pytest.mark.parametrize("distance", [10.0, 1.5])
def test_two_triangles(distance):
    V = np.vstack([triangle(), triangle((distance, 0.3, -0.2))])
    S = np.array([[0, 1, 2], [3, 4, 5]], dtype=np.int32)
    E, _ = check_against_oracle(2, V, S)
    assert E > 0.0


@pytest.mark.parametrize("distance", [10.0, 1.5])
def test_two_triangles_metric_product(distance):
    V = np.vstack([triangle(), triangle((distance, 0.3, -0.2))])
    S = np.array([[0, 1, 2], [3, 4, 5]], dtype=np.int32)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(2, V, S, threads=2)
    X = np.random.default_rng(3).standard_normal(V.shape)
    Y = rpb.TangentPointMetric0(Q, P).MultiplyMetric(M, 1.0, X)
    Y_ref = O.metric_multiply(X, Q, P)
    assert float(np.max(np.abs(Y - Y_ref))) <= 1e-5 * float(np.max(np.abs(Y_ref)))


def test_single_triangle_metric_product_is_zero():
    M = rpb.SimplicialMesh(triangle(), np.array([[0, 1, 2]], dtype=np.int32))
    Y = rpb.TangentPointMetric0(Q, P).MultiplyMetric(M, 1.0, np.ones((3, 3)))
    assert np.all(Y == 0.0)


def test_unreferenced_vertex_gets_zero_differential():
    rng = np.random.default_rng(5)
    n = 12
    t = np.linspace(0.0, 2.0 * np.pi, n, endpoint=False)
    V = np.stack([np.cos(t), np.sin(t), 0.1 * rng.standard_normal(n)], axis=1)
    S = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int32)
    V_extra = np.vstack([V, [[5.0, 5.0, 5.0]]])          # vertex n belongs to no edge
    E, D = check_against_oracle(1, V, S)
    E2, D2 = check_against_oracle(1, V_extra, S)
    assert E2 == pytest.approx(E, rel=1e-12)
    assert np.all(D2[n] == 0.0)
    assert float(np.max(np.abs(D2[:n] - D))) <= 1e-12 * float(np.max(np.abs(D)))


def test_three_edge_polygon():
    V = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.3, 0.8, 0.2]])
    S = np.array([[0, 1], [1, 2], [2, 0]], dtype=np.int32)
    check_against_oracle(1, V, S)


def test_simplex_index_out_of_range_is_rejected():
    V = triangle()
    for bad in ([[0, 1, 3]], [[0, -1, 2]]):
        with pytest.raises(rpb.RepulsorError):
            rpb.SimplicialMesh(V, np.array(bad, dtype=np.int32))
