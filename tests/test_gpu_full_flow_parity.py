"""The full-flow configuration at full size against the FP64 oracle: two linked tori (R=1,
r=0.3, 480 x 640 grids each, 1,228,800 triangles, the second rotated 90 degrees about x
and shifted by +1 along x, normal jitter N(0, 0.002^2)) with an icosphere level-5 obstacle
of radius 0.3 at (0, 0, 2). Energy within 1e-6 relative, differential within 1e-5 relative
in max norm, for TangentPointEnergy0 and TangentPointObstacleEnergy; the tree permutation
and the pattern sizes equal the oracle's. At this size the cluster moments come from FP64
prefix-sum differences over ranges of up to 1.2 M primitives, so this also bounds their
cancellation error."""
import os

import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes

pytestmark = pytest.mark.gpu

E_TOL, D_TOL = 1e-6, 1e-5
Q, P = 6.0, 12.0


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_linked_tori_with_obstacle_match_oracle_at_full_size():
    V, S = meshes.config_mesh(5)[1]
    assert S.shape[0] == 1_228_800
    Vo, So = meshes.icosphere(level=5, radius=0.3, centre=(0.0, 0.0, 2.0))
    M = rpb.SimplicialMesh(V, S)
    M.LoadObstacle(rpb.SimplicialMesh(Vo, So))
    tpe, tpo = rpb.TangentPointEnergy0(Q, P), rpb.TangentPointObstacleEnergy(Q, P)
    D = np.zeros_like(V)
    E = tpe.Differential(M, 1.0, 0.0, D)
    Do = np.zeros_like(V)
    Eo = tpo.Differential(M, 1.0, 0.0, Do)

    O = oracle.OracleMesh(2, V, S, threads=os.cpu_count() or 8)
    st, oc = M.stats(), O.counts()
    assert st["near_nnz"] == oc["near_nnz"] and st["far_nnz"] == oc["far_nnz"]
    assert st["verynear_nnz"] == oc["verynear_nnz"] and st["cluster_count"] == oc["clusters"]
    assert np.array_equal(M.tree()["perm"], O.tree()["perm"])
    E_ref, D_ref = O.differential(Q, P)
    assert abs(E - E_ref) <= E_TOL * abs(E_ref), (E, E_ref)
    assert rel_max(D, D_ref) <= D_TOL, rel_max(D, D_ref)

    O.load_obstacle(oracle.OracleMesh(2, Vo, So))
    Eo_ref, Do_ref = O.obstacle_differential(Q, P)
    assert abs(Eo - Eo_ref) <= E_TOL * abs(Eo_ref), (Eo, Eo_ref)
    assert rel_max(Do, Do_ref) <= D_TOL, rel_max(Do, Do_ref)
