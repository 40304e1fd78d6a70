"""The meshes the reference ships (Meshes/ of HenrikSchumacher/Repulsor: TwoSpheres.hpp of
its example program, two tori and a sphere in its mesh text format), read through the
reader of that format, as inputs of the parity suite.

CPU: the text format reader/writer (exact round trip, malformed files rejected); the
committed fixture equals the reference's files read with that reader (when the reference
tree is present); the host tree builder equals the oracle bit for bit on every mesh,
including the very-near pairs between the two spheres and the mesh x obstacle lists of
the example.
GPU: energy (1e-6), differential (1e-5) and metric product (1e-5) against the oracle on
every mesh; the example's obstacle energy and differential, whose lists hold 25 very-near
pairs, against the oracle; very-near results reproducible bit for bit; the device
traversal's patterns equal the host builder's."""
import os

import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes
from repulsor_b200.meshio import read_mesh_file, write_mesh_file

REFERENCE_MESHES = "/root/reference/Meshes"
E_TOL, D_TOL, M_TOL = 1e-6, 1e-5, 1e-5
Q, P = 6.0, 12.0
NAMES = ["twospheres", "twospheres_union", "torus2400", "torus38400", "sphere40560"]


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_mesh_file_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(7)
    V = rng.standard_normal((50, 3)) * 10.0 ** rng.integers(-8, 8, (50, 1))
    S = rng.integers(0, 50, (30, 3)).astype(np.int32)
    path = tmp_path / "m.txt"
    write_mesh_file(path, V, S)
    dom, amb, V2, S2 = read_mesh_file(path)
    assert (dom, amb) == (2, 3)
    assert np.array_equal(V2, V) and np.array_equal(S2, S)
    head = open(path).read().splitlines()[:5]
    assert head[0] == "domain_dimension\t2" and head[3] == "simplex_count\t30"
    assert "E" in head[4] and head[4].endswith("\t")


def test_mesh_file_reader_accepts_reference_header_names_and_rejects_malformed(tmp_path):
    p = tmp_path / "curve.txt"
    p.write_text("dom_dim 1\namb_dim 3\nvertex_count 3\nsimplex_count 3\n"
                 "0. 0. 0.\n1 0 0\n0 1 0\n0 1\n1 2\n2 0\n")
    dom, amb, V, S = read_mesh_file(p)
    assert dom == 1 and V.shape == (3, 3) and S.tolist() == [[0, 1], [1, 2], [2, 0]]
    (tmp_path / "short.txt").write_text("dom_dim 1\namb_dim 3\nvertex_count 3\nsimplex_count 3\n0 0 0\n")
    with pytest.raises(ValueError):
        read_mesh_file(tmp_path / "short.txt")
    (tmp_path / "bad.txt").write_text("dom_dim 1\namb_dim 3\nvertex_count 2\nsimplex_count 1\n0 0 0\n1 1 1\n0 5\n")
    with pytest.raises(ValueError):
        read_mesh_file(tmp_path / "bad.txt")


@pytest.mark.skipif(not os.path.isdir(REFERENCE_MESHES), reason="reference tree not present")
def test_fixture_equals_the_reference_files():
    import importlib.util

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_reference_meshes.py")
    spec = importlib.util.spec_from_file_location("make_reference_meshes", here)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    fresh = mod.load_all(os.path.dirname(REFERENCE_MESHES))
    fixture = np.load(os.path.join(os.path.dirname(here), "reference_meshes.npz"))
    assert set(fresh) == set(fixture.files)
    for k in fresh:
        assert np.array_equal(fresh[k], fixture[k]), k


@pytest.mark.parametrize("name", NAMES)
def test_host_tree_equals_oracle_on_reference_meshes(name):
    V, S = meshes.reference_mesh(name)
    T = rpb.HostTree(V, S)
    O = oracle.OracleMesh(2, V, S, threads=8)
    t, to = T.tree(), O.tree()
    for k in ("perm", "C_begin", "C_end", "C_left", "C_right"):
        assert np.array_equal(t[k], to[k]), k
    for which in ("near", "far", "verynear", "inter"):
        rp, ci = T.pattern(which)
        rpo, cio = O.pattern(which)
        assert np.array_equal(rp, rpo) and np.array_equal(ci, cio), which
    if name == "twospheres_union":
        assert O.counts()["verynear_nnz"] == 50 and O.counts()["inter_nnz"] == 0


def test_host_obstacle_lists_equal_oracle_on_the_example():
    V, S = meshes.reference_mesh("twospheres")
    VO, SO = meshes.reference_mesh("twospheres_obstacle")
    T, TO = rpb.HostTree(V, S), rpb.HostTree(VO, SO)
    O, OO = oracle.OracleMesh(2, V, S), oracle.OracleMesh(2, VO, SO)
    O.load_obstacle(OO)
    counts = O.obstacle_counts()
    assert counts["verynear"] == 25 and counts["inter"] == 0
    for which in ("near", "far", "verynear", "inter"):
        rp, ci, _ = T.obstacle_pattern(V, S, TO, VO, SO, which)
        rpo, cio = O.obstacle_pattern(which)
        assert np.array_equal(rp, rpo) and np.array_equal(ci, cio), which


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_energy_differential_metric_match_oracle_on_reference_meshes(name):
    V, S = meshes.reference_mesh(name)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(2, V, S, threads=8)
    tpe, tpm = rpb.TangentPointEnergy0(Q, P), rpb.TangentPointMetric0(Q, P)
    E = tpe.Value(M)
    E_ref = O.energy(Q, P)
    assert abs(E - E_ref) <= E_TOL * abs(E_ref), (E, E_ref)
    D = np.zeros_like(V)
    E2 = tpe.Differential(M, 1.0, 0.0, D)
    _, D_ref = O.differential(Q, P)
    assert abs(E2 - E_ref) <= E_TOL * abs(E_ref)
    assert rel_max(D, D_ref) <= D_TOL, rel_max(D, D_ref)
    rng = np.random.default_rng(11)
    for X in (rng.standard_normal(V.shape), np.sin(2 * V)):
        Y = tpm.MultiplyMetric(M, 1.0, X)
        assert rel_max(Y, O.metric_multiply(X, Q, P)) <= M_TOL
    # the device traversal built the patterns the host builder builds
    T = rpb.HostTree(V, S)
    for which in ("near", "far", "verynear", "inter"):
        a, b = M.pattern(which), T.pattern(which)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), which


@pytest.mark.gpu
def test_very_near_pairs_are_reproducible_and_enter_every_product():
    V, S = meshes.reference_mesh("twospheres_union")
    M = rpb.SimplicialMesh(V, S)
    assert M.stats()["verynear_nnz"] == 50
    tpe, tpm = rpb.TangentPointEnergy0(Q, P), rpb.TangentPointMetric0(Q, P)
    D1, D2 = np.zeros_like(V), np.zeros_like(V)
    E1 = tpe.Differential(M, 1.0, 0.0, D1)
    E2 = tpe.Differential(M, 1.0, 0.0, D2)
    assert E1 == E2 and np.array_equal(D1, D2)
    X = np.random.default_rng(2).standard_normal(V.shape)
    Y_all = tpm.MultiplyMetric(M, 1.0, X)
    Y_novf = tpm.MultiplyMetric(M, 1.0, X, VF_flag=False)
    O = oracle.OracleMesh(2, V, S, threads=8)
    dvf = Y_all - Y_novf
    dvf_ref = O.metric_multiply(X, Q, P, flags=7) - O.metric_multiply(X, Q, P, flags=6)
    assert np.max(np.abs(dvf_ref)) > 0
    assert rel_max(dvf, dvf_ref) <= M_TOL
    # symmetric operator with the very-near blocks
    Z = np.random.default_rng(3).standard_normal(V.shape)
    AZ = tpm.MultiplyMetric(M, 1.0, Z)
    assert abs((Z * Y_all).sum() - (X * AZ).sum()) <= 1e-5 * np.sqrt(abs((X * Y_all).sum() * (Z * AZ).sum()))


@pytest.mark.gpu
def test_example_obstacle_energy_with_very_near_pairs_matches_oracle():
    V, S = meshes.reference_mesh("twospheres")
    VO, SO = meshes.reference_mesh("twospheres_obstacle")
    M = rpb.SimplicialMesh(V, S)
    M.LoadObstacle(rpb.SimplicialMesh(VO, SO))
    assert M.obstacle_stats()["verynear_nnz"] == 25
    O, OO = oracle.OracleMesh(2, V, S, threads=8), oracle.OracleMesh(2, VO, SO)
    O.load_obstacle(OO)
    tpo = rpb.TangentPointObstacleEnergy(Q, P)
    E = tpo.Value(M)
    E_ref = O.obstacle_energy(Q, P)
    assert abs(E - E_ref) <= E_TOL * abs(E_ref), (E, E_ref)
    D = np.zeros_like(V)
    E2 = tpo.Differential(M, 1.0, 0.0, D)
    _, D_ref = O.obstacle_differential(Q, P)
    assert abs(E2 - E_ref) <= E_TOL * abs(E_ref)
    assert rel_max(D, D_ref) <= D_TOL, rel_max(D, D_ref)
    D2 = np.zeros_like(V)
    assert tpo.Differential(M, 1.0, 0.0, D2) == E2 and np.array_equal(D, D2)


@pytest.mark.gpu
def test_very_near_pairs_in_contact_are_reported_not_refined_forever():
    """The lists are classified on the construction-time coordinates; after a
    SemiStaticUpdate that pushes the lower sphere 0.01 into the upper one (0.0078 apart at
    construction), the very-near pairs intersect and their energy is infinite. The
    evaluation must end and report it (NaN results, RepulsorError), and a later update that
    separates the spheres again must give the regular energy back."""
    V, S = meshes.reference_mesh("twospheres_union")
    M = rpb.SimplicialMesh(V, S)
    tpe = rpb.TangentPointEnergy0(Q, P)
    E0 = tpe.Value(M)
    W = V.copy()
    W[162:, 2] += 0.01
    M.SemiStaticUpdate(W)
    with pytest.raises(rpb.RepulsorError, match="touch or intersect"):
        tpe.Value(M)
    M.SemiStaticUpdate(V)
    assert tpe.Value(M) == E0
