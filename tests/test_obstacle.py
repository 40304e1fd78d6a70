"""TangentPointObstacleEnergy: the obstacle lists of the host builder against the oracle
(bit-exact, CPU), the oracle's obstacle energy against identities of the mathematics
(all-pairs union identity, finite differences, CPU), and the GPU energy and differential
against the oracle (GPU)."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes

E_TOL = 1e-6       # relative energy, as for TangentPointEnergy0
D_TOL = 1e-5       # relative differential in the max norm


def _circle(n, radius, centre, seed=0):
    rng = np.random.default_rng(seed)
    t = 2 * np.pi * np.arange(n) / n
    V = np.stack([radius * np.cos(t), radius * np.sin(t), np.zeros(n)], 1) + np.asarray(centre)
    V += rng.normal(0, 1e-4 * radius, V.shape)
    S = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1).astype(np.int32)
    return V, S


def _case(name):
    if name == "torus_close_sphere":
        V, S = meshes.torus(R=1.0, r=0.3, n_major=48, n_minor=32, jitter=0.002, seed=11)
        VO, SO = meshes.icosphere(level=2, radius=0.1, centre=(1.0, 0.0, 0.45))
        return 2, V, S, VO, SO
    if name == "linked_tori_sphere":
        V, S = meshes.linked_tori(n_major=48, n_minor=64, seed=1005)
        VO, SO = meshes.icosphere(level=2, radius=0.3, centre=(0.0, 0.0, 2.0))
        return 2, V, S, VO, SO
    if name == "knot_circle":
        V, S = meshes.torus_knot(n=400, seed=1001)
        VO, SO = _circle(150, 0.2, (0.0, 0.0, 0.55))
        return 1, V, S, VO, SO
    raise KeyError(name)


CASES = ["torus_close_sphere", "linked_tori_sphere", "knot_circle"]


@pytest.fixture(scope="module", params=CASES)
def case(request):
    dom, V, S, VO, SO = _case(request.param)
    om = oracle.OracleMesh(dom, V, S, threads=8)
    oo = oracle.OracleMesh(dom, VO, SO, threads=8)
    om.load_obstacle(oo)
    return request.param, dom, V, S, VO, SO, om, oo


def test_obstacle_lists_match_oracle(case):
    name, dom, V, S, VO, SO, om, oo = case
    tm = rpb.HostTree(V, S)
    to = rpb.HostTree(VO, SO)
    for which in ("near", "far", "verynear", "inter"):
        rp, ci, counts = tm.obstacle_pattern(V, S, to, VO, SO, which)
        rp_o, ci_o = om.obstacle_pattern(which)
        np.testing.assert_array_equal(rp, rp_o)
        np.testing.assert_array_equal(ci, ci_o)
    c = om.obstacle_counts()
    assert c["far"] > 0
    if name == "torus_close_sphere":
        assert c["near"] > 0


def test_oracle_obstacle_union_identity():
    """All pairs at primitive level: E_union = E_mesh + E_obstacle + 2 E_cross, where the
    cross sum carries the obstacle energy's symmetry factor 1/2."""
    dom, V, S, VO, SO = _case("torus_close_sphere")
    V, S = meshes.torus(R=1.0, r=0.3, n_major=16, n_minor=12, jitter=0.002, seed=3)
    om = oracle.OracleMesh(dom, V, S, threads=8)
    oo = oracle.OracleMesh(dom, VO, SO, threads=8)
    om.load_obstacle(oo)
    U = oracle.OracleMesh(dom, np.vstack([V, VO]), np.vstack([S, SO + V.shape[0]]), threads=8)
    cross = (U.allpairs_energy() - om.allpairs_energy() - oo.allpairs_energy()) / 2
    assert abs(om.obstacle_allpairs_energy() - cross) <= 1e-12 * abs(cross)


def test_oracle_obstacle_differential_finite_differences(case):
    name, dom, V, S, VO, SO, om, oo = case
    en, D = om.obstacle_differential()
    assert en > 0
    rng = np.random.default_rng(4)
    dX = rng.normal(size=V.shape)
    h = 1e-6 * np.abs(V).max()
    mp = oracle.OracleMesh(dom, V, S, threads=8)
    mp.load_obstacle(oo)
    vals = []
    for sgn in (1, -1):
        mp.semistatic_update(V + sgn * h * dX)
        vals.append(mp.obstacle_energy())
    fd = (vals[0] - vals[1]) / (2 * h)
    an = (D * dX).sum()
    assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-12 * en), (fd, an)


@pytest.mark.gpu
def test_gpu_obstacle_energy_and_differential_match_oracle(case):
    name, dom, V, S, VO, SO, om, oo = case
    M = rpb.SimplicialMesh(V, S)
    O = rpb.SimplicialMesh(VO, SO)
    M.LoadObstacle(O)
    st = M.obstacle_stats()
    assert st == {k + "_nnz": v for k, v in om.obstacle_counts().items()}
    tpo = rpb.TangentPointObstacleEnergy(6.0, 12.0)
    E = tpo.Value(M)
    E_ref = om.obstacle_energy()
    assert abs(E - E_ref) <= E_TOL * abs(E_ref), (E, E_ref)
    D = tpo.Differential(M)
    _, D_ref = om.obstacle_differential()
    assert np.abs(D - D_ref).max() <= D_TOL * np.abs(D_ref).max()
    # alpha/beta/ldY form accumulates onto the self-energy's differential
    Y = rpb.TangentPointEnergy0(6.0, 12.0).Differential(M).copy()
    Y0 = Y.copy()
    tpo.Differential(M, 2.0, 1.0, Y)
    np.testing.assert_allclose(Y, Y0 + 2.0 * D, rtol=0, atol=1e-12 * np.abs(Y0 + 2.0 * D).max())


@pytest.mark.gpu
def test_gpu_obstacle_zero_without_obstacle():
    V, S = meshes.icosphere(level=2)
    M = rpb.SimplicialMesh(V, S)
    tpo = rpb.TangentPointObstacleEnergy(6.0, 12.0)
    assert tpo.Value(M) == 0.0
    Y = np.ones((V.shape[0], 3))
    assert tpo.Differential(M, 1.0, 0.5, Y) == 0.0
    np.testing.assert_array_equal(Y, 0.5)
