"""TangentPointEnergy0 Value / Differential on the B200 through the C ABI, against
the FP64 oracle. Tolerances: energy 1e-6 relative; differential 1e-5 relative in
max norm (||D_gpu - D_ref||_inf / ||D_ref||_inf)."""
import ctypes

import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
D_TOL = 1e-5
Q, P = 6.0, 12.0


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _pair(cfg, small):
    dom, (V, S) = meshes.config_mesh(cfg, small=small)
    M = rpb.SimplicialMesh(V, S)
    O = oracle.OracleMesh(dom, V, S, threads=8)
    return dom, V, S, M, O


@pytest.mark.parametrize("cfg", [1, 2, 3])
@pytest.mark.parametrize("small", [True, False])
def test_energy_and_differential_match_oracle(cfg, small):
    dom, V, S, M, O = _pair(cfg, small)
    tpe = rpb.TangentPointEnergy0(Q, P)
    E = tpe.Value(M)
    E_ref = O.energy(Q, P)
    assert abs(E - E_ref) <= E_TOL * abs(E_ref), (E, E_ref)
    D = np.zeros((V.shape[0], 3))
    E2 = tpe.Differential(M, 1.0, 0.0, D)
    E2_ref, D_ref = O.differential(Q, P)
    assert abs(E2 - E2_ref) <= E_TOL * abs(E2_ref)
    assert rel_max(D, D_ref) <= D_TOL, rel_max(D, D_ref)


def test_differential_alpha_beta_and_ldY():
    dom, V, S, M, O = _pair(2, True)
    tpe = rpb.TangentPointEnergy0(Q, P)
    _, D_ref = O.differential(Q, P)
    Y = np.random.default_rng(0).standard_normal((V.shape[0], 5))
    Y0 = Y.copy()
    tpe.Differential(M, 0.5, 2.0, Y)
    assert rel_max(Y[:, :3], 0.5 * D_ref + 2.0 * Y0[:, :3]) <= D_TOL
    assert np.array_equal(Y[:, 3:], Y0[:, 3:])      # columns beyond AMB_DIM untouched


def test_differential_into_pinned_host_rows():
    """Y in page-locked host memory (torch pin_memory), with ldY = 3 and 5: the rows equal
    those of a pageable Y and the columns beyond AMB_DIM stay untouched."""
    import torch

    dom, V, S, M, O = _pair(2, True)
    tpe = rpb.TangentPointEnergy0(Q, P)
    D = np.zeros((V.shape[0], 3))
    E = tpe.Differential(M, 0.5, 0.0, D)
    for width in (3, 5):
        Yt = torch.full((V.shape[0], width), 7.0, dtype=torch.float64).pin_memory()
        Y = Yt.numpy()
        E2 = tpe.Differential(M, 0.5, 0.0, Y)
        assert E2 == E
        assert np.array_equal(Y[:, :3], D)
        assert np.all(Y[:, 3:] == 7.0)


def test_cached_differential_and_value_consistency():
    dom, V, S, M, O = _pair(1, True)
    tpe = rpb.TangentPointEnergy0(Q, P)
    D = tpe.Differential(M)
    assert D.shape == (V.shape[0], 3)
    assert tpe.Differential(M) is D                  # cached on the mesh like the reference
    assert tpe.Value(M) == pytest.approx(O.energy(Q, P), rel=E_TOL)


def test_semistatic_update_matches_oracle():
    dom, V, S, M, O = _pair(3, True)
    rng = np.random.default_rng(7)
    V2 = V + 1e-3 * rng.standard_normal(V.shape)
    M.SemiStaticUpdate(V2)
    O.semistatic_update(V2)
    tpe = rpb.TangentPointEnergy0(Q, P)
    D = np.zeros_like(V2)
    E = tpe.Differential(M, 1.0, 0.0, D)
    E_ref, D_ref = O.differential(Q, P)
    assert abs(E - E_ref) <= E_TOL * abs(E_ref)
    assert rel_max(D, D_ref) <= D_TOL


@pytest.mark.parametrize("cfg", [2, 3])
def test_full_size_invariants(cfg):
    """Size-independent properties at the benchmark size: translation invariance
    sum_v dE/dx_v = 0 and Euler homogeneity sum_v x_v . dE/dx_v = (2n + q - p) E."""
    dom, (V, S) = meshes.config_mesh(cfg)
    M = rpb.SimplicialMesh(V, S)
    tpe = rpb.TangentPointEnergy0(Q, P)
    D = np.zeros_like(V)
    E = tpe.Differential(M, 1.0, 0.0, D)
    scale = np.abs(D).sum()
    assert np.all(np.abs(D.sum(axis=0)) <= 1e-6 * scale)
    assert abs((V * D).sum() - (2 * dom + Q - P) * E) <= 1e-5 * abs(E)


def test_other_exponents_generic_path():
    dom, V, S, M, O = _pair(2, True)
    for q, p in [(4.0, 8.0), (6.0, 13.0), (2.5, 7.0)]:
        tpe = rpb.TangentPointEnergy0(q, p)
        D = np.zeros_like(V)
        E = tpe.Differential(M, 1.0, 0.0, D)
        E_ref, D_ref = O.differential(q, p)
        assert abs(E - E_ref) <= 1e-5 * abs(E_ref), (q, p)
        assert rel_max(D, D_ref) <= 1e-4, (q, p)


def test_energy_rejects_bad_exponents():
    dom, V, S, M, O = _pair(1, True)
    with pytest.raises(rpb.RepulsorError):
        rpb.TangentPointEnergy0(1.0, 4.0).Value(M)


@pytest.mark.parametrize("cfg", [1, 2, 3])
def test_densities_match_oracle(cfg):
    """EnergyBase::SimplexDensities / VertexDensities against the oracle; the simplex
    densities weighted by the simplex weights sum to the energy."""
    dom, (V, S) = meshes.config_mesh(cfg, small=True)
    M = rpb.SimplicialMesh(V, S)
    om = oracle.OracleMesh(dom, V, S, threads=8)
    tpe = rpb.TangentPointEnergy0(6.0, 12.0)
    E, rho = tpe.SimplexDensities(M)
    E_ref, rho_ref = om.simplex_densities()
    assert abs(E - E_ref) <= E_TOL * abs(E_ref)
    assert np.abs(rho - rho_ref).max() <= D_TOL * np.abs(rho_ref).max()
    Ev, rv = tpe.VertexDensities(M)
    _, rv_ref = om.vertex_densities()
    assert np.abs(rv - rv_ref).max() <= D_TOL * np.abs(rv_ref).max()
    Pn, _ = om.primitive_data()
    a = np.zeros(S.shape[0])
    a[om.tree()["perm"]] = Pn[:, 0]
    assert abs((a * rho).sum() - E) <= 1e-6 * abs(E)


def test_differential_in_a_cuda_graph_matches_direct_call():
    """SemiStaticUpdateDevice + DifferentialDevice without an energy readback capture into
    a CUDA graph; replaying it (and rpb_tpe0_energy_device) gives the direct results."""
    torch = pytest.importorskip("torch")
    from repulsor_b200 import _capi

    dom, (V, S) = meshes.config_mesh(2, small=True)
    M = rpb.SimplicialMesh(V, S)
    tpe = rpb.TangentPointEnergy0(6.0, 12.0)
    D_ref = np.zeros_like(V)
    E_ref = tpe.Differential(M, 1.0, 0.0, D_ref)
    s = torch.cuda.Stream()
    M.set_stream(s.cuda_stream)
    Vd = torch.tensor(V * 1.0, device="cuda")
    Yd = torch.zeros((V.shape[0], 3), dtype=torch.float64, device="cuda")
    Ed = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = _capi.load()

    def step():
        M.SemiStaticUpdateDevice(Vd.data_ptr())
        tpe.DifferentialDevice(M, Yd.data_ptr(), 3, 1.0, 0.0, want_energy=False)
        _capi.check(lib.rpb_tpe0_energy_device(M._h, ctypes.c_void_p(Ed.data_ptr())), "energy_device")

    with torch.cuda.stream(s):
        step()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        step()
    Yd.zero_()
    Ed.zero_()
    with torch.cuda.stream(s):
        g.replay()
    torch.cuda.synchronize()
    assert abs(float(Ed.item()) - E_ref) <= 1e-12 * abs(E_ref)
    np.testing.assert_allclose(Yd.cpu().numpy(), D_ref, rtol=0, atol=1e-12 * np.abs(D_ref).max())
