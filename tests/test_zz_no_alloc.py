"""rpb_tpe0_value_noalloc: the energy entry point for callers that cannot allocate device
memory when they need the energy (hosts whose device memory belongs to a fixed-size arena
or pool, real-time loops that forbid allocation after start-up). Its result must match the
regular TangentPointEnergy0.Value entry point (rpb_tpe0_value) and the FP64 oracle within
the energy tolerance of the other GPU tests, on two calls in a row (the shared static
scratch keeps the previous call's contents, so the second call checks that everything that
must start at zero is cleared). Meshes it cannot evaluate (too large, very-near pairs, a
cluster count that does not fit the mesh) must be rejected with RPB_EINVAL."""
import ctypes

import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import _capi, meshes

pytestmark = pytest.mark.gpu

E_TOL = 1e-6       # relative, as in tests/test_gpu_energy.py
MAX_SIMPLICES = 40960


def _device_arrays(torch, M, V, S):
    t = M.tree()
    nrp, nci = M.pattern("near")
    frp, fci = M.pattern("far")
    dev = torch.device("cuda", 0)
    return dict(
        V=torch.tensor(V, dtype=torch.float64, device=dev),
        S=torch.tensor(S, dtype=torch.int32, device=dev),
        perm=torch.tensor(t["perm"], dtype=torch.int32, device=dev),
        C_begin=torch.tensor(t["C_begin"], dtype=torch.int32, device=dev),
        C_end=torch.tensor(t["C_end"], dtype=torch.int32, device=dev),
        nrp=torch.tensor(nrp, dtype=torch.int64, device=dev),
        nci=torch.tensor(nci, dtype=torch.int32, device=dev),
        frp=torch.tensor(frp, dtype=torch.int64, device=dev),
        fci=torch.tensor(fci, dtype=torch.int32, device=dev),
        nC=len(t["C_begin"]),
        vf=int(M.stats()["verynear_nnz"]),
    )


def _call(lib, d, dom, nV, nS, q, p, out, stream, nC=None, vf=None):
    vp = ctypes.c_void_p
    return lib.rpb_tpe0_value_noalloc(dom, vp(d["V"].data_ptr()), nV, vp(d["S"].data_ptr()), nS,
                                      vp(d["perm"].data_ptr()), vp(d["C_begin"].data_ptr()),
                                      vp(d["C_end"].data_ptr()), d["nC"] if nC is None else nC,
                                      vp(d["nrp"].data_ptr()), vp(d["nci"].data_ptr()), vp(d["frp"].data_ptr()),
                                      vp(d["fci"].data_ptr()), d["vf"] if vf is None else vf,
                                      q, p, vp(out.data_ptr()), vp(stream))


@pytest.mark.parametrize("cfg,small,q,p", [(1, False, 6.0, 12.0), (2, True, 6.0, 12.0), (3, True, 6.0, 12.0),
                                           (2, False, 6.0, 12.0), (2, True, 4.0, 8.0), (1, True, 5.0, 9.0)])
def test_noalloc_energy_matches_regular_entry_point_and_oracle(cfg, small, q, p):
    torch = pytest.importorskip("torch")
    dom, (V, S) = meshes.config_mesh(cfg, small=small)
    M = rpb.SimplicialMesh(V, S)
    assert M.stats()["verynear_nnz"] == 0
    E_gpu = rpb.TangentPointEnergy0(q, p).Value(M)
    E_orc = oracle.OracleMesh(dom, V, S, threads=8).energy(q, p)
    d = _device_arrays(torch, M, V, S)
    lib = _capi.load()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        _capi.check(_call(lib, d, dom, V.shape[0], S.shape[0], q, p, out, stream), "rpb_tpe0_value_noalloc")
        torch.cuda.synchronize()
        E = float(out.item())
        assert abs(E - E_gpu) <= E_TOL * abs(E_gpu), (E, E_gpu)
        assert abs(E - E_orc) <= E_TOL * abs(E_orc), (E, E_orc)


def test_noalloc_rejects_meshes_beyond_the_scratch_size():
    torch = pytest.importorskip("torch")
    V, S = meshes.icosphere(level=6)          # 81,920 triangles > 40,960
    assert S.shape[0] > MAX_SIMPLICES
    lib = _capi.load()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    vp = ctypes.c_void_p(dummy.data_ptr())
    st = lib.rpb_tpe0_value_noalloc(2, vp, V.shape[0], vp, S.shape[0], vp, vp, vp, 2 * S.shape[0] - 1, vp, vp, vp, vp,
                                    0, 6.0, 12.0, vp, ctypes.c_void_p(0))
    assert st == _capi.RPB_EINVAL
    assert "scratch size" in lib.rpb_last_error().decode()


def test_noalloc_rejects_very_near_pairs_and_foreign_trees():
    torch = pytest.importorskip("torch")
    # two interpenetrating icospheres: the very-near list is not empty
    Va, Sa = meshes.icosphere(level=3, radius=0.5, centre=(-0.45, 0.0, 0.0))
    Vb, Sb = meshes.icosphere(level=3, radius=0.5, centre=(0.45, 0.01, 0.0))
    V, S = np.vstack([Va, Vb]), np.vstack([Sa, Sb + Va.shape[0]]).astype(np.int32)
    M = rpb.SimplicialMesh(V, S)
    d = _device_arrays(torch, M, V, S)
    assert d["vf"] > 0
    lib = _capi.load()
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _call(lib, d, 2, V.shape[0], S.shape[0], 6.0, 12.0, out, stream) == _capi.RPB_EINVAL
    assert "very-near" in lib.rpb_last_error().decode()
    # a cluster count no tree of this mesh can have
    assert _call(lib, d, 2, V.shape[0], S.shape[0], 6.0, 12.0, out, stream, nC=2 * S.shape[0], vf=0) == _capi.RPB_EINVAL
    assert "2 nS - 1" in lib.rpb_last_error().decode()
    torch.cuda.synchronize()
