"""rpb_tpe0_value_noalloc: the energy entry point for callers that cannot allocate device
memory (inside CUDA graph capture, under a fixed memory arena, in loops that forbid
allocation). Its result must match the regular TangentPointEnergy0.Value entry point
(rpb_tpe0_value) within the energy tolerance of the other GPU tests, on two calls in a
row (the shared static scratch keeps the previous call's contents, so the second call
checks that everything that must start at zero is cleared)."""
import ctypes

import numpy as np
import pytest

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
    )


def _call(lib, d, dom, nV, nS, q, p, out, stream):
    vp = ctypes.c_void_p
    return lib.rpb_tpe0_value_noalloc(dom, vp(d["V"].data_ptr()), nV, vp(d["S"].data_ptr()), nS,
                                      vp(d["perm"].data_ptr()), vp(d["C_begin"].data_ptr()),
                                      vp(d["C_end"].data_ptr()), d["nC"], vp(d["nrp"].data_ptr()),
                                      vp(d["nci"].data_ptr()), vp(d["frp"].data_ptr()), vp(d["fci"].data_ptr()),
                                      q, p, vp(out.data_ptr()), vp(stream))


@pytest.mark.parametrize("cfg,small", [(1, False), (2, True), (3, True), (2, False)])
def test_noalloc_energy_matches_regular_entry_point(cfg, small):
    torch = pytest.importorskip("torch")
    dom, (V, S) = meshes.config_mesh(cfg, small=small)
    M = rpb.SimplicialMesh(V, S)
    assert M.stats()["verynear_nnz"] == 0
    E_ref = rpb.TangentPointEnergy0(6.0, 12.0).Value(M)
    d = _device_arrays(torch, M, V, S)
    lib = _capi.load()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        _capi.check(_call(lib, d, dom, V.shape[0], S.shape[0], 6.0, 12.0, out, stream), "rpb_tpe0_value_noalloc")
        torch.cuda.synchronize()
        E = float(out.item())
        assert abs(E - E_ref) <= E_TOL * abs(E_ref), (E, E_ref)


def test_noalloc_rejects_meshes_beyond_the_scratch_size():
    torch = pytest.importorskip("torch")
    V, S = meshes.icosphere(level=6)          # 81,920 triangles > 40,960
    assert S.shape[0] > MAX_SIMPLICES
    lib = _capi.load()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    vp = ctypes.c_void_p(dummy.data_ptr())
    st = lib.rpb_tpe0_value_noalloc(2, vp, V.shape[0], vp, S.shape[0], vp, vp, vp, 2 * S.shape[0] - 1, vp, vp, vp, vp,
                                    6.0, 12.0, vp, ctypes.c_void_p(0))
    assert st == _capi.RPB_EINVAL
    assert "scratch size" in lib.rpb_last_error().decode()
