"""repulsor_b200 -- B200 implementation of Repulsor's multipole-accelerated
tangent-point path behind Repulsor's own interface.

Host-side mirror of the reference classes (HenrikSchumacher/Repulsor):

* ``SimplicialMesh``        src/SimplicialMesh.hpp (construction builds the cluster
                            tree and block cluster tree, src/SimplicialMesh.hpp:470-607)
* ``TangentPointEnergy0``   src/Energies/TangentPointEnergy0.hpp with the EnergyBase
                            interface (Value / Differential, src/Energies/EnergyBase.hpp:40-121)
* ``TangentPointMetric0``   src/Metrics/TangentPointMetric0.hpp with the MetricBase
                            interface (MultiplyMetric / MultiplyPreconditioner / Solve,
                            src/Metrics/MetricBase.hpp:31-134)

Every call goes through the C ABI of ``librepulsor_b200.so`` (include/repulsor_b200.h).
Arguments follow the reference: ``Y = alpha * result + beta * Y``, ``nrhs`` must be the
ambient dimension 3, and argument errors raise ``RepulsorError`` where the reference
prints an error and does nothing.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from .meshio import read_mesh_file, write_mesh_file
from ._capi import (PRECOND_HYBRID, PRECOND_LEARNED, PRECOND_NONE, PRECOND_REFERENCE, RepulsorError, Settings, Stats,
                    check, dptr, iptr, lptr)

__all__ = [
    "SimplicialMesh",
    "HostTree",
    "TangentPointEnergy0",
    "TangentPointMetric0",
    "TangentPointObstacleEnergy",
    "SimplicialMesh_Factory",
    "TangentPointEnergy0_Factory",
    "TangentPointMetric0_Factory",
    "TangentPointObstacleEnergy_Factory",
    "read_mesh_file",
    "write_mesh_file",
    "RepulsorError",
    "PRECOND_NONE",
    "PRECOND_REFERENCE",
    "PRECOND_LEARNED",
    "PRECOND_HYBRID",
    "default_settings",
]


def default_settings(**overrides) -> Settings:
    """Reference defaults (src/Settings.hpp:5-54) with optional overrides."""
    s = Settings()
    check(_capi.load().rpb_default_settings(ctypes.byref(s)), "rpb_default_settings")
    for k, v in overrides.items():
        setattr(s, k, v)
    return s


class SimplicialMesh:
    """SimplicialMesh<DOM_DIM, 3, double, int, size_t> on a CUDA device.

    ``V``: (n_v, 3) float64 vertex coordinates, ``S``: (n_s, dom+1) int32 simplices.
    The tree is built from these (frozen) coordinates and kept across
    ``SemiStaticUpdate`` calls, as in the reference.
    """

    def __init__(self, V, S, charges=None, settings: Settings | None = None, device: int = 0, **overrides):
        lib = _capi.load()
        V = np.ascontiguousarray(V, dtype=np.float64)
        S = np.ascontiguousarray(S, dtype=np.int32)
        if V.ndim != 2 or V.shape[1] != 3:
            raise RepulsorError(_capi.RPB_EINVAL, "SimplicialMesh: V.Dim(1) != AMB_DIM = 3")
        if S.ndim != 2 or S.shape[1] not in (2, 3):
            raise RepulsorError(_capi.RPB_EINVAL, "SimplicialMesh: simplices.Dim(1) must be 2 (curves) or 3 (surfaces)")
        self.dom = S.shape[1] - 1
        self.nV = V.shape[0]
        self.nS = S.shape[0]
        if settings is None:
            settings = default_settings(device=device, **overrides)
        ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        h = ctypes.c_void_p()
        check(lib.rpb_mesh_create(self.dom, 3, dptr(V), self.nV, iptr(S), self.nS,
                                  None if ch is None else dptr(ch), ctypes.byref(settings), ctypes.byref(h)),
              "SimplicialMesh")
        self._h = h
        self._V = V
        self._S = S
        self._cache = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_owned", True) and _capi is not None and _capi._lib is not None:
            _capi._lib.rpb_mesh_destroy(h)
            self._h = None

    # --- reference accessors -------------------------------------------------------------
    def DomDim(self):
        return self.dom

    def AmbDim(self):
        return 3

    def VertexCount(self):
        return self.nV

    def SimplexCount(self):
        return self.nS

    def VertexCoordinates(self):
        return self._V

    def ClearCache(self):
        self._cache.clear()

    def WriteToFile(self, path):
        """SimplicialMesh::WriteToFile (src/SimplicialMesh.hpp:780-818): the current
        coordinates and the simplices in the reference's mesh text format."""
        write_mesh_file(path, self._V, self._S)

    def MaximumSafeStepSize(self, velocities, max_time: float, TOL: float = 0.0625) -> float:
        """SimplicialMesh::MaximumSafeStepSize (src/SimplicialMesh.hpp:441-468): the largest
        t <= max_time for which moving every vertex by t * velocities (n_v x 3) keeps the
        primitives without a common vertex apart (construction-time coordinates, as the
        reference's collision tree uses)."""
        vel = np.ascontiguousarray(velocities, dtype=np.float64)
        if vel.shape != (self.nV, 3):
            raise ValueError(f"velocities must be ({self.nV}, 3)")
        t = ctypes.c_double()
        check(_capi.load().rpb_mesh_maximum_safe_step_size(self._h, dptr(vel), float(max_time), float(TOL),
                                                           ctypes.byref(t)), "MaximumSafeStepSize")
        return t.value

    def SemiStaticUpdate(self, V, transp: bool = False):
        """New coordinates with the same tree and pair lists (src/SimplicialMesh.hpp:354-376)."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        check(_capi.load().rpb_mesh_semistatic_update(self._h, dptr(V), int(bool(transp))), "SemiStaticUpdate")
        self._V = V if not transp else np.ascontiguousarray(V.reshape(3, -1).T)
        self._cache.clear()

    def SemiStaticUpdateDevice(self, V_dev_ptr: int):
        """SemiStaticUpdate from a device pointer (n_v x 3 float64) on the mesh stream."""
        check(_capi.load().rpb_mesh_semistatic_update_device(self._h, ctypes.c_void_p(V_dev_ptr)),
              "SemiStaticUpdateDevice")
        self._cache.clear()

    def LoadObstacle(self, obstacle: "SimplicialMesh"):
        """SimplicialMesh::LoadObstacle (src/SimplicialMesh.hpp:697-719): the mesh takes the
        obstacle over (the obstacle object stays usable for reading, the mesh destroys it)."""
        check(_capi.load().rpb_mesh_load_obstacle(self._h, obstacle._h), "LoadObstacle")
        obstacle._owned = False
        self._obstacle = obstacle
        self._cache.clear()

    def obstacle_stats(self) -> dict:
        c = np.zeros(4, np.int64)
        check(_capi.load().rpb_mesh_obstacle_stats(self._h, lptr(c)), "rpb_mesh_obstacle_stats")
        return dict(zip(["near_nnz", "far_nnz", "verynear_nnz", "inter_nnz"], c.tolist()))

    def obstacle_pattern(self, which: str):
        """'near' | 'far' | 'verynear' | 'inter' -> (rowptr int64, colidx int32) of the obstacle lists."""
        w = {"near": 0, "far": 1, "verynear": 2, "inter": 3}[which]
        rows = self.stats()["cluster_count"] if which == "far" else self.nS
        nnz = self.obstacle_stats()[which + "_nnz"]
        rp = np.zeros(rows + 1, np.int64)
        ci = np.zeros(max(nnz, 1), np.int32)
        check(_capi.load().rpb_mesh_obstacle_pattern(self._h, w, lptr(rp), iptr(ci)), "rpb_mesh_obstacle_pattern")
        return rp, ci[:nnz]

    # --- B200 extras ---------------------------------------------------------------------
    def stats(self) -> dict:
        st = Stats()
        check(_capi.load().rpb_mesh_stats(self._h, ctypes.byref(st)), "rpb_mesh_stats")
        return {name: getattr(st, name) for name, _ in Stats._fields_}

    def build_info(self) -> dict:
        """Where the cluster tree and the block cluster tree were built (True: on the GPU,
        False: on host threads after the device work failed)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        check(_capi.load().rpb_mesh_build_info(self._h, ctypes.byref(a), ctypes.byref(b)), "rpb_mesh_build_info")
        return {"cluster_tree_on_device": bool(a.value), "block_tree_on_device": bool(b.value)}

    def stream(self) -> int:
        p = ctypes.c_void_p()
        check(_capi.load().rpb_mesh_get_stream(self._h, ctypes.byref(p)), "rpb_mesh_get_stream")
        return p.value or 0

    def set_stream(self, stream_ptr: int | None):
        check(_capi.load().rpb_mesh_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)), "rpb_mesh_set_stream")

    def tree(self) -> dict:
        st = self.stats()
        N, NC = st["simplex_count"], st["cluster_count"]
        perm = np.zeros(N, np.int32)
        arr = [np.zeros(NC, np.int32) for _ in range(4)]
        check(_capi.load().rpb_mesh_tree(self._h, iptr(perm), *[iptr(a) for a in arr]), "rpb_mesh_tree")
        return dict(perm=perm, C_begin=arr[0], C_end=arr[1], C_left=arr[2], C_right=arr[3])

    def pattern(self, which: str):
        """'near' | 'far' | 'verynear' | 'inter' -> (rowptr int64, colidx int32), full symmetric CSR."""
        w = {"near": 0, "far": 1, "verynear": 2, "inter": 3}[which]
        st = self.stats()
        rows = st["cluster_count"] if which == "far" else st["simplex_count"]
        nnz = st[{"near": "near_nnz", "far": "far_nnz", "verynear": "verynear_nnz", "inter": "inter_nnz"}[which]]
        rp = np.zeros(rows + 1, np.int64)
        ci = np.zeros(max(nnz, 1), np.int32)
        check(_capi.load().rpb_mesh_pattern(self._h, w, lptr(rp), iptr(ci)), "rpb_mesh_pattern")
        return rp, ci[:nnz]


class HostTree:
    """Cluster tree + block cluster tree built on the host only (no device needed)."""

    def __init__(self, V, S, settings: Settings | None = None, **overrides):
        lib = _capi.load()
        V = np.ascontiguousarray(V, dtype=np.float64)
        S = np.ascontiguousarray(S, dtype=np.int32)
        self.dom = S.shape[1] - 1
        if settings is None:
            settings = default_settings(**overrides)
        h = ctypes.c_void_p()
        check(lib.rpb_tree_build_host(self.dom, dptr(V), V.shape[0], iptr(S), S.shape[0], ctypes.byref(settings),
                                      ctypes.byref(h)), "rpb_tree_build_host")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _capi is not None and _capi._lib is not None:
            _capi._lib.rpb_tree_host_destroy(h)
            self._h = None

    def stats(self) -> dict:
        st = Stats()
        check(_capi.load().rpb_tree_host_stats(self._h, ctypes.byref(st)), "rpb_tree_host_stats")
        return {name: getattr(st, name) for name, _ in Stats._fields_}

    def tree(self) -> dict:
        st = self.stats()
        N, NC = st["simplex_count"], st["cluster_count"]
        perm = np.zeros(N, np.int32)
        arr = [np.zeros(NC, np.int32) for _ in range(4)]
        check(_capi.load().rpb_tree_host_arrays(self._h, iptr(perm), *[iptr(a) for a in arr]), "rpb_tree_host_arrays")
        return dict(perm=perm, C_begin=arr[0], C_end=arr[1], C_left=arr[2], C_right=arr[3])

    def pattern(self, which: str):
        w = {"near": 0, "far": 1, "verynear": 2, "inter": 3}[which]
        st = self.stats()
        rows = st["cluster_count"] if which == "far" else st["simplex_count"]
        nnz = st[{"near": "near_nnz", "far": "far_nnz", "verynear": "verynear_nnz", "inter": "inter_nnz"}[which]]
        rp = np.zeros(rows + 1, np.int64)
        ci = np.zeros(max(nnz, 1), np.int32)
        check(_capi.load().rpb_tree_host_pattern(self._h, w, lptr(rp), iptr(ci)), "rpb_tree_host_pattern")
        return rp, ci[:nnz]

    def obstacle_pattern(self, V, S, obstacle: "HostTree", VO, SO, which: str):
        """Obstacle list `which` of this tree (built from V, S) against `obstacle` (built
        from VO, SO), as rpb_mesh_load_obstacle builds it: (rowptr, colidx, counts)."""
        lib = _capi.load()
        w = {"near": 0, "far": 1, "verynear": 2, "inter": 3}[which]
        V = np.ascontiguousarray(V, dtype=np.float64)
        S = np.ascontiguousarray(S, dtype=np.int32)
        VO = np.ascontiguousarray(VO, dtype=np.float64)
        SO = np.ascontiguousarray(SO, dtype=np.int32)
        counts = np.zeros(4, np.int64)
        args = (self._h, dptr(V), iptr(S), obstacle._h, dptr(VO), iptr(SO), w, lptr(counts))
        check(lib.rpb_tree_host_obstacle_pattern(*args, None, None), "rpb_tree_host_obstacle_pattern")
        st = self.stats()
        rows = st["cluster_count"] if which == "far" else st["simplex_count"]
        nnz = int(counts[w])
        rp = np.zeros(rows + 1, np.int64)
        ci = np.zeros(max(nnz, 1), np.int32)
        check(lib.rpb_tree_host_obstacle_pattern(*args, lptr(rp), iptr(ci)), "rpb_tree_host_obstacle_pattern")
        return rp, ci[:nnz], dict(zip(["near", "far", "verynear", "inter"], counts.tolist()))

    def h1_solve(self, V, S, B):
        """X = H1^{-1} B on the host (nested-dissection sparse Cholesky)."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        S = np.ascontiguousarray(S, dtype=np.int32)
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.zeros_like(B)
        check(_capi.load().rpb_h1_solve_host(self._h, dptr(V), iptr(S), dptr(B), dptr(X), B.shape[1]),
              "rpb_h1_solve_host")
        return X


def _as_mesh(M):
    if not isinstance(M, SimplicialMesh):
        raise RepulsorError(_capi.RPB_EINVAL, "Input could not be downcast to compatible type")
    return M


class TangentPointEnergy0:
    """TangentPointEnergy0(q, p) or TangentPointEnergy0(p) with q = p, p = 2p
    (src/Energies/TangentPointEnergy0.hpp:35-45)."""

    def __init__(self, q, p=None):
        if p is None:
            q, p = float(q), 2.0 * float(q)
        self.q = float(q)
        self.p = float(p)

    def ClassName(self):
        return f"TangentPointEnergy0({self.q},{self.p})"

    def Value(self, M: SimplicialMesh) -> float:
        """EnergyBase::Value, cached on the mesh (src/Energies/EnergyBase.hpp:40-56)."""
        M = _as_mesh(M)
        tag = self.ClassName() + "::Value"
        if tag not in M._cache:
            e = ctypes.c_double()
            check(_capi.load().rpb_tpe0_value(M._h, self.q, self.p, ctypes.byref(e)), "Value")
            M._cache[tag] = e.value
        return M._cache[tag]

    def Differential(self, M: SimplicialMesh, alpha=None, beta=0.0, Y=None):
        """Without alpha: cached differential (n_v x 3) (src/Energies/EnergyBase.hpp:62-87).
        With alpha: Y = alpha * dE + beta * Y into the given array, returns the energy
        (src/Energies/EnergyBase.hpp:90-104)."""
        M = _as_mesh(M)
        lib = _capi.load()
        if alpha is None:
            tag = self.ClassName() + "::Differential"
            if tag not in M._cache:
                D = np.zeros((M.nV, 3))
                e = ctypes.c_double()
                check(lib.rpb_tpe0_differential(M._h, self.q, self.p, 1.0, 0.0, dptr(D), 3, ctypes.byref(e)),
                      "Differential")
                M._cache[tag] = D
                M._cache.setdefault(self.ClassName() + "::Value", e.value)
            return M._cache[tag]
        if Y is None:
            Y = np.zeros((M.nV, 3))
        if Y.dtype != np.float64 or not Y.flags.c_contiguous or Y.shape[0] != M.nV or Y.shape[1] < 3:
            raise RepulsorError(_capi.RPB_EINVAL, "Differential: Y must be a C-contiguous float64 (n_v, ldY>=3) array")
        e = ctypes.c_double()
        check(lib.rpb_tpe0_differential(M._h, self.q, self.p, float(alpha), float(beta), dptr(Y), Y.shape[1],
                                        ctypes.byref(e)), "Differential")
        return e.value

    def SimplexDensities(self, M: SimplicialMesh, density=None):
        """Energy density per simplex into `density` (n_s, original order); returns the
        energy (src/Energies/EnergyBase.hpp:129-137). Without `density`, returns
        (energy, densities)."""
        return self._densities(M, density, "simplex")

    def VertexDensities(self, M: SimplicialMesh, density=None):
        """Energy density per vertex into `density` (n_v); returns the energy
        (src/Energies/EnergyBase.hpp:140-148). Without `density`, returns (energy, densities)."""
        return self._densities(M, density, "vertex")

    def _densities(self, M, density, kind):
        M = _as_mesh(M)
        n = M.nS if kind == "simplex" else M.nV
        given = density is not None
        out = density if given else np.zeros(n)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != n:
            raise RepulsorError(_capi.RPB_EINVAL, f"{kind} densities need a contiguous float64 array of {n} values")
        e = ctypes.c_double()
        fn = _capi.load().rpb_tpe0_simplex_densities if kind == "simplex" else _capi.load().rpb_tpe0_vertex_densities
        check(fn(M._h, self.q, self.p, dptr(out), ctypes.byref(e)), f"{kind.capitalize()}Densities")
        return e.value if given else (e.value, out)

    def DifferentialDevice(self, M: SimplicialMesh, Y_dev_ptr: int, ldY: int = 3, alpha=1.0, beta=0.0,
                           want_energy: bool = True):
        """Y (device pointer, n_v x ldY float64) = alpha dE + beta Y on the mesh stream.
        Returns the energy (synchronizing) or, with want_energy=False, None without any
        synchronization (the call can then be captured into a CUDA graph)."""
        e = ctypes.c_double()
        check(_capi.load().rpb_tpe0_differential_device(M._h, self.q, self.p, float(alpha), float(beta),
                                                        ctypes.c_void_p(Y_dev_ptr), ldY,
                                                        ctypes.byref(e) if want_energy else None),
              "DifferentialDevice")
        return e.value if want_energy else None


class TangentPointObstacleEnergy:
    """TangentPointObstacleEnergy(q, p) of a mesh against its loaded obstacle
    (src/Energies/TangentPointObstacleEnergy.hpp:48-96); 0 without an obstacle."""

    def __init__(self, q, p=None):
        if p is None:
            q, p = float(q), 2.0 * float(q)
        self.q = float(q)
        self.p = float(p)

    def ClassName(self):
        return f"TangentPointObstacleEnergy({self.q},{self.p})"

    def Value(self, M: SimplicialMesh) -> float:
        M = _as_mesh(M)
        tag = self.ClassName() + "::Value"
        if tag not in M._cache:
            e = ctypes.c_double()
            check(_capi.load().rpb_tpoe_value(M._h, self.q, self.p, ctypes.byref(e)), "Value")
            M._cache[tag] = e.value
        return M._cache[tag]

    def Differential(self, M: SimplicialMesh, alpha=None, beta=0.0, Y=None):
        """As TangentPointEnergy0.Differential; derivatives with respect to M's vertices."""
        M = _as_mesh(M)
        lib = _capi.load()
        if alpha is None:
            tag = self.ClassName() + "::Differential"
            if tag not in M._cache:
                D = np.zeros((M.nV, 3))
                e = ctypes.c_double()
                check(lib.rpb_tpoe_differential(M._h, self.q, self.p, 1.0, 0.0, dptr(D), 3, ctypes.byref(e)),
                      "Differential")
                M._cache[tag] = D
                M._cache.setdefault(self.ClassName() + "::Value", e.value)
            return M._cache[tag]
        if Y is None:
            Y = np.zeros((M.nV, 3))
        if Y.dtype != np.float64 or not Y.flags.c_contiguous or Y.shape[0] != M.nV or Y.shape[1] < 3:
            raise RepulsorError(_capi.RPB_EINVAL, "Differential: Y must be a C-contiguous float64 (n_v, ldY>=3) array")
        e = ctypes.c_double()
        check(lib.rpb_tpoe_differential(M._h, self.q, self.p, float(alpha), float(beta), dptr(Y), Y.shape[1],
                                        ctypes.byref(e)), "Differential")
        return e.value

    def DifferentialDevice(self, M: SimplicialMesh, Y_dev_ptr: int, ldY: int = 3, alpha=1.0, beta=0.0) -> float:
        e = ctypes.c_double()
        check(_capi.load().rpb_tpoe_differential_device(M._h, self.q, self.p, float(alpha), float(beta),
                                                        ctypes.c_void_p(Y_dev_ptr), ldY, ctypes.byref(e)),
              "DifferentialDevice")
        return e.value


class TangentPointMetric0:
    """TangentPointMetric0(q, p) or TangentPointMetric0(p) with q = p, p = 2p
    (src/Metrics/TangentPointMetric0.hpp:31-45)."""

    def __init__(self, q, p=None):
        if p is None:
            q, p = float(q), 2.0 * float(q)
        self.q = float(q)
        self.p = float(p)
        self.iter = 0
        self.rel_residuals = np.zeros(3)

    def ClassName(self):
        return f"TangentPointMetric0({self.q},{self.p})"

    @staticmethod
    def _check_nrhs(nrhs, tag):
        if nrhs != 3:
            raise RepulsorError(_capi.RPB_EINVAL, f"{tag}: nrhs = {nrhs} != 3 = AMB_DIM")

    def MultiplyMetric(self, M, alpha, X, beta=0.0, Y=None, VF_flag=True, NF_flag=True, FF_flag=True):
        """Y = alpha * A X + beta * Y (src/Metrics/MetricDimRestricted.hpp:109-139)."""
        M = _as_mesh(M)
        X = np.ascontiguousarray(X, dtype=np.float64)
        self._check_nrhs(X.shape[1], "MultiplyMetric")
        if Y is None:
            Y = np.zeros((M.nV, 3))
        flags = (1 if VF_flag else 0) | (2 if NF_flag else 0) | (4 if FF_flag else 0)
        check(_capi.load().rpb_tpm0_multiply(M._h, self.q, self.p, float(alpha), dptr(X), X.shape[1], float(beta),
                                             dptr(Y), Y.shape[1], X.shape[1], flags), "MultiplyMetric")
        return Y

    def MultiplyMetricDevice(self, M, alpha, X_dev_ptr, beta, Y_dev_ptr, ldX=3, ldY=3, flags=7):
        check(_capi.load().rpb_tpm0_multiply_device(M._h, self.q, self.p, float(alpha), ctypes.c_void_p(X_dev_ptr),
                                                    ldX, float(beta), ctypes.c_void_p(Y_dev_ptr), ldY, 3, flags),
              "MultiplyMetricDevice")

    def MultiplyPreconditioner(self, M, alpha, X, beta=0.0, Y=None):
        """Y = alpha * H1^{-1} L_{2-s} H1^{-1} X + beta * Y (src/Metrics/TangentPointMetric0.hpp:88-126)."""
        M = _as_mesh(M)
        X = np.ascontiguousarray(X, dtype=np.float64)
        self._check_nrhs(X.shape[1], "MultiplyPreconditioner")
        if Y is None:
            Y = np.zeros((M.nV, 3))
        check(_capi.load().rpb_tpm0_precondition(M._h, self.q, self.p, float(alpha), dptr(X), X.shape[1],
                                                 float(beta), dptr(Y), Y.shape[1], X.shape[1]),
              "MultiplyPreconditioner")
        return Y

    def Solve(self, M, alpha, B, beta=0.0, X=None, max_iter=1000, tolerance=1e-6, precond=PRECOND_REFERENCE,
              strict=True):
        """X = alpha * A^{-1} B + beta * X (src/Metrics/MetricDimRestricted.hpp:232-289).

        The iterate after max_iter iterations is returned in every case; with strict=True
        a missed tolerance raises RepulsorError (RPB_ENOTCONV) after the statistics
        (Solver_IterationCount, Solver_RelativeResiduals) have been recorded."""
        M = _as_mesh(M)
        B = np.ascontiguousarray(B, dtype=np.float64)
        self._check_nrhs(B.shape[1], "Solve")
        if X is None:
            X = np.zeros((M.nV, 3))
        it = ctypes.c_int()
        rr = np.zeros(3)
        st = _capi.load().rpb_tpm0_solve(M._h, self.q, self.p, float(alpha), dptr(B), B.shape[1], float(beta),
                                         dptr(X), X.shape[1], B.shape[1], int(max_iter), float(tolerance),
                                         int(precond), ctypes.byref(it), dptr(rr))
        self.iter = it.value
        self.rel_residuals = rr
        if st != _capi.RPB_ENOTCONV or strict:
            check(st, "Solve")
        return X

    def Solver_IterationCount(self):
        return self.iter

    @staticmethod
    def SolveInfo(M) -> dict:
        """Statistics of the last Solve on M: iterations, restarts, fallback_iteration (-1: the
        learned preconditioner never fell back), supernode_levels, factor_seconds, factor_nnz,
        factor_on_device (1: the H1 factor's numeric phase ran on the GPU)."""
        info = _capi.SolveInfo()
        check(_capi.load().rpb_tpm0_solve_info(_as_mesh(M)._h, ctypes.byref(info)), "rpb_tpm0_solve_info")
        return {name: getattr(info, name) for name, _ in _capi.SolveInfo._fields_}

    def Solver_RelativeResiduals(self):
        return self.rel_residuals

    def MetricNorm(self, M, X):
        """sqrt(<X, A X>) (src/Metrics/MetricBase.hpp:79-100)."""
        Y = self.MultiplyMetric(M, 1.0, X)
        return float(np.sqrt(np.sum(np.asarray(X) * Y)))

    def PreconditionerNorm(self, M, X):
        Y = self.MultiplyPreconditioner(M, 1.0, X)
        return float(np.sqrt(np.sum(np.asarray(X) * Y)))


class SimplicialMesh_Factory:
    """SimplicialMesh_Factory<MeshBase_T, min_dom, max_dom, min_amb, max_amb>
    (src/SimplicialMesh/SimplicialMesh_Factory.hpp:8-246): meshes whose dimensions lie in
    the factory's ranges; this build has domain dimensions 1 and 2 in ambient dimension 3."""

    def __init__(self, min_dom=1, max_dom=2, min_amb=3, max_amb=3):
        self.min_dom, self.max_dom, self.min_amb, self.max_amb = min_dom, max_dom, min_amb, max_amb

    def Make(self, vertex_coords, vertex_count, amb_dim, vertex_coords_ColMajorQ, simplices, simplex_count,
             simplex_size, simplices_ColMajorQ, thread_count=1, **settings):
        dom_dim = simplex_size - 1
        if not self.min_dom <= dom_dim <= self.max_dom:
            raise RepulsorError(_capi.RPB_EINVAL, "SimplicialMesh_Factory::Make: dom_dim is out of range.")
        if not self.min_amb <= amb_dim <= self.max_amb:
            raise RepulsorError(_capi.RPB_EINVAL, "SimplicialMesh_Factory::Make: amb_dim is out of range.")
        if amb_dim != 3 or dom_dim not in (1, 2):
            raise RepulsorError(_capi.RPB_EINVAL, f"SimplicialMesh_Factory cannot create SimplicialMesh with domain "
                                f"dimension {dom_dim} and ambient dimension {amb_dim}.")
        V = np.asarray(vertex_coords, dtype=np.float64).reshape(-1)
        S = np.asarray(simplices).reshape(-1)
        V = V.reshape(amb_dim, vertex_count).T if vertex_coords_ColMajorQ else V.reshape(vertex_count, amb_dim)
        S = S.reshape(simplex_size, simplex_count).T if simplices_ColMajorQ else S.reshape(simplex_count, simplex_size)
        return SimplicialMesh(V, S.astype(np.int32), thread_count=max(1, int(thread_count)), **settings)

    def Make_FromFile(self, path, thread_count=1, **settings):
        """Reads a mesh in the reference's text format (read_mesh_file) and makes it."""
        dom, amb, V, S = read_mesh_file(path)
        return self.Make(V, V.shape[0], amb, False, S, S.shape[0], dom + 1, False, thread_count, **settings)


class TangentPointEnergy0_Factory:
    """Runtime dispatch on (dom_dim, amb_dim) (src/Energies/TangentPointEnergy/TP_Factory.hpp:24-44)."""

    @staticmethod
    def Make(dom_dim, amb_dim, q, p):
        if amb_dim != 3 or dom_dim not in (1, 2):
            raise RepulsorError(_capi.RPB_EINVAL, "TangentPointEnergy0_Factory: only (1,3) and (2,3) are built")
        return TangentPointEnergy0(q, p)


class TangentPointMetric0_Factory:
    @staticmethod
    def Make(dom_dim, amb_dim, q, p):
        if amb_dim != 3 or dom_dim not in (1, 2):
            raise RepulsorError(_capi.RPB_EINVAL, "TangentPointMetric0_Factory: only (1,3) and (2,3) are built")
        return TangentPointMetric0(q, p)


class TangentPointObstacleEnergy_Factory:
    """Make(dom_dim_S, dom_dim_T, amb_dim, q, p) (src/Energies/TangentPointEnergy/TPO_Factory.hpp:8-95);
    the mesh and the obstacle must have the same domain dimension in this build."""

    @staticmethod
    def Make(dom_dim_S, dom_dim_T, amb_dim, q, p):
        if amb_dim != 3 or dom_dim_S not in (1, 2) or dom_dim_T != dom_dim_S:
            raise RepulsorError(_capi.RPB_EINVAL, "TangentPointObstacleEnergy_Factory: only equal domain dimensions "
                                "1 or 2 in ambient dimension 3 are built")
        return TangentPointObstacleEnergy(q, p)
