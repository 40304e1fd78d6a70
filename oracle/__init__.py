"""ORACLE -- test infrastructure only.

ctypes binding of the CPU FP64 restatement of Repulsor's tangent-point path
(``oracle/tp0_oracle.cpp``) plus the numpy/scipy pieces of the solve (sparse
factorization of the H1 metric, left-preconditioned GMRES and PCG). Used by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtp0_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_int64)


def build():
    """Compile the oracle library with make (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def use_timed_build():
    """Use the build with the reference's optimization flags (-O3 -ffast-math, see the
    Makefile) for this process; only bench.py's CPU baseline does, before its first call.
    Returns the library path."""
    global _LIB_PATH
    if _lib is not None:
        raise RuntimeError("the oracle library is already loaded")
    _LIB_PATH = os.path.join(_HERE, "_build", "libtp0_oracle_timed.so")
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.oracle_create.restype = ctypes.c_void_p
    lib.oracle_create.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, ctypes.c_int, _dp,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.oracle_counts.argtypes = [ctypes.c_void_p, _lp]
    lib.oracle_tree.argtypes = [ctypes.c_void_p, _ip, _ip, _ip, _ip, _ip]
    lib.oracle_pattern.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _ip]
    lib.oracle_cluster_data.argtypes = [ctypes.c_void_p, _dp]
    lib.oracle_primitive_data.argtypes = [ctypes.c_void_p, _dp, _dp]
    lib.oracle_semistatic_update.argtypes = [ctypes.c_void_p, _dp]
    lib.oracle_energy.restype = ctypes.c_double
    lib.oracle_energy.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    lib.oracle_differential.restype = ctypes.c_double
    lib.oracle_differential.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _dp, ctypes.c_int]
    lib.oracle_moment_derivatives.argtypes = [ctypes.c_void_p, _dp, _dp]
    lib.oracle_partial_derivatives.restype = ctypes.c_double
    lib.oracle_partial_derivatives.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                               ctypes.c_int, _dp, _dp]
    lib.oracle_row_derivatives.restype = ctypes.c_double
    lib.oracle_row_derivatives.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                           ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _dp, _dp]
    lib.oracle_pair_opcounts.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, _lp]
    lib.oracle_maximum_safe_step_size.restype = ctypes.c_double
    lib.oracle_maximum_safe_step_size.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_double]
    lib.oracle_collect.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int]
    lib.oracle_allpairs_energy.restype = ctypes.c_double
    lib.oracle_allpairs_energy.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    lib.oracle_metric_values.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]
    lib.oracle_metric_multiply.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           _dp, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int]
    lib.oracle_pseudo_laplacian_multiply.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp,
                                                     ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int]
    lib.oracle_h1_triplet_count.restype = ctypes.c_int64
    lib.oracle_h1_triplet_count.argtypes = [ctypes.c_void_p]
    lib.oracle_h1_triplets.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _ip, _ip, _dp]
    for name in ("oracle_simplex_densities", "oracle_vertex_densities"):
        getattr(lib, name).restype = ctypes.c_double
        getattr(lib, name).argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp]
    lib.oracle_load_obstacle.restype = ctypes.c_int
    lib.oracle_load_obstacle.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.oracle_obstacle_counts.argtypes = [ctypes.c_void_p, _lp]
    lib.oracle_obstacle_pattern.argtypes = [ctypes.c_void_p, ctypes.c_int, _lp, _ip]
    for name in ("oracle_obstacle_energy", "oracle_obstacle_allpairs_energy"):
        getattr(lib, name).restype = ctypes.c_double
        getattr(lib, name).argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    lib.oracle_obstacle_differential.restype = ctypes.c_double
    lib.oracle_obstacle_differential.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_double, _dp, ctypes.c_int]
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _l(a):
    return a.ctypes.data_as(_lp)


def pair_opcounts(dom, far, q=6.0, p=12.0):
    """Arithmetic of one unique pair of the energy + differential traversal (FF loop body
    if far, else the NF loop body for simplices of dimension dom), counted by the oracle's
    operation-counting scalar: {"add", "mul", "div", "sqrt", "pow", "flops"} with flops =
    add + mul + div + sqrt + pow (the source has no fused multiply-adds)."""
    out = np.zeros(5, dtype=np.int64)
    _load().oracle_pair_opcounts(int(dom), int(bool(far)), float(q), float(p), _l(out))
    c = dict(zip(("add", "mul", "div", "sqrt", "pow"), (int(v) for v in out)))
    c["flops"] = sum(c.values())
    return c


class OracleMesh:
    """FP64 CPU restatement of ``SimplicialMesh`` + ``TangentPointEnergy0`` /
    ``TangentPointMetric0`` for one mesh (tree and block cluster tree built on
    construction, as ``GetBlockClusterTree`` does, src/SimplicialMesh.hpp:584-607)."""

    def __init__(self, dom, V, S, theta_far=0.5, theta_near=10.0, max_refinement=30, threads=1, charges=None):
        lib = _load()
        self.dom = int(dom)
        self.V = np.ascontiguousarray(V, dtype=np.float64)
        self.S = np.ascontiguousarray(S, dtype=np.int32)
        self.nV = self.V.shape[0]
        self.nS = self.S.shape[0]
        ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        self._h = lib.oracle_create(self.dom, _d(self.V), self.nV, _i(self.S), self.nS,
                                    None if ch is None else _d(ch), theta_far, theta_near, max_refinement, threads)
        if not self._h:
            raise ValueError("oracle_create rejected the mesh")
        self._h1 = None

    def __del__(self):
        if getattr(self, "_h", None):
            _load().oracle_destroy(self._h)
            self._h = None

    def set_threads(self, threads):
        _load().oracle_set_threads(self._h, int(threads))

    # --- obstacle (TangentPointObstacleEnergy) -------------------------------------------
    def load_obstacle(self, obstacle):
        """Non-symmetric block cluster tree against another OracleMesh (kept referenced)."""
        if _load().oracle_load_obstacle(self._h, obstacle._h) != 0:
            raise ValueError("obstacle domain dimension differs from the mesh's")
        self._obstacle = obstacle

    def obstacle_counts(self):
        out = np.zeros(4, dtype=np.int64)
        _load().oracle_obstacle_counts(self._h, _l(out))
        return dict(zip(["near", "far", "verynear", "inter"], out.tolist()))

    def obstacle_pattern(self, which):
        w = {"near": 0, "far": 1, "verynear": 2, "inter": 3}[which]
        rows = self.counts()["clusters"] if which == "far" else self.nS
        nnz = self.obstacle_counts()[which]
        rp = np.zeros(rows + 1, dtype=np.int64)
        ci = np.zeros(max(nnz, 1), dtype=np.int32)
        _load().oracle_obstacle_pattern(self._h, w, _l(rp), _i(ci))
        return rp, ci[:nnz]

    def obstacle_energy(self, q=6.0, p=12.0):
        return _load().oracle_obstacle_energy(self._h, q, p)

    def obstacle_differential(self, q=6.0, p=12.0, alpha=1.0, beta=0.0, Y=None):
        Y = np.zeros((self.nV, 3)) if Y is None else Y
        en = _load().oracle_obstacle_differential(self._h, q, p, alpha, beta, _d(Y), 3)
        return en, Y

    def obstacle_allpairs_energy(self, q=6.0, p=12.0):
        return _load().oracle_obstacle_allpairs_energy(self._h, q, p)

    def counts(self):
        out = np.zeros(7, dtype=np.int64)
        _load().oracle_counts(self._h, _l(out))
        keys = ["primitives", "clusters", "near_nnz", "far_nnz", "verynear_nnz", "inter_nnz", "depth"]
        return dict(zip(keys, out.tolist()))

    def tree(self):
        c = self.counts()
        N, NC = c["primitives"], c["clusters"]
        perm = np.zeros(N, np.int32)
        arr = [np.zeros(NC, np.int32) for _ in range(4)]
        _load().oracle_tree(self._h, _i(perm), *[_i(a) for a in arr])
        return dict(perm=perm, C_begin=arr[0], C_end=arr[1], C_left=arr[2], C_right=arr[3])

    def pattern(self, which):
        """which: 'near' | 'far' | 'verynear' | 'inter' -> (rowptr int64, colidx int32) full symmetric CSR."""
        w = {"near": 0, "far": 1, "verynear": 2, "inter": 3}[which]
        c = self.counts()
        rows = c["clusters"] if which == "far" else c["primitives"]
        nnz = c[{"near": "near_nnz", "far": "far_nnz", "verynear": "verynear_nnz", "inter": "inter_nnz"}[which]]
        rp = np.zeros(rows + 1, np.int64)
        ci = np.zeros(max(nnz, 1), np.int32)
        _load().oracle_pattern(self._h, w, _l(rp), _i(ci))
        return rp, ci[:nnz]

    def cluster_data(self):
        NC = self.counts()["clusters"]
        out = np.zeros((NC, 10))
        _load().oracle_cluster_data(self._h, _d(out))
        return out

    def primitive_data(self):
        nd = 1 + (self.dom + 1) * 3 + 6
        Pn = np.zeros((self.nS, nd))
        Pf = np.zeros((self.nS, 10))
        _load().oracle_primitive_data(self._h, _d(Pn), _d(Pf))
        return Pn, Pf

    def semistatic_update(self, V):
        self.V = np.ascontiguousarray(V, dtype=np.float64)
        _load().oracle_semistatic_update(self._h, _d(self.V))
        self._h1 = None

    def energy(self, q=6.0, p=12.0):
        return _load().oracle_energy(self._h, q, p)

    def differential(self, q=6.0, p=12.0, alpha=1.0, beta=0.0, Y=None):
        if Y is None:
            Y = np.zeros((self.nV, 3))
        en = _load().oracle_differential(self._h, q, p, alpha, beta, _d(Y), Y.shape[1])
        return en, Y

    def partial_derivatives(self, shard, shards, q=6.0, p=12.0):
        """Shard `shard` of `shards` (upper-triangle rows split like the reference's
        threads): its near (N x NEAR_DIM) and far (N_C x 10) derivative slices in tree
        order before collection, and its energy part."""
        nd = 1 + (self.dom + 1) * 3 + 6
        Dn = np.zeros((self.nS, nd))
        Df = np.zeros((self.counts()["clusters"], 10))
        e = _load().oracle_partial_derivatives(self._h, q, p, shard, shards, _d(Dn), _d(Df))
        return Dn, Df, e

    def row_derivatives(self, near_rows, far_rows, q=6.0, p=12.0):
        """Slices of a disjoint row partition: rows near_rows = [first, last) of the full
        Near() pattern and far_rows of Far(), each pair evaluated from its row with only
        the row's derivative accumulated (zero outside the rows), and the energy of the
        pairs with j > i in those rows. Summed over a partition of all rows they equal
        the unsharded slices."""
        nd = 1 + (self.dom + 1) * 3 + 6
        Dn = np.zeros((self.nS, nd))
        Df = np.zeros((self.counts()["clusters"], 10))
        e = _load().oracle_row_derivatives(self._h, q, p, int(near_rows[0]), int(near_rows[1]), int(far_rows[0]),
                                           int(far_rows[1]), _d(Dn), _d(Df))
        if np.isnan(e):
            raise ValueError("row-owned slices are not built for meshes with very-near pairs")
        return Dn, Df, e

    def collect(self, Dn, Df, alpha=1.0, beta=0.0, Y=None):
        """Y = alpha dE + beta Y from summed derivative slices (collection, chain rule,
        vertex scatter)."""
        Y = np.zeros((self.nV, 3)) if Y is None else Y
        Dn = np.ascontiguousarray(Dn, dtype=np.float64)
        Df = np.ascontiguousarray(Df, dtype=np.float64)
        _load().oracle_collect(self._h, _d(Dn), _d(Df), alpha, beta, _d(Y), Y.shape[1])
        return Y

    def maximum_safe_step_size(self, velocities, max_time, tol=0.0625):
        """Largest step t <= max_time along the vertex velocities (n_v x 3) that keeps
        non-adjacent primitives of the (construction-time) mesh apart."""
        vel = np.ascontiguousarray(velocities, dtype=np.float64)
        return _load().oracle_maximum_safe_step_size(self._h, _d(vel), float(max_time), float(tol))

    def moment_derivatives(self):
        nd = 1 + (self.dom + 1) * 3 + 6
        Dn = np.zeros((self.nS, nd))
        Df = np.zeros((self.nS, 10))
        _load().oracle_moment_derivatives(self._h, _d(Dn), _d(Df))
        return Dn, Df

    def simplex_densities(self, q=6.0, p=12.0):
        out = np.zeros(self.nS)
        en = _load().oracle_simplex_densities(self._h, q, p, _d(out))
        return en, out

    def vertex_densities(self, q=6.0, p=12.0):
        out = np.zeros(self.nV)
        en = _load().oracle_vertex_densities(self._h, q, p, _d(out))
        return en, out

    def allpairs_energy(self, q=6.0, p=12.0):
        return _load().oracle_allpairs_energy(self._h, q, p)

    def metric_values(self, q=6.0, p=12.0):
        c = self.counts()
        nf = np.zeros(2 * c["near_nnz"] + 1)
        ff = np.zeros(2 * c["far_nnz"] + 1)
        nfd = np.zeros(2 * c["primitives"])
        ffd = np.zeros(2 * c["clusters"])
        _load().oracle_metric_values(self._h, q, p, _d(nf), _d(ff), _d(nfd), _d(ffd))
        return nf[:-1].reshape(-1, 2), ff[:-1].reshape(-1, 2), nfd.reshape(-1, 2), ffd.reshape(-1, 2)

    def metric_multiply(self, X, q=6.0, p=12.0, alpha=1.0, beta=0.0, Y=None, flags=7):
        X = np.ascontiguousarray(X, dtype=np.float64)
        if Y is None:
            Y = np.zeros((self.nV, 3))
        _load().oracle_metric_multiply(self._h, q, p, alpha, _d(X), X.shape[1], beta, _d(Y), Y.shape[1], flags)
        return Y

    def pseudo_laplacian_multiply(self, X, s, alpha=1.0, beta=0.0, Y=None):
        X = np.ascontiguousarray(X, dtype=np.float64)
        if Y is None:
            Y = np.zeros((self.nV, 3))
        _load().oracle_pseudo_laplacian_multiply(self._h, s, alpha, _d(X), X.shape[1], beta, _d(Y), Y.shape[1])
        return Y

    # --- H1 metric and the reference preconditioner -------------------------------------------
    def h1_matrix(self, ws=1.0, wm=1.0):
        """Stiffness + mass matrix of src/SimplicialMesh/H1Metric.hpp:36-169 (scipy CSR)."""
        import scipy.sparse as sp

        n = _load().oracle_h1_triplet_count(self._h)
        I = np.zeros(n, np.int32)
        J = np.zeros(n, np.int32)
        A = np.zeros(n)
        _load().oracle_h1_triplets(self._h, ws, wm, _i(I), _i(J), _d(A))
        return sp.csr_matrix((A, (I, J)), shape=(self.nV, self.nV))

    def h1_solve(self, X):
        if self._h1 is None:
            import scipy.sparse.linalg as spla

            self._h1 = spla.splu(self.h1_matrix().tocsc())
        return self._h1.solve(np.ascontiguousarray(X))

    def precondition(self, X, q=6.0, p=12.0, alpha=1.0):
        """TangentPointMetric0::multiply_preconditioner (src/Metrics/TangentPointMetric0.hpp:88-126):
        Y = H1^{-1} . PseudoLaplacian(2 - s) . H1^{-1} (alpha X), s = (p - n)/q."""
        s_tp = (p - self.dom) / q
        Z = self.h1_solve(alpha * np.asarray(X))
        if alpha != 0:
            Z = self.pseudo_laplacian_multiply(Z, 2.0 - s_tp)
        return self.h1_solve(Z)


def pcg(apply_A, apply_P, B, tol=1e-6, max_iter=1000, X0=None):
    """Preconditioned CG (FP64) column-block version; stops when the true residual
    ||B - A X|| / ||B|| <= tol for every column. Returns (X, iterations, rel_res)."""
    B = np.asarray(B, dtype=np.float64)
    X = np.zeros_like(B) if X0 is None else X0.copy()
    R = B - apply_A(X)
    Z = apply_P(R)
    Pd = Z.copy()
    rz = np.einsum("ij,ij->j", R, Z)
    nb = np.linalg.norm(B, axis=0)
    it = 0
    rel = np.linalg.norm(R, axis=0) / nb
    while it < max_iter and np.max(rel) > tol:
        AP = apply_A(Pd)
        alpha = rz / np.einsum("ij,ij->j", Pd, AP)
        X += Pd * alpha
        R -= AP * alpha
        Z = apply_P(R)
        rz_new = np.einsum("ij,ij->j", R, Z)
        Pd = Z + Pd * (rz_new / rz)
        rz = rz_new
        it += 1
        rel = np.linalg.norm(R, axis=0) / nb
    rel_true = np.linalg.norm(B - apply_A(X), axis=0) / nb
    return X, it, rel_true


def gmres_left(apply_A, apply_P, B, tol=1e-6, max_iter=100, restart=None):
    """Left-preconditioned restarted GMRES per column (the reference's solver kind,
    src/Metrics/MetricDimRestricted.hpp:281-288); stops on the preconditioned
    residual. Returns (X, total_iterations, true relative residual per column)."""
    B = np.asarray(B, dtype=np.float64)
    n, m = B.shape
    restart = restart or max_iter
    X = np.zeros_like(B)
    total = 0
    for c in range(m):
        def A1(v):
            t = np.zeros((n, m)); t[:, c] = v
            return apply_A(t)[:, c]

        def P1(v):
            t = np.zeros((n, m)); t[:, c] = v
            return apply_P(t)[:, c]

        x = np.zeros(n)
        pb = P1(B[:, c])
        nb = np.linalg.norm(pb)
        it = 0
        while it < max_iter:
            r = P1(B[:, c] - A1(x))
            beta = np.linalg.norm(r)
            if beta <= tol * nb:
                break
            k = min(restart, max_iter - it)
            Q = np.zeros((n, k + 1)); H = np.zeros((k + 1, k))
            Q[:, 0] = r / beta
            g = np.zeros(k + 1); g[0] = beta
            cs = np.zeros(k); sn = np.zeros(k)
            jj = 0
            for j in range(k):
                w = P1(A1(Q[:, j]))
                for i in range(j + 1):
                    H[i, j] = Q[:, i] @ w
                    w -= H[i, j] * Q[:, i]
                H[j + 1, j] = np.linalg.norm(w)
                if H[j + 1, j] > 0:
                    Q[:, j + 1] = w / H[j + 1, j]
                for i in range(j):
                    t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                    H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                    H[i, j] = t
                den = np.hypot(H[j, j], H[j + 1, j])
                cs[j] = H[j, j] / den; sn[j] = H[j + 1, j] / den
                H[j, j] = den; H[j + 1, j] = 0
                g[j + 1] = -sn[j] * g[j]; g[j] = cs[j] * g[j]
                jj = j + 1
                it += 1
                if abs(g[j + 1]) <= tol * nb:
                    break
            y = np.linalg.solve(np.triu(H[:jj, :jj]), g[:jj])
            x += Q[:, :jj] @ y
        total = max(total, it)
        X[:, c] = x
    rel_true = np.linalg.norm(B - apply_A(X), axis=0) / np.linalg.norm(B, axis=0)
    return X, total, rel_true
