"""Seeded synthetic meshes for the tangent-point workloads.

Every generator returns ``(V, S)`` with ``V`` a C-contiguous ``(n_v, 3)`` float64
array of vertex coordinates and ``S`` a C-contiguous ``(n_s, dom_dim + 1)`` int32
array of simplices, the row-major layout that Repulsor's ``SimplicialMesh``
constructor reads (``src/SimplicialMesh.hpp:154-185``).

The random streams come from ``numpy.random.default_rng(seed)`` (PCG64), which is
bit-reproducible across platforms, so the same seed gives the same mesh on the
development host and on the GPU host.

Workloads (sizes and distributions of the five benchmark configurations):

* ``torus_knot``      closed (2,3) torus-knot polygon, 2,000 edges, jitter N(0, 1e-3^2)
* ``torus``           R=1, r=0.4 torus, 160 x 120 grid, 38,400 triangles, normal jitter N(0, 0.002^2)
* ``icosphere_sh``    level-L icosphere displaced radially by a real spherical-harmonic
                      field of degrees 1..8 with coefficients N(0, (0.05/l)^2)
* ``linked_tori``     two R=1, r=0.3 tori (480 x 640 grids), the second rotated 90 deg
                      about x and shifted by +1 along x, normal jitter N(0, 0.002^2)
* ``icosphere``       plain level-L icosphere of a given radius and centre (obstacle)

``reference_mesh`` returns the meshes the reference itself ships (its Meshes/ directory),
from a committed fixture.
"""
from __future__ import annotations

import math
import os

import numpy as np

__all__ = [
    "reference_mesh",
    "torus_knot",
    "torus",
    "icosphere",
    "icosphere_sh",
    "linked_tori",
    "random_rhs",
    "config_mesh",
]


def torus_knot(n: int = 2000, jitter: float = 1e-3, seed: int = 1001):
    """(2,3) torus knot x(t) = ((1+0.4cos3t)cos2t, (1+0.4cos3t)sin2t, 0.4 sin3t).

    ``n`` equispaced samples t_i = 2 pi i / n, each vertex jittered by i.i.d.
    N(0, jitter^2) per coordinate, edges i -> (i+1) mod n.
    """
    rng = np.random.default_rng(seed)
    t = 2.0 * math.pi * np.arange(n, dtype=np.float64) / n
    rad = 1.0 + 0.4 * np.cos(3.0 * t)
    V = np.stack([rad * np.cos(2.0 * t), rad * np.sin(2.0 * t), 0.4 * np.sin(3.0 * t)], axis=1)
    V = V + jitter * rng.standard_normal(V.shape)
    i = np.arange(n, dtype=np.int32)
    S = np.stack([i, (i + 1) % n], axis=1).astype(np.int32)
    return np.ascontiguousarray(V), np.ascontiguousarray(S)


def _torus_grid(R, r, n_major, n_minor):
    th = 2.0 * math.pi * np.arange(n_major, dtype=np.float64) / n_major
    ph = 2.0 * math.pi * np.arange(n_minor, dtype=np.float64) / n_minor
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    normal = np.stack([np.cos(PH) * np.cos(TH), np.cos(PH) * np.sin(TH), np.sin(PH)], axis=-1)
    centre = np.stack([R * np.cos(TH), R * np.sin(TH), np.zeros_like(TH)], axis=-1)
    P = centre + r * normal
    idx = np.arange(n_major * n_minor, dtype=np.int64).reshape(n_major, n_minor)
    i00 = idx
    i10 = np.roll(idx, -1, axis=0)
    i11 = np.roll(np.roll(idx, -1, axis=0), -1, axis=1)
    i01 = np.roll(idx, -1, axis=1)
    tri_a = np.stack([i00, i10, i11], axis=-1).reshape(-1, 3)
    tri_b = np.stack([i00, i11, i01], axis=-1).reshape(-1, 3)
    S = np.empty((2 * tri_a.shape[0], 3), dtype=np.int64)
    S[0::2] = tri_a
    S[1::2] = tri_b
    return P.reshape(-1, 3), normal.reshape(-1, 3), S.astype(np.int32)


def torus(R: float = 1.0, r: float = 0.4, n_major: int = 160, n_minor: int = 120,
          jitter: float = 0.002, seed: int = 1002):
    """Torus with each grid quad split into two triangles, vertices displaced along
    the normal by i.i.d. N(0, jitter^2)."""
    rng = np.random.default_rng(seed)
    V, N, S = _torus_grid(R, r, n_major, n_minor)
    V = V + (jitter * rng.standard_normal(V.shape[0]))[:, None] * N
    return np.ascontiguousarray(V), np.ascontiguousarray(S)


def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    V = np.array([
        [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
        [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
        [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
    ], dtype=np.float64)
    F = np.array([
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
    ], dtype=np.int64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    return V, F


def _unit_icosphere(level: int):
    V, F = _icosahedron()
    for _ in range(level):
        nv = V.shape[0]
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]], axis=0)
        e = np.sort(e, axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        ukey, inv = np.unique(key, return_inverse=True)
        a = ukey // (nv + 1)
        b = ukey % (nv + 1)
        mid = 0.5 * (V[a] + V[b])
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + nv  # midpoints of edges (01, 12, 20) per face
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([
            np.stack([F[:, 0], m01, m20], axis=1),
            np.stack([F[:, 1], m12, m01], axis=1),
            np.stack([F[:, 2], m20, m12], axis=1),
            np.stack([m01, m12, m20], axis=1),
        ], axis=0)
        V = np.concatenate([V, mid], axis=0)
    return V, F.astype(np.int32)


def icosphere(level: int = 5, radius: float = 1.0, centre=(0.0, 0.0, 0.0)):
    """Plain icosphere (20 * 4^level triangles) of the given radius and centre."""
    V, F = _unit_icosphere(level)
    V = radius * V + np.asarray(centre, dtype=np.float64)[None, :]
    return np.ascontiguousarray(V), np.ascontiguousarray(F)


def _real_sh_field(lmax: int, coeff_scale: float, rng, xyz):
    """f(x) = sum_{l=1..lmax} sum_{m=-l..l} c_lm Y_lm(x), c_lm ~ N(0, (coeff_scale/l)^2).

    Real orthonormal spherical harmonics built from associated Legendre functions.
    """
    from scipy.special import lpmv

    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    rr = np.sqrt(x * x + y * y + z * z)
    ct = np.clip(z / rr, -1.0, 1.0)
    phi = np.arctan2(y, x)
    f = np.zeros_like(x)
    for l in range(1, lmax + 1):
        c = rng.standard_normal(2 * l + 1) * (coeff_scale / l)
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            P = lpmv(am, l, ct)
            if m == 0:
                Y = norm * P
            elif m > 0:
                Y = math.sqrt(2.0) * norm * P * np.cos(am * phi)
            else:
                Y = math.sqrt(2.0) * norm * P * np.sin(am * phi)
            f += c[m + l] * Y
    return f


def icosphere_sh(level: int = 6, lmax: int = 8, coeff_scale: float = 0.05, seed: int = 1003):
    """Icosphere displaced radially by a random real spherical-harmonic field of
    degrees 1..lmax with coefficients N(0, (coeff_scale/l)^2)."""
    rng = np.random.default_rng(seed)
    V, F = _unit_icosphere(level)
    f = _real_sh_field(lmax, coeff_scale, rng, V)
    V = V * (1.0 + f)[:, None]
    return np.ascontiguousarray(V), np.ascontiguousarray(F)


def linked_tori(n_major: int = 480, n_minor: int = 640, R: float = 1.0, r: float = 0.3,
                jitter: float = 0.002, seed: int = 1005):
    """Two linked tori; the second is rotated 90 degrees about x and shifted +1 in x."""
    rng = np.random.default_rng(seed)
    V1, N1, S1 = _torus_grid(R, r, n_major, n_minor)
    V1 = V1 + (jitter * rng.standard_normal(V1.shape[0]))[:, None] * N1
    V2, N2, S2 = _torus_grid(R, r, n_major, n_minor)
    V2 = V2 + (jitter * rng.standard_normal(V2.shape[0]))[:, None] * N2
    rot = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, -1.0], [0.0, 1.0, 0.0]])
    V2 = V2 @ rot.T + np.array([1.0, 0.0, 0.0])
    V = np.concatenate([V1, V2], axis=0)
    S = np.concatenate([S1, S2 + V1.shape[0]], axis=0).astype(np.int32)
    return np.ascontiguousarray(V), np.ascontiguousarray(S)


def random_rhs(n_v: int, seed: int, project: bool = True):
    """i.i.d. N(0,1) vertex field (n_v x 3).

    With ``project`` the per-component mean is removed. The tangent-point metric
    annihilates constant vector fields (translations), so only right-hand sides
    orthogonal to them admit a solution; the mean removal is that projection.
    """
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n_v, 3))
    if project:
        B -= B.mean(axis=0, keepdims=True)
    return np.ascontiguousarray(B)


def config_mesh(cfg: int, small: bool = False):
    """Mesh of benchmark configuration ``cfg`` (1..5); ``small`` gives a reduced
    instance of the same family for fast tests."""
    if cfg == 1:
        return (1, torus_knot(n=400 if small else 2000, seed=1001))
    if cfg == 2:
        return (2, torus(n_major=40 if small else 160, n_minor=30 if small else 120, seed=1002))
    if cfg == 3:
        return (2, icosphere_sh(level=3 if small else 6, seed=1003))
    if cfg == 5:
        return (2, linked_tori(n_major=48 if small else 480, n_minor=64 if small else 640, seed=1005))
    raise ValueError(f"no single mesh for configuration {cfg}")


_REFERENCE_NPZ = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                              "reference_meshes.npz")


def reference_mesh(name: str):
    """A mesh shipped with the reference (Meshes/ of HenrikSchumacher/Repulsor), from the
    committed fixture tests/golden/reference_meshes.npz: "torus2400", "torus38400",
    "sphere40560", "twospheres" (the example's mesh), "twospheres_obstacle" (its
    obstacle) or "twospheres_union" (both spheres as one mesh: 25 very-near pairs).
    Returns (V, S)."""
    d = np.load(_REFERENCE_NPZ)
    if name == "twospheres_union":
        V, S = d["twospheres_V"], d["twospheres_S"]
        VO, SO = d["twospheres_obstacle_V"], d["twospheres_obstacle_S"]
        return np.vstack([V, VO]), np.vstack([S, SO + V.shape[0]]).astype(np.int32)
    return np.array(d[f"{name}_V"]), np.array(d[f"{name}_S"])
