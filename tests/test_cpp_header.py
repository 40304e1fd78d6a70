"""The header-only C++20 mirror (include/repulsor_b200/Repulsor.hpp): it compiles with
-std=c++20 -Wall -Wextra -Werror against the C ABI and links to librepulsor_b200.so (CPU),
and the driver tests/cpp/header_api.cpp, which uses it the way Repulsor's own example
drivers use the reference classes, returns the same numbers as the Python mirror (GPU)."""
import os
import subprocess

import numpy as np
import pytest

import repulsor_b200 as rpb
from repulsor_b200 import _capi, meshes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "header_api.cpp")
LIBDIR = os.path.dirname(_capi.LIB_PATH)


def _build(tmp_path):
    exe = str(tmp_path / "header_api")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", LIBDIR, "-lrepulsor_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_header_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


def _write_mesh(path, V, S):
    with open(path, "w") as f:
        f.write(f"{V.shape[0]} {S.shape[0]} {S.shape[1] - 1}\n")
        np.savetxt(f, V, fmt="%.17g")
        np.savetxt(f, S, fmt="%d")


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [1, 2])
def test_header_driver_matches_python_mirror(tmp_path, cfg):
    exe = _build(tmp_path)
    dom, (V, S) = meshes.config_mesh(cfg, small=True)
    mesh_file = str(tmp_path / "mesh.txt")
    _write_mesh(mesh_file, V, S)
    out = subprocess.run([exe, mesh_file], check=True, capture_output=True, text=True)
    lines = out.stdout.split()
    E, dmax, ysum, iters, rmax = float(lines[0]), float(lines[1]), float(lines[2]), int(lines[3]), float(lines[4])
    Ed, Eo = float(lines[5]), float(lines[6])
    assert "nrhs = 2 != 3 = AMB_DIM" in out.stderr          # print-and-return error path

    M = rpb.SimplicialMesh(V, S)
    tpe = rpb.TangentPointEnergy0(6.0, 12.0)
    tpm = rpb.TangentPointMetric0(6.0, 12.0)
    E_py = tpe.Value(M)
    D = tpe.Differential(M)
    Y = tpm.MultiplyMetric(M, 1.0, D)
    B = D - D.mean(0)
    tpm.Solve(M, 1.0, B, max_iter=20000, tolerance=1e-6, precond=rpb.PRECOND_NONE)
    assert abs(E - E_py) <= 1e-12 * abs(E_py)
    assert abs(dmax - np.abs(D).max()) <= 1e-12 * np.abs(D).max()
    assert abs(ysum - Y.sum()) <= 1e-9 * np.abs(Y).sum()
    assert iters == tpm.Solver_IterationCount()
    assert rmax <= 1e-6
    assert abs(Ed - E_py) <= 1e-6 * abs(E_py)          # the densities kernel sums in another order
    Mo = rpb.SimplicialMesh(V, S)
    VO = V.copy()
    VO[:, 2] += 3.0
    Mo.LoadObstacle(rpb.SimplicialMesh(VO, S))
    Eo_py = rpb.TangentPointObstacleEnergy(6.0, 12.0).Value(Mo)
    assert Eo > 0 and abs(Eo - Eo_py) <= 1e-12 * abs(Eo_py)
