"""The header-only C++20 mirror (include/repulsor_b200/Repulsor.hpp): both drivers compile
with -std=c++20 -Wall -Wextra -Werror against the C ABI and link to librepulsor_b200.so
(CPU); tests/cpp/header_api.cpp (concrete classes, a mesh file read by the factory's
Make_FromFile) and tests/cpp/example_main.cpp (Repulsor's Example/main.cpp call for call:
SimplicialMeshBase / EnergyBase / MetricBase and the four factories on the reference's
own TwoSpheres input) return the same numbers as the Python mirror (GPU)."""
import os
import subprocess

import numpy as np
import pytest

import repulsor_b200 as rpb
from repulsor_b200 import _capi, meshes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(_capi.LIB_PATH)


def _build(tmp_path, name="header_api"):
    exe = str(tmp_path / name)
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), src,
           "-L", LIBDIR, "-lrepulsor_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("name", ["header_api", "example_main"])
def test_header_compiles_and_links(tmp_path, name):
    exe = _build(tmp_path, name)
    assert os.path.exists(exe)


def _write_mesh(path, V, S):
    rpb.write_mesh_file(path, V, S)


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


def _run_example(tmp_path, *extra):
    exe = _build(tmp_path, "example_main")
    V, S = meshes.reference_mesh("twospheres")
    VO, SO = meshes.reference_mesh("twospheres_obstacle")
    fm, fo = str(tmp_path / "mesh.txt"), str(tmp_path / "obstacle.txt")
    _write_mesh(fm, V, S)
    _write_mesh(fo, VO, SO)
    try:
        out = subprocess.run([exe, fm, fo, "1", "0.25", *extra], check=True, capture_output=True, text=True,
                             timeout=300)
    except subprocess.TimeoutExpired as e:
        raise AssertionError(f"example driver did not finish; its progress: {e.stderr}") from e
    got = dict(line.split() for line in out.stdout.splitlines())
    return {k: float(v) for k, v in got.items()}, out.stderr, (V, S, VO, SO)


def _python_example(V, S, VO, SO, obstacle_first):
    M = rpb.SimplicialMesh(V, S, far_field_separation=0.25, thread_count=1)
    if obstacle_first:
        M.LoadObstacle(rpb.SimplicialMesh(VO, SO))
    tpe, tpm = rpb.TangentPointEnergy0(6.0, 12.0), rpb.TangentPointMetric0(6.0, 12.0)
    r = {"energy": tpe.Value(M)}
    diff = tpe.Differential(M).copy()
    r["differential_max"] = np.abs(diff).max()
    grad = tpm.Solve(M, 1.0, diff, max_iter=100, tolerance=1e-5, strict=False)
    r["solve_iterations"] = tpm.Solver_IterationCount()
    r["solve_relative_residual_max"] = max(tpm.Solver_RelativeResiduals())
    r["gradient_max"] = np.abs(grad).max()
    r["step_size"] = M.MaximumSafeStepSize(-grad, 1.0)
    M.SemiStaticUpdate(V - r["step_size"] * grad)
    r["energy_new"] = tpe.Value(M)
    if not obstacle_first:
        M.LoadObstacle(rpb.SimplicialMesh(VO, SO))
    return M, r


def _close(a, b, tol=1e-12):
    return abs(a - b) <= tol * max(abs(b), 1e-300)


@pytest.mark.gpu
def test_example_driver_reports_the_obstacle_intersection_of_the_example_order(tmp_path):
    """Example/main.cpp on its own input (Meshes/TwoSpheres.hpp) in its own order: the mesh
    moves along the gradient (far-field theta 0.25 as the example sets it; leaf size 1, the
    only leaf size of this build, instead of the example's 2) and only then loads the
    obstacle, 0.0078 away before the step. The moved sphere intersects the obstacle, so
    very-near (mesh, obstacle) pairs are in contact and the obstacle energy is infinite:
    the driver must finish and report this (the reference's quadrature would refine those
    pairs to its level limit), and the Python mirror must raise the same error."""
    f, err, (V, S, VO, SO) = _run_example(tmp_path)
    M, r = _python_example(V, S, VO, SO, obstacle_first=False)
    for k in ("energy", "differential_max", "gradient_max", "step_size", "energy_new"):
        assert _close(f[k], r[k], 1e-10), (k, f[k], r[k])
    assert int(f["solve_iterations"]) == r["solve_iterations"]
    assert f["energy_decreased"] == 1 and f["metric_xax_nonnegative"] == 1
    assert "touch or intersect" in err
    with pytest.raises(rpb.RepulsorError, match="touch or intersect"):
        rpb.TangentPointObstacleEnergy(6.0, 12.0).Value(M)


@pytest.mark.gpu
def test_example_driver_with_the_obstacle_loaded_first_matches_python_mirror(tmp_path):
    """The same program with the obstacle loaded right after the mesh: the step size then
    keeps the mesh off the obstacle, and every printed quantity equals the Python mirror's."""
    f, err, (V, S, VO, SO) = _run_example(tmp_path, "obstacle_first")
    M, r = _python_example(V, S, VO, SO, obstacle_first=True)
    tpo = rpb.TangentPointObstacleEnergy(6.0, 12.0)
    eo = tpo.Value(M)
    do = tpo.Differential(M)
    for k in ("energy", "differential_max", "gradient_max", "step_size", "energy_new"):
        assert _close(f[k], r[k], 1e-10), (k, f[k], r[k])
    # Differential's energy comes from the pair kernel with derivatives, Value's from the one
    # without: the same sum in other FP32 orders
    assert f["energy_pointer"] == pytest.approx(r["energy"], rel=1e-8)
    assert int(f["solve_iterations"]) == r["solve_iterations"]
    assert _close(f["solve_relative_residual_max"], r["solve_relative_residual_max"], 1e-5)
    assert 0 < f["step_size"] <= 1 and f["energy_decreased"] == 1
    assert int(f["obstacle_vertex_count"]) == VO.shape[0] and int(f["obstacle_simplex_count"]) == SO.shape[0]
    assert _close(f["obstacle_energy"], eo, 1e-10) and eo > 0
    assert _close(f["obstacle_differential_max"], np.abs(do).max(), 1e-10)
    assert "ERROR" not in err
