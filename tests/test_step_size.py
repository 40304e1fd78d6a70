"""MaximumSafeStepSize (rpb_mesh_maximum_safe_step_size): the oracle restatement on known
answers (CPU) and the GPU path against the oracle (GPU). Both search a bisection grid with
relative tolerance TOL, the reference's sequential traversal (the oracle) starting later
pairs from the running minimum and the GPU every pair from max_time, so they agree to TOL."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from repulsor_b200 import meshes  # noqa: E402

TOL = 0.0625


def _two_spheres(level=2, gap=1.0):
    """Two icospheres of radius 0.5 whose centres are 1 + gap apart on the x axis, moving
    towards each other at unit speed: the gap closes at t = gap / 2."""
    Va, Sa = meshes.icosphere(level=level, radius=0.5, centre=(-(1.0 + gap) / 2, 0.0, 0.0))
    Vb, Sb = meshes.icosphere(level=level, radius=0.5, centre=((1.0 + gap) / 2, 0.0, 0.0))
    V = np.vstack([Va, Vb])
    S = np.vstack([Sa, Sb + Va.shape[0]]).astype(np.int32)
    vel = np.zeros_like(V)
    vel[:Va.shape[0], 0] = 1.0
    vel[Va.shape[0]:, 0] = -1.0
    return V, S, vel


def _linked_tori():
    dom, (V, S) = meshes.config_mesh(5, small=True)
    vel = np.zeros_like(V)
    half = V.shape[0] // 2
    vel[:half, 0] = 1.0                     # the first torus moves through the second's hole
    vel[half:, 0] = -1.0
    return V, S, vel


def test_oracle_two_spheres_known_answer():
    V, S, vel = _two_spheres()
    O = oracle.OracleMesh(2, V, S, threads=4)
    # polyhedral spheres: the gap between their extreme faces closes slightly after 0.5
    t = O.maximum_safe_step_size(vel, 1.0, TOL)
    assert 0.5 * (1 - TOL) <= t <= 0.5 + 0.02
    assert O.maximum_safe_step_size(vel, 0.3, TOL) == 0.3           # no contact before max_time
    assert O.maximum_safe_step_size(np.zeros_like(V), 1.0, TOL) == 1.0
    assert O.maximum_safe_step_size(-vel, 1.0, TOL) == 1.0          # moving apart


def _sphere_and_obstacle():
    """An icosphere of radius 0.5 at (-1, 0, 0) moving at unit speed towards a resting
    obstacle icosphere of radius 0.5 at (1, 0, 0): the gap of 1 closes at t = 1."""
    V, S = meshes.icosphere(level=2, radius=0.5, centre=(-1.0, 0.0, 0.0))
    Vo, So = meshes.icosphere(level=2, radius=0.5, centre=(1.0, 0.0, 0.0))
    vel = np.zeros_like(V)
    vel[:, 0] = 1.0
    return V, S, Vo, So, vel


def test_oracle_obstacle_known_answer():
    V, S, Vo, So, vel = _sphere_and_obstacle()
    O = oracle.OracleMesh(2, V, S, threads=4)
    Ob = oracle.OracleMesh(2, Vo, So, threads=4)
    assert O.maximum_safe_step_size(vel, 2.0, TOL) == 2.0           # alone it moves freely
    O.load_obstacle(Ob)
    t = O.maximum_safe_step_size(vel, 2.0, TOL)
    assert 1.0 * (1 - TOL) <= t <= 1.0 + 0.04


def test_oracle_step_is_safe_and_tight_on_linked_tori():
    V, S, vel = _linked_tori()
    O = oracle.OracleMesh(2, V, S, threads=4)
    t = O.maximum_safe_step_size(vel, 1.0, TOL)
    assert 0.0 < t < 1.0
    # a tighter tolerance refines the same contact from below
    t2 = O.maximum_safe_step_size(vel, 1.0, TOL / 8)
    assert t2 >= t * (1 - TOL) and abs(t2 - t) <= TOL * t2


@pytest.mark.gpu
def test_gpu_step_size_with_obstacle_matches_oracle():
    import repulsor_b200 as rpb

    V, S, Vo, So, vel = _sphere_and_obstacle()
    O = oracle.OracleMesh(2, V, S, threads=4)
    Ob = oracle.OracleMesh(2, Vo, So, threads=4)
    O.load_obstacle(Ob)
    M = rpb.SimplicialMesh(V, S)
    M.LoadObstacle(rpb.SimplicialMesh(Vo, So))
    t_ref = O.maximum_safe_step_size(vel, 2.0, TOL)
    t = M.MaximumSafeStepSize(vel, 2.0, TOL)
    assert abs(t - t_ref) <= TOL * max(t, t_ref), (t, t_ref)
    assert 1.0 * (1 - TOL) <= t <= 1.04


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["spheres", "tori", "static"])
def test_gpu_step_size_matches_oracle(case):
    import repulsor_b200 as rpb

    if case == "tori":
        V, S, vel = _linked_tori()
    else:
        V, S, vel = _two_spheres()
        if case == "static":
            vel = np.zeros_like(V)
    O = oracle.OracleMesh(2, V, S, threads=4)
    M = rpb.SimplicialMesh(V, S)
    for max_time in (1.0, 0.3):
        t_ref = O.maximum_safe_step_size(vel, max_time, TOL)
        t = M.MaximumSafeStepSize(vel, max_time, TOL)
        assert 0.0 < t <= max_time
        assert abs(t - t_ref) <= TOL * max(t, t_ref), (case, max_time, t, t_ref)
    # the mesh's later coordinates do not move the collision geometry (as in the reference)
    t1 = M.MaximumSafeStepSize(vel, 1.0, TOL)
    M.SemiStaticUpdate(V + 0.01)
    assert M.MaximumSafeStepSize(vel, 1.0, TOL) == t1
    with pytest.raises(rpb.RepulsorError):
        M.MaximumSafeStepSize(vel, -1.0)
