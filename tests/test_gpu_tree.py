"""The block cluster tree built at mesh creation runs its dual traversal on the GPU
(rpb_gputree.cu, host/bct_rules.hpp); its four patterns must equal the host builder's
(HostTree, itself checked bit-exactly against the oracle in test_tree_parity.py) entry
for entry, including very-near and intersecting pairs."""
import numpy as np
import pytest

import repulsor_b200 as rpb
from repulsor_b200 import meshes


def _overlapping_spheres():
    # two icospheres that interpenetrate and nearly touch: very-near and intersecting pairs
    Va, Sa = meshes.icosphere(level=3, radius=0.5, centre=(-0.45, 0.0, 0.0))
    Vb, Sb = meshes.icosphere(level=3, radius=0.5, centre=(0.45, 0.01, 0.0))
    return 2, np.vstack([Va, Vb]), np.vstack([Sa, Sb + Va.shape[0]]).astype(np.int32)


CASES = {
    "curve": lambda: (1,) + meshes.config_mesh(1, small=True)[1],
    "torus": lambda: (2,) + meshes.config_mesh(2, small=True)[1],
    "icosphere": lambda: (2,) + meshes.config_mesh(3, small=True)[1],
    "linked_tori": lambda: (2,) + meshes.config_mesh(5, small=True)[1],
    "overlapping": _overlapping_spheres,
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_device_traversal_equals_host_builder(case):
    dom, V, S = CASES[case]()
    M = rpb.SimplicialMesh(V, S)
    H = rpb.HostTree(V, S)
    tm, th = M.tree(), H.tree()
    for k in th:
        np.testing.assert_array_equal(tm[k], th[k])
    for which in ("near", "far", "verynear", "inter"):
        rp_m, ci_m = M.pattern(which)
        rp_h, ci_h = H.pattern(which)
        np.testing.assert_array_equal(rp_m, rp_h, err_msg=which)
        np.testing.assert_array_equal(ci_m[:rp_m[-1]], ci_h[:rp_h[-1]], err_msg=which)
    if case == "overlapping":
        st = M.stats()
        assert st["verynear_nnz"] > 0 and st["inter_nnz"] > 0
