"""The cluster tree and the block cluster tree built at mesh creation run on the GPU
(rpb_gputree.cu: the level-by-level longest-axis splits with the median fallback on the
host, then the dual traversal with host/bct_rules.hpp); the permutation, the clusters and
the four patterns must equal the host builder's (HostTree, itself checked bit-exactly
against the oracle in test_tree_parity.py) entry for entry, including very-near and
intersecting pairs. The cases include meshes whose splits take the median fallback on
clusters of more than three primitives (the full torus, the 96 x 128 linked tori)."""
import numpy as np
import pytest

import repulsor_b200 as rpb
from repulsor_b200 import meshes


def _overlapping_spheres():
    # two icospheres that interpenetrate and nearly touch: very-near and intersecting pairs
    Va, Sa = meshes.icosphere(level=3, radius=0.5, centre=(-0.45, 0.0, 0.0))
    Vb, Sb = meshes.icosphere(level=3, radius=0.5, centre=(0.45, 0.01, 0.0))
    return 2, np.vstack([Va, Vb]), np.vstack([Sa, Sb + Va.shape[0]]).astype(np.int32)


def _few(n):
    # n triangles of a strip: the smallest trees (one leaf, one split, ...)
    V, S = meshes.torus(n_major=8, n_minor=4)
    return 2, V, S[:n].copy()


def _long_chain():
    # a strip of 400 small triangles along x in [0, 1] whose first triangle lies far out at
    # x = 100: the root split moves only that one above the box centre, and the reference's
    # in-place pass carries it along a chain of 399 swaps (the device finishes such chains by
    # pointer jumping)
    n = 400
    xs = np.concatenate([[100.0], np.linspace(0.0, 1.0, n - 1)])
    V = np.zeros((3 * n, 3))
    for i, x in enumerate(xs):
        V[3 * i] = (x, 0.0, 0.0)
        V[3 * i + 1] = (x + 1e-3, 0.0, 1e-3)
        V[3 * i + 2] = (x, 1e-3, 5e-4)
    S = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    return 2, V, S


CASES = {
    "curve": lambda: (1,) + meshes.config_mesh(1, small=True)[1],
    "curve_full": lambda: (1,) + meshes.config_mesh(1)[1],
    "torus": lambda: (2,) + meshes.config_mesh(2, small=True)[1],
    "torus_full": lambda: (2,) + meshes.config_mesh(2)[1],
    "icosphere": lambda: (2,) + meshes.config_mesh(3, small=True)[1],
    "linked_tori": lambda: (2,) + meshes.config_mesh(5, small=True)[1],
    "linked_tori_96x128": lambda: (2,) + meshes.linked_tori(96, 128),
    "overlapping": _overlapping_spheres,
    "one_triangle": lambda: _few(1),
    "two_triangles": lambda: _few(2),
    "five_triangles": lambda: _few(5),
    "long_chain": _long_chain,
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_device_traversal_equals_host_builder(case):
    dom, V, S = CASES[case]()
    M = rpb.SimplicialMesh(V, S)
    H = rpb.HostTree(V, S)
    assert M.build_info() == {"cluster_tree_on_device": True, "block_tree_on_device": True}
    tm, th = M.tree(), H.tree()
    assert M.stats()["tree_depth"] == H.stats()["tree_depth"]
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
