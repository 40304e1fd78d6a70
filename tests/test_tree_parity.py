"""Bit-exact parity of the product's host cluster tree and block cluster tree with
the oracle restatement (permutation, cluster arrays, near/far/very-near/intersection
patterns)."""
import numpy as np
import pytest

import oracle
import repulsor_b200 as rpb
from repulsor_b200 import meshes


def _compare(dom, V, S, **kw):
    T = rpb.HostTree(V, S, **kw)
    O = oracle.OracleMesh(dom, V, S, theta_far=kw.get("far_field_separation", 0.5),
                          theta_near=kw.get("near_field_separation", 10.0))
    a, b = T.tree(), O.tree()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    for w in ("near", "far", "verynear", "inter"):
        ra, ca = T.pattern(w)
        rb, cb = O.pattern(w)
        assert np.array_equal(ra, rb), w
        assert np.array_equal(ca, cb), w
    return T, O


@pytest.mark.parametrize("cfg", [1, 2, 3])
@pytest.mark.parametrize("small", [True, False])
def test_tree_and_pair_lists_bit_exact(cfg, small):
    dom, (V, S) = meshes.config_mesh(cfg, small=small)
    T, O = _compare(dom, V, S)
    st = T.stats()
    assert st["cluster_count"] == 2 * st["simplex_count"] - 1    # split_threshold = 1: singleton leaves


def test_tree_parity_other_theta():
    dom, (V, S) = meshes.config_mesh(2, small=True)
    _compare(dom, V, S, far_field_separation=0.35)


def test_tree_structure_invariants():
    dom, (V, S) = meshes.config_mesh(3, small=True)
    t = rpb.HostTree(V, S).tree()
    N = S.shape[0]
    assert sorted(t["perm"].tolist()) == list(range(N))
    L, R = t["C_left"], t["C_right"]
    internal = L >= 0
    # depth-first numbering: left child follows its parent, ranges split contiguously
    assert np.all(L[internal] == np.nonzero(internal)[0] + 1)
    assert np.all(t["C_end"][L[internal]] == t["C_begin"][R[internal]])
    assert np.all(t["C_end"][~internal] - t["C_begin"][~internal] == 1)


def test_pair_lists_partition_all_pairs_small():
    """Every unordered primitive pair is covered exactly once by near, very-near,
    intersection or a far cluster pair (the admissible-block partition)."""
    dom, (V, S) = meshes.config_mesh(1, small=True)
    T = rpb.HostTree(V, S)
    t = T.tree()
    N = S.shape[0]
    cover = np.zeros((N, N), np.int32)
    for w in ("near", "verynear", "inter"):
        rp, ci = T.pattern(w)
        for i in range(N):
            for j in ci[rp[i]:rp[i + 1]]:
                if j > i:
                    cover[i, j] += 1
    rp, ci = T.pattern("far")
    for I in range(len(rp) - 1):
        for J in ci[rp[I]:rp[I + 1]]:
            if J > I:
                for i in range(t["C_begin"][I], t["C_end"][I]):
                    for j in range(t["C_begin"][J], t["C_end"][J]):
                        cover[min(i, j), max(i, j)] += 1
    iu = np.triu_indices(N, 1)
    assert np.all(cover[iu] == 1)
