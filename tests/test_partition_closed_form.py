"""The closed form of the reference's in-place longest-axis partition that the device cluster
tree uses (repulsor_b200/csrc/rpb_gputree.cu, after AABB_LongestAxisSplit.hpp:181-199),
restated in numpy and checked against the sequential pass on seeded random flag patterns
(CPU): the r-th primitive below the box centre ends at r, a primitive above it at p >= nL
stays, one above it at p < nL follows p -> i_p -> i_{i_p} ... until the position reaches nL
(i_r: the position of the r-th primitive below the centre), both by direct chain following
and by the pointer jumping the device falls back to for long chains."""
import numpy as np


def sequential(flags):
    a = list(range(len(flags)))
    s = 0
    for i in range(len(flags)):
        if flags[a[i]]:
            a[s], a[i] = a[i], a[s]
            s += 1
    return a, s


def closed_form(flags, jump):
    f = np.asarray(flags, bool)
    n, nl = len(f), int(f.sum())
    rank = np.cumsum(f) - f
    ipos = np.nonzero(f)[0]
    dest = np.arange(n)
    dest[f] = rank[f]
    nxt = np.arange(n)
    nxt[:nl] = ipos
    if jump:
        for _ in range(max(1, int(np.ceil(np.log2(max(n, 2)))) + 1)):
            nxt[:nl] = np.where(nxt[:nl] < nl, nxt[nxt[:nl]], nxt[:nl])
    for p in np.nonzero(~f[:nl])[0]:
        q = p
        while q < nl:
            q = nxt[q]
        dest[p] = q
    out = [None] * n
    for i in range(n):
        out[dest[i]] = i
    return out, nl


def test_closed_form_matches_the_sequential_partition():
    rng = np.random.default_rng(7)
    for _ in range(3000):
        n = int(rng.integers(1, 60))
        flags = list(rng.random(n) < rng.random())
        ref = sequential(flags)
        assert closed_form(flags, jump=False) == ref
        assert closed_form(flags, jump=True) == ref


def test_long_chain_case():
    # one primitive above the centre at the front: a chain through every later position
    flags = [False] + [True] * 399
    out, nl = closed_form(flags, jump=True)
    assert (out, nl) == sequential(flags)
    assert out[-1] == 0
