"""The algorithmic flops per pair that bench.py's roofline uses are the oracle's counted
ones: the FF and NF loop bodies evaluated once with an operation-counting scalar."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle  # noqa: E402


def test_bench_flops_per_pair_are_the_oracle_counts():
    far = oracle.pair_opcounts(2, far=True)
    near = oracle.pair_opcounts(2, far=False)
    assert far["flops"] == bench.FLOPS_FAR_PAIR
    assert near["flops"] == bench.FLOPS_NEAR_PAIR
    # integer exponents q/2 = 3, p/2 = 6: powers by multiplication, one reciprocal
    assert far["pow"] == near["pow"] == 0 and far["div"] == near["div"] == 1


def test_counts_follow_the_simplex_dimension():
    # curves spread dE/dx over two hull slots instead of three and average two corners
    assert oracle.pair_opcounts(1, far=True) == oracle.pair_opcounts(2, far=True)
    assert oracle.pair_opcounts(1, far=False)["flops"] < oracle.pair_opcounts(2, far=False)["flops"]
    # non-integer exponents: the powers become pow calls
    c = oracle.pair_opcounts(2, far=True, q=5.0, p=11.0)
    assert c["pow"] == 3
