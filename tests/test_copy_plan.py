"""The automatic copy-overlap plan of host-buffer solves (host logic, no GPU):
groups are contiguous, each later group joins the trailing updates before its
first block column is solved, joins never go backwards, and block sizes whose
128-row update tiles would straddle a group boundary get one group."""
import pytest

import cholesky_gpu_b200 as mp


@pytest.mark.parametrize("n", [256, 1000, 2048, 4096, 8192, 16384, 30000])
@pytest.mark.parametrize("b", [32, 64, 96, 128, 256])
def test_automatic_plans_are_valid(n, b):
    cuts, join = mp.copy_plan(n, b)
    nb = -(-n // b)
    assert len(cuts) == len(join) <= 7
    if b % 128 != 0 or nb < 4:
        assert cuts == []
        return
    prev_c, prev_j = 0, 0
    for c, j in zip(cuts, join):
        assert prev_c < c < nb
        assert 0 <= j <= c - 1 and j >= prev_j
        prev_c, prev_j = c, j


def test_large_problems_overlap_the_copy():
    cuts, join = mp.copy_plan(8192, 256)
    assert len(cuts) >= 2     # n = 8192: the copy (~2.7 ms) is worth splitting
