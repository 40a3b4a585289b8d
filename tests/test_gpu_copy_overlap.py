"""Host-buffer solves with the copy of A overlapped with the factorization.

A's block columns cross the link in groups; a group that arrives after some
steps joins the trailing updates once the earlier panels' updates have been
applied to it in step order.  Each tile of C thus sees the same sequence of
FP32 reduce-adds as in the factorization of a fully copied matrix, so the
factor must be identical bit for bit, including every step's precision, for
every plan: early and late joins, a join one step before the group's first
block column (the head update then waits for the catch-up), a ragged last
block, and each trailing-update family (FP32 SIMT, one tensor-core format,
the device-dispatched switching ladder).
"""
import numpy as np
import pytest
import torch

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import matgen

pytestmark = pytest.mark.gpu

LADDER = dict(precision="switching", eps_prime=1e-5, ladder=["e4m3", "fp16", "fp16x2"])


@pytest.mark.parametrize("n,b,opts,cuts,join", [
    (2048, 256, LADDER, [2, 4, 6], [0, 2, 4]),
    (2048, 256, LADDER, [3, 5], [1, 4]),                       # joins at c0 - 1
    (1000, 128, dict(precision="fp32"), [2, 5], [1, 3]),       # ragged last block, SIMT update
    (1536, 128, dict(precision="e4m3"), [3, 7, 9], [2, 5, 8]),
    (1536, 128, dict(precision="mxfp8"), [1, 2, 3, 4, 6, 8, 10], [0, 1, 2, 3, 4, 6, 9]),
    (2048, 256, LADDER, None, None),                           # the automatic plan
])
def test_streamed_factor_is_bit_identical(cuda, n, b, opts, cuts, join):
    kappa = 1e2 if opts.get("precision") in ("e4m3", "mxfp8") else 1e5
    A = matgen.spd_matrix(n, kappa, 51)
    B = matgen.rhs(n, 1, 52).to(torch.float64)
    f_dev = mp.Factor(n, block_size=b, **opts)
    f_dev.compute(A.cuda())
    L_dev = f_dev.lower().cpu().numpy()
    i_dev = f_dev.info()
    f_host = mp.Factor(n, block_size=b, **opts)
    if cuts is not None:
        f_host.set_copy_plan(cuts, join)
    A_pin, B_pin = A.pin_memory(), B.pin_memory()
    # call 1 launches the factorization directly, call 2 (same buffer, same
    # plan) captures it as a CUDA graph, call 3 relaunches that graph; all
    # reuse the copy stream and the panel history
    for _ in range(3):
        X, rep = f_host.solve_host(A_pin, B_pin, rel_tol=1e-10)
        assert rep.converged
        i_host = f_host.info()
        assert i_host.step_prec == i_dev.step_prec
        assert i_host.step_fp64 == i_dev.step_fp64
        L_host = f_host.lower().cpu().numpy()
        bad = np.argwhere(L_host != L_dev)
        assert bad.size == 0, (bad[:5], L_host[tuple(bad[0])], L_dev[tuple(bad[0])])


def test_copy_plan_is_validated(cuda):
    f = mp.Factor(2048, block_size=256, precision="fp16x2")
    with pytest.raises(mp.MpcholError):
        f.set_copy_plan([3], [3])          # joins after its first block column is needed
    with pytest.raises(mp.MpcholError):
        f.set_copy_plan([5, 3], [1, 2])    # cuts not increasing
    with pytest.raises(mp.MpcholError):
        f.set_copy_plan([2, 4], [1, 0])    # join steps decreasing
    f.set_copy_plan([], [])                # one group: copy, then factor
    f.set_copy_plan(None)
    g = mp.Factor(2048, block_size=64, precision="fp16x2")
    with pytest.raises(mp.MpcholError):
        g.set_copy_plan([4], [2])          # 128-row tiles would straddle groups


@pytest.mark.parametrize("opts", [LADDER, dict(precision="fp32")])
def test_factor_graph_relaunch_is_bit_identical(cuda, opts):
    """Repeated compute() on one factor object: the first call launches the
    kernels directly, the second captures the factorization as a CUDA graph,
    later calls relaunch it.  Every factor must be the same bits."""
    n = 1536
    A = matgen.spd_matrix(n, 1e5, 61).cuda()
    f = mp.Factor(n, block_size=256, **opts)
    ref = None
    for _ in range(4):
        f.compute(A)
        L = f.lower().cpu().numpy()
        if ref is None:
            ref, prec = L, f.info().step_prec
        else:
            assert np.array_equal(L, ref)
            assert f.info().step_prec == prec
