"""Batched factor + PCG of many uneven systems against the single-system path
and the FP64 dense oracle.

The batched kernels run the same arithmetic as the single-system ones (only
the staging and the work distribution differ), so every system's factor must
equal, bit for bit, the factor mpchol_factor computes for it alone.  Every
solution is checked against the FP64 dense Cholesky solve.
"""
import numpy as np
import pytest
import torch

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import matgen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def systems(count, lo, hi, seed, kmax=1e4):
    ns = matgen.batch_sizes(count, lo, hi, seed)
    kappas = matgen.batch_kappas(count, 1e1 if kmax <= 1e2 else 1e2, kmax, seed + 1)
    As = [matgen.spd_matrix(int(n), float(k), 100 + i).numpy() for i, (n, k) in enumerate(zip(ns, kappas))]
    return [int(n) for n in ns], As


@pytest.mark.parametrize("precision,b,nrhs", [("fp16", 128, 4), ("e4m3", 128, 1),
                                               ("fp16x2", 256, 2), ("mxfp8", 128, 1)])
def test_batch_factor_equals_single_and_solves(cuda, precision, b, nrhs):
    # FP8 factors need well-conditioned systems for PCG to finish in a few
    # hundred iterations
    ns, As = systems(10, 64, 700, 5, kmax=1e2 if precision in ("e4m3", "mxfp8") else 1e4)
    ns[3] = 64          # a one-step system
    As[3] = matgen.spd_matrix(64, 1e2, 77).numpy()
    Ad = [torch.from_numpy(A).cuda() for A in As]
    bt = mp.Batch(ns, nrhs=nrhs, block_size=b, precision=precision)
    bt.factor(Ad)
    st, rows, _ = bt.info()
    assert all(s_ == 0 for s_ in st), st
    for i, A in enumerate(Ad):
        f = mp.factor(A, block_size=b, precision=precision)
        assert torch.equal(bt.lower(i), f.lower()), f"system {i} (n={ns[i]}) factor differs"
    g = np.random.default_rng(9)
    Bs = [g.standard_normal((n, nrhs)) for n in ns]
    Bd = [torch.from_numpy(B).cuda() for B in Bs]
    Xs, reps, status = bt.pcg(Ad, Bd, rel_tol=1e-10, max_it=600)
    print(precision, [r.iterations for r in reps])
    assert status == 0
    for i, (A, B, X, r) in enumerate(zip(As, Bs, Xs, reps)):
        Xh = X.cpu().numpy()
        res = np.linalg.norm(B - A.astype(np.float64) @ Xh, axis=0) / np.linalg.norm(B, axis=0)
        assert r.converged and res.max() <= 1.5e-10, (i, ns[i], r, res.max())
        Xd = O.dense_solve(A, B)
        assert np.linalg.norm(Xh - Xd) / np.linalg.norm(Xd) < 1e4 * 1e-9
        assert r.iterations >= 1


def test_batch_matches_single_pcg_iterations(cuda):
    ns, As = systems(6, 100, 500, 11)
    Ad = [torch.from_numpy(A).cuda() for A in As]
    bt = mp.Batch(ns, nrhs=1, block_size=128, precision="fp16").factor(Ad)
    Bs = [torch.from_numpy(np.random.default_rng(i).standard_normal(n)).cuda() for i, n in enumerate(ns)]
    Xs, reps, status = bt.pcg(Ad, Bs, rel_tol=1e-10, max_it=300, check_every=2)
    assert status == 0
    for i, A in enumerate(Ad):
        f = mp.factor(A, block_size=128, precision="fp16")
        X1, r1 = f.pcg(A, Bs[i], rel_tol=1e-10, max_it=300, check_every=2)
        # same preconditioner, same recurrences: the counts agree up to the
        # pair granularity of the batched loop and the restart points
        assert abs(reps[i].iterations - r1.iterations) <= 3, (i, reps[i], r1)
        assert torch.allclose(Xs[i], X1, rtol=0, atol=1e-8 * X1.abs().max().item())
