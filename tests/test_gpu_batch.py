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
                                               ("fp16x2", 256, 2), ("mxfp8", 128, 1),
                                               ("fp16", 128, 8)])
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


def test_batch_of_512_systems(cuda):
    """The batch at the scale of the 512-system workload (orders U[64, 512],
    kappa up to 1e4, one rhs, FP16 trailing updates, block 128): every system
    reaches a 1e-10 FP64 true residual, and a sample of eight systems keeps
    the factor of the single-system path bit for bit."""
    count = 512
    ns = [int(n) for n in matgen.batch_sizes(count, 64, 512, 21)]
    kappas = matgen.batch_kappas(count, 1e2, 1e4, 22)
    Ad = [matgen.spd_matrix(n, float(k), 1000 + i, device="cuda") for i, (n, k) in enumerate(zip(ns, kappas))]
    bt = mp.Batch(ns, nrhs=1, block_size=128, precision="fp16").factor(Ad)
    st, rows, _ = bt.info()
    assert all(s_ == 0 for s_ in st), [i for i, s_ in enumerate(st) if s_ != 0]
    g = torch.Generator(device="cpu").manual_seed(23)
    Bd = [torch.randn(n, generator=g, dtype=torch.float64).cuda() for n in ns]
    Xs, reps, status = bt.pcg(Ad, Bd, rel_tol=1e-10, max_it=400)
    assert status == 0
    worst = 0.0
    for i, (A, B, X, r) in enumerate(zip(Ad, Bd, Xs, reps)):
        res = (torch.linalg.norm(B - A.double() @ X) / torch.linalg.norm(B)).item()
        assert r.converged and res <= 1.5e-10, (i, ns[i], r, res)
        worst = max(worst, res)
    print(f"512 systems: worst FP64 residual {worst:.2e}, iterations "
          f"{min(r.iterations for r in reps)}-{max(r.iterations for r in reps)}")
    for i in np.random.default_rng(24).choice(count, 8, replace=False):
        f = mp.factor(Ad[i], block_size=128, precision="fp16")
        assert torch.equal(bt.lower(int(i)), f.lower()), f"system {i} (n={ns[i]}) factor differs"
