"""FP8 / MXFP8 factors the preconditioned solve wins back, the coherence rule
of the switching criterion, the non-finite-pivot guard, equilibration, the
adjoint solve and the reference-literal switching mode -- on the GPU, against
the oracle and the FP64 dense solve.

The kernel matrix here is the RBF workload's shape at a size the oracle
factors in a second: 2048 points in [0,1]^784 with 80 % zero coordinates,
the median pairwise distance as lengthscale, nugget 1e-3 (condition number
about 2e4).  Its first panel is the matrix's constant mode, which an FP8
update cannot carry (the coherence rule sends that step to FP16X2); every
later step runs in MXFP8.
"""
import numpy as np
import pytest
import torch

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import _lib, matgen
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LADDER = ["mxfp8", "fp16", "fp16x2"]


@pytest.fixture(scope="module")
def rbf2048():
    X = torch.from_numpy(matgen.mnist_like_points(2048, 784, 4))
    ell = matgen.median_pairwise_distance(X)
    return matgen.rbf_matrix(X, ell, 1e-3).numpy()


def oracle_factor(A, f, force=True):
    info = f.info()
    kw = O.factor_kwargs(f.opts)
    if force:
        kw["precision"] = O.SWITCHING
        return O.blocked_chol(A, force_prec=info.step_prec, force_fp64=info.step_fp64, **kw), info
    return O.blocked_chol(A, **kw), info


def test_coherence_rule_picks_mxfp8_after_the_constant_mode(cuda, rbf2048):
    """Switching with ladder {MXFP8, FP16, FP16X2}, eps' = 2: the GPU's step
    precisions equal the oracle's own decisions (coherence ratio and Schur
    ratio recomputed on the CPU), step 0 is FP16X2, the rest MXFP8; the
    factor matches the oracle's restatement and PCG reaches 1e-10 on the
    FP64 true residual in about the oracle's iteration count."""
    A = rbf2048
    n = A.shape[0]
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision="switching",
                  eps_prime=2.0, ladder=LADDER)
    ref, info = oracle_factor(A, f, force=False)
    assert info.status == 0 and ref["status"] == 0
    gpu_steps = info.step_prec[:-1]
    assert list(ref["step_prec"][:-1]) == gpu_steps
    assert gpu_steps[0] == _lib.PREC_FP16X2
    assert all(p == _lib.PREC_MXFP8 for p in gpu_steps[1:])
    Lg = f.lower().cpu().numpy()
    err = np.linalg.norm(Lg - ref["L"]) / np.linalg.norm(ref["L"])
    print(f"rbf n={n} steps {gpu_steps}: factor rel Frobenius vs oracle {err:.2e}")
    # MXFP8 steps: a one-ulp FP32 difference in a panel value (accumulation
    # order) can move an E4M3 code by one step (2^-4 relative); measured
    # 2.9e-3 on the B200
    assert err < 1e-2
    B = matgen.rhs(n, 2, 5).numpy()
    Ad = torch.from_numpy(A).cuda()
    X, rep = f.pcg(Ad, torch.from_numpy(B).cuda(), rel_tol=1e-10, max_it=100)
    print(f"  pcg it={rep.iterations} rel={rep.rel_residual:.2e} be={rep.backward_error:.2e}")
    assert rep.converged and rep.rel_residual <= 1e-10
    Xd = O.dense_solve(A, B)
    assert np.linalg.norm(X.cpu().numpy() - Xd) / np.linalg.norm(Xd) < 1e-6
    _, it_o, _ = O.pcg(A, ref["L"], B, 1e-10, 100)
    assert abs(rep.iterations - it_o) <= max(3, it_o // 4)


def test_coherence_rule_off_lets_step0_take_mxfp8_and_the_guard_reports_it(cuda, rbf2048):
    """Without the coherence rule the ratio test alone gives step 0 to MXFP8;
    the constant mode's rounding error then makes the Schur complement
    indefinite, the floored pivots overflow the next blocks, and the factor
    reports NOT_SPD (a non-finite pivot) -- as the oracle does -- instead of
    handing PCG a factor that breaks down.  PCG refuses the failed factor."""
    A = rbf2048
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision="switching",
                  eps_prime=2.0, ladder=LADDER, coherence=0)
    ref, info = oracle_factor(A, f, force=False)
    assert info.step_prec[0] == _lib.PREC_MXFP8
    assert ref["status"] == _lib.ERR_NOT_SPD
    assert info.status == _lib.ERR_NOT_SPD and info.fail_row >= 256
    B = matgen.rhs(A.shape[0], 1, 5).cuda()
    with pytest.raises(mp.MpcholError) as e:
        f.pcg(torch.from_numpy(A).cuda(), B, rel_tol=1e-10, max_it=50)
    assert e.value.status == _lib.ERR_NOT_SPD
    with pytest.raises(mp.MpcholError) as e:
        f.save()
    assert e.value.status == _lib.ERR_NOT_SPD


@pytest.mark.parametrize("prec", ["e4m3", "mxfp8"])
def test_fp8_factor_with_shifts_is_won_back_at_kappa_1e4(cuda, prec):
    """A fixed FP8 factor of a kappa = 1e4 SPD matrix with rounding-error
    diagonal shifts of 4 u_p sum L^2: the factor matches the oracle, and PCG
    reaches 1e-10 (about 160 iterations, against 6 for FP16)."""
    n = 1024
    A = matgen.spd_matrix(n, 1e4, 1).numpy()
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision=prec, pert=4.0)
    ref, info = oracle_factor(A, f)
    assert info.status == 0 and ref["status"] == 0 and info.n_perturbed == 0
    Lg = f.lower().cpu().numpy()
    err = np.linalg.norm(Lg - ref["L"]) / np.linalg.norm(ref["L"])
    B = matgen.rhs(n, 1, 2).numpy()
    Ad = torch.from_numpy(A).cuda()
    X, rep = f.pcg(Ad, torch.from_numpy(B).cuda(), rel_tol=1e-10, max_it=400)
    _, it_o, _ = O.pcg(A, ref["L"], B, 1e-10, 400)
    print(f"{prec} kappa=1e4: factor err vs oracle {err:.2e}, it {rep.iterations} (oracle {it_o})")
    assert err < 5e-3          # measured 1.5e-3 (E4M3) and 1.6e-3 (MXFP8) on the B200
    assert rep.converged and rep.rel_residual <= 1e-10
    assert abs(rep.iterations - it_o) <= max(10, it_o // 5)


def test_equilibrated_factor_matches_oracle_on_a_badly_scaled_matrix(cuda):
    """S A S with S = diag(10^U(-1, 1)): equilibration (powers of two) gives
    the oracle's factor (scaled, factored, rows scaled back) and PCG on the
    unscaled operator converges.  (A wider scaling makes 1e-10 unreachable
    for any solver: with S spanning 10^6 the FP64 residual of the scaled
    system bottoms out near 5e-10, at a backward error of 4e-23.)"""
    n = 768
    A0 = matgen.spd_matrix(n, 1e3, 21).double().numpy()
    s = 10.0 ** np.random.default_rng(3).uniform(-1, 1, n)
    A = (A0 * s[:, None] * s[None, :]).astype(np.float32)
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=128, precision="fp16x2", equilibrate=1)
    ref, info = oracle_factor(A, f)
    assert info.status == 0 and ref["status"] == 0
    Lg = f.lower().cpu().numpy()
    err = np.linalg.norm((Lg - ref["L"]) / s[:, None]) / np.linalg.norm(ref["L"] / s[:, None])
    print(f"equilibrated fp16x2: row-normalised factor err vs oracle {err:.2e}")
    assert err < 3e-5
    d, _ = f.diags()
    dd = d.cpu().numpy()
    assert dd.min() >= 0.5 and dd.max() < 2.0
    B = matgen.rhs(n, 1, 4)
    Ad = torch.from_numpy(A).cuda()
    X, rep = f.pcg(Ad, B.cuda(), rel_tol=1e-10)
    assert rep.converged and rep.rel_residual <= 1e-10


def test_adjoint_solve_reuses_the_factor(cuda):
    """mpchol_adjoint_solve: lambda = A^-1 g by PCG on the forward factor and
    the dense cotangent -(lambda x^T + x lambda^T) / 2, against FP64."""
    n = 640
    A = matgen.spd_matrix(n, 1e4, 51).double()
    B = matgen.rhs(n, 2, 52)
    G = matgen.rhs(n, 2, 53)
    Ad = A.cuda()
    f = mp.factor(A.float().cuda(), block_size=128, precision="fp16x2")
    X, rep = f.pcg(Ad, B.cuda(), rel_tol=1e-12)
    assert rep.converged
    Lam, GA, arep = f.adjoint_solve(Ad, X, G.cuda(), rel_tol=1e-12, grad_a=True)
    assert arep.converged and arep.rel_residual <= 1e-12
    lam_d = O.dense_solve(A.numpy(), G.numpy())
    lam = Lam.cpu().numpy()
    assert np.linalg.norm(lam - lam_d) / np.linalg.norm(lam_d) < 1e-8
    x = X.cpu().numpy()
    want = -0.5 * (lam @ x.T + x @ lam.T)
    got = np.tril(GA.cpu().numpy())
    np.testing.assert_allclose(got, np.tril(want), rtol=1e-10, atol=1e-12 * np.abs(want).max())


def test_reference_literal_switching_mode_matches_oracle(cuda):
    """switch_mode = 1 (the reference's can_switch comparison with its machine
    epsilons, src/kernels_macros.cuh:191-211): the GPU's per-step choices are
    the oracle's, and the factor matches its restatement."""
    n = 1536
    A = matgen.spd_matrix(n, 1e4, 8).numpy()
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision="switching",
                  switch_mode=1, eps_prime=1e-4)
    ref, info = oracle_factor(A, f, force=False)
    assert info.status == 0 and ref["status"] == 0
    print(f"literal mode steps {info.step_prec}")
    assert list(ref["step_prec"][:-1]) == info.step_prec[:-1]
    assert set(info.step_prec[:-1]) <= {_lib.PREC_FP32, _lib.PREC_FP16, _lib.PREC_E4M3}
    forced, _ = oracle_factor(A, f)
    Lg = f.lower().cpu().numpy()
    err = np.linalg.norm(Lg - forced["L"]) / np.linalg.norm(forced["L"])
    assert err < 5e-2


@pytest.mark.parametrize("low", ["mxfp6e2m3", "mxfp6e3m2", "mxfp4"])
def test_fp6_fp4_steps_on_the_kernel_matrix(cuda, rbf2048, low):
    """FP6/FP4 trailing updates (OCP MX element formats) in a switching
    ladder on the RBF matrix: the GPU's decisions are the oracle's, the factor
    matches its restatement, and PCG wins the factor back to 1e-10."""
    A = rbf2048
    n = A.shape[0]
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision="switching",
                  eps_prime=2.0, eps_coherence=0.25, ladder=[low, "fp16", "fp16x2"])
    ref, info = oracle_factor(A, f, force=False)
    assert info.status == 0 and ref["status"] == 0
    assert list(ref["step_prec"][:-1]) == info.step_prec[:-1]
    lowid = _lib.PREC_BY_NAME[low]
    nlow = sum(p == lowid for p in info.step_prec[:-1])
    Lg = f.lower().cpu().numpy()
    err = np.linalg.norm(Lg - ref["L"]) / np.linalg.norm(ref["L"])
    B = matgen.rhs(n, 2, 5).numpy()
    Ad = torch.from_numpy(A).cuda()
    X, rep = f.pcg(Ad, torch.from_numpy(B).cuda(), rel_tol=1e-10, max_it=300)
    _, it_o, _ = O.pcg(A, ref["L"], B, 1e-10, 300)
    print(f"{low}: steps {info.step_prec[:-1]} ({nlow} {low}), factor err {err:.2e}, "
          f"it {rep.iterations} (oracle {it_o})")
    assert nlow >= 1
    assert err < 5e-2
    assert rep.converged and rep.rel_residual <= 1e-10
    assert abs(rep.iterations - it_o) <= max(3, it_o // 4)
