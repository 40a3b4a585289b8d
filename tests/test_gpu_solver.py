"""Factor and solver parity against the CPU oracle and the FP64 dense solve.

Factor parity: the GPU factor is compared with the oracle's blocked
restatement run with the same per-step precisions and FP64-diagonal flags (read
back from the GPU), by relative Frobenius error of the lower triangle with a
per-precision bar.  Solutions are checked against the FP64 dense Cholesky
solve, with the FP64 true residual, backward error and iteration count.
"""
import ctypes

import numpy as np
import pytest
import torch

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import _lib, matgen
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# relative Frobenius bar of ||L_gpu - L_oracle|| / ||L_oracle|| per step precision
FACTOR_TOL = {O.FP32: 1e-5, O.FP16: 1e-3, O.E4M3: 5e-2, O.E5M2: 5e-2, O.MXFP8: 5e-2,
              O.FP16X2: 3e-5}


def factor_parity(A: np.ndarray, **opts):
    f = mp.factor(torch.from_numpy(A).cuda(), **opts)
    info = f.info()
    Lg = f.lower().cpu().numpy()
    # the oracle with the factor's own options (library defaults included),
    # run with the GPU's per-step precisions and FP64-diagonal flags
    kw = O.factor_kwargs(f.opts)
    kw["precision"] = O.SWITCHING
    ref = O.blocked_chol(A, force_prec=info.step_prec, force_fp64=info.step_fp64, **kw)
    Lo = ref["L"]
    err = np.linalg.norm(Lg - Lo) / np.linalg.norm(Lo)
    return f, info, ref, err


@pytest.mark.parametrize("n,b,prec", [
    (1024, 128, "fp16"),    # the small plain-method workload (block 128, FP16 trailing)
    (1000, 128, "fp32"),    # ragged: n not a multiple of b
    (512, 256, "fp32"),
    (768, 256, "e4m3"),
    (640, 128, "e5m2"),
    (768, 256, "mxfp8"),    # block-scaled MX trailing updates (kind::mxf8f6f4)
    (1000, 128, "mxfp8"),   # ragged, K = 128
    (1024, 256, "fp16x2"),  # split FP16: FP32-class factor on tensor cores
    (96, 256, "fp32"),      # n < b: a single diagonal block
])
def test_factor_matches_oracle(cuda, n, b, prec):
    A = matgen.spd_matrix(n, 1e2 if prec in ("e4m3", "e5m2", "mxfp8") else 1e4, 1).numpy()
    f, info, ref, err = factor_parity(A, block_size=b, precision=prec)
    assert info.status == 0 and ref["status"] == 0
    worst = max([O.FP32] + [p for p in info.step_prec[:-1]], key=lambda p: FACTOR_TOL[p])
    print(f"n={n} b={b} {prec}: steps {info.step_prec} rel Frobenius {err:.2e}")
    assert err < FACTOR_TOL[worst], err


def test_switching_decisions_match_oracle_rule(cuda):
    n, b = 1536, 256
    A = matgen.spd_matrix(n, 1e6, 3).numpy()
    # rounding-error diagonal shifts on (without them FP16 steps make this
    # kappa = 1e6 factor indefinite; the oracle breaks down the same way)
    f, info, ref, err = factor_parity(A, block_size=b, eps_prime=0.05, diag_pert=1, pert=1.0)
    assert info.status == 0 and info.n_perturbed == 0
    # FP16 steps at kappa = 1e6: two correct factorizations differ by up to
    # ~kappa(L) * u16 in the trailing blocks
    assert err < 5e-3
    # re-derive each step's choice from the oracle's own tracker on the GPU's
    # precision path: the rule must agree step by step
    r2 = O.blocked_chol(A, block_size=b, precision=O.SWITCHING, eps_prime=0.05, diag_pert=1,
                        pert=1.0)
    assert list(r2["step_prec"][:-1]) == list(info.step_prec[:-1])
    d, dt = f.diags()
    # dtilde = d - sum L^2 loses digits to cancellation when it is small
    # (d ~ 1 here): compare with an absolute floor
    np.testing.assert_allclose(dt.cpu().numpy(), ref["dtilde"], rtol=1e-3, atol=2e-5)


def test_factor_matches_oracle_at_full_c2_size(cuda):
    """The C2 configuration at its full size: n = 8192, kappa = 1e6 (seed 3),
    block 256, switching {E4M3, FP16, FP16X2} at eps' = 1e-5 -- the bench's
    spd line.  The oracle (OpenMP restatement on the host cores) re-derives
    every step's precision on its own and restates the factor; PCG on the GPU
    reaches 1e-10 in the oracle PCG's iteration count on the GPU's factor."""
    n, b = 8192, 256
    A = matgen.spd_matrix(n, 1e6, 3).numpy()
    opts = dict(block_size=b, precision="switching", eps_prime=1e-5,
                ladder=["e4m3", "fp16", "fp16x2"])
    f, info, ref, err = factor_parity(A, **opts)
    kw = O.factor_kwargs(f.opts)
    own = O.blocked_chol(A, **kw)
    assert info.status == 0 and own["status"] == 0
    assert list(own["step_prec"][:-1]) == info.step_prec[:-1]
    print(f"C2 n={n}: steps {set(info.step_prec[:-1])}, rel Frobenius vs oracle {err:.2e}")
    # FP16X2 steps at kappa = 1e6: two FP32-class factorizations differ by
    # about kappa(L) * u32 in the last blocks
    assert err < 1e-3
    B = matgen.rhs(n, 1, 100).numpy()
    Ad = torch.from_numpy(A).cuda()
    X, rep = f.pcg(Ad, torch.from_numpy(B).cuda(), rel_tol=1e-10, max_it=100)
    assert rep.converged and rep.rel_residual <= 1e-10
    _, it_o, _ = O.pcg(A, f.lower().cpu().numpy(), B, 1e-10, 100)
    print(f"  pcg it={rep.iterations} (oracle {it_o}) rel={rep.rel_residual:.2e}")
    assert abs(rep.iterations - it_o) <= 1


def test_not_spd_reports_failing_row(cuda):
    A = matgen.spd_matrix(512, 10.0, 4).numpy()
    A[300, 300] = -1.0
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=128, precision="fp32", diag_pert=0)
    info = f.info()
    assert info.status == _lib.ERR_NOT_SPD and info.fail_row == 300


def test_fp64_diagonal_fallback_flags_blocks(cuda):
    # kappa = 1e4 keeps two FP32 factorizations within 1e-5 of each other
    # (their difference scales like kappa(L) * u); floor = 0.99 flags almost
    # every block after the first for the FP64 diagonal POTRF
    A = matgen.spd_matrix(768, 1e4, 6).numpy()
    f, info, ref, err = factor_parity(A, block_size=128, precision="fp32", floor=0.99)
    assert info.n_fp64_blocks >= 3
    assert err < 1e-5


def test_apply_precond_matches_oracle_potrs(cuda):
    n = 1000
    A = matgen.spd_matrix(n, 1e4, 2).numpy()
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=128, precision="fp16")
    L = f.lower().cpu().numpy()
    R = np.random.default_rng(0).standard_normal((n, 3))
    Z = f.apply_precond(torch.from_numpy(R).cuda()).cpu().numpy()
    want = O.potrs(L, R)
    # the solves apply FP32-rounded inverses of the 1024-row diagonal
    # super-blocks (FP64 vectors and accumulation): agreement to ~1e-6
    err = np.abs(Z - want).max() / np.abs(want).max()
    print(f"apply_precond rel err {err:.2e}")
    assert err < 1e-5
    # and the applied operator is symmetric: u^T M^-1 v == v^T M^-1 u
    u = np.random.default_rng(1).standard_normal(n)
    v = np.random.default_rng(2).standard_normal(n)
    Mu = f.apply_precond(torch.from_numpy(u).cuda()).cpu().numpy()
    Mv = f.apply_precond(torch.from_numpy(v).cuda()).cpu().numpy()
    assert abs(v @ Mu - u @ Mv) <= 1e-10 * abs(v @ Mu)


@pytest.mark.parametrize("n,nrhs", [(2100, 8), (1024, 8)])
def test_apply_precond_8_rhs_matches_oracle_potrs(cuda, n, nrhs):
    """The triangular solves with 8 right-hand sides (the FP64 tensor-core
    tile pass of the persistent solve), ragged super-blocks included."""
    A = matgen.spd_matrix(n, 1e4, 12).numpy()
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision="fp16x2")
    L = f.lower().cpu().numpy()
    R = np.random.default_rng(3).standard_normal((n, nrhs))
    Z = f.apply_precond(torch.from_numpy(R).cuda()).cpu().numpy()
    want = O.potrs(L, R)
    err = np.abs(Z - want).max() / np.abs(want).max()
    print(f"apply_precond n={n} nrhs={nrhs} rel err {err:.2e}")
    assert err < 1e-5


@pytest.mark.parametrize("n,b,prec,kappa,nrhs", [
    (1024, 128, "fp16", 1e4, 1),     # plain-method workload
    (1024, 128, "fp32", 1e4, 2),
    (2048, 256, "switching", 1e6, 1),
    (2048, 256, "fp16x2", 1e6, 1),
    (1000, 128, "fp32", 1e3, 8),
    (1024, 128, "mxfp8", 1e3, 2),
])
def test_pcg_reaches_1e10_and_matches_dense_solve(cuda, n, b, prec, kappa, nrhs):
    A = matgen.spd_matrix(n, kappa, 1).numpy()
    B = matgen.rhs(n, nrhs, 2).numpy()
    Ad = torch.from_numpy(A).cuda()
    f = mp.factor(Ad, block_size=b, precision=prec, eps_prime=0.05)
    X, rep = f.pcg(Ad, torch.from_numpy(B).cuda(), rel_tol=1e-10, max_it=300)
    X = X.cpu().numpy()
    print(f"n={n} {prec} kappa={kappa:.0e}: it={rep.iterations} rel={rep.rel_residual:.2e} "
          f"be={rep.backward_error:.2e}")
    assert rep.converged and rep.rel_residual <= 1e-10
    res = np.linalg.norm(B - A.astype(np.float64) @ X, axis=0) / np.linalg.norm(B, axis=0)
    assert res.max() <= 1.5e-10
    Xd = O.dense_solve(A, B)
    assert np.linalg.norm(X - Xd) / np.linalg.norm(Xd) < kappa * 1e-9
    # the oracle's PCG on the GPU's factor takes a comparable number of iterations
    _, it_o, _ = O.pcg(A, f.lower().cpu().numpy(), B if nrhs > 1 else B, 1e-10, 300)
    assert abs(rep.iterations - it_o) <= max(3, it_o // 5)


def test_pcg_fp64_operator(cuda):
    n = 512
    A32 = matgen.spd_matrix(n, 1e3, 9)
    A64 = A32.double().cuda()
    B = matgen.rhs(n, 1, 3).cuda()
    f = mp.factor(A32.cuda(), block_size=128, precision="fp16")
    X, rep = f.pcg(A64, B, rel_tol=1e-12)
    assert rep.converged and rep.rel_residual <= 1e-12


def test_pcg_maxit_is_reported(cuda):
    n = 512
    A = matgen.spd_matrix(n, 1e6, 9).cuda()
    B = matgen.rhs(n, 1, 3).cuda()
    f = mp.factor(A, block_size=128, precision="fp16")
    X, rep = f.pcg(A, B, rel_tol=1e-14, max_it=2, check_every=1)
    assert rep.status == _lib.PCG_MAXIT and not rep.converged and rep.iterations == 2


def test_reference_shaped_precond_cg(cuda):
    n = 768
    A = matgen.spd_matrix(n, 1e4, 12).double().cuda()
    b = matgen.rhs(n, 1, 13).cuda()
    x = torch.zeros_like(b)
    rc = mp.precond_CG(A, x, b, n, 128, 0.0, eps_prime=0.05, rel_tol=1e-10, max_it=200)
    assert rc == 0
    r = b - A @ x
    assert (r.norm() / b.norm()).item() <= 1e-10
    # reference default rel_tol = 0: runs max_it and reports "not converged"
    x2 = torch.zeros_like(b)
    assert mp.precond_CG(A, x2, b, n, 128, 0.0, eps_prime=0.05, rel_tol=0.0, max_it=5) == -1


def test_reference_shaped_switching_chol(cuda):
    n = 512
    A = matgen.spd_matrix(n, 1e3, 14)
    dA = A.clone().cuda()            # symmetric: row-major storage == column-major
    d = torch.zeros(n, device="cuda")
    dt = torch.zeros(n, device="cuda")
    assert mp.switching_chol(dA, n, 128, d, dt, 0.05) == 0
    Lg = dA.cpu().numpy().T          # column-major result viewed back
    Lg = np.tril(Lg)
    L64 = np.linalg.cholesky(A.double().numpy())
    assert np.linalg.norm(Lg - L64) / np.linalg.norm(L64) < 2e-3
    np.testing.assert_allclose(d.cpu().numpy(), np.diag(A.numpy()))


@pytest.mark.parametrize("n,nrhs", [(1000, 2), (768, 1)])
def test_solve_host_matches_device_path(cuda, n, nrhs):
    """mpchol_solve_host (host buffers, lower triangle copied by block columns)
    gives the device path's solution: same factor, same operator, the same PCG
    iteration count (within one).  The solutions agree to 1e-8 relative: the operator and
    preconditioner products combine partial sums with FP64 atomics, whose
    order varies from run to run (differences ~1e-10 relative)."""
    A = matgen.spd_matrix(n, 1e4, 41)
    B = matgen.rhs(n, nrhs, 42).to(torch.float64)
    opts = dict(block_size=256, precision="switching", eps_prime=1e-5,
                ladder=["e4m3", "fp16", "fp16x2"])
    f_dev = mp.Factor(n, **opts)
    f_dev.compute(A.cuda())
    Xd, rd = f_dev.pcg(A.cuda(), B.cuda(), rel_tol=1e-10)
    f_host = mp.Factor(n, **opts)
    for _ in range(2):   # the second call reuses the buffers the first allocated
        Xh, rh = f_host.solve_host(A.pin_memory(), B.pin_memory(), rel_tol=1e-10)
        assert rh.converged and abs(rh.iterations - rd.iterations) <= 1
        assert Xh.device.type == "cpu" and Xh.shape == B.shape
        err = np.linalg.norm(Xh.numpy() - Xd.cpu().numpy()) / np.linalg.norm(Xd.cpu().numpy())
        assert err < 1e-8, err
    xd = O.dense_solve(A.numpy().astype(np.float64), B.numpy())
    assert np.linalg.norm(Xh.numpy() - xd) / np.linalg.norm(xd) < 1e-6


@pytest.mark.parametrize("n", [1000, 999])
def test_reported_backward_error_matches_numpy(cuda, n):
    """The report's backward error ||b - Ax|| / (||A||_F ||x|| + ||b||) matches
    numpy's.  n = 1000 takes ||A||_F from the first operator product (staged
    SYMV, columns 16-byte aligned); n = 999 (odd leading dimension) from the
    separate norm kernel."""
    A = matgen.spd_matrix(n, 1e4, 31)
    b = matgen.rhs(n, 1, 32)
    f = mp.factor(A.cuda(), block_size=256, precision="fp16x2")
    X, rep = f.pcg(A.cuda(), b.cuda(), rel_tol=1e-10)
    assert rep.converged
    A64 = A.double().numpy()
    x = X.cpu().numpy()
    bb = b.numpy()
    be = np.linalg.norm(bb - A64 @ x) / (np.linalg.norm(A64) * np.linalg.norm(x) + np.linalg.norm(bb))
    assert rep.backward_error == pytest.approx(be, rel=0.05), (rep.backward_error, be)


def test_factor_save_load_round_trip(cuda):
    """A factor saved before a solve, restored into a new object, gives the
    same L bits, step precisions, status word (floored pivots) and PCG solve
    without refactoring; a solve does not change the factor's status word, so
    a factor saved after the solve carries the same status; the target's
    storage outside L's lower triangle is never read (NaN-filled before the
    load); a blob of another order or block size is refused."""
    n = 1000
    # kappa = 1e6 with a pivot floor of 1e-3 d_i: a few hundred pivots are
    # raised to the floor (a modified-Cholesky preconditioner, still SPD)
    A = matgen.spd_matrix(n, 1e6, 71)
    B = matgen.rhs(n, 2, 72).to(torch.float64)
    opts = dict(block_size=256, precision="switching", eps_prime=1e-5, pivot_floor=1e-3,
                ladder=["e4m3", "fp16", "fp16x2"])
    f = mp.Factor(n, **opts)
    f.compute(A.cuda())
    fi = f.info()
    assert fi.status == 0 and fi.n_perturbed > 0
    blob = f.save()                          # before any solve
    X1, r1 = f.pcg(A.cuda(), B.cuda(), rel_tol=1e-10, max_it=400)
    assert f.info().n_perturbed == fi.n_perturbed
    assert f.save() == blob                  # the solve left the factor's state alone
    assert mp.factor_blob_info(blob) == (n, 256)
    g = mp.Factor(n, **opts)
    p = ctypes.c_void_p()
    ld = ctypes.c_int()
    nn = ctypes.c_int()
    g.lib.mpchol_factor_lower(g.handle, ctypes.byref(p), ctypes.byref(ld), ctypes.byref(nn))
    from cholesky_gpu_b200.api import _wrap_device
    _wrap_device(p.value, (n, ld.value), torch.float32).fill_(float("nan"))
    g.load(blob)
    assert torch.equal(g.lower(), f.lower())
    gi = g.info()
    assert gi.step_prec == fi.step_prec and gi.step_fp64 == fi.step_fp64
    assert gi.status == fi.status and gi.n_perturbed == fi.n_perturbed
    X2, r2 = g.pcg(A.cuda(), B.cuda(), rel_tol=1e-10, max_it=400)
    # same factor bits; the solves themselves sum their FP64 products with
    # atomics in no fixed order, so at kappa = 1e6 the count may differ by one
    assert r1.converged and r2.converged and abs(r2.iterations - r1.iterations) <= 1
    x1, x2 = X1.cpu().numpy(), X2.cpu().numpy()
    assert np.linalg.norm(x2 - x1) / np.linalg.norm(x1) < 1e-8
    with pytest.raises(mp.MpcholError):
        mp.Factor(n + 1, **opts).load(blob)
    with pytest.raises(mp.MpcholError):
        mp.Factor(n, **dict(opts, block_size=128)).load(blob)
