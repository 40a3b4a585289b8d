"""RBF kernel matrix builder and the differentiable solve against FP64 oracles.

Oracle: oracle.rbf_kernel_f64 / rbf_loss_grads_f64 (dense FP64 Cholesky), whose
analytic gradients are pinned against FP64 central finite differences in
tests/test_oracle.py.  Bars: the FP64 kernel matrix to 1e-13 relative; the
gradients to 1e-6 relative (the target for the differentiation workload).
"""
import numpy as np
import pytest
import torch

from cholesky_gpu_b200 import autograd as AG
from cholesky_gpu_b200 import matgen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("n,d,kind", [(300, 7, "gauss"), (160, 784, "mnist"), (64, 1, "gauss")])
def test_rbf_build_matches_fp64(cuda, n, d, kind):
    X = (matgen.gaussian_points(n, d, 6) if kind == "gauss"
         else matgen.mnist_like_points(n, d, 4))
    ell = 4.0 if kind == "gauss" else 9.0
    lam = 1e-2
    K64, K32 = AG.rbf_build(torch.from_numpy(X).cuda(), ell, lam, lower_only=False)
    want, _ = O.rbf_kernel_f64(X, ell, lam)
    got = K64.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    # the FP32 copy is the FP64 value rounded
    assert np.array_equal(K32.cpu().numpy(), got.astype(np.float32))
    # lower-only build writes only the lower triangle
    L64, _ = AG.rbf_build(torch.from_numpy(X).cuda(), ell, lam, fp32=False, lower_only=True)
    L = L64.cpu().numpy()
    low = np.tril(np.ones((n, n), bool))
    assert np.array_equal(L[low], got[low]) and not np.any(L[~low])


def test_rbf_grad_contraction_matches_dense(cuda):
    n, d, ell = 203, 5, 1.7
    g = np.random.default_rng(3)
    X = g.standard_normal((n, d)).astype(np.float32)
    a = g.standard_normal(n)
    b = g.standard_normal(n)
    P, s = AG.rbf_grad_contract(torch.from_numpy(X).cuda(), ell, torch.from_numpy(a).cuda(),
                                torch.from_numpy(b).cuda())
    K, r2 = O.rbf_kernel_f64(X, ell, 0.0)
    Xd = X.astype(np.float64)
    Z = np.concatenate([a[:, None], b[:, None], a[:, None] * Xd, b[:, None] * Xd], 1)
    assert rel(P.cpu().numpy(), K @ Z) < 1e-13
    s_want = float(a @ (K * r2) @ b)
    assert abs(s.item() - s_want) <= 1e-12 * abs(s_want)


@pytest.mark.parametrize("precision,n,d", [("e4m3", 512, 64), ("fp16", 640, 16),
                                            ("mxfp8", 2048, 64), ("fp16x2", 3072, 32)])
def test_rbf_solve_gradients_match_fp64(cuda, precision, n, d):
    """Loss 1/2 y^T K^-1 y of the differentiation workload's construction
    (x ~ N(0, I_d), l = 4, nugget = 1e-2, y ~ N(0,1)) at a size the dense
    oracle finishes in seconds."""
    X = matgen.gaussian_points(n, d, 6)
    y = np.random.default_rng(7).standard_normal(n)
    ell0, lam0 = 4.0, 1e-2
    Xt = torch.from_numpy(X).cuda().requires_grad_(True)
    ell = torch.tensor(ell0, dtype=torch.float64, requires_grad=True)
    lam = torch.tensor(lam0, dtype=torch.float64, requires_grad=True)
    yt = torch.from_numpy(y).cuda().requires_grad_(True)
    x = AG.rbf_solve(Xt, ell, lam, yt, block_size=128, precision=precision, rel_tol=1e-12)
    loss = 0.5 * (yt * x).sum()
    loss.backward()
    dX, d_ell, d_lam, xw = O.rbf_loss_grads_f64(X, ell0, lam0, y)
    print(f"{precision}: |dX| rel {rel(Xt.grad.cpu().numpy(), dX):.2e}  "
          f"dl {d_ell:.6e} vs {ell.grad.item():.6e}  dlam {d_lam:.6e} vs {lam.grad.item():.6e}")
    assert abs(loss.item() - O.rbf_loss_f64(X, ell0, lam0, y)) <= 1e-9 * abs(loss.item())
    assert rel(yt.grad.cpu().numpy(), xw) < 1e-6
    assert rel(Xt.grad.cpu().numpy(), dX) < 1e-6
    assert abs(ell.grad.item() - d_ell) <= 1e-6 * abs(d_ell)
    assert abs(lam.grad.item() - d_lam) <= 1e-6 * abs(d_lam)
    # and against FP64 central finite differences of the oracle loss (h = 1e-5)
    h = 1e-5
    fd_ell = (O.rbf_loss_f64(X, ell0 + h, lam0, y) - O.rbf_loss_f64(X, ell0 - h, lam0, y)) / (2 * h)
    fd_lam = (O.rbf_loss_f64(X, ell0, lam0 + h, y) - O.rbf_loss_f64(X, ell0, lam0 - h, y)) / (2 * h)
    assert abs(ell.grad.item() - fd_ell) <= 1e-6 * abs(fd_ell)
    assert abs(lam.grad.item() - fd_lam) <= 1e-6 * abs(fd_lam)
