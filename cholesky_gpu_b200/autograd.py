"""Differentiable RBF kernel solve: x = K(X, l, nugget)^-1 y.

A ``torch.autograd.Function`` over the C ABI.  Forward builds K in FP64 (the
PCG operator) and FP32 (what the factor reads) with ``mpchol_rbf_build``,
factors the FP32 copy with the mixed-precision factor and solves with PCG on
the FP64 operator.  Backward runs one adjoint PCG solve a = K^-1 (dL/dx) that
reuses the forward's factor as its preconditioner, then
``mpchol_rbf_grad`` recomputes the K tiles from X to contract the cotangent
G_K = -(a x^T + x a^T) / 2 into the gradients for X, the lengthscale, the
nugget and y.  There is no counterpart in the reference (its RBF file is a
stub, src/RBF.cu:1-45).  The adjoint solve is the C ABI's mpchol_adjoint_solve,
so a caller outside Python can compose the same backward pass.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .api import Factor, _stream_handle
from ._lib import check, load


def rbf_build(X: torch.Tensor, lengthscale: float, nugget: float, fp64: bool = True,
              fp32: bool = True, lower_only: bool = True):
    """K_ij = exp(-||x_i - x_j||^2 / (2 l^2)) + nugget delta_ij for the rows
    of X (n x d FP32 CUDA tensor).  Returns (K64, K32); each is an n x n
    tensor whose storage is column-major (symmetric: the lower triangle holds
    K when lower_only)."""
    if not X.is_cuda or X.dtype != torch.float32 or X.dim() != 2:
        raise ValueError("X must be an n x d float32 CUDA tensor")
    Xc = X.contiguous()
    n, d = Xc.shape
    K64 = torch.zeros((n, n), dtype=torch.float64, device=X.device) if fp64 else None
    K32 = torch.zeros((n, n), dtype=torch.float32, device=X.device) if fp32 else None
    lib = load()
    check(lib.mpchol_rbf_build(Xc.data_ptr(), n, d, d, float(lengthscale), float(nugget),
                               None if K64 is None else K64.data_ptr(),
                               None if K32 is None else K32.data_ptr(), n, int(lower_only),
                               _stream_handle()), "mpchol_rbf_build")
    # the library wrote column-major storage: view it as such
    return (None if K64 is None else K64.t(), None if K32 is None else K32.t())


def rbf_grad_contract(X: torch.Tensor, lengthscale: float, a: torch.Tensor, b: torch.Tensor):
    """P = K_rbf [a, b, a*X, b*X] (n x (2 + 2d)) and s = sum a_i b_j K_ij r_ij^2,
    with K recomputed from X (FP64)."""
    Xc = X.contiguous()
    n, d = Xc.shape
    lib = load()
    P = torch.empty((2 + 2 * d, n), dtype=torch.float64, device=X.device)   # column-major n x NC
    s = torch.empty((1,), dtype=torch.float64, device=X.device)
    work = torch.empty((lib.mpchol_rbf_grad_work_elems(n),), dtype=torch.float64, device=X.device)
    ac = a.contiguous().double()
    bc = b.contiguous().double()
    check(lib.mpchol_rbf_grad(Xc.data_ptr(), n, d, d, float(lengthscale), ac.data_ptr(),
                              bc.data_ptr(), P.data_ptr(), s.data_ptr(), work.data_ptr(),
                              _stream_handle()), "mpchol_rbf_grad")
    return P.t(), s[0]


class RBFSolve(torch.autograd.Function):
    """x = K(X, lengthscale, nugget)^-1 y with a mixed-precision preconditioner."""

    @staticmethod
    def forward(ctx, X, lengthscale, nugget, y, opts):
        opts = dict(opts or {})
        rel_tol = opts.pop("rel_tol", 1e-12)
        max_it = opts.pop("max_it", 500)
        ell = float(lengthscale)
        lam = float(nugget)
        K64, K32 = rbf_build(X.detach(), ell, lam)
        n = X.shape[0]
        f = Factor(n, **opts)
        f.compute(K32)
        yd = y.detach().double()
        x, rep = f.pcg(K64, yd, rel_tol=rel_tol, max_it=max_it)
        if not rep.converged:
            raise RuntimeError(f"forward PCG did not converge: {rep}")
        ctx.factor, ctx.K64 = f, K64
        ctx.solve = (rel_tol, max_it)
        ctx.report = rep
        ctx.save_for_backward(X.detach(), yd, x)
        ctx.ell, ctx.lam = ell, lam
        ctx.param_meta = [(t.device, t.dtype) if torch.is_tensor(t) else None
                          for t in (lengthscale, nugget)]
        ctx.y_dtype = y.dtype
        return x.to(y.dtype)

    @staticmethod
    def backward(ctx, gx):
        X, y, x = ctx.saved_tensors
        rel_tol, max_it = ctx.solve
        ell = ctx.ell
        g = gx.detach().double()
        # adjoint solve, preconditioned by the forward's factor (the C ABI's
        # mpchol_adjoint_solve; the matrix cotangent stays implicit)
        a, _, rep = ctx.factor.adjoint_solve(ctx.K64, x, g, rel_tol=rel_tol, max_it=max_it)
        if not rep.converged:
            raise RuntimeError(f"adjoint PCG did not converge: {rep}")
        ctx.adjoint_report = rep
        A2 = a.reshape(a.shape[0], -1)
        X2 = x.reshape(x.shape[0], -1)
        n, d = X.shape
        Xd = X.double()
        dX = torch.zeros((n, d), dtype=torch.float64, device=X.device)
        s_tot = torch.zeros((), dtype=torch.float64, device=X.device)
        for r in range(A2.shape[1]):
            ar, br = A2[:, r], X2[:, r]
            P, s = rbf_grad_contract(X, ell, ar, br)
            Ka, Kb = P[:, 0], P[:, 1]
            KaX, KbX = P[:, 2:2 + d], P[:, 2 + d:]
            dX += (Xd * (ar * Kb + br * Ka).unsqueeze(1) - ar.unsqueeze(1) * KbX
                   - br.unsqueeze(1) * KaX) / (ell * ell)
            s_tot = s_tot + s
        d_ell = -s_tot / ell ** 3
        d_lam = -(A2 * X2).sum()
        dy = a.to(ctx.y_dtype)
        (le, lt), (ne, nt) = [m if m is not None else (None, None) for m in ctx.param_meta]
        d_ell = d_ell.to(device=le, dtype=lt) if le is not None else None
        d_lam = d_lam.to(device=ne, dtype=nt) if ne is not None else None
        return dX.to(X.dtype), d_ell, d_lam, dy, None


def rbf_solve(X: torch.Tensor, lengthscale, nugget, y: torch.Tensor, **opts) -> torch.Tensor:
    """Differentiable x = K^-1 y; lengthscale and nugget may be tensors that
    require grad.  opts: factor options (block_size, precision, ...) plus
    rel_tol / max_it for both PCG solves."""
    ell = lengthscale if torch.is_tensor(lengthscale) else torch.tensor(float(lengthscale),
                                                                        dtype=torch.float64)
    lam = nugget if torch.is_tensor(nugget) else torch.tensor(float(nugget), dtype=torch.float64)
    return RBFSolve.apply(X, ell, lam, y, opts)
