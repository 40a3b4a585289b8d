"""Seeded synthetic inputs for the solver's workloads.

The reference generates its SPD test matrices as A = Q^T diag(sigma) Q with Q
from a QR factorization of a random matrix and one of four spectra
(src/matgen.cuh:98-298, src/kernels_macros.cuh:635-716).  The workloads here
follow that construction with their own seeded RNG: Q from QR of an N(0,1)
matrix, sigma geometric from 1 to 1/kappa.  The RBF workloads stand in for
MNIST (whose images are not available) with MNIST-shaped data: 784-dim points,
80 % zeros, the rest U(0,1).

Generation is input preparation, not part of any timed region.  Random draws
come from numpy's PCG64 so CPU and GPU runs see identical matrices; the dense
algebra (QR, products) runs in FP64 with torch on the requested device.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _rng(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


def geometric_spectrum(n: int, kappa: float) -> np.ndarray:
    """sigma_i = kappa^(-i/(n-1)), i = 0..n-1 (src/kernels_macros.cuh:669-675)."""
    if n == 1:
        return np.ones(1)
    return kappa ** (-np.arange(n, dtype=np.float64) / (n - 1))


def spd_matrix(n: int, kappa: float, seed: int, device: str | torch.device = "cpu",
               spectrum: str = "geometric") -> torch.Tensor:
    """A = Q diag(sigma) Q^T in FP64, exactly symmetric, then rounded to FP32.

    Returns an n x n float32 tensor on `device` (symmetric, so row- and
    column-major storage coincide)."""
    g = _rng(seed)
    G = torch.from_numpy(g.standard_normal((n, n))).to(device=device, dtype=torch.float64)
    Q, R = torch.linalg.qr(G)
    Q = Q * torch.sign(torch.diagonal(R)).unsqueeze(0)
    if spectrum == "geometric":
        sig = geometric_spectrum(n, kappa)
    elif spectrum == "arithmetic":
        sig = 1.0 - (1.0 - 1.0 / kappa) * np.arange(n) / max(n - 1, 1)
    elif spectrum == "logrand":
        sig = 10.0 ** (-math.log10(kappa) * g.random(n))
        sig[0], sig[-1] = 1.0, 1.0 / kappa
    elif spectrum == "clustered":
        sig = np.ones(n)
        sig[-1] = 1.0 / kappa
    else:
        raise ValueError(spectrum)
    s = torch.from_numpy(sig).to(device=device, dtype=torch.float64)
    A = (Q * s.unsqueeze(0)) @ Q.t()
    A = 0.5 * (A + A.t())
    return A.to(torch.float32).contiguous()


def rhs(n: int, nrhs: int, seed: int, device: str | torch.device = "cpu") -> torch.Tensor:
    """B ~ N(0,1), n x nrhs FP64 (a vector when nrhs == 1)."""
    B = torch.from_numpy(_rng(seed).standard_normal((n, nrhs))).to(device=device)
    return B[:, 0].contiguous() if nrhs == 1 else B.contiguous()


def mnist_like_points(n: int, d: int, seed: int, zero_frac: float = 0.8) -> np.ndarray:
    """n points in [0,1]^d: each coordinate 0 with probability zero_frac, else U(0,1)."""
    g = _rng(seed)
    X = g.random((n, d)).astype(np.float32)
    X[g.random((n, d)) < zero_frac] = 0.0
    return X


def gaussian_points(n: int, d: int, seed: int) -> np.ndarray:
    return _rng(seed).standard_normal((n, d)).astype(np.float32)


def median_pairwise_distance(X: torch.Tensor) -> float:
    """Exact median of the n(n-1)/2 pairwise Euclidean distances (FP64)."""
    Xd = X.to(torch.float64)
    sq = (Xd * Xd).sum(1)
    D2 = (sq.unsqueeze(1) + sq.unsqueeze(0) - 2.0 * Xd @ Xd.t()).clamp_min_(0.0)
    n = X.shape[0]
    iu = torch.triu_indices(n, n, 1, device=X.device)
    vals = D2[iu[0], iu[1]]
    del D2
    k = (vals.numel() + 1) // 2
    med2 = torch.kthvalue(vals, k).values.item()
    return math.sqrt(med2)


def rbf_matrix(X: torch.Tensor, ell: float, lam: float) -> torch.Tensor:
    """K_ij = exp(-||x_i - x_j||^2 / (2 ell^2)) + lam delta_ij, FP64 -> FP32."""
    Xd = X.to(torch.float64)
    sq = (Xd * Xd).sum(1)
    D2 = (sq.unsqueeze(1) + sq.unsqueeze(0) - 2.0 * Xd @ Xd.t()).clamp_min_(0.0)
    K = torch.exp(-D2 / (2.0 * ell * ell))
    K.diagonal().add_(lam)
    K = 0.5 * (K + K.t())
    return K.to(torch.float32).contiguous()


def batch_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    return _rng(seed).integers(lo, hi + 1, size=count)


def batch_kappas(count: int, lo: float, hi: float, seed: int) -> np.ndarray:
    g = _rng(seed)
    return 10.0 ** g.uniform(math.log10(lo), math.log10(hi), size=count)
