"""mpchol_potrf_static: the allocation-free diagonal-block POTRF.

Its factor is compared with the one mpchol_factor computes for the same block
(a single-step factorization runs the same diagonal kernel), on two calls in
a row so the second call sees the static scratch the first one left behind,
and with the oracle: the restated reference micro_cholesky
(src/micro_chol.hpp:14-44, FP32, unblocked) and an FP64 Cholesky.
The file is named to be collected last; it passes alone and after the rest.
"""
import ctypes

import numpy as np
import pytest
import torch

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import _lib, matgen
from oracle import oracle as O

# both paths run the same kernel on the same input: the bound is FP32-level
TOL = 1e-6
# against another FP32 Cholesky (the oracle's unblocked micro_cholesky, which
# orders its operations differently) and FP64: two FP32 factorizations of a
# kappa = 1e3 matrix differ by up to ~kappa * u32 = 6e-5
TOL_ORACLE = 1e-4


def static_potrf(A: np.ndarray, pivot_floor: float):
    lib = _lib.load()
    n = A.shape[0]
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()   # column-major storage
    info = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
    st = lib.mpchol_potrf_static(Ad.data_ptr(), n, n, ctypes.c_float(pivot_floor), info.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
    assert st == _lib.OK, _lib.load().mpchol_status_str(st)
    torch.cuda.synchronize()
    return np.tril(Ad.cpu().numpy().T), int(info.item())


def factor_lower(A: np.ndarray) -> np.ndarray:
    n = A.shape[0]
    f = mp.factor(torch.from_numpy(A).cuda(), block_size=256, precision="fp32",
                  pivot_floor=1e-7)
    assert f.info().status == 0
    return f.lower().cpu().numpy()[:n, :n]


@pytest.mark.gpu
def test_static_potrf_matches_factor_on_two_calls_in_a_row(cuda):
    for n, seed in ((256, 21), (200, 22)):       # full block, then a ragged one
        A = matgen.spd_matrix(n, 1e3, seed).numpy()
        L, info = static_potrf(A, 1e-7)
        assert info == 0
        Lf = factor_lower(A)
        err = np.linalg.norm(L - Lf) / np.linalg.norm(Lf)
        Lm, rc = O.micro_cholesky(A)
        L64 = np.linalg.cholesky(A.astype(np.float64))
        err_m = np.linalg.norm(L - Lm) / np.linalg.norm(Lm)
        err_64 = np.linalg.norm(L - L64) / np.linalg.norm(L64)
        print(f"n={n}: static vs factor {err:.2e}, vs micro_cholesky {err_m:.2e}, "
              f"vs FP64 {err_64:.2e}")
        assert err <= TOL
        assert rc == 0 and err_m <= TOL_ORACLE and err_64 <= TOL_ORACLE


@pytest.mark.gpu
def test_static_potrf_reports_the_failing_pivot(cuda):
    A = matgen.spd_matrix(128, 10.0, 23).numpy()
    A[77, 77] = -1.0
    _, info = static_potrf(A, 0.0)
    assert info == 78


def test_static_potrf_rejects_sizes_beyond_its_scratch():
    # argument checks return before any CUDA call, so this runs without a GPU
    lib = _lib.load()
    dummy = ctypes.c_void_p(16)
    info = ctypes.c_void_p(16)
    bad = _lib.ERR_BAD_ARG
    # (lda, n): n beyond the static scratch, lda < n, lda not a multiple of 4
    for lda, n in ((257, 257), (512, 300), (64, 100), (66, 64)):
        assert lib.mpchol_potrf_static(dummy, lda, n, ctypes.c_float(0.0), info, None) == bad
    assert lib.mpchol_potrf_static(dummy, 64, 64, ctypes.c_float(-1.0), info, None) == bad
