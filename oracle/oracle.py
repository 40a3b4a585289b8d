"""CPU oracle for the mpchol solver -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module,
and only as the checker.  It wraps the C restatement in mpchol_oracle.c
(built into oracle/_build/liboracle.so by oracle/Makefile) and adds the FP64
parts in numpy/scipy:

  * ``pcg``            -- the reference's PCG loop (src/mixed_cholesky.cu:143-217)
                          in FP64, with the stopping test on the true residual.
  * ``dense_solve``    -- FP64 dense Cholesky solve, the reference's
                          solveWithCuSolver (src/mixed_cholesky.cu:297-349).
  * ``ref_lofloat_*``  -- the reference's own lo_float.h conversions, when
                          oracle/_ref/ was built from the reference sources.

Parity of the number formats is pinned against tests/golden/ (vectors produced
by the reference's lo_float.h); the restatement also matched lo_float on all
2^32 float32 inputs when oracle/_ref was available.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LOFLOAT = HERE / "_ref" / "libref_lofloat.so"
REF_MICRO = HERE / "_ref" / "libref_micro.so"

FP32, FP16, E4M3, E5M2, MXFP8, SWITCHING, FP16X2, MXFP6E2M3, MXFP6E3M2, MXFP4 = range(10)
MX_FAMILY = (MXFP8, MXFP6E2M3, MXFP6E3M2, MXFP4)

_lib = None


class CholOpts(ctypes.Structure):
    _fields_ = [
        ("block_size", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("eps_prime", ctypes.c_float),
        ("floor_ratio", ctypes.c_float),
        ("diag_pert", ctypes.c_int),
        ("pert", ctypes.c_float),
        ("pivot_floor", ctypes.c_float),
        ("switch_mode", ctypes.c_int),
        ("ladder_len", ctypes.c_int),
        ("ladder", ctypes.c_int * 4),
        ("force_prec", ctypes.POINTER(ctypes.c_int)),
        ("force_fp64", ctypes.POINTER(ctypes.c_int)),
        ("coherence", ctypes.c_int),
        ("equilibrate", ctypes.c_int),
        ("eps_coherence", ctypes.c_float),
    ]


class CholInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("fail_row", ctypes.c_int),
                ("n_perturbed", ctypes.c_int), ("nsteps", ctypes.c_int)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        fp = ctypes.POINTER(ctypes.c_float)
        L.orc_f32_to_e4m3.restype = ctypes.c_uint8
        L.orc_f32_to_e4m3.argtypes = [ctypes.c_float, ctypes.c_int]
        L.orc_f32_to_e5m2.restype = ctypes.c_uint8
        L.orc_f32_to_e5m2.argtypes = [ctypes.c_float, ctypes.c_int]
        L.orc_f32_to_f16.restype = ctypes.c_uint16
        L.orc_f32_to_f16.argtypes = [ctypes.c_float]
        L.orc_quantize.argtypes = [fp, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]
        L.orc_quantize_hash.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
        L.orc_row_scale_exp.restype = ctypes.c_int
        L.orc_row_scale_exp.argtypes = [ctypes.c_float, ctypes.c_int]
        L.orc_mx_scale_exp.restype = ctypes.c_int
        L.orc_mx_scale_exp.argtypes = [ctypes.c_float]
        L.orc_mx_scale_exp_fmt.restype = ctypes.c_int
        L.orc_mx_scale_exp_fmt.argtypes = [ctypes.c_float, ctypes.c_int]
        L.orc_mx_round.restype = ctypes.c_float
        L.orc_mx_round.argtypes = [ctypes.c_float, ctypes.c_int]
        L.orc_blocked_chol.restype = ctypes.c_int
        L.orc_blocked_chol.argtypes = [fp, ctypes.c_int, ctypes.c_int, fp, fp, fp,
                                       ctypes.POINTER(CholOpts), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(CholInfo)]
        L.orc_micro_cholesky.restype = ctypes.c_int
        L.orc_micro_cholesky.argtypes = [fp, ctypes.c_int, ctypes.c_int]
        L.orc_chol_fp32_omp.restype = ctypes.c_int
        L.orc_chol_fp32_omp.argtypes = [fp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_gemv_f32_f64.argtypes = [fp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_potrs_f32_f64.argtypes = [fp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_choose_precision.restype = ctypes.c_int
        L.orc_choose_precision.argtypes = [fp, fp, ctypes.c_int, ctypes.c_float,
                                           ctypes.POINTER(CholOpts)]
        L.orc_coherence_ratio.restype = ctypes.c_float
        L.orc_coherence_ratio.argtypes = [fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, fp]
        _lib = L
    return _lib


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ---- number formats ---------------------------------------------------------

def quantize(x: np.ndarray, fmt: int) -> np.ndarray:
    """Elementwise RNE conversion (saturating for E4M3/E5M2) of float32 x."""
    x = np.ascontiguousarray(x, dtype=np.float32).ravel()
    out = np.empty(x.size, dtype=np.uint16 if fmt == FP16 else np.uint8)
    lib().orc_quantize(_fptr(x), out.ctypes.data_as(ctypes.c_void_p), x.size, fmt)
    return out


def quantize_hash(first: int, count: int, chunk: int, fmt: int) -> np.ndarray:
    nch = (count + chunk - 1) // chunk
    out = np.zeros(nch, dtype=np.uint64)
    lib().orc_quantize_hash(first, count, chunk, fmt,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return out


def row_scale_exp(amax: float, fmt: int) -> int:
    return lib().orc_row_scale_exp(float(amax), fmt)


def mx_scale_exp(amax: float, fmt: int = MXFP8) -> int:
    return lib().orc_mx_scale_exp_fmt(float(amax), fmt)


def mx_round(x: np.ndarray, fmt: int) -> np.ndarray:
    """RNE onto an MX element grid (E4M3, or the OCP FP6/FP4 element
    formats), saturating; float32 values."""
    x = np.ascontiguousarray(x, dtype=np.float32).ravel()
    f = lib().orc_mx_round
    return np.array([f(float(v), fmt) for v in x], dtype=np.float32)


def decode(codes: np.ndarray, fmt: int) -> np.ndarray:
    """Value of each code (NaN codes -> nan)."""
    c = codes.astype(np.int64)
    if fmt == FP16:
        return codes.astype(np.uint16).view(np.float16).astype(np.float32)
    if fmt == E4M3:
        s, e, m = c >> 7, (c >> 3) & 0xF, c & 7
        v = np.where(e == 0, m * 2.0 ** -9, (1 + m / 8.0) * 2.0 ** (e - 7))
        v = np.where((e == 15) & (m == 7), np.nan, v)
    else:
        s, e, m = c >> 7, (c >> 2) & 0x1F, c & 3
        v = np.where(e == 0, m * 2.0 ** -16, (1 + m / 4.0) * 2.0 ** (e - 15))
        v = np.where(e == 31, np.where(m == 0, np.inf, np.nan), v)
    return np.where(s == 1, -v, v).astype(np.float32)


def quantize_rows(P: np.ndarray, fmt: int) -> tuple[np.ndarray, np.ndarray]:
    """Panel quantization as the solver does it.  P is m x k float32.
    Returns (codes m x k, scales): per-row int exponents, or per-32-block
    E8M0 codes (m x k/32) for MXFP8."""
    P = np.asarray(P, dtype=np.float32)
    m, k = P.shape
    if fmt in MX_FAMILY:
        # codes: E4M3 codes of the element values (FP6/FP4 values rounded on
        # their own grid first -- exactly representable in E4M3)
        blocks = np.abs(P).reshape(m, k // 32, 32).max(axis=2)
        ex = np.vectorize(lambda a: mx_scale_exp(a, fmt), otypes=[np.int32])(blocks) \
            if blocks.size else np.zeros((m, k // 32), np.int32)
        inv = np.ldexp(np.float32(1.0), -np.repeat(ex, 32, axis=1)).astype(np.float32)
        xs = (P * inv).astype(np.float32)
        if fmt != MXFP8:
            xs = mx_round(xs, fmt).reshape(m, k)
        codes = quantize(xs, E4M3).reshape(m, k)
        return codes, (ex + 127).astype(np.uint8)
    amax = np.abs(P).max(axis=1) if k else np.zeros(m, np.float32)
    ex = np.array([row_scale_exp(a, fmt) for a in amax], dtype=np.int32)
    inv = np.ldexp(np.float32(1.0), -ex).astype(np.float32)[:, None]
    xs = (P * inv).astype(np.float32)
    if fmt == FP16X2:
        hi = quantize(xs, FP16).reshape(m, k)
        lo = quantize((xs - decode(hi, FP16)).astype(np.float32), FP16).reshape(m, k)
        return np.concatenate([hi, lo], axis=0), ex.astype(np.int8)
    codes = quantize(xs, fmt).reshape(m, k)
    return codes, ex.astype(np.int8)


# ---- reference library (built from the reference sources) -----------------

def have_ref() -> bool:
    return REF_LOFLOAT.exists()


def ref_lofloat(x: np.ndarray, fmt: int, saturate: bool = True) -> np.ndarray:
    L = ctypes.CDLL(str(REF_LOFLOAT))
    fn = L.ref_lofloat_e4m3 if fmt == E4M3 else L.ref_lofloat_e5m2
    fn.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]
    x = np.ascontiguousarray(x, dtype=np.float32).ravel()
    out = np.empty(x.size, dtype=np.uint8)
    fn(_fptr(x), out.ctypes.data_as(ctypes.c_void_p), x.size, int(saturate))
    return out


def ref_lofloat_small(x: np.ndarray, fmt: int) -> np.ndarray:
    """The reference lo_float's saturating RNE conversion of float32 x to
    float6_e2m3 (MXFP6E2M3), float6_e3m2 (MXFP6E3M2) or float4_e2m1 (MXFP4),
    as float32 values."""
    L = ctypes.CDLL(str(REF_LOFLOAT))
    fn = {MXFP6E2M3: L.ref_lofloat_f6e2m3, MXFP6E3M2: L.ref_lofloat_f6e3m2,
          MXFP4: L.ref_lofloat_f4e2m1}[fmt]
    fn.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_longlong]
    x = np.ascontiguousarray(x, dtype=np.float32).ravel()
    out = np.empty(x.size, dtype=np.float32)
    fn(_fptr(x), _fptr(out), x.size)
    return out


def ref_micro_cholesky(A: np.ndarray) -> tuple[np.ndarray, int]:
    """The reference's own micro_cholesky (src/micro_chol.hpp:14-44) on a copy
    of the column-major float32 matrix A."""
    L = ctypes.CDLL(str(REF_MICRO))
    L.ref_micro_cholesky.restype = ctypes.c_int
    L.ref_micro_cholesky.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int]
    F = np.array(A, dtype=np.float32, order="F", copy=True)
    rc = L.ref_micro_cholesky(_fptr(F), F.shape[0], F.shape[0])
    return np.tril(F), rc


# ---- factorization ----------------------------------------------------------

def make_opts(block_size=256, precision=SWITCHING, eps_prime=0.5, floor=0.0, diag_pert=0,
              pert=1.0, pivot_floor=1e-7, switch_mode=0, ladder=(E4M3, FP16, FP32),
              coherence=1, equilibrate=0, eps_coherence=0.0) -> CholOpts:
    o = CholOpts()
    o.block_size, o.precision, o.eps_prime, o.floor_ratio = block_size, precision, eps_prime, floor
    o.diag_pert, o.pert, o.pivot_floor, o.switch_mode = diag_pert, pert, pivot_floor, switch_mode
    o.coherence, o.equilibrate, o.eps_coherence = coherence, equilibrate, eps_coherence
    o.ladder_len = len(ladder)
    for i in range(4):
        o.ladder[i] = ladder[i] if i < len(ladder) else FP32
    return o


OPTS_FIELDS = ("block_size", "precision", "eps_prime", "floor", "diag_pert", "pert",
               "pivot_floor", "switch_mode")


def factor_kwargs(opts) -> dict:
    """make_opts keyword arguments equal to a library options struct (the
    ctypes mpchol_opts of cholesky_gpu_b200._lib, or any object with the same
    field names), so that the oracle restates a GPU factor with the options it
    was computed with -- the diagonal shifts and pivot floor included."""
    kw = {f: getattr(opts, f) for f in OPTS_FIELDS}
    kw["ladder"] = tuple(int(opts.ladder[i]) for i in range(int(opts.ladder_len)))
    kw["coherence"] = int(getattr(opts, "coherence", 0))
    kw["equilibrate"] = int(getattr(opts, "equilibrate", 0))
    kw["eps_coherence"] = float(getattr(opts, "eps_coherence", 0.0))
    return kw


def blocked_chol(A: np.ndarray, force_prec=None, force_fp64=None, **kw):
    """Blocked mixed-precision Cholesky restatement.  A is n x n float32
    (symmetric; lower triangle used).  Returns dict with L (lower, float32),
    d, dtilde, step_prec, step_fp64, status, fail_row, n_perturbed."""
    n = A.shape[0]
    o = make_opts(**kw)
    F = np.array(A, dtype=np.float32, order="F", copy=True)
    ex = None
    if o.equilibrate:
        # D A D with D = diag(2^-e_i) (exact power-of-two scaling), then the
        # factor's rows are scaled back by 2^e_i
        ex = equilibration_exponents(np.diag(F))
        F = np.asfortranarray(np.ldexp(F, -(ex[:, None] + ex[None, :])).astype(np.float32))
    d = np.ascontiguousarray(np.diag(F).astype(np.float32))
    dt = d.copy()
    sh = np.zeros(n, dtype=np.float32)
    ns = (n + o.block_size - 1) // o.block_size
    sp = np.zeros(ns, dtype=np.int32)
    s64 = np.zeros(ns, dtype=np.int32)
    keep = []
    if force_prec is not None:
        fp_arr = np.ascontiguousarray(force_prec, dtype=np.int32)
        keep.append(fp_arr)
        o.force_prec = fp_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    if force_fp64 is not None:
        f64_arr = np.ascontiguousarray(force_fp64, dtype=np.int32)
        keep.append(f64_arr)
        o.force_fp64 = f64_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    info = CholInfo()
    lib().orc_blocked_chol(_fptr(F), n, n, _fptr(d), _fptr(dt), _fptr(sh), ctypes.byref(o),
                           sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                           s64.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(info))
    L = np.tril(np.asarray(F))
    if ex is not None:
        L = np.ldexp(L, ex[:, None]).astype(np.float32)
    return dict(L=L, d=d, dtilde=dt, step_prec=sp, step_fp64=s64,
                status=info.status, fail_row=info.fail_row, n_perturbed=info.n_perturbed,
                eq_exp=ex)


def equilibration_exponents(diag: np.ndarray) -> np.ndarray:
    """e_i = floor((floor(log2 a_ii) + 1) / 2), clamped to [-63, 63], so that
    a_ii * 2^(-2 e_i) lies in [0.5, 2); 0 for a non-positive or non-finite
    diagonal entry.  (The diagonal scaling intent of src/kernels_macros.cuh:137-158.)"""
    a = np.asarray(diag, dtype=np.float32).astype(np.float64)
    ok = np.isfinite(a) & (a > 0)
    _, fe = np.frexp(np.where(ok, a, 1.0))
    E = fe.astype(np.int64) - 1                      # floor(log2 a)
    e = np.clip((E + 1) // 2, -63, 63)
    return np.where(ok, e, 0).astype(np.int32)


def coherence_ratio(P: np.ndarray, dtilde: np.ndarray) -> float:
    """(||P^T 1||^2 / m) / min dtilde of a solved panel P (m x b), as the
    factor's switching rule computes it."""
    P = np.asfortranarray(P, dtype=np.float32)
    dt = np.ascontiguousarray(dtilde, dtype=np.float32)
    m, bs = P.shape
    return float(lib().orc_coherence_ratio(_fptr(P), max(m, 1), m, bs, _fptr(dt)))


def choose_precision(d: np.ndarray, dtilde: np.ndarray, coh: float = 0.0, **kw) -> int:
    o = make_opts(**kw)
    d = np.ascontiguousarray(d, dtype=np.float32)
    dt = np.ascontiguousarray(dtilde, dtype=np.float32)
    return lib().orc_choose_precision(_fptr(d), _fptr(dt), d.size, float(coh), ctypes.byref(o))


def micro_cholesky(A: np.ndarray) -> tuple[np.ndarray, int]:
    F = np.array(A, dtype=np.float32, order="F", copy=True)
    rc = lib().orc_micro_cholesky(_fptr(F), F.shape[0], F.shape[0])
    return np.tril(F), rc


def chol_fp32_omp(A: np.ndarray, b: int = 256) -> tuple[np.ndarray, int]:
    F = np.array(A, dtype=np.float32, order="F", copy=True)
    rc = lib().orc_chol_fp32_omp(_fptr(F), F.shape[0], F.shape[0], b)
    return np.tril(F), rc


def num_threads() -> int:
    return lib().orc_num_threads()


# ---- FP64 solve side --------------------------------------------------------

def potrs(L: np.ndarray, r: np.ndarray) -> np.ndarray:
    """z = (L L^T)^-1 r with the float32 factor, FP64 vectors."""
    from scipy.linalg import solve_triangular
    L64 = np.asarray(L, dtype=np.float64)
    y = solve_triangular(L64, r, lower=True, check_finite=False)
    return solve_triangular(L64.T, y, lower=False, check_finite=False)


def pcg(A: np.ndarray, L: np.ndarray, b: np.ndarray, rel_tol: float = 1e-10, max_it: int = 200,
        x0_precond: bool = True):
    """The reference's PCG loop (src/mixed_cholesky.cu:143-217) in FP64 with
    A the (float32-valued) operator, M = L L^T, stopping when the true FP64
    residual ||b - A x|| / ||b|| <= rel_tol (checked every iteration here).
    Returns (x, iterations, rel_residual)."""
    A64 = np.asarray(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    x = potrs(L, b) if x0_precond else np.zeros_like(b)
    r = b - A64 @ x
    nb = np.linalg.norm(b, axis=0)
    it = 0
    if np.all(np.linalg.norm(r, axis=0) <= rel_tol * nb):
        return x, 0, float(np.max(np.linalg.norm(r, axis=0) / nb))
    z = potrs(L, r)
    p = z.copy()
    rho = np.sum(r * z, axis=0)
    while it < max_it:
        it += 1
        Ap = A64 @ p
        alpha = rho / np.sum(p * Ap, axis=0)
        x = x + alpha * p
        r = r - alpha * Ap
        rt = b - A64 @ x
        if np.all(np.linalg.norm(rt, axis=0) <= rel_tol * nb):
            break
        z = potrs(L, r)
        rho_new = np.sum(r * z, axis=0)
        p = z + (rho_new / rho) * p
        rho = rho_new
    rel = float(np.max(np.linalg.norm(b - A64 @ x, axis=0) / nb))
    return x, it, rel


def dense_solve(A: np.ndarray, b: np.ndarray) -> np.ndarray:
    """FP64 dense Cholesky solve (Dpotrf + Dpotrs), the FP64 oracle form."""
    from scipy.linalg import cho_factor, cho_solve
    c = cho_factor(np.asarray(A, dtype=np.float64), lower=True, check_finite=False)
    return cho_solve(c, np.asarray(b, dtype=np.float64), check_finite=False)


# ---- RBF kernel solve (FP64 dense oracle for the differentiable solve) -------

def rbf_kernel_f64(X: np.ndarray, ell: float, lam: float) -> tuple[np.ndarray, np.ndarray]:
    """(K, r2): K_ij = exp(-r2_ij / (2 ell^2)) + lam delta_ij in FP64, r2 from
    coordinate differences."""
    Xd = np.asarray(X, dtype=np.float64)
    r2 = ((Xd[:, None, :] - Xd[None, :, :]) ** 2).sum(-1)
    K = np.exp(-r2 / (2.0 * ell * ell))
    K[np.diag_indices_from(K)] += lam
    return K, r2


def rbf_loss_f64(X: np.ndarray, ell: float, lam: float, y: np.ndarray) -> float:
    """L = 1/2 y^T K^-1 y by FP64 dense Cholesky."""
    import scipy.linalg as sl
    K, _ = rbf_kernel_f64(X, ell, lam)
    c = sl.cho_factor(K, lower=True)
    yd = np.asarray(y, dtype=np.float64)
    return 0.5 * float(np.sum(yd * sl.cho_solve(c, yd)))


def rbf_loss_grads_f64(X: np.ndarray, ell: float, lam: float, y: np.ndarray):
    """Gradients of L = 1/2 y^T K^-1 y w.r.t. (X, ell, lam, y), FP64 dense:
    x = K^-1 y, G_K = -x x^T / 2; dL/dlam = tr G_K; dL/dell = sum G_K K r2 / ell^3;
    dL/dX_i = sum_j 2 G_K,ij K_ij (X_j - X_i) / ell^2; dL/dy = x."""
    import scipy.linalg as sl
    Xd = np.asarray(X, dtype=np.float64)
    K, r2 = rbf_kernel_f64(Xd, ell, lam)
    Kr = K - lam * np.eye(K.shape[0])
    c = sl.cho_factor(K, lower=True)
    yd = np.asarray(y, dtype=np.float64)
    x = sl.cho_solve(c, yd)
    x2 = x.reshape(x.shape[0], -1)
    G = -0.5 * x2 @ x2.T
    d_lam = float(np.trace(G))
    d_ell = float(np.sum(G * Kr * r2) / ell ** 3)
    W = 2.0 * G * Kr
    dX = (W @ Xd - W.sum(1)[:, None] * Xd) / (ell * ell)
    return dX, d_ell, d_lam, x
