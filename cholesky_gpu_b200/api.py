"""Python mirror of the reference's solver surface over the C ABI.

``precond_CG`` and ``switching_chol`` keep the reference's argument order and
meaning (src/mixed_cholesky.cu:76-78, src/switching_chol.cuh:19-22) with torch
CUDA tensors in place of raw device pointers; ``Factor`` exposes the
factor-object API of include/mpchol.h.  Every call runs the sm_100a library;
there is no CPU path here.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check, load


def _stream_handle(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _require_cuda(t: torch.Tensor, dtype: torch.dtype, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")


def _col_major(A: torch.Tensor) -> tuple[torch.Tensor, int]:
    """Return a tensor whose storage is column-major n x n and its ld.

    A symmetric matrix given in row-major torch layout has the same lower
    triangle as its column-major transpose, so A.t() is used without a copy
    when A is contiguous."""
    if A.dim() != 2 or A.shape[0] != A.shape[1]:
        raise ValueError("A must be square")
    if A.stride(0) == 1 and A.stride(1) >= A.shape[0]:
        return A, A.stride(1)
    At = A.t()
    if At.stride(0) == 1:
        return At, At.stride(1)
    At = A.t().contiguous().t()
    return At, At.stride(1)


@dataclass
class FactorInfo:
    status: int
    fail_row: int
    n_perturbed: int
    nsteps: int
    n_fp64_blocks: int
    steps_by_prec: list
    step_prec: list
    step_fp64: list


@dataclass
class Report:
    iterations: int
    converged: bool
    rel_residual: float
    backward_error: float
    precond_residual: float
    status: int


class Factor:
    """A factor object: blocked mixed-precision Cholesky of an SPD matrix."""

    def __init__(self, n: int, **opts):
        self.lib = load()
        self.n = n
        self.opts = _lib.default_opts(**opts)
        h = ctypes.c_void_p()
        check(self.lib.mpchol_factor_create(ctypes.byref(self.opts), n, ctypes.byref(h)),
              "mpchol_factor_create")
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.mpchol_factor_destroy(h)
            self.handle = None

    def compute(self, A: torch.Tensor) -> "Factor":
        _require_cuda(A, torch.float32, "A")
        Ac, lda = _col_major(A)
        check(self.lib.mpchol_factor_compute(self.handle, Ac.data_ptr(), lda, _stream_handle()),
              "mpchol_factor_compute")
        self._A_keepalive = Ac
        return self

    def info(self) -> FactorInfo:
        fi = _lib.FactorInfo()
        ns = (self.n + self.opts.block_size - 1) // self.opts.block_size
        prec = (ctypes.c_int * ns)()
        f64 = (ctypes.c_int * ns)()
        check(self.lib.mpchol_factor_info_get(self.handle, ctypes.byref(fi), prec, f64,
                                              _stream_handle()), "mpchol_factor_info_get")
        return FactorInfo(fi.status, fi.fail_row, fi.n_perturbed, fi.nsteps, fi.n_fp64_blocks,
                          list(fi.steps_by_prec), list(prec), list(f64))

    def lower(self) -> torch.Tensor:
        """The factor L as an n x n torch tensor (lower triangle; a copy)."""
        p = ctypes.c_void_p()
        ld = ctypes.c_int()
        n = ctypes.c_int()
        check(self.lib.mpchol_factor_lower(self.handle, ctypes.byref(p), ctypes.byref(ld),
                                           ctypes.byref(n)), "mpchol_factor_lower")
        buf = torch.empty((self.n, ld.value), dtype=torch.float32, device="cuda")
        nbytes = self.n * ld.value * 4
        torch.cuda.current_stream().synchronize()
        # device-to-device copy via cudaMemcpy through torch: wrap the raw pointer
        src = _wrap_device(p.value, (self.n, ld.value), torch.float32)
        buf.copy_(src)
        del nbytes
        return buf[:, : self.n].t().tril()

    def panel_codes(self, fmt: int):
        """The last trailing update's quantized panel in format fmt (a step
        candidate): (codes, scales, col0) as host numpy arrays; codes are rows x
        block (FP16X2: hi rows then lo rows, as uint16), scales int8 per row or
        (MXFP8) uint8 rows x block/32.  The panel covers L[col0+block:, col0:col0+block]."""
        import numpy as np
        pc, ps = ctypes.c_void_p(), ctypes.c_void_p()
        ldq, rows, col0 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self.lib.mpchol_factor_codes(self.handle, fmt, ctypes.byref(pc), ctypes.byref(ps),
                                           ctypes.byref(ldq), ctypes.byref(rows),
                                           ctypes.byref(col0)), "mpchol_factor_codes")
        torch.cuda.current_stream().synchronize()
        k, m = ldq.value, rows.value
        if fmt in (_lib.PREC_FP16, _lib.PREC_FP16X2):
            nrow = 2 * m if fmt == _lib.PREC_FP16X2 else m
            codes = _wrap_device(pc.value, (nrow, k), torch.int16).cpu().numpy().view(np.uint16)
        else:
            codes = _wrap_device(pc.value, (m, k), torch.uint8).cpu().numpy()
        if fmt == _lib.PREC_MXFP8:
            scales = _wrap_device(ps.value, (m, k // 32), torch.uint8).cpu().numpy()
        else:
            scales = _wrap_device(ps.value, (m,), torch.int8).cpu().numpy()
        return codes, scales, col0.value

    def diags(self) -> tuple[torch.Tensor, torch.Tensor]:
        pd = ctypes.c_void_p()
        pt = ctypes.c_void_p()
        check(self.lib.mpchol_factor_diags(self.handle, ctypes.byref(pd), ctypes.byref(pt)),
              "mpchol_factor_diags")
        torch.cuda.current_stream().synchronize()
        return (_wrap_device(pd.value, (self.n,), torch.float32).clone(),
                _wrap_device(pt.value, (self.n,), torch.float32).clone())

    def apply_precond(self, R: torch.Tensor) -> torch.Tensor:
        _require_cuda(R, torch.float64, "R")
        R2 = R.reshape(self.n, -1) if R.dim() == 1 else R
        nrhs = R2.shape[1]
        Rc = R2.t().contiguous()          # column-major n x nrhs
        Z = torch.empty_like(Rc)
        check(self.lib.mpchol_apply_precond(self.handle, Rc.data_ptr(), Z.data_ptr(), nrhs,
                                            _stream_handle()), "mpchol_apply_precond")
        Z = Z.t()
        return Z.reshape(R.shape) if R.dim() == 1 else Z

    def save(self) -> bytes:
        """The computed factor as a byte blob (header, L's lower block columns,
        per-step states, diagonals, status) that load() restores into a factor
        object of the same order and block size, so solves can reuse it
        without refactoring."""
        size = ctypes.c_size_t()
        check(self.lib.mpchol_factor_save(self.handle, None, 0, ctypes.byref(size), _stream_handle()),
              "mpchol_factor_save")
        buf = ctypes.create_string_buffer(size.value)
        check(self.lib.mpchol_factor_save(self.handle, buf, size.value, ctypes.byref(size),
                                          _stream_handle()), "mpchol_factor_save")
        return buf.raw

    def load(self, blob: bytes) -> "Factor":
        """Replace this object's factor by a saved one (same n and block size)."""
        data = bytes(blob)
        check(self.lib.mpchol_factor_load(self.handle, data, len(data), _stream_handle()),
              "mpchol_factor_load")
        return self

    def set_copy_plan(self, cuts=None, join=None) -> None:
        """Fix the copy groups of solve_host: cuts (block columns where groups
        start, increasing) and join (the step at which each later group joins
        the trailing updates); cuts=[] copies all of A before factoring, None
        restores the automatic plan."""
        if cuts is None:
            check(self.lib.mpchol_set_copy_plan(self.handle, 0, None, None), "mpchol_set_copy_plan")
            return
        ng = len(cuts) + 1
        if join is None or len(join) != len(cuts):
            raise ValueError("join needs one step per cut")
        c = (ctypes.c_int * max(1, len(cuts)))(*cuts)
        j = (ctypes.c_int * max(1, len(join)))(*join)
        check(self.lib.mpchol_set_copy_plan(self.handle, ng, c, j), "mpchol_set_copy_plan")

    def solve_host(self, A: torch.Tensor, B: torch.Tensor, rel_tol: float = 1e-10,
                   max_it: int = 200, x0_precond: bool = True,
                   check_every: int = 4) -> tuple[torch.Tensor, Report]:
        """Factor A and solve A X = B with A (FP32) and B (FP64, n or n x nrhs)
        in host memory (page-locked for full-speed copies).  Only A's lower
        triangle reaches the device, in groups of block columns that overlap
        the factorization (copy_plan).  Returns X on the host."""
        if A.device.type != "cpu" or B.device.type != "cpu":
            raise ValueError("solve_host takes host (CPU) tensors")
        if A.dtype != torch.float32 or B.dtype != torch.float64:
            raise ValueError("A must be float32 and B float64")
        Ac, lda = _col_major(A)
        Bc = _host_col_major(B, self.n)
        nrhs = Bc.shape[1]
        X = torch.empty((nrhs, self.n), dtype=torch.float64, pin_memory=A.is_pinned()).t()
        po = _lib.default_pcg_opts(rel_tol=rel_tol, max_it=max_it, x0_precond=int(x0_precond),
                                   check_every=check_every)
        rep = _lib.Report()
        st = self.lib.mpchol_solve_host(self.handle, Ac.data_ptr(), lda, Bc.data_ptr(),
                                        X.data_ptr(), nrhs, ctypes.byref(po), ctypes.byref(rep),
                                        _stream_handle())
        if st not in (_lib.OK, _lib.PCG_MAXIT):
            check(st, "mpchol_solve_host")
        Xo = X.reshape(B.shape) if B.dim() == 1 else X
        return Xo, Report(rep.iterations, bool(rep.converged), rep.rel_residual,
                          rep.backward_error, rep.precond_residual, st)

    def pcg(self, A: torch.Tensor, B: torch.Tensor, rel_tol: float = 1e-10, max_it: int = 200,
            x0_precond: bool = True, check_every: int = 4) -> tuple[torch.Tensor, Report]:
        """Solve A X = B (B: n or n x nrhs FP64 CUDA tensor) with PCG on this factor."""
        if A.dtype not in (torch.float32, torch.float64):
            raise ValueError("A must be float32 or float64")
        _require_cuda(B, torch.float64, "B")
        Ac, lda = _col_major(A)
        B2 = B.reshape(self.n, 1) if B.dim() == 1 else B
        nrhs = B2.shape[1]
        Bc = B2.t().contiguous()
        X = torch.empty_like(Bc)
        po = _lib.default_pcg_opts(rel_tol=rel_tol, max_it=max_it, x0_precond=int(x0_precond),
                                   check_every=check_every)
        rep = _lib.Report()
        fn = self.lib.mpchol_pcg if A.dtype == torch.float32 else self.lib.mpchol_pcg_f64
        st = fn(self.handle, Ac.data_ptr(), lda, Bc.data_ptr(), X.data_ptr(), nrhs,
                ctypes.byref(po), ctypes.byref(rep), _stream_handle())
        if st not in (_lib.OK, _lib.PCG_MAXIT):
            check(st, "mpchol_pcg")
        Xo = X.t()
        Xo = Xo.reshape(B.shape) if B.dim() == 1 else Xo
        return Xo, Report(rep.iterations, bool(rep.converged), rep.rel_residual,
                          rep.backward_error, rep.precond_residual, st)

    def adjoint_solve(self, A: torch.Tensor, X: torch.Tensor, G: torch.Tensor,
                      rel_tol: float = 1e-10, max_it: int = 200, grad_a: bool = False):
        """Backward of the solve X = A^-1 B: Lam = A^-1 G (G = dL/dX) by PCG
        with this factor as preconditioner (mpchol_adjoint_solve; A the FP64
        operator of the forward solve).  Returns (Lam, dL/dA or None, report);
        dL/dA = -(Lam X^T + X Lam^T) / 2 (lower triangle filled) when grad_a."""
        _require_cuda(A, torch.float64, "A")
        _require_cuda(X, torch.float64, "X")
        _require_cuda(G, torch.float64, "G")
        Ac, lda = _col_major(A)
        X2 = X.reshape(self.n, 1) if X.dim() == 1 else X
        G2 = G.reshape(self.n, 1) if G.dim() == 1 else G
        if X2.shape != G2.shape:
            raise ValueError("X and G must have the same shape")
        nrhs = G2.shape[1]
        Xc = X2.t().contiguous()
        Gc = G2.t().contiguous()
        Lam = torch.empty_like(Gc)
        GA = torch.zeros((self.n, self.n), dtype=torch.float64, device=A.device) if grad_a else None
        po = _lib.default_pcg_opts(rel_tol=rel_tol, max_it=max_it)
        rep = _lib.Report()
        st = self.lib.mpchol_adjoint_solve(self.handle, Ac.data_ptr(), lda, Xc.data_ptr(),
                                           Gc.data_ptr(), Lam.data_ptr(), nrhs,
                                           None if GA is None else GA.data_ptr(), self.n,
                                           ctypes.byref(po), ctypes.byref(rep), _stream_handle())
        if st not in (_lib.OK, _lib.PCG_MAXIT):
            check(st, "mpchol_adjoint_solve")
        L = Lam.t()
        L = L.reshape(G.shape) if G.dim() == 1 else L
        # the cotangent was written column-major: its transpose view is the matrix
        return L, (None if GA is None else GA.t()), Report(
            rep.iterations, bool(rep.converged), rep.rel_residual, rep.backward_error,
            rep.precond_residual, st)


def _host_col_major(M: torch.Tensor, n: int) -> torch.Tensor:
    """n x nrhs (or n) CPU FP64 tensor as column-major storage (no copy for one
    column or an already column-major view)."""
    M2 = M.reshape(n, 1) if M.dim() == 1 else M
    if M2.stride(0) == 1 and (M2.shape[1] == 1 or M2.stride(1) == n):
        return M2
    Mc = M2.t().contiguous()
    return Mc.t()


def _wrap_device(ptr: int, shape: tuple, dtype: torch.dtype) -> torch.Tensor:
    """View of library-owned device memory as a torch tensor (no copy)."""
    numel = 1
    for s in shape:
        numel *= s
    itemsize = torch.tensor([], dtype=dtype).element_size()

    class _Holder:
        __cuda_array_interface__ = {
            "shape": tuple(shape),
            "typestr": {torch.float32: "<f4", torch.float64: "<f8", torch.uint8: "|u1",
                        torch.int8: "|i1", torch.int16: "<i2"}[dtype],
            "data": (ptr, False),
            "version": 3,
            "strides": None,
        }

    del numel, itemsize
    return torch.as_tensor(_Holder(), device="cuda")


def factor_blob_info(blob: bytes) -> tuple[int, int]:
    """(n, block_size) of a factor blob from Factor.save(), after checking its
    header, sizes and checksum on the host; raises MpcholError if invalid."""
    lib = _lib.load()
    data = bytes(blob)
    n, b = ctypes.c_int(), ctypes.c_int()
    check(lib.mpchol_factor_blob_check(data, len(data), ctypes.byref(n), ctypes.byref(b)),
          "mpchol_factor_blob_check")
    return n.value, b.value


def copy_plan(n: int, block_size: int = 256) -> tuple[list[int], list[int]]:
    """The automatic copy groups of Factor.solve_host for order n: (cuts,
    join), block columns where groups 2.. start and the step each joins at;
    ([], []) means copy all of A, then factor.  Host-only."""
    lib = _lib.load()
    cuts = (ctypes.c_int * 8)()
    join = (ctypes.c_int * 8)()
    ng = lib.mpchol_copy_plan(n, block_size, cuts, join, 8)
    return list(cuts[: max(0, ng - 1)]), list(join[: max(0, ng - 1)])


def factor(A: torch.Tensor, **opts) -> Factor:
    """Factor the FP32 SPD matrix A (CUDA tensor) with the given options."""
    f = Factor(A.shape[0], **opts)
    return f.compute(A)


def solve(A: torch.Tensor, B: torch.Tensor, rel_tol: float = 1e-10, max_it: int = 200,
          **opts) -> tuple[torch.Tensor, Report, Factor]:
    """Factor A and run PCG on A X = B; returns (X, report, factor)."""
    f = factor(A if A.dtype == torch.float32 else A.float(), **opts)
    X, rep = f.pcg(A, B, rel_tol=rel_tol, max_it=max_it)
    return X, rep, f


# ---- reference-shaped entry points ------------------------------------------

def precond_CG(A: torch.Tensor, x: torch.Tensor, b: torch.Tensor, n: int, r: int,
               normA: float = 0.0, eps_prime: float = 0.0, flr: float = 0.0,
               perturb_diag: bool = False, microscal_size: int = 32,
               rel_tol: float = 0.0, max_it: int = 200) -> int:
    """The reference's precond_CG (src/mixed_cholesky.cu:76-78).

    A: n x n FP64 (column-major device storage; a symmetric row-major tensor is
    the same matrix), x written, b read, r the block size.  Returns 0 when
    converged, -1 when not, > 0 when the preconditioner failed (the failing
    row + 1, the reference's cuSOLVER info convention).  With the reference's
    rel_tol = 0 the loop runs max_it iterations.
    """
    _require_cuda(A, torch.float64, "A")
    _require_cuda(x, torch.float64, "x")
    _require_cuda(b, torch.float64, "b")
    Ac, lda = _col_major(A)
    if lda != n:
        Ac = Ac.t().contiguous().t()
    return load().mpchol_precond_cg(Ac.data_ptr(), x.data_ptr(), b.data_ptr(), n, r, normA,
                                    eps_prime, flr, int(perturb_diag), microscal_size, rel_tol,
                                    max_it, _stream_handle())


def switching_chol(d_A: torch.Tensor, n: int, b: int, d_diagVals: torch.Tensor,
                   updated_diag: torch.Tensor, eps_prime: float, perturb_diag: bool = False,
                   microscal_size: int = 32, scales: torch.Tensor | None = None) -> int:
    """The reference's switching_chol (src/switching_chol.cuh:19-22): in-place
    FP32 factor of the n x n column-major matrix d_A with block b.  Returns a
    status code (0 = ok) where the reference returns nothing."""
    _require_cuda(d_A, torch.float32, "d_A")
    if d_A.stride(0) != 1 and not d_A.is_contiguous():
        raise ValueError("d_A must be column-major or contiguous symmetric")
    return load().mpchol_switching_chol(d_A.data_ptr(), n, b, _ptr(d_diagVals),
                                        _ptr(updated_diag), eps_prime, int(perturb_diag),
                                        microscal_size, _stream_handle(), _ptr(scales))


class Batch:
    """Many independent SPD systems of uneven size, factored and solved with
    batched launches (every kernel serves all systems; the factorization is
    one CUDA graph launch, PCG runs the systems in lockstep)."""

    def __init__(self, ns, nrhs: int = 1, **opts):
        self.lib = load()
        self.ns = [int(v) for v in ns]
        self.count = len(self.ns)
        self.nrhs = nrhs
        self.opts = _lib.default_opts(**opts)
        arr = (ctypes.c_int * self.count)(*self.ns)
        h = ctypes.c_void_p()
        check(self.lib.mpchol_batch_create(ctypes.byref(self.opts), self.count, arr, nrhs,
                                           ctypes.byref(h)), "mpchol_batch_create")
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.mpchol_batch_destroy(h)
            self.handle = None

    def _mats(self, As, dtype=torch.float32):
        ptrs = (ctypes.c_void_p * self.count)()
        lds = (ctypes.c_int * self.count)()
        keep = []
        for i, A in enumerate(As):
            _require_cuda(A, dtype, f"A[{i}]")
            if A.shape[0] != self.ns[i]:
                raise ValueError(f"A[{i}] has order {A.shape[0]}, expected {self.ns[i]}")
            Ac, lda = _col_major(A)
            keep.append(Ac)
            ptrs[i] = Ac.data_ptr()
            lds[i] = lda
        return ptrs, lds, keep

    def factor(self, As) -> "Batch":
        ptrs, lds, keep = self._mats(As)
        check(self.lib.mpchol_batch_factor(self.handle, ptrs, lds, _stream_handle()),
              "mpchol_batch_factor")
        self._keep = keep
        return self

    def info(self):
        st = (ctypes.c_int * self.count)()
        row = (ctypes.c_int * self.count)()
        npert = (ctypes.c_int * self.count)()
        check(self.lib.mpchol_batch_info(self.handle, st, row, npert, _stream_handle()),
              "mpchol_batch_info")
        return list(st), list(row), list(npert)

    def lower(self, i: int) -> torch.Tensor:
        p = ctypes.c_void_p()
        ld = ctypes.c_int()
        n = ctypes.c_int()
        check(self.lib.mpchol_batch_lower(self.handle, i, ctypes.byref(p), ctypes.byref(ld),
                                          ctypes.byref(n)), "mpchol_batch_lower")
        torch.cuda.current_stream().synchronize()
        src = _wrap_device(p.value, (n.value, ld.value), torch.float32)
        return src.clone()[:, : n.value].t().tril()

    def pcg(self, As, Bs, rel_tol: float = 1e-10, max_it: int = 200, x0_precond: bool = True,
            check_every: int = 4):
        """Solve A_i X_i = B_i for every system; B_i: n_i x nrhs (or n_i) FP64."""
        ptrs, lds, keep = self._mats(As)
        bp = (ctypes.c_void_p * self.count)()
        xp = (ctypes.c_void_p * self.count)()
        Xs, Bc = [], []
        for i, B in enumerate(Bs):
            _require_cuda(B, torch.float64, f"B[{i}]")
            B2 = B.reshape(self.ns[i], -1)
            if B2.shape[1] != self.nrhs:
                raise ValueError(f"B[{i}] has {B2.shape[1]} columns, expected {self.nrhs}")
            Bt = B2.t().contiguous()            # column-major n x nrhs
            X = torch.empty_like(Bt)
            Bc.append(Bt)
            Xs.append(X)
            bp[i] = Bt.data_ptr()
            xp[i] = X.data_ptr()
        po = _lib.default_pcg_opts(rel_tol=rel_tol, max_it=max_it, x0_precond=int(x0_precond),
                                   check_every=check_every)
        reps = (_lib.Report * self.count)()
        st = self.lib.mpchol_batch_pcg(self.handle, ptrs, lds, bp, xp, ctypes.byref(po), reps,
                                       _stream_handle())
        if st not in (_lib.OK, _lib.PCG_MAXIT):
            check(st, "mpchol_batch_pcg")
        out = []
        for i, X in enumerate(Xs):
            Xo = X.t()
            out.append(Xo.reshape(Bs[i].shape) if Bs[i].dim() == 1 else Xo)
        reports = [Report(r.iterations, bool(r.converged), r.rel_residual, r.backward_error,
                          r.precond_residual, st) for r in reps]
        return out, reports, st
