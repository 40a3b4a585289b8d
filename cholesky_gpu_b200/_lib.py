"""ctypes binding of ``libmpchol.so`` (the C ABI declared in include/mpchol.h).

The shared library is the product; this module only declares its symbols.
Loading fails loudly when the library is missing -- there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmpchol.so"

# mpchol_status
OK = 0
ERR_BAD_ARG = 1
ERR_NOT_SPD = 2
ERR_CUDA = 3
ERR_ALLOC = 4
PCG_MAXIT = 5
PCG_BREAKDOWN = 6
ERR_TIMEOUT = 7
ERR_NOT_SUPPORTED = 8

# mpchol_precision
PREC_FP32 = 0
PREC_FP16 = 1
PREC_E4M3 = 2
PREC_E5M2 = 3
PREC_MXFP8 = 4
PREC_SWITCHING = 5
PREC_FP16X2 = 6
PREC_MXFP6_E2M3 = 7
PREC_MXFP6_E3M2 = 8
PREC_MXFP4 = 9
PREC_NAMES = {PREC_FP32: "fp32", PREC_FP16: "fp16", PREC_E4M3: "e4m3", PREC_E5M2: "e5m2",
              PREC_MXFP8: "mxfp8", PREC_SWITCHING: "switching", PREC_FP16X2: "fp16x2",
              PREC_MXFP6_E2M3: "mxfp6e2m3", PREC_MXFP6_E3M2: "mxfp6e3m2", PREC_MXFP4: "mxfp4"}
PREC_BY_NAME = {v: k for k, v in PREC_NAMES.items()}


class Opts(ctypes.Structure):
    _fields_ = [
        ("block_size", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("eps_prime", ctypes.c_float),
        ("floor", ctypes.c_float),
        ("diag_pert", ctypes.c_int),
        ("pert", ctypes.c_float),
        ("pivot_floor", ctypes.c_float),
        ("switch_mode", ctypes.c_int),
        ("ladder_len", ctypes.c_int),
        ("ladder", ctypes.c_int * 4),
        ("left", ctypes.c_int),
        ("coherence", ctypes.c_int),
        ("equilibrate", ctypes.c_int),
        ("eps_coherence", ctypes.c_float),
    ]


class FactorInfo(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("fail_row", ctypes.c_int),
        ("n_perturbed", ctypes.c_int),
        ("nsteps", ctypes.c_int),
        ("n_fp64_blocks", ctypes.c_int),
        ("steps_by_prec", ctypes.c_int * 10),
    ]


class PcgOpts(ctypes.Structure):
    _fields_ = [
        ("rel_tol", ctypes.c_double),
        ("max_it", ctypes.c_int),
        ("x0_precond", ctypes.c_int),
        ("check_every", ctypes.c_int),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("rel_residual", ctypes.c_double),
        ("backward_error", ctypes.c_double),
        ("precond_residual", ctypes.c_double),
    ]


NPHASES = 10
PHASE_NAMES = ["potrf", "trsm", "quant", "syrk_f32", "syrk_tc", "symv", "trsv", "pcg_vec",
               "setup", "test"]


class Profile(ctypes.Structure):
    _fields_ = [
        ("ms", ctypes.c_double * NPHASES),
        ("calls", ctypes.c_longlong * NPHASES),
        ("launches", ctypes.c_longlong * NPHASES),
    ]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_ll = ctypes.c_longlong
_ull = ctypes.c_ulonglong

# name -> (restype, argtypes)
SIGNATURES = {
    "mpchol_status_str": (ctypes.c_char_p, [_i]),
    "mpchol_opts_default": (None, [ctypes.POINTER(Opts)]),
    "mpchol_pcg_opts_default": (None, [ctypes.POINTER(PcgOpts)]),
    "mpchol_last_error": (ctypes.c_char_p, []),
    "mpchol_profile_enable": (None, [_i]),
    "mpchol_profile_read": (_i, [ctypes.POINTER(Profile), _i]),
    "mpchol_kernel_launches": (ctypes.c_longlong, []),
    "mpchol_factor_create": (_i, [ctypes.POINTER(Opts), _i, ctypes.POINTER(_vp)]),
    "mpchol_factor_compute": (_i, [_vp, _vp, _i, _vp]),
    "mpchol_factor": (_i, [ctypes.POINTER(Opts), _i, _vp, _i, ctypes.POINTER(_vp), _vp]),
    "mpchol_factor_destroy": (_i, [_vp]),
    "mpchol_factor_info_get": (_i, [_vp, ctypes.POINTER(FactorInfo), _vp, _vp, _vp]),
    "mpchol_factor_lower": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "mpchol_factor_diags": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "mpchol_factor_prepare_solve": (_i, [_vp, _vp]),
    "mpchol_pcg": (_i, [_vp, _vp, _i, _vp, _vp, _i, ctypes.POINTER(PcgOpts), ctypes.POINTER(Report), _vp]),
    "mpchol_pcg_f64": (_i, [_vp, _vp, _i, _vp, _vp, _i, ctypes.POINTER(PcgOpts), ctypes.POINTER(Report), _vp]),
    "mpchol_adjoint_solve": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _i, _vp, _i, ctypes.POINTER(PcgOpts),
                                  ctypes.POINTER(Report), _vp]),
    "mpchol_solve_host": (_i, [_vp, _vp, _i, _vp, _vp, _i, ctypes.POINTER(PcgOpts), ctypes.POINTER(Report), _vp]),
    "mpchol_factor_codes": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "mpchol_set_copy_plan": (_i, [_vp, _i, _vp, _vp]),
    "mpchol_factor_save": (_i, [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), _vp]),
    "mpchol_factor_load": (_i, [_vp, _vp, ctypes.c_size_t, _vp]),
    "mpchol_factor_blob_check": (_i, [_vp, ctypes.c_size_t, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "mpchol_copy_plan": (_i, [_i, _i, _vp, _vp, _i]),
    "mpchol_apply_precond": (_i, [_vp, _vp, _vp, _i, _vp]),
    "mpchol_symv": (_i, [_vp, _i, _i, _vp, _vp, _i, _vp]),
    "mpchol_precond_cg": (_i, [_vp, _vp, _vp, _i, _i, _d, _f, _f, _i, _i, _d, _i, _vp]),
    "mpchol_switching_chol": (_i, [_vp, _i, _i, _vp, _vp, _f, _i, _i, _vp, _vp]),
    "mpchol_quantize": (_i, [_vp, _vp, _ll, _i, _vp]),
    "mpchol_quantize_rows": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp]),
    "mpchol_quantize_hash": (_i, [_ull, _ull, _ull, _i, _vp, _vp]),
    "mpchol_syrk_update": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _i, _vp]),
    "mpchol_potrf_static": (_i, [_vp, _i, _i, ctypes.c_float, _vp, _vp]),
    "mpchol_rbf_build": (_i, [_vp, _i, _i, _i, ctypes.c_double, ctypes.c_double, _vp, _vp, _i, _i,
                              _vp]),
    "mpchol_rbf_grad_work_elems": (_i, [_i]),
    "mpchol_batch_create": (_i, [ctypes.POINTER(Opts), _i, _vp, _i, _vp]),
    "mpchol_batch_factor": (_i, [_vp, _vp, _vp, _vp]),
    "mpchol_batch_info": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "mpchol_batch_lower": (_i, [_vp, _i, _vp, _vp, _vp]),
    "mpchol_batch_pcg": (_i, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(PcgOpts), _vp, _vp]),
    "mpchol_batch_destroy": (_i, [_vp]),
    "mpchol_rbf_grad": (_i, [_vp, _i, _i, _i, ctypes.c_double, _vp, _vp, _vp, _vp, _vp, _vp]),
}

_LIB = None


def load() -> ctypes.CDLL:
    """Load libmpchol.so (building it first if the sources are present and the
    library is missing).  Raises if it cannot be loaded."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        if os.environ.get("MPCHOL_NO_BUILD"):
            raise RuntimeError(f"{LIB_PATH} is missing and building is disabled")
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class MpcholError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        lib = load()
        msg = lib.mpchol_status_str(status).decode()
        last = lib.mpchol_last_error().decode()
        super().__init__(f"{what}: {msg} (status {status})" + (f"; {last}" if last else ""))
        self.status = status


def check(status: int, what: str = "") -> int:
    if status != OK:
        raise MpcholError(status, what)
    return status


def default_opts(**kw) -> Opts:
    o = Opts()
    load().mpchol_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = PREC_BY_NAME[v]
        if k == "ladder":
            seq = [PREC_BY_NAME[x] if isinstance(x, str) else int(x) for x in v]
            o.ladder_len = len(seq)
            for i in range(4):
                o.ladder[i] = seq[i] if i < len(seq) else PREC_FP32
            continue
        setattr(o, k, v)
    return o


def default_pcg_opts(**kw) -> PcgOpts:
    o = PcgOpts()
    load().mpchol_pcg_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
