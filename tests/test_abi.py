"""C-ABI library: loads, exports every declared symbol, host-side checks.

No compute calls here (no GPU needed): argument validation happens before any
CUDA call, so the error paths are exercised on the CPU.
"""
import ctypes
import re

import pytest

from cholesky_gpu_b200 import _lib

from .conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "mpchol.h").read_text()
    return sorted(set(re.findall(r"MPCHOL_API\s+[\w\s\*]+?\b(mpchol_\w+)\s*\(", text)))


def test_library_loads_and_exports_all_declared_symbols():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "ctypes table and header disagree"


def test_refcompat_header_mentions_reference_signatures():
    text = (ROOT / "include" / "mpchol_refcompat.h").read_text()
    assert "int precond_CG(double* A, double* x, double* b, int n, int r, double normA" in text
    assert "void switching_chol(float* d_A, int n, int b" in text


def test_status_strings():
    lib = _lib.load()
    for code in range(9):
        s = lib.mpchol_status_str(code).decode()
        assert s and s != "unknown status"
    assert lib.mpchol_status_str(99).decode() == "unknown status"


def test_default_options():
    o = _lib.default_opts()
    assert o.block_size == 256 and o.diag_pert == 1
    assert o.precision == _lib.PREC_SWITCHING
    assert list(o.ladder)[: o.ladder_len] == [_lib.PREC_E4M3, _lib.PREC_FP16, _lib.PREC_FP32]
    p = _lib.default_pcg_opts()
    assert p.rel_tol == 1e-10 and p.max_it == 200 and p.x0_precond == 1


@pytest.mark.parametrize("kw,status", [
    (dict(block_size=100), _lib.ERR_BAD_ARG),
    (dict(block_size=512), _lib.ERR_BAD_ARG),
    (dict(precision=10), _lib.ERR_BAD_ARG),
    (dict(precision="switching", ladder=["mxfp8", "mxfp4"]), _lib.ERR_NOT_SUPPORTED),
    (dict(left=2), _lib.ERR_BAD_ARG),
    (dict(coherence=2), _lib.ERR_BAD_ARG),
    (dict(equilibrate=-1), _lib.ERR_BAD_ARG),
    (dict(diag_pert=1, pivot_floor=0.0), _lib.ERR_BAD_ARG),
    (dict(switch_mode=3), _lib.ERR_BAD_ARG),
    (dict(precision="e4m3", block_size=64), _lib.ERR_NOT_SUPPORTED),
    (dict(precision="mxfp8", block_size=96), _lib.ERR_NOT_SUPPORTED),
])
def test_option_validation_without_gpu(kw, status):
    lib = _lib.load()
    o = _lib.default_opts(**kw)
    h = ctypes.c_void_p()
    assert lib.mpchol_factor_create(ctypes.byref(o), 1024, ctypes.byref(h)) == status
    assert not h.value


def test_null_and_size_arguments_rejected():
    lib = _lib.load()
    assert lib.mpchol_factor_create(None, 16, None) == _lib.ERR_BAD_ARG
    o = _lib.default_opts()
    h = ctypes.c_void_p()
    assert lib.mpchol_factor_create(ctypes.byref(o), 0, ctypes.byref(h)) == _lib.ERR_BAD_ARG
    assert lib.mpchol_quantize(None, None, -1, 2, None) == _lib.ERR_BAD_ARG
    assert lib.mpchol_quantize_hash(0, 16, 0, 2, None, None) == _lib.ERR_BAD_ARG
    assert lib.mpchol_factor_destroy(None) == _lib.ERR_BAD_ARG
    assert lib.mpchol_precond_cg(None, None, None, 4, 2, 0.0, 0.0, 0.0, 0, 32, 0.0, 10, None) < 0


def test_smoke_checks_the_factor_with_its_own_options():
    """smoke() restates its factor with the oracle under the options the
    factor was computed with: the library defaults (rounding-error shifts,
    pivot floor, coherence rule) plus the smoke case's block size and
    precision -- not the oracle's own defaults."""
    import __graft_entry__ as ge
    from oracle import oracle as O
    opts = _lib.default_opts(**ge.SMOKE_OPTS)
    kw = ge.smoke_oracle_kwargs(opts)
    d = _lib.default_opts()
    assert kw["diag_pert"] == d.diag_pert == 1
    assert kw["pert"] == pytest.approx(d.pert) and kw["pivot_floor"] == pytest.approx(d.pivot_floor)
    assert kw["block_size"] == ge.SMOKE_OPTS["block_size"]
    assert kw["precision"] == O.SWITCHING and kw["coherence"] == d.coherence
    # the oracle accepts exactly these keywords
    O.make_opts(**kw)
