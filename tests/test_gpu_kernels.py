"""Kernel-level parity of the sm_100a library against the CPU oracle.

Every call goes through the C ABI (libmpchol.so).  Bars: bit-exact for the
quantizers (codes and scale exponents); FP32-accumulation tolerance for the
trailing updates; FP64 tolerance for the PCG operator and preconditioner.
"""
import ctypes

import numpy as np
import pytest
import torch

from cholesky_gpu_b200 import _lib, matgen
from oracle import oracle as O

from .conftest import ROOT

pytestmark = pytest.mark.gpu


def stream():
    return torch.cuda.current_stream().cuda_stream


def gpu_quantize(x: np.ndarray, fmt: int) -> np.ndarray:
    lib = _lib.load()
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    q = torch.empty(x.size, dtype=torch.int16 if fmt == O.FP16 else torch.uint8, device="cuda")
    _lib.check(lib.mpchol_quantize(xd.data_ptr(), q.data_ptr(), x.size, fmt, stream()))
    out = q.cpu().numpy()
    return out.view(np.uint16) if fmt == O.FP16 else out


@pytest.mark.parametrize("fmt", [O.E4M3, O.E5M2, O.FP16])
def test_quantize_matches_oracle_on_golden_and_random(cuda, fmt):
    g = np.load(ROOT / "tests" / "golden" / "quant_golden.npz")
    x = g["inputs"].view(np.float32)
    rnd = np.random.default_rng(1)
    x = np.concatenate([x, (rnd.standard_normal(1 << 20) * np.exp(rnd.uniform(-30, 20, 1 << 20)))
                        .astype(np.float32)])
    got = gpu_quantize(x, fmt)
    want = O.quantize(x, fmt)
    fin = np.isfinite(x)
    assert np.array_equal(got[fin], want[fin])
    # NaN inputs give a NaN code (hardware emits the OCP encoding)
    nanv = O.decode(got[np.isnan(x)], fmt)
    assert np.all(np.isnan(nanv))
    if fmt != O.FP16:
        key = "e4m3_sat" if fmt == O.E4M3 else "e5m2_sat"
        gi = np.isfinite(g["inputs"].view(np.float32))
        assert np.array_equal(got[: gi.size][gi], g[key][gi])


@pytest.mark.parametrize("fmt", [O.E4M3, O.E5M2, O.FP16])
def test_quantize_exhaustive_all_float32_patterns(cuda, fmt):
    """All 2^32 inputs: GPU and oracle fold the codes of each 2^24-pattern
    chunk into a hash (non-finite inputs as class tokens); 256 words compared."""
    lib = _lib.load()
    chunk = 1 << 24
    h = torch.zeros(256, dtype=torch.int64, device="cuda")
    _lib.check(lib.mpchol_quantize_hash(0, 1 << 32, chunk, fmt, h.data_ptr(), stream()))
    got = h.cpu().numpy().view(np.uint64)
    want = O.quantize_hash(0, 1 << 32, chunk, fmt)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"chunks differing: {bad[:8]}"


def gpu_quantize_rows(P: np.ndarray, fmt: int):
    lib = _lib.load()
    m, k = P.shape
    Pd = torch.from_numpy(np.asfortranarray(P).T.copy()).cuda()   # column-major storage
    half = fmt in (O.FP16, O.FP16X2)
    q = torch.zeros(m * k * (2 if fmt == O.FP16X2 else 1), dtype=torch.int16 if half else torch.uint8,
                    device="cuda")
    sc = torch.zeros(m * (k // 32 if fmt in O.MX_FAMILY else 1), dtype=torch.uint8, device="cuda")
    _lib.check(lib.mpchol_quantize_rows(Pd.data_ptr(), m, k, m, fmt, q.data_ptr(), sc.data_ptr(),
                                        stream()))
    codes = q.cpu().numpy().reshape(-1, k)
    if half:
        codes = codes.view(np.uint16)
    s = sc.cpu().numpy()
    s = s.reshape(m, k // 32) if fmt in O.MX_FAMILY else s.view(np.int8)
    return codes, s


def panel(m, k, seed):
    g = np.random.default_rng(seed)
    P = (g.standard_normal((m, k)) * np.exp(g.uniform(-6, 6, (m, 1)))).astype(np.float32)
    P[3, :] = 0.0                                     # an all-zero row
    P[5, 7] = 3.0e5                                   # an outlier inside a row
    P[9, :] *= np.float32(1e-30)                      # a tiny row (subnormal-scale values)
    return P


@pytest.mark.parametrize("fmt", [O.E4M3, O.E5M2, O.FP16, O.MXFP8, O.FP16X2])
@pytest.mark.parametrize("m,k", [(300, 256), (129, 128), (64, 64)])
def test_quantize_rows_matches_oracle(cuda, fmt, m, k):
    P = panel(m, k, 7 + k)
    codes, s = gpu_quantize_rows(P, fmt)
    wc, ws = O.quantize_rows(P, fmt)
    assert np.array_equal(s.astype(np.int64), ws.astype(np.int64))
    assert np.array_equal(codes, wc)


def syrk_ref(C, Q, s, fmt, m, k):
    if fmt == O.MXFP8:
        vals = O.decode(Q, O.E4M3).astype(np.float64) * np.repeat(2.0 ** (s.astype(np.int64) - 127), 32, 1)
        prod = vals @ vals.T
    elif fmt == O.FP16X2:
        hi = O.decode(Q[:m], O.FP16).astype(np.float64)
        lo = O.decode(Q[m:], O.FP16).astype(np.float64)
        sc = 2.0 ** s.astype(np.float64)
        prod = (hi @ hi.T + hi @ lo.T + lo @ hi.T) * sc[:, None] * sc[None, :]
    else:
        vals = O.decode(Q, fmt).astype(np.float64)
        sc = 2.0 ** s.astype(np.float64)
        prod = (vals @ vals.T) * sc[:, None] * sc[None, :]
    out = C.astype(np.float64).copy()
    low = np.tril(np.ones((m, m), bool))
    out[low] -= prod[low]
    return out


@pytest.mark.parametrize("fmt", [O.E4M3, O.E5M2, O.FP16, O.FP16X2, O.MXFP8])
@pytest.mark.parametrize("m,k", [(640, 256), (300, 128), (1000, 256), (2500, 256)])
def test_tensor_core_syrk_matches_oracle(cuda, fmt, m, k):
    lib = _lib.load()
    P = panel(m, k, 3)
    P[5, 7] = 1.0
    codes, s = gpu_quantize_rows(P, fmt)
    g = np.random.default_rng(4)
    C = g.standard_normal((m, m)).astype(np.float32)
    Cd = torch.from_numpy(C.T.copy()).cuda()    # column-major
    Qd = torch.from_numpy(codes.view(np.int16) if fmt in (O.FP16, O.FP16X2) else codes).cuda()
    Sd = torch.from_numpy(s.view(np.uint8)).cuda()
    _lib.check(lib.mpchol_syrk_update(Cd.data_ptr(), m, m, k, fmt, Qd.data_ptr(), Sd.data_ptr(),
                                      None, 0, stream()))
    got = Cd.cpu().numpy().T
    want = syrk_ref(C, codes, s, fmt, m, k)
    low = np.tril(np.ones((m, m), bool))
    scale = np.abs(want[low]).max()
    err = np.abs(got[low] - want[low]).max() / scale
    print(f"tc syrk fmt={fmt} m={m} k={k} max rel err {err:.3e}")
    # FP32 accumulation in TMEM; the FP8 MMA (plain and block-scaled MX)
    # accumulates with reduced internal precision, so its bar is looser.
    # (FP16X2 accumulates three products per K step: slightly more rounding)
    assert err < {O.FP16: 2e-6, O.FP16X2: 5e-6}.get(fmt, 1e-4), err
    # upper triangle untouched
    assert np.array_equal(got[~low], C[~low])


@pytest.mark.parametrize("fmt", [O.MXFP8, O.FP16, O.E4M3])
@pytest.mark.parametrize("m,k", [(700, 512), (1300, 1024)])
def test_tensor_core_syrk_wide_panels(cuda, fmt, m, k):
    """The kernel-level SYRK with 512- and 1024-wide quantized panels (codes
    and scales from the oracle's quantizer): MXFP8 takes one E8M0 scale per
    32 columns across all K chunks (tensor-memory scale columns per chunk and
    accumulator buffer)."""
    lib = _lib.load()
    P = panel(m, k, 5)
    codes, s = O.quantize_rows(P, fmt)
    g = np.random.default_rng(6)
    C = g.standard_normal((m, m)).astype(np.float32)
    Cd = torch.from_numpy(C.T.copy()).cuda()
    Qd = torch.from_numpy(np.ascontiguousarray(codes.view(np.int16) if fmt == O.FP16 else codes)).cuda()
    Sd = torch.from_numpy(np.ascontiguousarray(s.view(np.uint8))).cuda()
    _lib.check(lib.mpchol_syrk_update(Cd.data_ptr(), m, m, k, fmt, Qd.data_ptr(), Sd.data_ptr(),
                                      None, 0, stream()))
    got = Cd.cpu().numpy().T
    want = syrk_ref(C, codes, s, fmt, m, k)
    low = np.tril(np.ones((m, m), bool))
    err = np.abs(got[low] - want[low]).max() / np.abs(want[low]).max()
    print(f"tc syrk fmt={fmt} m={m} k={k} max rel err {err:.3e}")
    assert err < {O.FP16: 4e-6}.get(fmt, 2e-4), err
    assert np.array_equal(got[~low], C[~low])


@pytest.mark.parametrize("m,k", [(640, 256), (333, 96)])
def test_fp32_syrk_matches_fp64(cuda, m, k):
    lib = _lib.load()
    g = np.random.default_rng(8)
    P = g.standard_normal((m, k)).astype(np.float32)
    C = g.standard_normal((m, m)).astype(np.float32)
    Cd = torch.from_numpy(C.T.copy()).cuda()
    Pd = torch.from_numpy(P.T.copy()).cuda()
    _lib.check(lib.mpchol_syrk_update(Cd.data_ptr(), m, m, k, O.FP32, None, None, Pd.data_ptr(), m,
                                      stream()))
    got = Cd.cpu().numpy().T
    want = C.astype(np.float64) - P.astype(np.float64) @ P.astype(np.float64).T
    low = np.tril(np.ones((m, m), bool))
    err = np.abs(got[low] - want[low]).max() / np.abs(want[low]).max()
    assert err < 1e-6, err


# (1024, 8), (1000, 8), (2100, 8): the staged kernel's 8-rhs path on the FP64
# tensor cores (ragged last tile for 1000 and 2100); (257, 8) the unstaged one
@pytest.mark.parametrize("n,nrhs", [(1000, 1), (1024, 4), (257, 8), (64, 2), (1024, 8), (1000, 8),
                                    (2100, 8)])
def test_symv_matches_fp64(cuda, n, nrhs):
    lib = _lib.load()
    A = matgen.spd_matrix(n, 1e3, 5).numpy()
    X = np.random.default_rng(1).standard_normal((n, nrhs))
    Ad = torch.from_numpy(A).cuda()
    Xd = torch.from_numpy(X.T.copy()).cuda()
    Yd = torch.empty_like(Xd)
    _lib.check(lib.mpchol_symv(Ad.data_ptr(), n, n, Xd.data_ptr(), Yd.data_ptr(), nrhs, stream()))
    got = Yd.cpu().numpy().T
    want = A.astype(np.float64) @ X
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-13


@pytest.mark.parametrize("n", [640, 1000])
def test_fused_panel_codes_match_oracle(cuda, n):
    """The panel solve writes the step's panel in every candidate format from
    shared memory; those codes and scales must equal the oracle's quantization
    of the solved panel (read back from L) bit for bit.  n = 1000 leaves a
    partial 32-row slab at the bottom of the panel."""
    import cholesky_gpu_b200 as mp
    A = matgen.spd_matrix(n, 1e3, 17)
    f = mp.Factor(n, block_size=256, precision="switching", eps_prime=1e-5,
                  ladder=["e4m3", "e5m2", "mxfp8", "fp16x2"])
    f.compute(A.cuda())
    L = f.lower().cpu().numpy()
    for fmt in (O.E4M3, O.E5M2, O.MXFP8, O.FP16X2):
        codes, scales, s0 = f.panel_codes(fmt)
        P = np.ascontiguousarray(L[s0 + 256:, s0:s0 + 256])
        wc, ws = O.quantize_rows(P, fmt)
        assert codes.shape == wc.shape
        bad = np.nonzero(codes != wc)
        assert bad[0].size == 0, (fmt, bad[0][:5], bad[1][:5])
        assert np.array_equal(scales.astype(np.int32), ws.astype(np.int32)), fmt


@pytest.mark.parametrize("fmt", [O.MXFP6E2M3, O.MXFP6E3M2, O.MXFP4])
@pytest.mark.parametrize("m,k", [(300, 256), (129, 128)])
def test_fp6_fp4_quantize_rows_matches_oracle(cuda, fmt, m, k):
    """MX quantization with FP6/FP4 elements: block scales 2^(floor(log2
    amax) - emax_elem) and the element values (E4M3 codes of the
    FP6/FP4-rounded values) equal the oracle's bit for bit."""
    P = panel(m, k, 11 + k)
    codes, s = gpu_quantize_rows(P, fmt)
    wc, ws = O.quantize_rows(P, fmt)
    assert np.array_equal(s.astype(np.int64), ws.astype(np.int64))
    assert np.array_equal(codes, wc)


@pytest.mark.parametrize("fmt", [O.MXFP6E2M3, O.MXFP6E3M2, O.MXFP4])
def test_fp6_fp4_syrk_matches_oracle(cuda, fmt):
    """The trailing update with FP6/FP4 element values through the
    block-scaled E4M3 MMA equals the FP64 product of the dequantized panel."""
    lib = _lib.load()
    m, k = 700, 256
    P = panel(m, k, 21)
    codes, s = gpu_quantize_rows(P, fmt)
    g = np.random.default_rng(22)
    C = g.standard_normal((m, m)).astype(np.float32)
    Cd = torch.from_numpy(C.T.copy()).cuda()
    # the operands stay referenced until the update has run (a temporary's
    # device memory could be handed to the next allocation meanwhile)
    Qd = torch.from_numpy(codes).cuda()
    Sd = torch.from_numpy(s.view(np.uint8)).cuda()
    _lib.check(lib.mpchol_syrk_update(Cd.data_ptr(), m, m, k, fmt, Qd.data_ptr(), Sd.data_ptr(),
                                      None, 0, stream()))
    got = Cd.cpu().numpy().T
    want = syrk_ref(C, codes, s, O.MXFP8, m, k)
    low = np.tril(np.ones((m, m), bool))
    err = np.abs(got[low] - want[low]).max() / np.abs(want[low]).max()
    assert err < 2e-4, err
