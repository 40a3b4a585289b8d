"""The CPU oracle, pinned against the reference's own outputs.

* number formats: bit-exact against tests/golden/quant_golden.npz, which was
  produced by the reference's lo_float.h (tests/golden/gen_golden.py), and,
  when oracle/_ref is built here, directly against that library;
* the reference CPU POTRF (src/micro_chol.hpp) vs the restatement;
* the blocked factor and PCG against FP64 dense algebra;
* the switching decision rule on hand-made diagonals.
"""
import numpy as np
import pytest

from cholesky_gpu_b200 import matgen
from oracle import oracle as O

from .conftest import ROOT

GOLDEN = ROOT / "tests" / "golden" / "quant_golden.npz"


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("fmt,key", [(O.E4M3, "e4m3"), (O.E5M2, "e5m2")])
@pytest.mark.parametrize("sat", [True, False])
def test_oracle_matches_golden_lofloat(golden, fmt, key, sat):
    x = golden["inputs"].view(np.float32)
    want = golden[f"{key}_{'sat' if sat else 'nosat'}"]
    lib = O.lib()
    fn = lib.orc_f32_to_e4m3 if fmt == O.E4M3 else lib.orc_f32_to_e5m2
    got = np.array([fn(float(v), int(sat)) for v in x], dtype=np.uint8)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, [(hex(golden["inputs"][i]), want[i], got[i]) for i in bad[:5]]


def test_golden_covers_edge_cases(golden):
    x = golden["inputs"].view(np.float32)
    assert np.isnan(x).any() and np.isinf(x).any() and (x == 0).any()
    assert (np.abs(x[np.isfinite(x)]) > 448).any()              # saturation region
    assert ((np.abs(x) < 2.0 ** -6) & (x != 0)).any()           # E4M3 subnormals
    assert x.size > 50000


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref (reference lo_float build) not present")
@pytest.mark.parametrize("fmt", [O.E4M3, O.E5M2])
def test_oracle_matches_reference_lofloat_strided_sweep(fmt):
    pats = np.arange(0, 1 << 32, 4099, dtype=np.uint64).astype(np.uint32)
    x = pats.view(np.float32)
    ref = O.ref_lofloat(x, fmt, True)
    got = O.quantize(x, fmt)
    fin = np.isfinite(x)
    assert np.array_equal(ref[fin], got[fin])


def test_fp16_matches_numpy_rne():
    g = np.random.default_rng(3)
    x = (g.standard_normal(200000) * np.exp(g.uniform(-20, 12, 200000))).astype(np.float32)
    x = np.concatenate([x, np.float32([65504, 65520, 65519.99, 1e-8, 6e-8, -0.0])])
    got = O.quantize(x, O.FP16)
    want = x.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("fmt,maxv", [(O.E4M3, 448.0), (O.E5M2, 57344.0), (O.FP16, 65504.0)])
def test_row_scale_is_smallest_non_saturating_power_of_two(fmt, maxv):
    g = np.random.default_rng(5)
    for a in np.concatenate([np.exp(g.uniform(-80, 80, 2000)), [maxv, maxv * 1.0001, 1.0]]):
        a = np.float32(a)
        e = O.row_scale_exp(a, fmt)
        assert a * 2.0 ** -e <= maxv
        if e > -126:   # exponents are clamped so 2^e and 2^-e stay normal floats
            assert a * 2.0 ** -(e - 1) > maxv
    assert O.row_scale_exp(0.0, fmt) == 0


def test_mx_scale_follows_ocp_rule():
    for a, e in [(1.0, -8), (448.0, 0), (511.9, 0), (512.0, 1), (2.0 ** -130, -127), (0.0, -127)]:
        assert O.mx_scale_exp(a) == e


def test_decode_roundtrip_all_codes():
    for fmt in (O.E4M3, O.E5M2):
        codes = np.arange(256, dtype=np.uint8)
        v = O.decode(codes, fmt)
        fin = np.isfinite(v)
        assert np.array_equal(O.quantize(v[fin], fmt), codes[fin] if fmt == O.E5M2 else codes[fin])


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not present")
def test_micro_cholesky_restatement_matches_reference_bitwise():
    A = matgen.spd_matrix(96, 1e3, 11).numpy()
    Lr, rc = O.ref_micro_cholesky(A)
    Lo, rc2 = O.micro_cholesky(A)
    assert rc == 0 and rc2 == 0
    assert np.array_equal(Lr, Lo)


def test_blocked_fp32_factor_matches_fp64_cholesky():
    A = matgen.spd_matrix(384, 1e4, 7).numpy()
    r = O.blocked_chol(A, block_size=128, precision=O.FP32)
    assert r["status"] == 0
    L64 = np.linalg.cholesky(A.astype(np.float64))
    err = np.linalg.norm(r["L"] - L64) / np.linalg.norm(L64)
    assert err < 1e-5, err
    # the tracker equals the true Schur diagonals at the start of each block:
    # after the last panel it holds the final pivots' squares
    Lf = r["L"].astype(np.float64)
    np.testing.assert_allclose(r["dtilde"][256:], (Lf[256:, 256:] ** 2).sum(1), rtol=2e-3)


def test_blocked_reduces_to_unblocked_when_one_block():
    A = matgen.spd_matrix(64, 1e2, 9).numpy()
    r = O.blocked_chol(A, block_size=64, precision=O.FP32)
    Lu, _ = O.micro_cholesky(A)
    assert np.array_equal(r["L"], Lu)


def test_not_spd_is_reported_with_row():
    A = matgen.spd_matrix(256, 10.0, 4).numpy()
    A[200, 200] = -1.0
    r = O.blocked_chol(A, block_size=64, precision=O.FP32)
    assert r["status"] == 2 and r["fail_row"] == 200


def test_pcg_fp32_factor_reaches_1e10_and_matches_dense_solve():
    n = 512
    A = matgen.spd_matrix(n, 1e4, 1).numpy()
    b = matgen.rhs(n, 1, 2).numpy()
    r = O.blocked_chol(A, block_size=128, precision=O.FP16)
    x, it, rel = O.pcg(A, r["L"], b, 1e-10, 200)
    assert rel <= 1e-10 and it > 1
    xd = O.dense_solve(A, b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-6


def test_switching_rule_picks_lowest_admissible_precision():
    d = np.ones(8, np.float32)
    # max d/dtilde = 2: E4M3 (u=1/16) admissible when eps' >= 1/8
    dt = np.full(8, 0.5, np.float32)
    assert O.choose_precision(d, dt, eps_prime=0.2) == O.E4M3
    assert O.choose_precision(d, dt, eps_prime=0.1) == O.FP16
    assert O.choose_precision(d, dt, eps_prime=1e-5) == O.FP32
    dt[3] = 0.0   # exhausted pivot forbids everything but FP32
    assert O.choose_precision(d, dt, eps_prime=100.0) == O.FP32
    # a ladder without FP32 falls back to its own most precise (last) entry
    dt[3] = 0.5
    lad = (O.E4M3, O.FP16, O.FP16X2)
    assert O.choose_precision(d, dt, eps_prime=1e-9, ladder=lad) == O.FP16X2
    assert O.choose_precision(d, dt, eps_prime=1e-6, ladder=lad) == O.FP16X2
    assert O.choose_precision(d, dt, eps_prime=0.2, ladder=lad) == O.E4M3


def test_reference_literal_rule():
    d = np.ones(4, np.float32)
    dt = np.array([0.9, 0.9, 0.9, 0.9], np.float32)
    # FP16 row condition: 2^-10 * 0.9 >= eps' -> true for eps' = 5e-4
    assert O.choose_precision(d, dt, eps_prime=5e-4, switch_mode=1) == O.FP16
    assert O.choose_precision(d, dt, eps_prime=1e-2, switch_mode=1) == O.E4M3
    assert O.choose_precision(d, dt, eps_prime=1e-9, switch_mode=1) == O.FP32


def test_rbf_oracle_gradients_match_central_differences():
    """Pins the FP64 gradient formulas of the RBF solve oracle (loss
    1/2 y^T K^-1 y) against FP64 central differences, h = 1e-5."""
    g = np.random.default_rng(0)
    n, d, ell, lam, h = 40, 3, 1.3, 0.1, 1e-5
    X = g.standard_normal((n, d))
    y = g.standard_normal(n)
    dX, d_ell, d_lam, x = O.rbf_loss_grads_f64(X, ell, lam, y)
    L = lambda X_, e_, l_: O.rbf_loss_f64(X_, e_, l_, y)  # noqa: E731
    assert abs((L(X, ell + h, lam) - L(X, ell - h, lam)) / (2 * h) - d_ell) <= 1e-7 * abs(d_ell)
    assert abs((L(X, ell, lam + h) - L(X, ell, lam - h)) / (2 * h) - d_lam) <= 1e-7 * abs(d_lam)
    for (i, k) in ((5, 1), (0, 0), (39, 2)):
        E = np.zeros_like(X)
        E[i, k] = h
        fd = (L(X + E, ell, lam) - L(X - E, ell, lam)) / (2 * h)
        assert abs(fd - dX[i, k]) <= 1e-6 * max(abs(dX[i, k]), 1e-3)


@pytest.mark.parametrize("fmt,name", [(O.MXFP6E3M2, "f6e3m2"), (O.MXFP4, "f4e2m1"),
                                      (O.MXFP6E2M3, "f6e2m3")])
def test_fp6_fp4_element_rounding_matches_lo_float(fmt, name):
    """The oracle's FP6/FP4 element rounding (OCP E2M3, E3M2, E2M1: RNE,
    saturating) against the reference lo_float's float6_e2m3 / float6_e3m2 /
    float4_e2m1 conversions (golden vectors).  lo_float reserves two codes
    the OCP formats use as numbers: float4_e2m1's -0 (0x8) and float6_e2m3's
    +-7.0 (0x1e, 0x3e) are NaN there.  Where lo_float returns that NaN for a
    finite input, the oracle must return the OCP value (-0 or +-7.0);
    everywhere else the two agree exactly."""
    g = np.load(GOLDEN)
    x = g["small_inputs"].view(np.float32)
    want = g[name]
    got = O.mx_round(x, fmt)
    fin = np.isfinite(x)
    assert np.all(np.isnan(got[np.isnan(x)]))
    special = fin & np.isnan(want)
    if fmt == O.MXFP4:
        assert np.all(got[special] == 0.0) and np.all(np.signbit(got[special]))
    elif fmt == O.MXFP6E2M3:
        assert np.all(np.abs(got[special]) == 7.0)
    else:
        assert not special.any()
    ok = fin & ~special
    assert np.array_equal(got[ok], want[ok])
    assert ok.sum() > 25000
