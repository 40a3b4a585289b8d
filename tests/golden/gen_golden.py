"""Generate tests/golden/quant_golden.npz from the reference's own lo_float.h.

Run in a checkout that has the reference sources and the oracle/_ref build
(`make -C oracle ref`).  The vectors pin the float32 -> E4M3 / E5M2
conversions (lo_float ConvertFrom<kSaturate, kTruncate=false>, RNE) that the
oracle restates and the GPU quantizer must reproduce bit for bit:

  * every float32 whose low 16 bits are zero (covers all exponents/top bits),
  * the neighbourhood (+-3 ulps) of every rounding midpoint between adjacent
    E4M3 and E5M2 values, including the subnormal and saturation boundaries,
  * 20000 seeded random finite values spread over the E4M3/E5M2 range,
  * +-0, +-inf, NaN.

Output arrays: inputs (uint32 bit patterns), e4m3_sat, e4m3_nosat, e5m2_sat,
e5m2_nosat (uint8 codes); small_inputs (uint32, |x| <= 64 and the specials)
with f6e2m3, f6e3m2, f4e2m1 (the saturating conversions to lo_float's
float6_e2m3, float6_e3m2 and float4_e2m1, as float32 values).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402


def midpoints(fmt: int) -> np.ndarray:
    codes = np.arange(256, dtype=np.uint8)
    vals = O.decode(codes, fmt).astype(np.float64)
    v = np.unique(vals[np.isfinite(vals) & (vals >= 0)])
    mids = (v[:-1] + v[1:]) / 2.0
    top = v[-1] * 1.0625  # beyond the largest finite value
    return np.concatenate([mids, [top, v[-1]], v]).astype(np.float32)


def main() -> None:
    if not O.have_ref():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    pats = [np.arange(0, 1 << 32, 1 << 16, dtype=np.uint64).astype(np.uint32)]
    for fmt in (O.E4M3, O.E5M2):
        m = midpoints(fmt).view(np.uint32).astype(np.int64)
        nb = (m[:, None] + np.arange(-3, 4)[None, :]).ravel()
        nb = nb[(nb >= 0) & (nb < (1 << 31))].astype(np.uint32)
        pats += [nb, nb | np.uint32(0x80000000)]
    g = np.random.default_rng(20241203)
    r = (g.standard_normal(20000) * np.exp(g.uniform(-25, 13, 20000))).astype(np.float32)
    pats.append(r.view(np.uint32))
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan], dtype=np.float32).view(np.uint32)
    pats.append(specials)
    inputs = np.unique(np.concatenate(pats))
    x = inputs.view(np.float32)
    out = dict(inputs=inputs)
    out["e4m3_sat"] = O.ref_lofloat(x, O.E4M3, True)
    out["e4m3_nosat"] = O.ref_lofloat(x, O.E4M3, False)
    out["e5m2_sat"] = O.ref_lofloat(x, O.E5M2, True)
    out["e5m2_nosat"] = O.ref_lofloat(x, O.E5M2, False)
    # the 6- and 4-bit element formats (OCP MX FP6/FP4): every float32 whose
    # low 16 bits are zero inside [-64, 64], the neighbourhood of every
    # rounding midpoint of each grid, and the random set scaled into range
    small = [np.arange(0, 1 << 32, 1 << 16, dtype=np.uint64).astype(np.uint32)]
    for fmt in (O.MXFP6E2M3, O.MXFP6E3M2, O.MXFP4):
        grid = np.unique(np.abs(O.ref_lofloat_small(
            np.linspace(-40, 40, 200001).astype(np.float32), fmt)))
        grid = grid[np.isfinite(grid)].astype(np.float64)
        mids = np.concatenate([(grid[:-1] + grid[1:]) / 2.0, grid, [grid[-1] * 1.07]])
        m = mids.astype(np.float32).view(np.uint32).astype(np.int64)
        nb = (m[:, None] + np.arange(-3, 4)[None, :]).ravel()
        nb = nb[(nb >= 0) & (nb < (1 << 31))].astype(np.uint32)
        small += [nb, nb | np.uint32(0x80000000)]
    small.append((r / np.float32(1 << 20)).view(np.uint32))
    small.append(specials)
    sin = np.unique(np.concatenate(small))
    xs = sin.view(np.float32)
    keep = ~np.isfinite(xs) | (np.abs(xs) <= 64.0)
    sin = sin[keep]
    xs = sin.view(np.float32)
    out["small_inputs"] = sin
    out["f6e2m3"] = O.ref_lofloat_small(xs, O.MXFP6E2M3)
    out["f6e3m2"] = O.ref_lofloat_small(xs, O.MXFP6E3M2)
    out["f4e2m1"] = O.ref_lofloat_small(xs, O.MXFP4)
    dst = Path(__file__).resolve().parent / "quant_golden.npz"
    np.savez_compressed(dst, **out)
    print(f"{dst}: {inputs.size} inputs")


if __name__ == "__main__":
    main()
