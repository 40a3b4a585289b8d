"""The left-looking schedule (opts.left = 1, settings.json "left"): block
column k receives the updates of panels 0..k-1 just before it is factored.
Every tile of the trailing matrix receives the same FP32 updates in the same
order as in the right-looking schedule, so the two factors -- and the per-step
precisions the switching rule picks -- must agree bit for bit; the
left-looking factor is also checked against the oracle and solved with."""
import numpy as np
import pytest
import torch

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import matgen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,b,opts", [
    (1536, 256, dict(precision="switching", eps_prime=0.05, ladder=["e4m3", "fp16", "fp16x2"])),
    (1000, 128, dict(precision="fp16x2")),             # ragged last block
    (1280, 256, dict(precision="mxfp8")),
    (900, 128, dict(precision="fp32")),
])
def test_left_looking_factor_equals_right_looking(cuda, n, b, opts):
    A = matgen.spd_matrix(n, 1e4 if opts["precision"] != "mxfp8" else 1e2, 31).numpy()
    Ad = torch.from_numpy(A).cuda()
    fr = mp.factor(Ad, block_size=b, **opts)
    fl = mp.factor(Ad, block_size=b, left=1, **opts)
    ir, il = fr.info(), fl.info()
    assert ir.status == 0 and il.status == 0
    assert il.step_prec == ir.step_prec and il.n_perturbed == ir.n_perturbed
    assert torch.equal(fl.lower(), fr.lower())
    # and it is the oracle's factor
    kw = O.factor_kwargs(fl.opts)
    kw["precision"] = O.SWITCHING
    ref = O.blocked_chol(A, force_prec=il.step_prec, force_fp64=il.step_fp64, **kw)
    Lg = fl.lower().cpu().numpy()
    err = np.linalg.norm(Lg - ref["L"]) / np.linalg.norm(ref["L"])
    print(f"left n={n} b={b} {opts['precision']}: steps {il.step_prec}, err vs oracle {err:.2e}")
    assert err < 5e-2
    B = matgen.rhs(n, 2, 32).cuda()
    X, rep = fl.pcg(Ad, B, rel_tol=1e-10, max_it=300)
    assert rep.converged and rep.rel_residual <= 1e-10
    # a second factorization on the same object replays the captured graph
    fl.compute(Ad)
    assert torch.equal(fl.lower(), fr.lower())
