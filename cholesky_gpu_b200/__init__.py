"""mpchol: mixed-precision blocked Cholesky preconditioner + FP64-checked PCG
for NVIDIA B200 (sm_100a), behind a plain C ABI (include/mpchol.h).

The compute path is ``libmpchol.so`` (hand-written sm_100a kernels); this
package is its Python face: ``Factor`` / ``factor`` / ``solve`` and the
reference-shaped ``precond_CG`` / ``switching_chol``.
"""
from ._lib import (  # noqa: F401
    PREC_E4M3, PREC_E5M2, PREC_FP16, PREC_FP32, PREC_MXFP8, PREC_SWITCHING, PREC_NAMES,
    MpcholError, load,
)
from .api import (  # noqa: F401
    Batch, Factor, FactorInfo, Report, copy_plan, factor, factor_blob_info, precond_CG, solve,
    switching_chol,
)
from .autograd import RBFSolve, rbf_build, rbf_solve  # noqa: F401

__all__ = ["Factor", "FactorInfo", "Report", "factor", "solve", "precond_CG", "switching_chol",
           "copy_plan", "factor_blob_info", "load", "MpcholError"]
