"""The drop-in shim as C++: a reference-style caller compiled against
include/mpchol_refcompat.h and linked with libmpchol.so.

The caller makes the reference's own calls -- precond_CG as its main() does
(src/mixed_cholesky.cu:430-431) and switching_chol with the handle arguments
of src/switching_chol.cuh:19-22 -- with arguments the library rejects before
any CUDA call, so it runs on a machine without a GPU: precond_CG returns
-(100 + MPCHOL_ERR_BAD_ARG) and the status of the void switching_chol is read
back through mpchol_refcompat_last_status().
"""
import shutil
import subprocess

import pytest

from cholesky_gpu_b200 import _lib

from .conftest import ROOT

CALLER = r"""
#include <cstdio>
#include "mpchol_refcompat.h"

int main() {
  cublasHandle_t cublasH = nullptr;
  cusolverDnHandle_t cusolverH = nullptr;
  cublasLtHandle_t cublasltH = nullptr;
  cudaStream_t stream = nullptr;
  double* d_A = nullptr;
  double* x = nullptr;
  double* b = nullptr;
  double inf_norm_A = 1.0;
  const int N = 64, r = 32;
  // the reference's call, unchanged (null device buffers: rejected on the host)
  int success = precond_CG(d_A, x, b, N, r, inf_norm_A, cublasH, cusolverH, stream, 0.1f, 0.0f, true);
  // default arguments of the reference signature
  int success2 = precond_CG(d_A, x, b, N, r, inf_norm_A, cublasH, cusolverH, stream);
  switching_chol(nullptr, N, r, nullptr, nullptr, 0.1f, false, 32, cusolverH, cublasltH, cublasH,
                 stream, nullptr);
  const int st = mpchol_refcompat_last_status();
  std::printf("%d %d %d\n", success, success2, st);
  const int want = -(100 + MPCHOL_ERR_BAD_ARG);
  return (success == want && success2 == want && st == MPCHOL_ERR_BAD_ARG) ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs a C++ compiler")
def test_reference_style_caller_compiles_links_and_runs(tmp_path):
    lib = _lib.load()              # builds libmpchol.so when it is missing
    del lib
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    libdir = _lib.LIB_PATH.parent
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(src), "-o", str(exe),
           f"-L{libdir}", "-l:libmpchol.so", f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    want = -(100 + _lib.ERR_BAD_ARG)
    assert out.stdout.split() == [str(want), str(want), str(_lib.ERR_BAD_ARG)]
