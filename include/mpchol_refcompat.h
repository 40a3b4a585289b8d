/*
 * Drop-in replacements for the reference's driver surface, with its exact
 * signatures, implemented over the mpchol C ABI (include/mpchol.h).
 *
 *   precond_CG      src/mixed_cholesky.cu:76-78
 *   switching_chol  src/switching_chol.cuh:19-22
 *
 * A caller of the reference (e.g. its main(), src/mixed_cholesky.cu:355-501)
 * includes this header instead of mixed_cholesky.cu / switching_chol.cuh and
 * links libmpchol.so.  The library handles are accepted and ignored (no
 * cuBLAS/cuSOLVER link is needed) and, unlike the reference
 * (src/mixed_cholesky.cu:221-223), they and the stream are never destroyed.
 *
 * Semantics kept: A is an FP64 device matrix (column-major, ld = n) cast to
 * FP32 for the factor, the PCG operator is the FP64 A, x0 = M^-1 b, the
 * return value is 0 (converged) / -1 (not converged) / > 0 (preconditioner
 * failed, failing row + 1).  Semantics changed on purpose: convergence is
 * tested on the FP64 true residual ||b - A x|| / ||b|| with tolerance
 * MPCHOL_REFCOMPAT_REL_TOL (the reference hard-codes rel_tol = 0, i.e. always
 * max_it = 200 iterations, src/mixed_cholesky.cu:81-82 -- define the macro to
 * 0.0 to get that behaviour); library errors return -(100 + mpchol_status).
 */
#ifndef MPCHOL_REFCOMPAT_H_
#define MPCHOL_REFCOMPAT_H_

#include "mpchol.h"

#ifndef MPCHOL_REFCOMPAT_REL_TOL
#define MPCHOL_REFCOMPAT_REL_TOL 1e-10
#endif
#ifndef MPCHOL_REFCOMPAT_MAX_IT
#define MPCHOL_REFCOMPAT_MAX_IT 200
#endif

#ifdef __cplusplus
#include <cstdint>

/* Opaque handle types with the same spelling as cuBLAS / cuSOLVER / cuBLASLt
 * / CUDA runtime, so reference call sites compile unchanged. */
typedef struct cublasContext* cublasHandle_t;
typedef struct cusolverDnContext* cusolverDnHandle_t;
typedef struct cublasLtContext* cublasLtHandle_t;
typedef struct CUstream_st* cudaStream_t;

inline int precond_CG(double* A, double* x, double* b, int n, int r, double normA,
                      cublasHandle_t& cublasH, cusolverDnHandle_t& cusolverH,
                      cudaStream_t& stream, float eps_prime = 0.0f, float flr = 0.0f,
                      bool perturb_diag = false, int microscal_size = 32) {
  (void)cublasH;
  (void)cusolverH;
  return mpchol_precond_cg(A, x, b, n, r, normA, eps_prime, flr, perturb_diag ? 1 : 0,
                           microscal_size, MPCHOL_REFCOMPAT_REL_TOL, MPCHOL_REFCOMPAT_MAX_IT,
                           stream);
}

/* The reference's switching_chol returns nothing, so a failure (a
 * non-positive pivot, a bad argument) cannot reach its caller through the
 * signature.  The shim keeps the mpchol_status of the calling thread's last
 * switching_chol here; a caller that wants it reads it after the call. */
inline int& mpchol_refcompat_status_slot() {
  static thread_local int status = 0;
  return status;
}
inline int mpchol_refcompat_last_status() { return mpchol_refcompat_status_slot(); }

inline void switching_chol(float* d_A, int n, int b, float* d_diagVals, float* updated_diag,
                           float eps_prime, bool perturb_diag, int microscal_size,
                           cusolverDnHandle_t cusolverH, cublasLtHandle_t cublasltH,
                           cublasHandle_t cublasH, cudaStream_t stream, uint8_t* scales) {
  (void)cusolverH;
  (void)cublasltH;
  (void)cublasH;
  mpchol_refcompat_status_slot() =
      mpchol_switching_chol(d_A, n, b, d_diagVals, updated_diag, eps_prime,
                            perturb_diag ? 1 : 0, microscal_size, stream, scales);
}
#endif /* __cplusplus */

#endif /* MPCHOL_REFCOMPAT_H_ */
