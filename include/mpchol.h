/*
 * mpchol -- mixed-precision blocked Cholesky preconditioner + FP64-checked PCG
 * for NVIDIA B200 (sm_100a).  Plain C ABI: no C++ or torch types cross it.
 *
 * Conventions
 *   - Matrices are column-major, lower triangle significant (as in the
 *     reference, src/micro_chol.hpp:18-20, src/sChol.cuh:278-279).
 *   - All pointers named d* are device pointers; h* are host pointers.
 *   - Every call is ordered on the caller's stream; the library never
 *     synchronizes the device except where a call is documented to return a
 *     host-visible result (reports, info), and then only that stream.
 *   - Errors are status codes.  The library never calls exit(), never destroys
 *     caller-owned handles or streams, and its kernels never trap.
 *   - Objects are re-entrant across different factor objects; one stream per
 *     object at a time.
 *
 * Reference interfaces replaced (paths inside SudhanvaKulkarni123/Cholesky_GPU):
 *   precond_CG      src/mixed_cholesky.cu:76-78   -> mpchol_precond_cg, mpchol_factor + mpchol_pcg
 *   switching_chol  src/switching_chol.cuh:19-22  -> mpchol_switching_chol, mpchol_factor
 *   solveWithCuSolver src/mixed_cholesky.cu:297   -> (oracle only; FP64 dense solve on CPU)
 *   convert_fp32_to_mxe4m3 / convertFloatToHalf  src/fp8_utils.cuh:27-130,
 *                   src/kernels_macros.cuh:115-124 -> mpchol_quantize*, fused in the factor
 */
#ifndef MPCHOL_H_
#define MPCHOL_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MPCHOL_API __attribute__((visibility("default")))
#else
#define MPCHOL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* mpchol_stream_t; /* == cudaStream_t */

typedef enum {
  MPCHOL_OK = 0,
  MPCHOL_ERR_BAD_ARG = 1,
  MPCHOL_ERR_NOT_SPD = 2,      /* non-positive pivot; see info.fail_row */
  MPCHOL_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  MPCHOL_ERR_ALLOC = 4,        /* device allocation failed */
  MPCHOL_PCG_MAXIT = 5,        /* PCG stopped at max_it without reaching rel_tol */
  MPCHOL_PCG_BREAKDOWN = 6,    /* p^T A p <= 0 or NaN, or rho NaN */
  MPCHOL_ERR_TIMEOUT = 7,      /* a bounded device-side wait ran out */
  MPCHOL_ERR_NOT_SUPPORTED = 8 /* option combination not built */
} mpchol_status;

/* Storage precision of a trailing update (and policy ids). */
typedef enum {
  MPCHOL_PREC_FP32 = 0,
  MPCHOL_PREC_FP16 = 1,
  MPCHOL_PREC_E4M3 = 2,   /* per-row power-of-two scaled E4M3 (RNE, satfinite) */
  MPCHOL_PREC_E5M2 = 3,   /* per-row power-of-two scaled E5M2 */
  MPCHOL_PREC_MXFP8 = 4,  /* OCP MX: E4M3 + E8M0 scale per 32 elements along K */
  MPCHOL_PREC_SWITCHING = 5, /* per-step choice by the switching criterion */
  MPCHOL_PREC_FP16X2 = 6,    /* two-term FP16 split (hi + lo, per-row scaled): FP32-class
                                accuracy on FP16 tensor cores */
  /* OCP MX with FP6 / FP4 elements (E8M0 scale per 32 elements along K,
   * scale 2^(floor(log2 amax) - emax_elem), round to nearest even, saturating,
   * no Inf/NaN codes).  The element values are exactly representable in E4M3
   * and are stored and multiplied as E4M3 codes by the block-scaled MMA, so
   * the products are those of FP6/FP4 operands with FP8 storage and speed.
   * A switching ladder holds at most one MX format (MXFP8 or one of these). */
  MPCHOL_PREC_MXFP6_E2M3 = 7,   /* u = 2^-4, largest element 7.5 */
  MPCHOL_PREC_MXFP6_E3M2 = 8,   /* u = 2^-3, largest element 28 */
  MPCHOL_PREC_MXFP4 = 9         /* E2M1, u = 2^-2, largest element 6 */
} mpchol_precision;

/* Factorization options.  Field names follow the reference's settings.json
 * "factorization_settings" keys (src/settings.json:7-12) where one exists. */
typedef struct {
  int block_size;      /* b: diagonal block / panel width (64..256, multiple of 32) */
  int precision;       /* mpchol_precision policy */
  float eps_prime;     /* switching threshold eps' */
  float floor;         /* rows with dtilde_i <= floor * d_i flag their diagonal block for FP64 POTRF */
  int diag_pert;       /* 1: shift pivots by pert * (accumulated rounding estimate) and floor them */
  float pert;          /* shift multiplier (diag_pert) */
  float pivot_floor;   /* diag_pert: pivots <= pivot_floor * d_i are raised to pivot_floor * d_i */
  int switch_mode;     /* 0: build criterion (lowest ladder precision with u_p*max(d/dtilde) <= eps');
                          1: reference-literal can_switch comparison (src/kernels_macros.cuh:191-211) */
  int ladder_len;      /* switching ladder, lowest precision first (default {E4M3, FP16, FP32});
                          a step no entry qualifies for takes the last (most precise) entry */
  int ladder[4];
  int left;            /* settings.json "left".  0: right-looking with a one-block look-ahead.
                          1: left-looking -- block column k receives the updates of panels
                          0..k-1 (kept quantized, about 7 n b bytes per step) just before it is
                          factored; the factor is identical bit for bit, the schedule has no
                          look-ahead and one launch per (panel, block column) pair.  Batches:
                          0 only. */
  int coherence;       /* switch_mode 0 only.  1 (default): a ladder entry p must also satisfy
                          u_p * ||P^T 1||^2 / m <= eps' * min_i dtilde_i, where P is the step's
                          m x b panel: a panel whose columns share one sign pattern across the
                          trailing rows (the constant mode of a kernel matrix) turns rounding
                          errors into a coherent rank-2 perturbation of norm ~u_p ||P^T 1||^2/m,
                          which the per-row ratio test cannot see.  0: ratio test only. */
  int equilibrate;     /* 1: factor D A D with D = diag(2^-e_i), e_i = floor((floor(log2 a_ii)
                          + 1) / 2) clamped to [-63, 63] (0 for a non-positive a_ii), so the
                          scaled diagonal lies in [0.5, 2); when the factorization ends L's rows
                          are scaled back by 2^e_i (exact), so L L^T still approximates A and
                          the solves are unchanged.  mpchol_factor_diags then returns the scaled
                          diagonals.  The diagonal equilibration intent of
                          src/kernels_macros.cuh:137-158.  0 (default): off. */
  float eps_coherence; /* threshold of the coherence test (coherence = 1): a ladder entry p
                          needs u_p * ||P^T 1||^2 / (m min_i dtilde_i) <= eps_coherence;
                          0 (default) uses eps_prime.  A small value keeps the large, coherent
                          updates of the first steps in the higher precisions and gives the
                          later, smaller ones to FP8, which costs fewer PCG iterations than
                          the same number of early FP8 steps. */
} mpchol_opts;

/* Per-factor results, filled by mpchol_factor_info (synchronizes the stream). */
typedef struct {
  int status;          /* mpchol_status of the factorization */
  int fail_row;        /* NOT_SPD: global row of the failed pivot */
  int n_perturbed;     /* pivots raised by diag_pert */
  int nsteps;          /* ceil(n / b) */
  int n_fp64_blocks;   /* diagonal blocks factored in FP64 */
  int steps_by_prec[10];/* number of trailing updates done in each mpchol_precision */
} mpchol_factor_info;

typedef struct {
  double rel_tol;      /* stop when the FP64 true residual ||b-Ax||/||b|| <= rel_tol (every rhs) */
  int max_it;          /* iteration cap (the reference uses 200, src/mixed_cholesky.cu:82) */
  int x0_precond;      /* 1: x0 = M^-1 b as the reference (src/mixed_cholesky.cu:145-149); 0: x0 = 0 */
  int check_every;     /* iterations between host convergence checks (>= 1) when
                          the iterations are launched directly (see mpchol_pcg) */
} mpchol_pcg_opts;

typedef struct {
  int iterations;          /* PCG iterations taken */
  int converged;           /* 1 if every rhs met rel_tol on the true residual */
  double rel_residual;     /* max over rhs of ||b - A x|| / ||b||, FP64, recomputed from x */
  double backward_error;   /* max over rhs of ||b - A x|| / (||A||_F ||x|| + ||b||) */
  double precond_residual; /* max over rhs of sqrt(r^T z)/||b|| (the reference's stopping quantity) */
} mpchol_report;

typedef struct mpchol_factor mpchol_factor_t;

/* Phases of the per-phase event timers (mpchol_profile_*). */
enum {
  MPCHOL_PH_POTRF = 0,     /* diagonal-block Cholesky */
  MPCHOL_PH_TRSM = 1,      /* panel solve + Schur-diagonal / switching statistics */
  MPCHOL_PH_QUANT = 2,     /* precision decision + panel quantization */
  MPCHOL_PH_SYRK_F32 = 3,  /* FP32 trailing update */
  MPCHOL_PH_SYRK_TC = 4,   /* tensor-core trailing update */
  MPCHOL_PH_SYMV = 5,      /* PCG operator A p */
  MPCHOL_PH_TRSV = 6,      /* PCG preconditioner triangular solves */
  MPCHOL_PH_PCG_VEC = 7,   /* PCG FP64 dots / updates */
  MPCHOL_PH_SETUP = 8,     /* diagonal extraction, solve-side setup */
  MPCHOL_PH_TEST = 9,      /* kernel-level test entry points */
  MPCHOL_NPHASES = 10
};

typedef struct {
  double ms[MPCHOL_NPHASES];          /* summed event time per phase */
  long long calls[MPCHOL_NPHASES];    /* timed calls per phase */
  long long launches[MPCHOL_NPHASES]; /* kernels launched per phase since load (all calls) */
} mpchol_profile;

/* ---- status / defaults ------------------------------------------------- */
MPCHOL_API const char* mpchol_status_str(int status);
MPCHOL_API void mpchol_opts_default(mpchol_opts* opts);
MPCHOL_API void mpchol_pcg_opts_default(mpchol_pcg_opts* opts);
/* Per-phase CUDA-event timers (the reference's phase timers,
 * src/hChol.cuh:22-31, src/sChol.cuh:150-154).  While enabled, every kernel
 * group the library launches is bracketed by events on its stream;
 * mpchol_profile_read waits for those events and sums them per phase. */
MPCHOL_API void mpchol_profile_enable(int on);
MPCHOL_API mpchol_status mpchol_profile_read(mpchol_profile* out, int reset);
/* Total number of kernels the library has launched in this process. */
MPCHOL_API long long mpchol_kernel_launches(void);
/* Last CUDA error text recorded by the library in this process ("" if none). */
MPCHOL_API const char* mpchol_last_error(void);

/* ---- factorization (switching_chol, src/switching_chol.cuh:19-227) ---- */
/* Allocate a factor object (device workspace for order n). */
MPCHOL_API mpchol_status mpchol_factor_create(const mpchol_opts* opts, int n, mpchol_factor_t** out);
/* Copy the lower triangle of dA (n x n, lda >= n) into the object and factor
 * it on `stream`.  Asynchronous: failures inside kernels are reported by
 * mpchol_factor_info.  The second and later calls on one object run the
 * factorization as a CUDA graph the object captures (on a private stream) and
 * keeps; the first launches the kernels directly.  The factor is the same
 * either way. */
MPCHOL_API mpchol_status mpchol_factor_compute(mpchol_factor_t* f, const float* dA, int lda, mpchol_stream_t stream);
/* create + compute. */
MPCHOL_API mpchol_status mpchol_factor(const mpchol_opts* opts, int n, const float* dA, int lda,
                            mpchol_factor_t** out, mpchol_stream_t stream);
MPCHOL_API mpchol_status mpchol_factor_destroy(mpchol_factor_t* f);
/* Synchronizes `stream`; fills info; hStepPrec (nullable, length nsteps)
 * receives each step's trailing-update precision, hStepFp64 (nullable) the
 * FP64-diagonal flags. */
MPCHOL_API mpchol_status mpchol_factor_info_get(const mpchol_factor_t* f, mpchol_factor_info* info,
                                     int* hStepPrec, int* hStepFp64, mpchol_stream_t stream);
/* Device pointer to the factor L (lower triangle valid; upper unspecified). */
MPCHOL_API mpchol_status mpchol_factor_lower(const mpchol_factor_t* f, const float** dL, int* ldl, int* n);
/* ---- factor serialization (reuse without refactoring) ------------------ */
/* A computed factor as a host byte blob: a 64-byte header (magic "MPCHOLF1",
 * version 1, n, block size, step count, payload sizes, a 64-bit checksum of
 * the payload), then L's lower block columns packed (each block column from
 * its diagonal down, column by column, FP32), the per-step states (chosen
 * precision, FP64-diagonal flag, switching statistics), the diagonals d and
 * d-tilde, and the status word (perturbed pivots, failure).  The panel codes
 * are not saved: PCG needs only L.  The blob is for the same library build
 * and byte order.
 * mpchol_factor_save: *size receives the blob size; blob == NULL only
 * queries it; cap < size is MPCHOL_ERR_BAD_ARG.  Synchronizes `stream`
 * (the factor must have been computed on it or before it).  A factor whose
 * factorization failed is not saved: save returns its status (NOT_SPD,
 * TIMEOUT) and writes nothing.
 * mpchol_factor_load: replaces the factor of f (same n and block size as the
 * blob, else MPCHOL_ERR_BAD_ARG) and its solve-side data is rebuilt on the
 * next solve; synchronizes `stream`.  A blob whose saved status is not OK
 * is loaded and its status returned, so the caller learns the factor is
 * unusable (the solves refuse it too).
 * mpchol_factor_blob_check: host-only validation of a blob (magic, version,
 * sizes, n <= MPCHOL_BLOB_MAX_N, checksum); writes n and the block size.
 * No counterpart in the reference, which refactors for every solve. */
#define MPCHOL_BLOB_MAX_N (1 << 24)
MPCHOL_API mpchol_status mpchol_factor_save(const mpchol_factor_t* f, void* blob, size_t cap,
                                            size_t* size, mpchol_stream_t stream);
MPCHOL_API mpchol_status mpchol_factor_load(mpchol_factor_t* f, const void* blob, size_t size,
                                            mpchol_stream_t stream);
MPCHOL_API mpchol_status mpchol_factor_blob_check(const void* blob, size_t size, int* n,
                                                  int* block_size);
/* Inspection of the last trailing update's quantized panel (the codes the
 * panel solve of the factorization's last step wrote for format fmt, one of
 * the step's candidates): dCodes, K-major, *rows rows of *ldq codes (FP16X2:
 * the hi rows, then the lo rows), and dScales (per-row pow-2 exponents, int8,
 * or for MXFP8 *ldq/32 E8M0 bytes per row).  The panel holds L's rows
 * [*col0 + ldq, n) of columns [*col0, *col0 + ldq).  No counterpart in the
 * reference: it lets tests check the fused quantization against the oracle. */
MPCHOL_API mpchol_status mpchol_factor_codes(const mpchol_factor_t* f, int fmt, const void** dCodes,
                                             const void** dScales, int* ldq, int* rows, int* col0);
/* Device pointers to the tracked diagonals d (original) and dtilde (Schur). */
MPCHOL_API mpchol_status mpchol_factor_diags(const mpchol_factor_t* f, const float** dD, const float** dDtilde);
/* Prepare the solve-side data (diagonal-block inverses).  Called implicitly
 * by the first mpchol_pcg / mpchol_apply_precond. */
MPCHOL_API mpchol_status mpchol_factor_prepare_solve(mpchol_factor_t* f, mpchol_stream_t stream);

/* ---- PCG (precond_CG, src/mixed_cholesky.cu:76-229) ---------------------- */
/* Solve A X = B for nrhs (1..8) right-hand sides with M = L L^T.  dA is the
 * FP32 operator (full symmetric storage), dB/dX are n x nrhs FP64 (ld = n).
 * The iterations run in a device-side loop (a CUDA graph the object keeps)
 * that stops when the recursive residual meets the tolerance or max_it is
 * reached; `stream` is synchronized after each such loop and the answer is
 * re-checked on the true residual (restarting from it if needed).  When the
 * runtime refuses the graph, or profiling is on, iterations are launched
 * directly and `stream` is synchronized every check_every iterations.
 * report may be NULL.  A factor whose factorization failed (NOT_SPD,
 * TIMEOUT) is not used: the solve returns the factor's status without
 * iterating.  The solve has a device status word of its own (breakdown,
 * timeouts), so mpchol_factor_info_get reports the factorization's status,
 * failing row and perturbed-pivot count before and after any solve. */
MPCHOL_API mpchol_status mpchol_pcg(mpchol_factor_t* f, const float* dA, int lda, const double* dB,
                         double* dX, int nrhs, const mpchol_pcg_opts* opts, mpchol_report* report,
                         mpchol_stream_t stream);
/* Same with an FP64 operator (the reference's Dgemv on FP64 A). */
MPCHOL_API mpchol_status mpchol_pcg_f64(mpchol_factor_t* f, const double* dA, int lda, const double* dB,
                             double* dX, int nrhs, const mpchol_pcg_opts* opts,
                             mpchol_report* report, mpchol_stream_t stream);
/* Adjoint solve of a differentiable solve x = A^-1 b (A symmetric, the FP64
 * operator dA of the forward solve).  Given the forward solution dX and the
 * cotangent dG = dL/dx (both n x nrhs FP64, ld = n), solves A lambda = dG by
 * PCG preconditioned by the forward's factor f -- no refactoring -- and
 * writes dLam = lambda, which is dL/db.  The matrix cotangent is
 * dL/dA = -(lambda x^T + x lambda^T) / 2 summed over the rhs: its factors are
 * dLam and dX; dGradA (nullable; n x n FP64, ld = ldg >= n) receives it
 * densely, lower triangle only.  Returns like mpchol_pcg.  The backward pass
 * of a differentiable solve for callers outside Python (the torch wrapper
 * composes the same steps); no counterpart in the reference. */
MPCHOL_API mpchol_status mpchol_adjoint_solve(mpchol_factor_t* f, const double* dA, int lda,
                                              const double* dX, const double* dG, double* dLam,
                                              int nrhs, double* dGradA, int ldg,
                                              const mpchol_pcg_opts* opts, mpchol_report* report,
                                              mpchol_stream_t stream);
/* Factor and solve from host memory: the step precond_CG
 * (src/mixed_cholesky.cu:76-229) performs on device buffers, for a caller
 * whose matrix and right-hand sides are in host memory.  hA: FP32 symmetric,
 * column-major, leading dimension lda; only its lower triangle is read, and
 * only that part is copied to the device (the diagonal-down part of each
 * block column, about half of A, one 2-D copy per block column), once into an
 * operator buffer the factor object keeps and once, device to device, into
 * the factor's storage.  hB / hX: n x nrhs FP64 (ld = n), nrhs 1..8.
 * Page-locked host buffers let the copies run at full link speed.
 * When block_size is a multiple of 128 the copy overlaps the factorization:
 * the block columns cross the link in groups on a library stream, step 0
 * starts once the first group (and the diagonal of A, read on the host) is on
 * the device, and each later group joins the trailing updates after
 * receiving the earlier panels' updates in step order -- the factor is
 * identical bit for bit to the one computed after a full copy.  The groups
 * come from a timeline model of the copy and the factor steps
 * (mpchol_copy_plan) unless mpchol_set_copy_plan fixed them.  The first call
 * on a factor object allocates the operator and vector buffers (n x lda FP32,
 * 2 x n x 8 FP64), and with copy overlap the quantized panels of the steps
 * that late groups catch up with (about 7 n b bytes per step); later calls
 * allocate nothing.  Returns like mpchol_pcg; the stream is synchronized
 * before returning.  No counterpart in the reference (its precond_CG takes
 * device buffers). */
MPCHOL_API mpchol_status mpchol_solve_host(mpchol_factor_t* f, const float* hA, int lda,
                                           const double* hB, double* hX, int nrhs,
                                           const mpchol_pcg_opts* opts, mpchol_report* report,
                                           mpchol_stream_t stream);
/* Copy groups of mpchol_solve_host.  ngroups <= 0: the automatic plan;
 * ngroups == 1: copy all of A, then factor; ngroups 2..8: block columns
 * [0, cuts[0]), [cuts[0], cuts[1]), ..., group g >= 1 joining at step
 * join[g-1] (0 <= join[g-1] <= cuts[g-1] - 1, non-decreasing).  Needs
 * block_size % 128 == 0, equilibrate == 0 and left == 0 for ngroups > 1
 * (MPCHOL_ERR_NOT_SUPPORTED); an equilibrated or left-looking factor copies
 * all of A first. */
MPCHOL_API mpchol_status mpchol_set_copy_plan(mpchol_factor_t* f, int ngroups, const int* cuts,
                                              const int* join);
/* The automatic plan for order n and block_size: returns the number of
 * groups and writes up to cap cuts / join steps (host only, no device). */
MPCHOL_API int mpchol_copy_plan(int n, int block_size, int* cuts, int* join, int cap);
/* dZ = (L L^T)^-1 dR for nrhs vectors (n x nrhs, ld = n), i.e. Dpotrs
 * (src/mixed_cholesky.cu:204-206) on the FP32 factor with FP64 vectors. */
MPCHOL_API mpchol_status mpchol_apply_precond(mpchol_factor_t* f, const double* dR, double* dZ, int nrhs,
                                   mpchol_stream_t stream);
/* dY = A dX for symmetric FP32 A (lower triangle read), FP64 vectors,
 * nrhs columns (ld = n): the Dgemv of src/mixed_cholesky.cu:185-191. */
MPCHOL_API mpchol_status mpchol_symv(const float* dA, int lda, int n, const double* dX, double* dY, int nrhs,
                          mpchol_stream_t stream);

/* ---- reference-shaped entry points (used by include/mpchol_refcompat.h) -- */
/* precond_CG semantics: dA FP64 n x n (device, ld = n), dX written, dB read,
 * block size r.  Returns 0 if converged, -1 if not, > 0 if the
 * preconditioner failed (the reference's convention, src/mixed_cholesky.cu:149,225),
 * and -(100 + status) for library errors.  normA is accepted and unused, as
 * in the reference.  Convergence uses the FP64 true residual with tolerance
 * rel_tol (the reference's rel_tol = 0 means "run max_it iterations"). */
MPCHOL_API int mpchol_precond_cg(double* dA, double* dX, double* dB, int n, int r, double normA,
                      float eps_prime, float flr, int perturb_diag, int microscal_size,
                      double rel_tol, int max_it, mpchol_stream_t stream);
/* switching_chol semantics: in-place factor of the FP32 matrix dA (ld = n)
 * with block b; d_diagVals (n) receives the original diagonal and
 * updated_diag (n) the Schur-complement diagonal tracker (the reference's
 * caller fills both, src/mixed_cholesky.cu:128-131; here the library fills
 * them).  scales (nullable) receives the last MX step's E8M0 codes.
 * Returns an mpchol_status (the reference returns void). */
MPCHOL_API int mpchol_switching_chol(float* dA, int n, int b, float* d_diagVals, float* updated_diag,
                          float eps_prime, int perturb_diag, int microscal_size,
                          mpchol_stream_t stream, uint8_t* scales);

/* ---- quantizers (bit-exact vs lo_float ConvertFrom<kSaturate=true>) ----- */
/* Elementwise FP32 -> fmt (E4M3/E5M2: 1 byte, FP16: 2 bytes) with RNE +
 * satfinite, no scaling. */
MPCHOL_API mpchol_status mpchol_quantize(const float* dX, void* dQ, long long count, int fmt,
                              mpchol_stream_t stream);
/* Panel quantization as done inside the factor: dP is m x k column-major
 * (ld = ldp); dQ receives a row-major (K-major) m x k copy in fmt (FP16X2:
 * the m x k hi panel followed by the m x k lo panel); dScale
 * receives per-row int8 exponents (E4M3/E5M2/FP16, scale = 2^e, m bytes) or
 * per-32-block E8M0 codes (MXFP8, m x ceil(k/32) bytes, row-major). */
MPCHOL_API mpchol_status mpchol_quantize_rows(const float* dP, int m, int k, int ldp, int fmt, void* dQ,
                                   void* dScale, mpchol_stream_t stream);
/* Exhaustive-sweep helper: converts the raw bit patterns [first, first+count)
 * and folds each chunk of `chunk` codes into one 64-bit hash (non-finite
 * inputs folded as class tokens), dHash receives ceil(count/chunk) words. */
MPCHOL_API mpchol_status mpchol_quantize_hash(unsigned long long first, unsigned long long count,
                                   unsigned long long chunk, int fmt, unsigned long long* dHash,
                                   mpchol_stream_t stream);

/* ---- kernel-level entry points (tests and micro-benchmarks) ------------- */
/* Trailing update C -= s_i s_j (Q Q^T) on the lower triangle of the m x m
 * block dC (ld = ldc) from a quantized panel produced by
 * mpchol_quantize_rows (fmt) or, for FP32, from the column-major panel dP. */
MPCHOL_API mpchol_status mpchol_syrk_update(float* dC, int ldc, int m, int k, int fmt, const void* dQ,
                                 const void* dScale, const float* dP, int ldp,
                                 mpchol_stream_t stream);

/* ---- batches of independent systems of uneven size --------------------- */
/* No counterpart in the reference (one system per precond_CG call).  All
 * systems share the options (a fixed tensor-core precision: FP16, E4M3,
 * E5M2, MXFP8 or FP16X2; not FP32 or SWITCHING; no equilibration) and the
 * rhs count; every
 * kernel launch serves all of them.  ns[i] is the order of system i; arrays
 * passed to the calls below are indexed in that same (caller) order and hold
 * device pointers.  Matrices are FP32 column-major (ld lda[i]) with the lower
 * triangle read; B and X are n_i x nrhs FP64 column-major (ld n_i).
 *   mpchol_batch_factor: one CUDA graph launch factors every system (and
 *     forms the solve data); blocks the host until it has read the pointer
 *     tables.
 *   mpchol_batch_pcg: PCG of every system in lockstep (converged ones skip),
 *     FP64 true residual per system; reports[i] per system (may be NULL).
 *     Returns OK if every system converged, PCG_MAXIT otherwise. */
typedef struct mpchol_batch mpchol_batch_t;
MPCHOL_API mpchol_status mpchol_batch_create(const mpchol_opts* opts, int count, const int* ns,
                                             int nrhs, mpchol_batch_t** out);
MPCHOL_API mpchol_status mpchol_batch_factor(mpchol_batch_t* b, const float* const* dA,
                                             const int* lda, mpchol_stream_t stream);
/* the factor of system `index` (caller order): device pointer, ld, n */
MPCHOL_API mpchol_status mpchol_batch_lower(const mpchol_batch_t* b, int index, const float** dL,
                                            int* ldl, int* n);
/* per-system factor status (mpchol_status), failing row and floored-pivot count */
MPCHOL_API mpchol_status mpchol_batch_info(mpchol_batch_t* b, int* status, int* fail_row,
                                           int* n_perturbed, mpchol_stream_t stream);
MPCHOL_API mpchol_status mpchol_batch_pcg(mpchol_batch_t* b, const float* const* dA,
                                          const int* lda, const double* const* dB,
                                          double* const* dX, const mpchol_pcg_opts* opts,
                                          mpchol_report* reports, mpchol_stream_t stream);
MPCHOL_API mpchol_status mpchol_batch_destroy(mpchol_batch_t* b);

/* ---- Gaussian RBF kernel matrices (no reference arithmetic: src/RBF.cu is a stub)
 * dX: n points x d features, row-major FP32 (ld = ldx).  Writes
 *   K_ij = exp(-||x_i - x_j||^2 / (2 lengthscale^2)) + nugget * delta_ij
 * computed in FP64 from coordinate differences, column-major (ld = ldk) into
 * dK64 (FP64) and/or dK32 (FP32); either may be NULL.  lower_only = 1 writes
 * the lower triangle only (all the factor and the PCG operator read). */
MPCHOL_API mpchol_status mpchol_rbf_build(const float* dX, int n, int d, int ldx, double lengthscale,
                                          double nugget, double* dK64, float* dK32, int ldk,
                                          int lower_only, mpchol_stream_t stream);
/* Gradient contraction for a solve x = K^-1 y with adjoint a = K^-1 (dL/dx):
 * recomputes the K tiles from dX (FP64) and writes
 *   dP (n x (2 + 2d), column-major, ld = n) = K_rbf [a, b, a*X, b*X]
 *   dS (1 double) = sum_ij a_i b_j K_ij ||x_i - x_j||^2
 * (K_rbf without the nugget; b = x).  d <= 128.  dWork: at least
 * mpchol_rbf_grad_work_elems(n) doubles of caller scratch.  The gradients
 * follow: dL/dnugget = -a.b, dL/dlengthscale = -S / l^3, dL/dy = a,
 * dL/dX_i = (X_i (a_i P_i1 + b_i P_i0) - a_i P_i(b*X) - b_i P_i(a*X)) / l^2. */
MPCHOL_API int mpchol_rbf_grad_work_elems(int n);
MPCHOL_API mpchol_status mpchol_rbf_grad(const float* dX, int n, int d, int ldx, double lengthscale,
                                         const double* dA, const double* dB, double* dP, double* dS,
                                         double* dWork, mpchol_stream_t stream);

/* ---- allocation-free diagonal-block POTRF ------------------------------- */
/* No counterpart in the reference (its diagonal factor is cusolverDnSpotrf on
 * a workspace the caller allocates, src/switching_chol.cuh:86-95).
 * Factors the n x n block dA (column-major, ld = lda, lower triangle, FP32)
 * in place with the factorization's diagonal-block kernel and allocates
 * nothing: no cudaMalloc/cudaFree, no allocating library call.  For callers
 * that cannot allocate at the point of the call: cudaMalloc/cudaFree
 * synchronize the device (stalling every other stream), and a process whose
 * device memory is held by a caching allocator may have none to give.
 *   n <= MPCHOL_POTRF_STATIC_MAX (larger n: MPCHOL_ERR_BAD_ARG, nothing runs);
 *   dA 16-byte aligned and lda a multiple of 4 (TMA); lda >= n.
 *   pivot_floor > 0: pivots <= pivot_floor * A(i,i) are raised to that value
 *   (max(|pivot|, floor) repair); pivot_floor = 0: no repair.
 *   dInfo (device int): 0 on success, i + 1 if pivot i was not positive
 *   (pivot_floor = 0), -1 for another device-side error; written on `stream`.
 * Scratch is one static device array per device: calls that overlap in time
 * on one device race on it (order them on one stream).  The first call on
 * each device does one-time setup (symbol lookup); make it before any stream
 * capture. */
#define MPCHOL_POTRF_STATIC_MAX 256
MPCHOL_API mpchol_status mpchol_potrf_static(float* dA, int lda, int n, float pivot_floor,
                                             int* dInfo, mpchol_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MPCHOL_H_ */
