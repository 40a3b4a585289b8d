// Launchers of the PCG kernels (pcg.cu).
#pragma once
#include "common.cuh"

namespace mpchol {

int pcg_padded_nrhs(int nrhs);   // 1, 2, 4 or 8
int pcg_vgrid();                 // CTAs of the reduction kernels (partials per vector)

// ---- operator and preconditioner (solve.cu) ----
cudaError_t solve_init_attributes();
int solve_super_rows();
size_t solve_wsup_elems(int n);
int solve_setup_launches(int n);
template <typename TA>
cudaError_t launch_symv_skip(const TA* A, int lda, int n, const double* x, double* y, int nrhs,
                             const int* skip, cudaStream_t stream, double* fro = nullptr,
                             int nfro = 0);
// True when launch_symv_skip streams A through the staged kernel (FP32, 16-byte
// aligned columns); only then does it fill `fro` (per-CTA shares of ||A||_F^2).
template <typename TA>
bool symv_staged_ok(const TA* A, int lda);
// 128-block inverses into winv, then the super-block inverses into wsup.
cudaError_t launch_solve_setup(const float* L, int ldl, int n, float* wsup, cudaStream_t stream);
// out = L^-1 in (forward) or L^-T in (backward) through the super-block
// inverses wsup: one launch that prepares work <- in, out <- 0 and clears the
// counters, then one persistent cooperative launch; work is an n x nrhs
// scratch, counters trsv_counter_ints(n) ints.
size_t trsv_counter_ints(int n);
cudaError_t launch_trsv_persistent(bool backward, const float* L, int ldl, int n,
                                   const float* wsup, const double* in, double* out,
                                   double* work, int nrhs, int* counters, const int* skip,
                                   DevStatus* st, cudaStream_t stream);
cudaError_t launch_dot(const double* a, const double* b, int n, int nrhs, double* partials,
                       const int* skip, cudaStream_t stream);
cudaError_t launch_update_xr(double* x, double* r, const double* p, const double* Ap, int n,
                             int nrhs, const double* pAp_partials, const double* rho,
                             double* alpha_out, double* rr_partials, const int* skip,
                             DevStatus* st, cudaStream_t stream);
cudaError_t launch_update_p(double* p, const double* z, int n, int nrhs, const double* rz_partials,
                            const double* rho_old, double* rho_out, const double* rr_partials,
                            const double* bnorm2, double tol2, int* done, const int* skip,
                            int* iters, cudaStream_t stream);
cudaError_t launch_reduce_partials(const double* partials, double* out, int nrhs,
                                   cudaStream_t stream);
cudaError_t launch_residual(const double* b, const double* y, double* r, int n, int nrhs,
                            double* rr_partials, cudaStream_t stream);
cudaError_t launch_copy(const double* a, double* b, int n, int nrhs, cudaStream_t stream);
// Device-side PCG loop (a WHILE node of a CUDA graph): ctl[0] <- 0,
// ctl[1] <- max_iters before the loop; after each iteration the condition
// kernel copies rho[8..8+nr) to rho[0..nr) and sets the loop condition
// (continue while ctl[0] < ctl[1], *done == 0 and no recorded error).
cudaError_t launch_pcg_loop_init(int* ctl, int max_iters, cudaStream_t stream);
cudaError_t launch_pcg_loop_cond(cudaGraphConditionalHandle handle, int* ctl, const int* done,
                                 const DevStatus* st, double* rho, int nr, cudaStream_t stream);

// misc device utilities (util.cu)
cudaError_t launch_extract_diag(const float* A, int lda, int n, float* d, float* dtilde,
                                cudaStream_t stream);
cudaError_t launch_f64_to_f32(const double* src, int lds, float* dst, int ldd, int n,
                              cudaStream_t stream);
// Equilibration: ex[i] = exponent of row i from A's diagonal; then the lower
// triangle of columns [c0, c1) is scaled to D A D
// (unscale_rows = false) or the factor's rows scaled back by 2^ex[i] (true).
cudaError_t launch_equil_exps(const float* A, int lda, int n, int8_t* ex, cudaStream_t stream);
cudaError_t launch_equil_scale(float* A, int lda, int n, const int8_t* ex, int c0, int c1,
                               bool unscale_rows, cudaStream_t stream);
// G = -(Lam X^T + X Lam^T) / 2, lower triangle (n x nrhs column-major inputs).
cudaError_t launch_sym_outer(const double* lam, const double* x, int n, int nrhs, double* G,
                             int ldg, cudaStream_t stream);
template <typename TA>
cudaError_t launch_frob_lower(const TA* A, int lda, int n, double* partials, cudaStream_t stream);
cudaError_t launch_pad_columns(const double* src, int n, int ncols, double* dst, int ncols_pad,
                               cudaStream_t stream);

// RBF kernel matrix (FP64 arithmetic) and its gradient contraction.
int rbf_grad_max_features();
int rbf_grad_work_elems(int n);
cudaError_t launch_rbf_build(const float* X, int n, int d, int ldx, double lengthscale,
                             double nugget, double* K64, float* K32, int ldk, int lower_only,
                             cudaStream_t stream);
cudaError_t launch_rbf_grad(const float* X, int n, int d, int ldx, double lengthscale,
                            const double* a, const double* b, double* P, double* s, double* work,
                            cudaStream_t stream);

// ---- batched solve side (solve.cu, pcg.cu): every launch serves all systems
struct BatchSys;
cudaError_t launch_vec_slot_batched(const BatchSys* sys, int nsys, int src, int dst, int nr,
                                    int use_skip, cudaStream_t stream);
cudaError_t launch_symv_batched(const BatchSys* sys, int nsys, int ntiles, int xslot, int yslot,
                                int nr, int use_skip, cudaStream_t stream);
cudaError_t launch_solve_setup_batched(const BatchSys* sys, int nsys, int max_n,
                                       cudaStream_t stream);
cudaError_t launch_trsv_batched(bool backward, const BatchSys* sys, int nsys, int max_n,
                                int in_slot, int out_slot, int work_slot, int nr, int use_skip,
                                cudaStream_t stream);

cudaError_t launch_dot_batched(const BatchSys* sys, int nsys, int aslot, int bslot, int group,
                               int nr, int use_skip, cudaStream_t stream);
cudaError_t launch_update_xr_batched(const BatchSys* sys, int nsys, int cur, int nr,
                                     cudaStream_t stream);
cudaError_t launch_update_p_batched(const BatchSys* sys, int nsys, int cur, int nrhs, int nr,
                                    double tol2, cudaStream_t stream);
cudaError_t launch_reduce_batched(const BatchSys* sys, int nsys, int group, int off, int nr,
                                  int use_skip, cudaStream_t stream);
cudaError_t launch_residual_batched(const BatchSys* sys, int nsys, int nr, cudaStream_t stream);
cudaError_t launch_check_true_batched(const BatchSys* sys, int nsys, int nrhs, double tol2,
                                      cudaStream_t stream);
cudaError_t launch_count_open(const BatchSys* sys, int nsys, int* out, cudaStream_t stream);
cudaError_t launch_load_rhs_batched(const BatchSys* sys, int nsys, const double* const* B, int nrhs,
                                    int nr, cudaStream_t stream);
cudaError_t launch_store_x_batched(const BatchSys* sys, int nsys, double* const* X, int nrhs,
                                   int nr, cudaStream_t stream);
cudaError_t launch_frob_batched(const BatchSys* sys, int nsys, cudaStream_t stream);

}  // namespace mpchol
