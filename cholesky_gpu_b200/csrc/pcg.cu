// PCG FP64 recurrences with device-resident scalars.
//
// Replaces the reference's Ddot/Daxpy/Dscal/Dcopy/Dnrm2 calls in host pointer
// mode (two host syncs per iteration, src/mixed_cholesky.cu:171-216) with
// reduction and update kernels whose alpha, beta and rho never leave the
// device -- the intent of the reference's unused computeAlphaKernel /
// x_r_update / update_search_dir (src/kernels_macros.cuh:547-550,599-632).
// Reductions use a fixed grid and a fixed summation order (deterministic).
// All vectors are n x nrhs, column-major, ld = n, nrhs <= 8.
#include "common.cuh"
#include "kernels.cuh"
#include "pcg.cuh"

namespace mpchol {
namespace {

constexpr int NTH = 256;     // 8 warps

// ---- FP64 vector kernels ----------------------------------------------------
constexpr int VG = 296;   // fixed grid for reductions (2 x 148 SMs): deterministic order

template <int NR>
__device__ __forceinline__ void block_reduce_store(double (&v)[NR], double* partials) {
  __shared__ double s_red[NTH / 32][NR];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NR; ++k) s_red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < NR) {
    double s = 0.0;
    for (int w = 0; w < NTH / 32; ++w) s += s_red[w][threadIdx.x];
    partials[blockIdx.x * NR + threadIdx.x] = s;
  }
}

// Sum of the VG partials of each rhs, formed by the whole block with a fixed
// tree (two loads per thread, warp shuffles, then the eight warp sums in
// order), so every block -- and every launch -- gets the same bits.  Every
// thread of the block must call it; all receive the sums.
template <int NR>
__device__ __forceinline__ void sum_partials(const double* partials, double (&out)[NR]) {
  static_assert(VG <= 2 * NTH, "two partials per thread");
  __shared__ double s_w[NTH / 32][NR];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    double v = (t < VG) ? partials[t * NR + k] : 0.0;
    if (t + NTH < VG) v += partials[(t + NTH) * NR + k];
    v = warp_sum(v);
    if (lane == 0) s_w[warp][k] = v;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NTH / 32; ++w) s += s_w[w][k];
    out[k] = s;
  }
  __syncthreads();
}

template <int NR>
__global__ void __launch_bounds__(NTH)
dot_kernel(const double* __restrict__ a, const double* __restrict__ b, int n, double* partials,
           const int* skip) {
  if (skip != nullptr && *skip) return;
  double v[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = 0.0;
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += VG * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) v[k] = fma(a[(size_t)k * n + i], b[(size_t)k * n + i], v[k]);
  block_reduce_store<NR>(v, partials);
}

// alpha = rho / (p^T A p); x += alpha p; r -= alpha A p; partial ||r||^2.
// A right-hand side whose pAp or rho is zero (already converged exactly) or
// not finite takes alpha = 0; a negative pAp records PCG_BREAKDOWN.
template <int NR>
__global__ void __launch_bounds__(NTH)
update_xr_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                 const double* __restrict__ Ap, int n, const double* pAp_partials,
                 const double* rho, double* alpha_out, double* rr_partials, const int* skip,
                 DevStatus* st) {
  if (skip != nullptr && *skip) return;
  double pAp[NR], al[NR];
  sum_partials<NR>(pAp_partials, pAp);
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double a = rho[k] / pAp[k];
    al[k] = (pAp[k] != 0.0 && isfinite(a)) ? a : 0.0;
    if (!(pAp[k] >= 0.0) && threadIdx.x == 0 && blockIdx.x == 0) set_status(st, MPCHOL_PCG_BREAKDOWN, k);
  }
  if (blockIdx.x == 0 && threadIdx.x < NR) alpha_out[threadIdx.x] = al[threadIdx.x];
  double v[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = 0.0;
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += VG * NTH) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const size_t o = (size_t)k * n + i;
      x[o] = fma(al[k], p[o], x[o]);
      const double rn = fma(-al[k], Ap[o], r[o]);
      r[o] = rn;
      v[k] = fma(rn, rn, v[k]);
    }
  }
  block_reduce_store<NR>(v, rr_partials);
}

// rho_new = r^T z (from partials); beta = rho_new / rho_old; p = z + beta p.
// Writes rho_new to rho_out (a different buffer from rho_old) and, from the
// ||r||^2 partials, sets *done when every rhs has ||r|| <= tol * ||b||.
template <int NR>
__global__ void __launch_bounds__(NTH)
update_p_kernel(double* __restrict__ p, const double* __restrict__ z, int n,
                const double* rz_partials, const double* rho_old, double* rho_out,
                const double* rr_partials, const double* bnorm2, double tol2, int* done,
                const int* skip, int* iters) {
  if (skip != nullptr && *skip) return;
  double rz[NR], be[NR];
  sum_partials<NR>(rz_partials, rz);
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double b = rz[k] / rho_old[k];
    be[k] = (rho_old[k] != 0.0 && isfinite(b)) ? b : 0.0;
  }
  double rr[NR];
  sum_partials<NR>(rr_partials, rr);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int all = 1;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      rho_out[k] = rz[k];
      if (!(rr[k] <= tol2 * bnorm2[k])) all = 0;
    }
    *done = all;
    *iters += 1;
  }
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += VG * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const size_t o = (size_t)k * n + i;
      p[o] = fma(be[k], p[o], z[o]);
    }
}

// out = sum of partials (fixed order) for the first NR slots; used to form
// rho_0 = r_0^T z_0 and ||b||^2 on the device.
template <int NR>
__global__ void __launch_bounds__(NTH) reduce_partials_kernel(const double* partials, double* out) {
  double s[NR];
  sum_partials<NR>(partials, s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NR; ++k) out[k] = s[k];
}

// r = b - y (y = A x), partial ||r||^2
template <int NR>
__global__ void __launch_bounds__(NTH)
residual_kernel(const double* __restrict__ b, const double* __restrict__ y, double* __restrict__ r,
                int n, double* rr_partials) {
  double v[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = 0.0;
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += VG * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const size_t o = (size_t)k * n + i;
      const double rv = b[o] - y[o];
      r[o] = rv;
      v[k] = fma(rv, rv, v[k]);
    }
  block_reduce_store<NR>(v, rr_partials);
}

template <int NR>
__global__ void copy_kernel(const double* __restrict__ a, double* __restrict__ b, int n) {
  for (long long i = blockIdx.x * (long long)NTH + threadIdx.x; i < (long long)n * NR;
       i += (long long)VG * NTH)
    b[i] = a[i];
}

// ---- batched PCG (one launch for every system of a batch) ------------------
// grid (BATCH_VB, nsys): CTA (v, i) handles rows v*NTH + t, stride
// BATCH_VB*NTH, of system i.  Slots: 0 x, 1 r, 2 z, 3 p, 4 Ap, 5 b, 6 tmp,
// 7 work.  Partial groups: 0 pAp, 1 r^T r, 2 r^T z, 3 misc.  Scalars:
// rho[0] 0, rho[1] 8, alpha 16, ||b||^2 24, true ||r||^2 32, ||x||^2 40,
// ||A||_F^2 48, final r^T z 56.
namespace bslots { constexpr int X = 0, R = 1, Z = 2, P = 3, AP = 4, B = 5; }   // 6, 7: solve scratch

__device__ __forceinline__ double* bvec(const BatchSys& S, int slot, int nr) {
  return S.vec + (size_t)slot * S.n * nr;
}
__device__ __forceinline__ double* bpart(const BatchSys& S, int group) {
  return S.part + (size_t)group * BATCH_VB * 8;
}

template <int NR>
__device__ __forceinline__ void bsum(const double* part, double (&out)[NR]) {
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    double s = 0.0;
    for (int b = 0; b < BATCH_VB; ++b) s += part[b * NR + k];
    out[k] = s;
  }
}

template <int NR>
__device__ __forceinline__ void bstore(double (&v)[NR], double* part) {
  __shared__ double s_red[NTH / 32][NR];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NR; ++k) s_red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < NR) {
    double s = 0.0;
    for (int w = 0; w < NTH / 32; ++w) s += s_red[w][threadIdx.x];
    part[blockIdx.x * NR + threadIdx.x] = s;
  }
}

template <int NR>
__global__ void __launch_bounds__(NTH)
dot_batched_kernel(const BatchSys* __restrict__ sys, int aslot, int bslot_, int group, int use_skip) {
  const BatchSys& S = sys[blockIdx.y];
  if (use_skip && S.done[0]) return;
  const int n = S.n;
  const double* a = bvec(S, aslot, NR);
  const double* b = bvec(S, bslot_, NR);
  double v[NR] = {};
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += BATCH_VB * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) v[k] = fma(a[(size_t)k * n + i], b[(size_t)k * n + i], v[k]);
  bstore<NR>(v, bpart(S, group));
}

template <int NR>
__global__ void __launch_bounds__(NTH)
update_xr_batched_kernel(const BatchSys* __restrict__ sys, int cur) {
  const BatchSys& S = sys[blockIdx.y];
  if (S.done[0]) return;
  const int n = S.n;
  double pAp[NR], al[NR];
  bsum<NR>(bpart(S, 0), pAp);
  const double* rho = S.scal + 8 * cur;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double a = rho[k] / pAp[k];
    al[k] = (pAp[k] != 0.0 && isfinite(a)) ? a : 0.0;
    if (!(pAp[k] >= 0.0) && threadIdx.x == 0 && blockIdx.x == 0) set_status(S.st, MPCHOL_PCG_BREAKDOWN, k);
  }
  if (blockIdx.x == 0 && threadIdx.x < NR) S.scal[16 + threadIdx.x] = al[threadIdx.x];
  double* x = bvec(S, bslots::X, NR);
  double* r = bvec(S, bslots::R, NR);
  const double* p = bvec(S, bslots::P, NR);
  const double* Ap = bvec(S, bslots::AP, NR);
  double v[NR] = {};
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += BATCH_VB * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const size_t o = (size_t)k * n + i;
      x[o] = fma(al[k], p[o], x[o]);
      const double rn = fma(-al[k], Ap[o], r[o]);
      r[o] = rn;
      v[k] = fma(rn, rn, v[k]);
    }
  bstore<NR>(v, bpart(S, 1));
}

template <int NR>
__global__ void __launch_bounds__(NTH)
update_p_batched_kernel(const BatchSys* __restrict__ sys, int cur, int nrhs, double tol2) {
  const BatchSys& S = sys[blockIdx.y];
  if (S.done[0]) return;
  const int n = S.n;
  double rz[NR], be[NR], rr[NR];
  bsum<NR>(bpart(S, 2), rz);
  bsum<NR>(bpart(S, 1), rr);
  const double* rho_old = S.scal + 8 * cur;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double b = rz[k] / rho_old[k];
    be[k] = (rho_old[k] != 0.0 && isfinite(b)) ? b : 0.0;
  }
  // CTA 0 writes rho into the other buffer (no CTA of this launch reads it)
  // and the done flag; a CTA that already sees done = 1 skips the p update,
  // which no later iteration of a converged system reads
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int all = 1;
    for (int k = 0; k < NR; ++k) {
      S.scal[8 * (cur ^ 1) + k] = rz[k];
      if (k < nrhs && !(rr[k] <= tol2 * S.scal[24 + k])) all = 0;
    }
    S.done[1] += 1;
    S.done[0] = all;
  }
  double* p = bvec(S, bslots::P, NR);
  const double* z = bvec(S, bslots::Z, NR);
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += BATCH_VB * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const size_t o = (size_t)k * n + i;
      p[o] = fma(be[k], p[o], z[o]);
    }
}

// scal[off + k] = sum of the group's partials
template <int NR>
__global__ void reduce_batched_kernel(const BatchSys* __restrict__ sys, int group, int off,
                                      int use_skip) {
  const BatchSys& S = sys[blockIdx.y];
  if (use_skip && S.done[0]) return;
  if (threadIdx.x == 0) {
    double s[NR];
    bsum<NR>(bpart(S, group), s);
    for (int k = 0; k < NR; ++k) S.scal[off + k] = s[k];
  }
}

// r = b - Ap, partial ||r||^2 (group 1)
template <int NR>
__global__ void __launch_bounds__(NTH)
residual_batched_kernel(const BatchSys* __restrict__ sys) {
  const BatchSys& S = sys[blockIdx.y];
  const int n = S.n;
  const double* b = bvec(S, bslots::B, NR);
  const double* y = bvec(S, bslots::AP, NR);
  double* r = bvec(S, bslots::R, NR);
  double v[NR] = {};
  for (int i = blockIdx.x * NTH + threadIdx.x; i < n; i += BATCH_VB * NTH)
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const size_t o = (size_t)k * n + i;
      const double rv = b[o] - y[o];
      r[o] = rv;
      v[k] = fma(rv, rv, v[k]);
    }
  bstore<NR>(v, bpart(S, 1));
}

// done[0] = true residual of every rhs within tolerance (scal[32..] vs ||b||^2)
__global__ void check_true_batched_kernel(const BatchSys* __restrict__ sys, int nrhs, double tol2) {
  const BatchSys& S = sys[blockIdx.x];
  if (threadIdx.x != 0) return;
  int all = 1;
  for (int k = 0; k < nrhs; ++k)
    if (!(S.scal[32 + k] <= tol2 * S.scal[24 + k])) all = 0;
  S.done[0] = all;
}

__global__ void count_open_kernel(const BatchSys* __restrict__ sys, int nsys, int* out) {
  __shared__ int s_cnt;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < nsys; i += blockDim.x) c += (sys[i].done[0] == 0);
  atomicAdd(&s_cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = s_cnt;
}

// b slot <- the caller's B_i (n x nrhs, ld n), zero-padded to nr columns
__global__ void load_rhs_batched_kernel(const BatchSys* __restrict__ sys,
                                        const double* const* __restrict__ B, int nrhs, int nr) {
  const BatchSys& S = sys[blockIdx.y];
  const double* src = B[blockIdx.y];
  double* dst = bvec(S, bslots::B, nr);
  const long long cnt = (long long)S.n * nr;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cnt;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / S.n);
    dst[e] = k < nrhs ? src[e] : 0.0;
  }
}

// the caller's X_i (n x nrhs, ld n) <- x slot
__global__ void store_x_batched_kernel(const BatchSys* __restrict__ sys, double* const* __restrict__ X,
                                       int nrhs, int nr) {
  const BatchSys& S = sys[blockIdx.y];
  double* dst = X[blockIdx.y];
  const double* src = bvec(S, bslots::X, nr);
  const long long cnt = (long long)S.n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cnt;
       e += (long long)gridDim.x * blockDim.x)
    dst[e] = src[e];
}

// partial ||A||_F^2 of the operator's lower triangle (group 3, first column)
__global__ void __launch_bounds__(NTH)
frob_batched_kernel(const BatchSys* __restrict__ sys) {
  const BatchSys& S = sys[blockIdx.y];
  const int n = S.n;
  double v[1] = {0.0};
  // CTA x sums columns x, x + BATCH_VB, ... from the diagonal down
  for (int c = blockIdx.x; c < n; c += BATCH_VB) {
    const float* col = S.op + (size_t)c * S.op_ld;
    for (int r = c + threadIdx.x; r < n; r += NTH) {
      const double a = (double)col[r];
      v[0] += (r == c ? 1.0 : 2.0) * a * a;
    }
  }
  bstore<1>(v, bpart(S, 3));
}

}  // namespace

// ---- host launchers ---------------------------------------------------------
#define NR_DISPATCH(nrhs, CALL)            \
  switch (nrhs) {                          \
    case 1: { constexpr int NRC = 1; CALL; } break; \
    case 2: { constexpr int NRC = 2; CALL; } break; \
    case 4: { constexpr int NRC = 4; CALL; } break; \
    case 8: { constexpr int NRC = 8; CALL; } break; \
    default: return cudaErrorInvalidValue;          \
  }

int pcg_padded_nrhs(int nrhs) { return nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : 8; }
int pcg_vgrid() { return VG; }

cudaError_t launch_dot(const double* a, const double* b, int n, int nrhs, double* partials,
                       const int* skip, cudaStream_t stream) {
  NR_DISPATCH(nrhs, (dot_kernel<NRC><<<VG, NTH, 0, stream>>>(a, b, n, partials, skip)));
  return cudaGetLastError();
}

cudaError_t launch_update_xr(double* x, double* r, const double* p, const double* Ap, int n,
                             int nrhs, const double* pAp_partials, const double* rho,
                             double* alpha_out, double* rr_partials, const int* skip,
                             DevStatus* st, cudaStream_t stream) {
  NR_DISPATCH(nrhs, (update_xr_kernel<NRC><<<VG, NTH, 0, stream>>>(x, r, p, Ap, n, pAp_partials, rho, alpha_out, rr_partials, skip, st)));
  return cudaGetLastError();
}

cudaError_t launch_update_p(double* p, const double* z, int n, int nrhs, const double* rz_partials,
                            const double* rho_old, double* rho_out, const double* rr_partials,
                            const double* bnorm2, double tol2, int* done, const int* skip,
                            int* iters, cudaStream_t stream) {
  NR_DISPATCH(nrhs, (update_p_kernel<NRC><<<VG, NTH, 0, stream>>>(p, z, n, rz_partials, rho_old, rho_out, rr_partials, bnorm2, tol2, done, skip, iters)));
  return cudaGetLastError();
}

cudaError_t launch_reduce_partials(const double* partials, double* out, int nrhs,
                                   cudaStream_t stream) {
  NR_DISPATCH(nrhs, (reduce_partials_kernel<NRC><<<1, NTH, 0, stream>>>(partials, out)));
  return cudaGetLastError();
}

cudaError_t launch_residual(const double* b, const double* y, double* r, int n, int nrhs,
                            double* rr_partials, cudaStream_t stream) {
  NR_DISPATCH(nrhs, (residual_kernel<NRC><<<VG, NTH, 0, stream>>>(b, y, r, n, rr_partials)));
  return cudaGetLastError();
}

cudaError_t launch_copy(const double* a, double* b, int n, int nrhs, cudaStream_t stream) {
  NR_DISPATCH(nrhs, (copy_kernel<NRC><<<VG, NTH, 0, stream>>>(a, b, n)));
  return cudaGetLastError();
}

cudaError_t launch_dot_batched(const BatchSys* sys, int nsys, int aslot, int bslot, int group,
                               int nr, int use_skip, cudaStream_t stream) {
  NR_DISPATCH(nr, (dot_batched_kernel<NRC><<<dim3(BATCH_VB, nsys), NTH, 0, stream>>>(sys, aslot, bslot, group, use_skip)));
  return cudaGetLastError();
}
cudaError_t launch_update_xr_batched(const BatchSys* sys, int nsys, int cur, int nr,
                                     cudaStream_t stream) {
  NR_DISPATCH(nr, (update_xr_batched_kernel<NRC><<<dim3(BATCH_VB, nsys), NTH, 0, stream>>>(sys, cur)));
  return cudaGetLastError();
}
cudaError_t launch_update_p_batched(const BatchSys* sys, int nsys, int cur, int nrhs, int nr,
                                    double tol2, cudaStream_t stream) {
  NR_DISPATCH(nr, (update_p_batched_kernel<NRC><<<dim3(BATCH_VB, nsys), NTH, 0, stream>>>(sys, cur, nrhs, tol2)));
  return cudaGetLastError();
}
cudaError_t launch_reduce_batched(const BatchSys* sys, int nsys, int group, int off, int nr,
                                  int use_skip, cudaStream_t stream) {
  NR_DISPATCH(nr, (reduce_batched_kernel<NRC><<<dim3(1, nsys), 32, 0, stream>>>(sys, group, off, use_skip)));
  return cudaGetLastError();
}
cudaError_t launch_residual_batched(const BatchSys* sys, int nsys, int nr, cudaStream_t stream) {
  NR_DISPATCH(nr, (residual_batched_kernel<NRC><<<dim3(BATCH_VB, nsys), NTH, 0, stream>>>(sys)));
  return cudaGetLastError();
}
cudaError_t launch_check_true_batched(const BatchSys* sys, int nsys, int nrhs, double tol2,
                                      cudaStream_t stream) {
  check_true_batched_kernel<<<nsys, 32, 0, stream>>>(sys, nrhs, tol2);
  return cudaGetLastError();
}
cudaError_t launch_count_open(const BatchSys* sys, int nsys, int* out, cudaStream_t stream) {
  count_open_kernel<<<1, NTH, 0, stream>>>(sys, nsys, out);
  return cudaGetLastError();
}
cudaError_t launch_load_rhs_batched(const BatchSys* sys, int nsys, const double* const* B, int nrhs,
                                    int nr, cudaStream_t stream) {
  load_rhs_batched_kernel<<<dim3(8, nsys), NTH, 0, stream>>>(sys, B, nrhs, nr);
  return cudaGetLastError();
}
cudaError_t launch_store_x_batched(const BatchSys* sys, int nsys, double* const* X, int nrhs,
                                   int nr, cudaStream_t stream) {
  store_x_batched_kernel<<<dim3(8, nsys), NTH, 0, stream>>>(sys, X, nrhs, nr);
  return cudaGetLastError();
}
cudaError_t launch_frob_batched(const BatchSys* sys, int nsys, cudaStream_t stream) {
  frob_batched_kernel<<<dim3(BATCH_VB, nsys), NTH, 0, stream>>>(sys);
  return cudaGetLastError();
}


namespace {
// Loop control of the device-side PCG loop: ctl[0] counts the iterations run
// by this launch of the loop, ctl[1] is how many it may run.
__global__ void pcg_loop_init_kernel(int* ctl, int max_iters) {
  ctl[0] = 0;
  ctl[1] = max_iters;
}
// After each iteration: the new r^T z becomes the current one (rho[8..] ->
// rho[0..]), and the loop runs again only if the recursive residual has not
// met the tolerance, no error was recorded and the iteration budget is not
// spent.  The budget alone ends the loop, whatever the other flags hold.
__global__ void pcg_loop_cond_kernel(cudaGraphConditionalHandle handle, int* ctl, const int* done,
                                     const DevStatus* st, double* rho, int nr) {
  const int c = ctl[0] + 1;
  ctl[0] = c;
  for (int k = 0; k < nr; ++k) rho[k] = rho[8 + k];
  const bool more = c < ctl[1] && done[0] == 0 && st->code == 0;
  cudaGraphSetConditional(handle, more ? 1u : 0u);
}
}  // namespace

cudaError_t launch_pcg_loop_init(int* ctl, int max_iters, cudaStream_t stream) {
  pcg_loop_init_kernel<<<1, 1, 0, stream>>>(ctl, max_iters);
  return cudaGetLastError();
}
cudaError_t launch_pcg_loop_cond(cudaGraphConditionalHandle handle, int* ctl, const int* done,
                                 const DevStatus* st, double* rho, int nr, cudaStream_t stream) {
  pcg_loop_cond_kernel<<<1, 1, 0, stream>>>(handle, ctl, done, st, rho, nr);
  return cudaGetLastError();
}

}  // namespace mpchol
