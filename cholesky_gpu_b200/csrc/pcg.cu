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

constexpr int RB = 128;      // block rows / tile size
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

}  // namespace mpchol
