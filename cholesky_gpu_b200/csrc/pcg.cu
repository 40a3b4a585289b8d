// PCG building blocks: operator apply, preconditioner apply, FP64 recurrences.
//
// Replaces the reference's PCG loop library calls (src/mixed_cholesky.cu:153-216):
//   cublasDgemv on FP64 A              -> symv_kernel (lower triangle of FP32 or FP64 A,
//                                         FP64 vectors; reads n^2/2 elements, not n^2)
//   cusolverDnDpotrs on an FP64 copy L -> trsv_kernel (forward, backward) on the FP32
//                                         factor, FP64 vectors, no FP64 copy of L
//   Ddot/Daxpy/Dscal/Dcopy/Dnrm2 with host pointer mode (two host syncs per
//   iteration)                         -> dot_partial / update kernels with device-resident
//                                         alpha, beta, rho (the intent of
//                                         src/kernels_macros.cuh:547-550,599-632)
// All vectors are n x nrhs, column-major, ld = n, nrhs <= 8.
#include <cuda/atomic>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg.cuh"

namespace mpchol {
namespace {

constexpr int RB = 128;      // block rows / tile size
constexpr int NTH = 256;     // 8 warps
constexpr unsigned kFlagPolls = 1u << 22;

__device__ __forceinline__ void tile_of(int t, int& I, int& J) {
  int i = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (i * (i + 1) / 2 > t) --i;
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  I = i;
  J = t - i * (i + 1) / 2;
}

template <typename TA>
struct Vec4 { double v[4]; };

template <typename TA>
__device__ __forceinline__ void load4(const TA* p, int nvalid, double out[4]);
template <>
__device__ __forceinline__ void load4<float>(const float* p, int nvalid, double out[4]) {
  if (nvalid >= 4 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = (r < nvalid) ? (double)__ldg(p + r) : 0.0;
  }
}
template <>
__device__ __forceinline__ void load4<double>(const double* p, int nvalid, double out[4]) {
  if (nvalid >= 4 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    out[0] = a.x; out[1] = a.y; out[2] = b.x; out[3] = b.y;
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = (r < nvalid) ? __ldg(p + r) : 0.0;
  }
}

// ---- y += A x for symmetric A, lower triangle read once --------------------
// One CTA per 128 x 128 lower tile (I >= J): y_I += A_IJ x_J and, off the
// diagonal, y_J += A_IJ^T x_I.  Lane l covers rows 4l..4l+3 of the tile, warp w
// columns 16w..16w+15.  Results are added to y with FP64 atomics (y zeroed by
// the caller).
template <typename TA, int NR>
__global__ void __launch_bounds__(NTH)
symv_kernel(const TA* __restrict__ A, int lda, int n, const double* __restrict__ x,
            double* __restrict__ y, const int* skip) {
  if (skip != nullptr && *skip) return;
  __shared__ double s_xJ[RB * NR];
  __shared__ double s_xI[RB * NR];
  extern __shared__ double s_part_dyn[];
  double (*s_part)[RB * NR] = reinterpret_cast<double (*)[RB * NR]>(s_part_dyn);
  int I, J;
  tile_of(blockIdx.x, I, J);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i0 = I * RB, j0 = J * RB;
  for (int e = tid; e < RB * NR; e += NTH) {
    const int r = e / NR, k = e % NR;
    s_xJ[e] = (j0 + r < n) ? x[(size_t)k * n + j0 + r] : 0.0;
    s_xI[e] = (i0 + r < n) ? x[(size_t)k * n + i0 + r] : 0.0;
  }
  __syncthreads();
  double accI[4][NR];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < NR; ++k) accI[r][k] = 0.0;
  const bool diag = (I == J);
  const int rloc = 4 * lane;
  const int nvalid = min(4, n - (i0 + rloc));
#pragma unroll 2
  for (int cc = 0; cc < 16; ++cc) {
    const int c = warp * 16 + cc;
    const int gj = j0 + c;
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    if (gj < n && nvalid > 0) load4<TA>(A + (size_t)gj * lda + i0 + rloc, nvalid, a);
    if (diag) {
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (rloc + r < c) a[r] = 0.0;    // strictly upper part of the diagonal tile is not read
    }
    // y_I[rows] += a * x_J[c]
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      const double xc = s_xJ[c * NR + k];
#pragma unroll
      for (int r = 0; r < 4; ++r) accI[r][k] = fma(a[r], xc, accI[r][k]);
    }
    // y_J[c] += sum_rows a * x_I[rows]  (strictly lower only on the diagonal tile)
    double pd[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      double s = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const double ar = (diag && rloc + r == c) ? 0.0 : a[r];
        s = fma(ar, s_xI[(rloc + r) * NR + k], s);
      }
      pd[k] = warp_sum(s);
    }
    if (lane == 0 && gj < n) {
#pragma unroll
      for (int k = 0; k < NR; ++k) atomicAdd(&y[(size_t)k * n + gj], pd[k]);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < NR; ++k) s_part[warp][(rloc + r) * NR + k] = accI[r][k];
  __syncthreads();
  for (int e = tid; e < RB * NR; e += NTH) {
    const int r = e / NR, k = e % NR;
    if (i0 + r < n) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < NTH / 32; ++w) s += s_part[w][e];
      atomicAdd(&y[(size_t)k * n + i0 + r], s);
    }
  }
}

// ---- diagonal-block inverses for the triangular solves --------------------
// linv + I*RB*RB holds inv(L_II) (RB x RB, column-major, FP32), formed in FP64.
__global__ void __launch_bounds__(RB)
diag_inverse_kernel(const float* __restrict__ L, int ldl, int n, float* __restrict__ linv) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double* W = reinterpret_cast<double*>(sm_raw);            // [RB][RB+1]
  float* Ls = reinterpret_cast<float*>(W + RB * (RB + 1));  // [RB][RB+1]
  const int I = blockIdx.x, c = threadIdx.x;
  const int i0 = I * RB;
  const int nb = min(RB, n - i0);
  for (int e = c; e < RB * RB; e += RB) {
    const int col = e / RB, row = e % RB;
    float v;
    if (row < nb && col < nb) v = L[(size_t)(i0 + col) * ldl + i0 + row];
    else v = (row == col) ? 1.0f : 0.0f;
    Ls[col * (RB + 1) + row] = v;
  }
  __syncthreads();
  for (int i = 0; i < RB; ++i) {
    double w = 0.0;
    if (i >= c) {
      double acc = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) acc -= (double)Ls[k * (RB + 1) + i] * W[c * (RB + 1) + k];
      w = acc / (double)Ls[i * (RB + 1) + i];
    }
    W[c * (RB + 1) + i] = w;
  }
  __syncthreads();
  float* out = linv + (size_t)I * RB * RB;
  for (int e = c; e < RB * RB; e += RB) {
    const int col = e / RB, row = e % RB;
    out[e] = (float)W[col * (RB + 1) + row];
  }
}

__device__ __forceinline__ bool wait_flag(const int* flag, int epoch) {
  cuda::atomic_ref<const int, cuda::thread_scope_device> f(*flag);
  for (unsigned it = 0; it < kFlagPolls; ++it) {
    if (f.load(cuda::memory_order_acquire) == epoch) return true;
    __nanosleep(64);
  }
  return false;
}

// ---- triangular solves (forward L y = b, backward L^T z = b) --------------
// Persistent, dependency-ordered: each CTA takes the next block row from a
// ticket counter (so it only ever waits on block rows owned by CTAs already
// running), accumulates the off-diagonal tiles as their inputs are published
// (flags[J] == epoch), applies the diagonal-block inverse and publishes its
// own block.  Every wait is bounded; on timeout the status is set and the CTA
// returns.
template <int NR, bool BWD>
__global__ void __launch_bounds__(NTH)
trsv_kernel(const float* __restrict__ L, int ldl, int n, const float* __restrict__ linv,
            const double* __restrict__ rhs, double* __restrict__ out, int* flags, int epoch,
            int* ticket, const int* skip, DevStatus* st) {
  if (skip != nullptr && *skip) return;
  __shared__ double s_v[RB * NR];
  __shared__ double s_rhs[RB * NR];
  extern __shared__ double s_part_dyn[];
  double (*s_part)[RB * NR] = reinterpret_cast<double (*)[RB * NR]>(s_part_dyn);
  __shared__ int s_idx, s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NB = (n + RB - 1) / RB;
  if (tid == 0) { s_idx = atomicAdd(ticket, 1); s_bad = 0; }
  __syncthreads();
  const int idx = s_idx;
  if (idx >= NB) return;
  const int I = BWD ? NB - 1 - idx : idx;
  const int i0 = I * RB;
  const int rloc = 4 * lane;
  double acc[4][NR];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < NR; ++k) acc[r][k] = 0.0;
  // BWD keeps per-column sums for the warp's 16 columns in s_part[warp]
  if (BWD) {
    for (int e = tid; e < (NTH / 32) * RB * NR; e += NTH) (&s_part[0][0])[e] = 0.0;
    __syncthreads();
  }
  const int jbeg = BWD ? I + 1 : 0, jend = BWD ? NB : I;
  for (int J = jbeg; J < jend; ++J) {
    if (tid == 0) {
      if (!wait_flag(flags + J, epoch)) {
        s_bad = 1;
        set_status(st, MPCHOL_ERR_TIMEOUT, J);
      }
    }
    __syncthreads();
    if (s_bad) return;
    const int j0 = J * RB;
    for (int e = tid; e < RB * NR; e += NTH) {
      const int r = e / NR, k = e % NR;
      s_v[e] = (j0 + r < n) ? out[(size_t)k * n + j0 + r] : 0.0;
    }
    __syncthreads();
    if (!BWD) {
      // acc[rows of I] += L_IJ * v_J
      const int nvalid = min(4, n - (i0 + rloc));
#pragma unroll 4
      for (int cc = 0; cc < 16; ++cc) {
        const int c = warp * 16 + cc;
        double a[4] = {0.0, 0.0, 0.0, 0.0};
        if (j0 + c < n && nvalid > 0) load4<float>(L + (size_t)(j0 + c) * ldl + i0 + rloc, nvalid, a);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          const double vc = s_v[c * NR + k];
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[r][k] = fma(a[r], vc, acc[r][k]);
        }
      }
    } else {
      // column sums: for column c of block I, sum_rows L_JI[row][c] * v_J[row]
      const int nvalid = min(4, n - (j0 + rloc));
#pragma unroll 4
      for (int cc = 0; cc < 16; ++cc) {
        const int c = warp * 16 + cc;
        double a[4] = {0.0, 0.0, 0.0, 0.0};
        if (i0 + c < n && nvalid > 0) load4<float>(L + (size_t)(i0 + c) * ldl + j0 + rloc, nvalid, a);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          double sacc = 0.0;
#pragma unroll
          for (int r = 0; r < 4; ++r) sacc = fma(a[r], s_v[(rloc + r) * NR + k], sacc);
          sacc = warp_sum(sacc);
          if (lane == 0) s_part[warp][c * NR + k] += sacc;
        }
      }
    }
    __syncthreads();
  }
  // right-hand side minus the accumulated off-diagonal part
  if (!BWD) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < NR; ++k) s_part[warp][(rloc + r) * NR + k] = acc[r][k];
    __syncthreads();
  }
  for (int e = tid; e < RB * NR; e += NTH) {
    const int r = e / NR, k = e % NR;
    double s = 0.0;
    if (!BWD) {
#pragma unroll
      for (int w = 0; w < NTH / 32; ++w) s += s_part[w][e];
    } else {
      s = s_part[r / 16][e];          // column r belongs to warp r/16
    }
    s_rhs[e] = (i0 + r < n) ? rhs[(size_t)k * n + i0 + r] - s : 0.0;
  }
  __syncthreads();
  // diagonal block: out_I = inv(L_II) s_rhs (forward) or inv(L_II)^T s_rhs (backward)
  const float* W = linv + (size_t)I * RB * RB;
  if (!BWD) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < NR; ++k) acc[r][k] = 0.0;
#pragma unroll 4
    for (int cc = 0; cc < 16; ++cc) {
      const int c = warp * 16 + cc;
      double a[4];
      load4<float>(W + (size_t)c * RB + rloc, 4, a);
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        const double vc = s_rhs[c * NR + k];
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[r][k] = fma(a[r], vc, acc[r][k]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < NR; ++k) s_part[warp][(rloc + r) * NR + k] = acc[r][k];
    __syncthreads();
    for (int e = tid; e < RB * NR; e += NTH) {
      const int r = e / NR, k = e % NR;
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < NTH / 32; ++w) s += s_part[w][e];
      if (i0 + r < n) out[(size_t)k * n + i0 + r] = s;
    }
  } else {
#pragma unroll 4
    for (int cc = 0; cc < 16; ++cc) {
      const int c = warp * 16 + cc;
      double a[4];
      load4<float>(W + (size_t)c * RB + rloc, 4, a);
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        double sacc = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) sacc = fma(a[r], s_rhs[(rloc + r) * NR + k], sacc);
        sacc = warp_sum(sacc);
        if (lane == 0 && i0 + c < n) out[(size_t)k * n + i0 + c] = sacc;
      }
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    cuda::atomic_ref<int, cuda::thread_scope_device> f(flags[I]);
    f.store(epoch, cuda::memory_order_release);
  }
}

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

template <int NR>
__device__ __forceinline__ void sum_partials(const double* partials, double (&out)[NR]) {
  // every thread sums the VG partials in the same fixed order
#pragma unroll
  for (int k = 0; k < NR; ++k) out[k] = 0.0;
  for (int b = 0; b < VG; ++b)
#pragma unroll
    for (int k = 0; k < NR; ++k) out[k] += partials[b * NR + k];
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
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double rr[NR];
    sum_partials<NR>(rr_partials, rr);
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
__global__ void reduce_partials_kernel(const double* partials, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s[NR];
    sum_partials<NR>(partials, s);
#pragma unroll
    for (int k = 0; k < NR; ++k) out[k] = s[k];
  }
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

static size_t part_bytes(int nr) { return (size_t)(NTH / 32) * RB * nr * sizeof(double); }

int pcg_padded_nrhs(int nrhs) { return nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : 8; }
int pcg_vgrid() { return VG; }

template <typename TA>
cudaError_t launch_symv(const TA* A, int lda, int n, const double* x, double* y, int nrhs,
                        cudaStream_t stream) {
  return launch_symv_skip<TA>(A, lda, n, x, y, nrhs, nullptr, stream);
}

template <typename TA>
cudaError_t launch_symv_skip(const TA* A, int lda, int n, const double* x, double* y, int nrhs,
                             const int* skip, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(y, 0, sizeof(double) * (size_t)n * nrhs, stream);
  if (e != cudaSuccess) return e;
  const int T = ceil_div(n, RB);
  NR_DISPATCH(nrhs, ({
    const size_t dyn = part_bytes(NRC);
    e = cudaFuncSetAttribute(symv_kernel<TA, NRC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    symv_kernel<TA, NRC><<<T * (T + 1) / 2, NTH, dyn, stream>>>(A, lda, n, x, y, skip);
  }));
  return cudaGetLastError();
}
template cudaError_t launch_symv<float>(const float*, int, int, const double*, double*, int, cudaStream_t);
template cudaError_t launch_symv<double>(const double*, int, int, const double*, double*, int, cudaStream_t);
template cudaError_t launch_symv_skip<float>(const float*, int, int, const double*, double*, int, const int*, cudaStream_t);
template cudaError_t launch_symv_skip<double>(const double*, int, int, const double*, double*, int, const int*, cudaStream_t);

cudaError_t launch_diag_inverse(const float* L, int ldl, int n, float* linv, cudaStream_t stream) {
  const size_t smem = (size_t)RB * (RB + 1) * (sizeof(double) + sizeof(float));
  cudaError_t e = cudaFuncSetAttribute(diag_inverse_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  diag_inverse_kernel<<<ceil_div(n, RB), RB, smem, stream>>>(L, ldl, n, linv);
  return cudaGetLastError();
}

cudaError_t launch_trsv(bool backward, const float* L, int ldl, int n, const float* linv,
                        const double* rhs, double* out, int nrhs, int* flags, int epoch,
                        int* ticket, const int* skip, DevStatus* st, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  const int NB = ceil_div(n, RB);
  if (backward) {
    NR_DISPATCH(nrhs, ({
      const size_t dyn = part_bytes(NRC);
      e = cudaFuncSetAttribute(trsv_kernel<NRC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
      if (e != cudaSuccess) return e;
      trsv_kernel<NRC, true><<<NB, NTH, dyn, stream>>>(L, ldl, n, linv, rhs, out, flags, epoch, ticket, skip, st);
    }));
  } else {
    NR_DISPATCH(nrhs, ({
      const size_t dyn = part_bytes(NRC);
      e = cudaFuncSetAttribute(trsv_kernel<NRC, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
      if (e != cudaSuccess) return e;
      trsv_kernel<NRC, false><<<NB, NTH, dyn, stream>>>(L, ldl, n, linv, rhs, out, flags, epoch, ticket, skip, st);
    }));
  }
  return cudaGetLastError();
}

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
  NR_DISPATCH(nrhs, (reduce_partials_kernel<NRC><<<1, 32, 0, stream>>>(partials, out)));
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
