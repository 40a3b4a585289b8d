// Small device utilities of the solver: diagonal extraction, FP64 -> FP32
// cast, Frobenius norm of a symmetric matrix from its lower triangle,
// zero-padded copies of right-hand sides, the diagonal power-of-two
// equilibration of the factor's storage, and the dense matrix cotangent of an
// adjoint solve.
//
// extract_diag replaces the reference's extractDiagonal + D2D copy
// (src/kernels_macros.cuh:161-173, src/mixed_cholesky.cu:128-131);
// f64_to_f32 its convertDoubleToFloat (src/kernels_macros.cuh:78-86).
#include <algorithm>

#include "common.cuh"
#include "pcg.cuh"

namespace mpchol {
namespace {

__global__ void extract_diag_kernel(const float* __restrict__ A, int lda, int n, float* d,
                                    float* dtilde) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float v = A[(size_t)i * lda + i];
    d[i] = v;
    dtilde[i] = v;
  }
}

__global__ void f64_to_f32_kernel(const double* __restrict__ src, int lds, float* __restrict__ dst,
                                  int ldd, int n) {
  const long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / n), r = (int)(e % n);
    dst[(size_t)c * ldd + r] = (float)src[(size_t)c * lds + r];
  }
}

// ||A||_F^2 of a symmetric matrix from its lower triangle.  Block b takes
// the columns b, b + gridDim.x, ...; its threads stride down each column from
// the diagonal (coalesced, no index division).  One partial per block.
template <typename TA>
__global__ void frob_lower_kernel(const TA* __restrict__ A, int lda, int n, double* partials) {
  double s = 0.0, s4[4] = {0.0, 0.0, 0.0, 0.0};
  for (int c = blockIdx.x; c < n; c += gridDim.x) {
    const TA* col = A + (size_t)c * lda;
    if (threadIdx.x == 0) {
      const double v = (double)col[c];
      s += v * v;
    }
    // off-diagonal part of the column: four independent loads in flight
    int r = c + 1 + threadIdx.x;
    for (; r + 3 * (int)blockDim.x < n; r += 4 * blockDim.x)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double v = (double)col[r + u * blockDim.x];
        s4[u] = fma(v, v, s4[u]);
      }
    for (; r < n; r += blockDim.x) {
      const double v = (double)col[r];
      s4[0] = fma(v, v, s4[0]);
    }
  }
  s += 2.0 * ((s4[0] + s4[1]) + (s4[2] + s4[3]));
  __shared__ double red[8];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    partials[blockIdx.x] = t;
  }
}

// Diagonal power-of-two equilibration exponent of a_ii: e = floor((floor(log2
// a) + 1) / 2) clamped to [-63, 63] (a * 2^(-2e) in [0.5, 2)); 0 for a
// non-positive or non-finite a.
__device__ __forceinline__ int equil_exp(float a) {
  if (!(a > 0.0f) || isinf(a)) return 0;
  const int E = ilog2f_dev(a);
  const int e = (E + 1) >> 1;              // arithmetic shift: floor division by 2
  return e < -63 ? -63 : (e > 63 ? 63 : e);
}

__global__ void equil_exps_kernel(const float* __restrict__ A, int lda, int n, int8_t* ex) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    ex[i] = (int8_t)equil_exp(A[(size_t)i * lda + i]);
}

// mode 0: A(i, j) *= 2^-(e_i + e_j) on the lower triangle of columns
// [c0, c1) (D A D); mode 1: the factor's rows scaled back, L(i, j) *= 2^e_i.  Block b walks columns b, b + gridDim.x, ...; its threads stride
// down each column from the diagonal.  |e_i + e_j| <= 126, so each scale is
// an exact normal power of two and each product is exact unless it leaves
// the normal range.
__global__ void equil_scale_kernel(float* __restrict__ A, int lda, int n, const int8_t* __restrict__ ex,
                                   int c0, int c1, int mode) {
  for (int c = c0 + blockIdx.x; c < c1; c += gridDim.x) {
    const int ec = ex[c];
    float* col = A + (size_t)c * lda;
    for (int r = c + threadIdx.x; r < n; r += blockDim.x) {
      const int e = mode == 0 ? -(ec + ex[r]) : ex[r];
      col[r] *= pow2f(e);
    }
  }
}

// G = -(Lam X^T + X Lam^T) / 2 (lower triangle, ld ldg) for n x nrhs column-major
// Lam, X: the matrix cotangent of a solve x = A^-1 b.
__global__ void sym_outer_kernel(const double* __restrict__ lam, const double* __restrict__ x,
                                 int n, int nrhs, double* __restrict__ G, int ldg) {
  for (int c = blockIdx.x; c < n; c += gridDim.x) {
    for (int r = c + threadIdx.x; r < n; r += blockDim.x) {
      double v = 0.0;
      for (int k = 0; k < nrhs; ++k)
        v += lam[(size_t)k * n + r] * x[(size_t)k * n + c] + x[(size_t)k * n + r] * lam[(size_t)k * n + c];
      G[(size_t)c * ldg + r] = -0.5 * v;
    }
  }
}

__global__ void pad_columns_kernel(const double* __restrict__ src, int n, int ncols,
                                   double* __restrict__ dst, int ncols_pad) {
  const long long total = (long long)n * ncols_pad;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / n);
    dst[e] = (c < ncols) ? src[e] : 0.0;
  }
}

}  // namespace

cudaError_t launch_extract_diag(const float* A, int lda, int n, float* d, float* dtilde,
                                cudaStream_t stream) {
  extract_diag_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(A, lda, n, d, dtilde);
  return cudaGetLastError();
}

cudaError_t launch_equil_exps(const float* A, int lda, int n, int8_t* ex, cudaStream_t stream) {
  equil_exps_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(A, lda, n, ex);
  return cudaGetLastError();
}

cudaError_t launch_equil_scale(float* A, int lda, int n, const int8_t* ex, int c0, int c1,
                               bool unscale_rows, cudaStream_t stream) {
  if (c1 <= c0) return cudaSuccess;
  const int grid = std::min(c1 - c0, 148 * 8);
  equil_scale_kernel<<<grid, 256, 0, stream>>>(A, lda, n, ex, c0, c1, unscale_rows ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_sym_outer(const double* lam, const double* x, int n, int nrhs, double* G,
                             int ldg, cudaStream_t stream) {
  sym_outer_kernel<<<std::min(n, 148 * 8), 256, 0, stream>>>(lam, x, n, nrhs, G, ldg);
  return cudaGetLastError();
}

cudaError_t launch_f64_to_f32(const double* src, int lds, float* dst, int ldd, int n,
                              cudaStream_t stream) {
  f64_to_f32_kernel<<<148 * 8, 256, 0, stream>>>(src, lds, dst, ldd, n);
  return cudaGetLastError();
}

template <typename TA>
cudaError_t launch_frob_lower(const TA* A, int lda, int n, double* partials, cudaStream_t stream) {
  frob_lower_kernel<TA><<<pcg_vgrid(), 256, 0, stream>>>(A, lda, n, partials);
  return cudaGetLastError();
}
template cudaError_t launch_frob_lower<float>(const float*, int, int, double*, cudaStream_t);
template cudaError_t launch_frob_lower<double>(const double*, int, int, double*, cudaStream_t);

cudaError_t launch_pad_columns(const double* src, int n, int ncols, double* dst, int ncols_pad,
                               cudaStream_t stream) {
  pad_columns_kernel<<<148 * 4, 256, 0, stream>>>(src, n, ncols, dst, ncols_pad);
  return cudaGetLastError();
}

}  // namespace mpchol
