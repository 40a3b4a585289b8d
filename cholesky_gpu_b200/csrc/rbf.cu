// Gaussian RBF kernel matrices and their gradient contractions.
//
// The reference has only a stub for this (src/RBF.cu:1-45).  Forward:
//   K_ij = exp(-||x_i - x_j||^2 / (2 l^2)) + nugget * delta_ij
// from n points x_i (rows of X, FP32), formed in FP64 (differences, not the
// norm expansion, so close points lose no digits) and written as FP64 and/or
// FP32 column-major.  Backward: for a symmetric cotangent
// G_K = -(a b^T + b a^T) / 2 of the solve x = K^-1 y (a the adjoint solution,
// b = x), every gradient needs only
//   P = K_rbf [a, b, a*X, b*X]    (n x (2 + 2d), K_rbf without the nugget)
//   s = sum_ij a_i b_j K_ij r_ij^2
// which one kernel forms while recomputing the K tiles from X (K itself is
// never read back):
//   dL/dnugget = -a.b,   dL/dl = -s / l^3,   dL/dy = a,
//   dL/dX_i = (X_i (a_i (K b)_i + b_i (K a)_i) - a_i (K(b*X))_i - b_i (K(a*X))_i) / l^2.
#include "common.cuh"
#include "pcg.cuh"

namespace mpchol {
namespace {

constexpr int BT = 64;        // build tile (BT x BT outputs per CTA)
constexpr int BK = 16;        // feature chunk staged per step
constexpr int NTH = 256;

__global__ void __launch_bounds__(NTH)
rbf_build_kernel(const float* __restrict__ X, int n, int d, int ldx, double inv2l2, double nugget,
                 double* __restrict__ K64, float* __restrict__ K32, int ldk, int lower_only) {
  const int I = blockIdx.y, J = blockIdx.x;
  if (lower_only && J > I) return;
  __shared__ double xi[BK][BT + 1];
  __shared__ double xj[BK][BT + 1];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int i0 = I * BT, j0 = J * BT;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < d; k0 += BK) {
    for (int e = tid; e < BK * BT; e += NTH) {
      const int r = e / BK, k = e % BK;     // consecutive threads: consecutive features
      const int gi = i0 + r, gj = j0 + r, gk = k0 + k;
      xi[k][r] = (gi < n && gk < d) ? (double)X[(size_t)gi * ldx + gk] : 0.0;
      xj[k][r] = (gj < n && gk < d) ? (double)X[(size_t)gj * ldx + gk] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < BK; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = xi[k][tx * 4 + u]; b[u] = xj[k][ty * 4 + u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double df = a[u] - b[v];
          acc[u][v] = fma(df, df, acc[u][v]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int j = j0 + ty * 4 + v;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + tx * 4 + u;
      if (i < n && j < n && (!lower_only || i >= j)) {
        double kv = exp(-acc[u][v] * inv2l2);
        if (i == j) kv = 1.0 + nugget;
        if (K64) K64[(size_t)j * ldk + i] = kv;
        if (K32) K32[(size_t)j * ldk + i] = (float)kv;
      }
    }
  }
}

// Backward contraction.  One CTA owns RB_ rows and sweeps all column tiles,
// so P is written once (no atomics) and s is reduced in a fixed order.
constexpr int RB_ = 32;       // rows per CTA
constexpr int CB = 64;        // columns per sweep step
constexpr int MAXD = 128;     // largest feature count the kernel stages
constexpr int MAXC = (2 + 2 * MAXD + 7) / 8;   // P columns per thread (8 column groups)

__global__ void __launch_bounds__(NTH)
rbf_grad_kernel(const float* __restrict__ X, int n, int d, int ldx, double inv2l2,
                const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ P,
                double* __restrict__ s_part) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double* xiT = reinterpret_cast<double*>(sm_raw);        // [d][RB_]   (feature-major)
  double* xJ = xiT + (size_t)d * RB_;                      // [CB][d]    (row-major)
  double* kt = xJ + (size_t)CB * d;                        // [RB_][CB + 1]
  double* aJ = kt + RB_ * (CB + 1);                        // [CB]
  double* bJ = aJ + CB;                                    // [CB]
  __shared__ double s_red[NTH / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i0 = blockIdx.x * RB_;
  for (int e = tid; e < RB_ * d; e += NTH) {
    const int r = e / d, k = e % d;
    const int gi = i0 + r;
    xiT[k * RB_ + r] = (gi < n) ? (double)X[(size_t)gi * ldx + k] : 0.0;
  }
  const int my_i = tid % RB_;                  // row of this thread in the output phase
  const int grp = tid / RB_;                   // column group: columns grp, grp + 8, ...
  const int gi_me = i0 + my_i;
  const double a_me = (gi_me < n) ? a[gi_me] : 0.0;
  const int NC = 2 + 2 * d;
  double acc[MAXC];
#pragma unroll
  for (int q = 0; q < MAXC; ++q) acc[q] = 0.0;
  double s_acc = 0.0;
  for (int j0 = 0; j0 < n; j0 += CB) {
    __syncthreads();
    for (int e = tid; e < CB * d; e += NTH) {
      const int r = e / d, k = e % d;
      const int gj = j0 + r;
      xJ[r * d + k] = (gj < n) ? (double)X[(size_t)gj * ldx + k] : 0.0;
    }
    for (int e = tid; e < CB; e += NTH) {
      const int gj = j0 + e;
      aJ[e] = (gj < n) ? a[gj] : 0.0;
      bJ[e] = (gj < n) ? b[gj] : 0.0;
    }
    __syncthreads();
    // K tile: warp w handles columns w, w + 8, ...; lane = row
    for (int j = warp; j < CB; j += NTH / 32) {
      const int gj = j0 + j, gi = i0 + lane;
      double r2 = 0.0;
      for (int k = 0; k < d; ++k) {
        const double df = xiT[k * RB_ + lane] - xJ[j * d + k];
        r2 = fma(df, df, r2);
      }
      double kv = 0.0;
      if (gi < n && gj < n) {
        kv = exp(-r2 * inv2l2);
        s_acc += a_me * bJ[j] * kv * r2;
      }
      kt[lane * (CB + 1) + j] = kv;
    }
    __syncthreads();
    // P rows += K tile x [a, b, a*X, b*X] of the columns
    for (int j = 0; j < CB; ++j) {
      const double kij = kt[my_i * (CB + 1) + j];
      const double aj = aJ[j], bj = bJ[j];
      const double* xr = xJ + (size_t)j * d;
#pragma unroll
      for (int q = 0; q < MAXC; ++q) {
        const int c = grp + 8 * q;
        if (c < NC) {
          double z;
          if (c == 0) z = aj;
          else if (c == 1) z = bj;
          else if (c < 2 + d) z = aj * xr[c - 2];
          else z = bj * xr[c - 2 - d];
          acc[q] = fma(kij, z, acc[q]);
        }
      }
    }
  }
  if (gi_me < n) {
#pragma unroll
    for (int q = 0; q < MAXC; ++q) {
      const int c = grp + 8 * q;
      if (c < NC) P[(size_t)c * n + gi_me] = acc[q];
    }
  }
  s_acc = warp_sum(s_acc);
  if (lane == 0) s_red[warp] = s_acc;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < NTH / 32; ++w) t += s_red[w];
    s_part[blockIdx.x] = t;
  }
}

// s = sum of the per-CTA partials in index order (deterministic)
__global__ void sum_partials_kernel(const double* __restrict__ part, int count, double* out) {
  __shared__ double s_w[NTH / 32];
  double v = 0.0;
  for (int i = threadIdx.x; i < count; i += NTH) v += part[i];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NTH / 32; ++w) t += s_w[w];
    *out = t;
  }
}

size_t grad_smem(int d) {
  return ((size_t)d * RB_ + (size_t)CB * d + RB_ * (CB + 1) + 2 * CB) * sizeof(double);
}

}  // namespace

int rbf_grad_max_features() { return MAXD; }
int rbf_grad_work_elems(int n) { return ceil_div(n, RB_); }

cudaError_t launch_rbf_build(const float* X, int n, int d, int ldx, double lengthscale,
                             double nugget, double* K64, float* K32, int ldk, int lower_only,
                             cudaStream_t stream) {
  const double inv2l2 = 1.0 / (2.0 * lengthscale * lengthscale);
  const dim3 grid(ceil_div(n, BT), ceil_div(n, BT));
  rbf_build_kernel<<<grid, NTH, 0, stream>>>(X, n, d, ldx, inv2l2, nugget, K64, K32, ldk, lower_only);
  return cudaGetLastError();
}

cudaError_t launch_rbf_grad(const float* X, int n, int d, int ldx, double lengthscale,
                            const double* a, const double* b, double* P, double* s, double* work,
                            cudaStream_t stream) {
  const double inv2l2 = 1.0 / (2.0 * lengthscale * lengthscale);
  const size_t smem = grad_smem(d);
  cudaError_t e = cudaFuncSetAttribute(rbf_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int nb = ceil_div(n, RB_);
  rbf_grad_kernel<<<nb, NTH, smem, stream>>>(X, n, d, ldx, inv2l2, a, b, P, work);
  sum_partials_kernel<<<1, NTH, 0, stream>>>(work, nb, s);
  return cudaGetLastError();
}

}  // namespace mpchol
