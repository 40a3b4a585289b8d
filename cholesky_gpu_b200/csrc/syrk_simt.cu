// FP32 trailing update (SIMT FFMA), the "plain FP32" path.
//
// Replaces the reference's FP32 trailing GEMM LtSgemm (src/switching_chol.cuh:200-219,
// src/fp8_utils.cuh:231-302) and the CUTLASS FP32 GEMM of the uniform-precision
// prototype (src/sChol.cuh:284-306).  Unlike the reference it updates only the
// lower-triangle tiles (a SYRK, half the flops of the full GEMM it issues).
// 128 x 128 output tiles, 256 threads, 8 x 8 register tile per thread.
#include "common.cuh"
#include "kernels.cuh"

namespace mpchol {
namespace {

constexpr int BM = 128, BK = 8, NTH = 256;

__device__ __forceinline__ void tile_of(int t, int& I, int& J) {
  int i = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (i * (i + 1) / 2 > t) --i;
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  I = i;
  J = t - i * (i + 1) / 2;
}

__global__ void __launch_bounds__(NTH)
syrk_f32_kernel(float* __restrict__ C, int ldc, int m, int k, const float* __restrict__ P, int ldp,
                const int* prec_sel, DevStatus* st) {
  if (st != nullptr && st->code != 0) return;
  if (prec_sel != nullptr && *prec_sel != FP32) return;
  __shared__ __align__(16) float As[BK][BM];
  __shared__ __align__(16) float Bs[BK][BM];
  int I, J;
  tile_of(blockIdx.x, I, J);
  const int i0 = I * BM, j0 = J * BM;
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;    // rows follow tx (coalesced C access)
  float acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.0f;

  for (int k0 = 0; k0 < k; k0 += BK) {
#pragma unroll
    for (int e = tid; e < BK * BM; e += NTH) {
      const int kk = e / BM, r = e % BM;
      const int kc = k0 + kk;
      const int ia = i0 + r, jb = j0 + r;
      As[kk][r] = (ia < m && kc < k) ? P[(size_t)kc * ldp + ia] : 0.0f;
      Bs[kk][r] = (jb < m && kc < k) ? P[(size_t)kc * ldp + jb] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[kk][tx * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[kk][64 + tx * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[kk][ty * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[kk][64 + ty * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int j = j0 + (b < 4 ? ty * 4 + b : 64 + ty * 4 + (b - 4));
    if (j >= m) continue;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int i = i0 + (a < 4 ? tx * 4 + a : 64 + tx * 4 + (a - 4));
      if (i < m && i >= j) C[(size_t)j * ldc + i] -= acc[a][b];
    }
  }
}

}  // namespace

cudaError_t launch_syrk_f32(float* C, int ldc, int m, int k, const float* P, int ldp,
                            const int* prec_sel, DevStatus* st, cudaStream_t stream) {
  if (m <= 0) return cudaSuccess;
  const int T = ceil_div(m, BM);
  syrk_f32_kernel<<<T * (T + 1) / 2, NTH, 0, stream>>>(C, ldc, m, k, P, ldp, prec_sel, st);
  return cudaGetLastError();
}

}  // namespace mpchol
