// FP32 trailing update (SIMT FFMA), the "plain FP32" path.
//
// Replaces the reference's FP32 trailing GEMM LtSgemm (src/switching_chol.cuh:200-219,
// src/fp8_utils.cuh:231-302) and the CUTLASS FP32 GEMM of the uniform-precision
// prototype (src/sChol.cuh:284-306).  Unlike the reference it updates only the
// lower-triangle tiles (a SYRK, half the flops of the full GEMM it issues).
// 128 x 128 output tiles, 256 threads, 8 x 8 register tile per thread.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace mpchol {
namespace {

constexpr int BM = 128, BK = 8, NTH = 256;

__device__ __forceinline__ void group_sync(int group) {
  // named barrier of one 256-thread tile group (barrier 0 is __syncthreads)
  asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(NTH) : "memory");
}

// One 128 x 128 output tile (I, J) by the 256 threads of a tile group.
__device__ __forceinline__ void syrk_f32_tile(float* __restrict__ C, int ldc, int m, int k,
                                              const float* __restrict__ P, int ldp, int I, int J,
                                              float (*As)[BM], float (*Bs)[BM], int tid, int group) {
  const int i0 = I * BM, j0 = J * BM;
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
    group_sync(group);
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
    group_sync(group);
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

// One tile per CTA.
__global__ void __launch_bounds__(NTH)
syrk_f32_kernel(float* __restrict__ C, int ldc, int m, int k, const float* __restrict__ P, int ldp,
                const int* prec_sel, DevStatus* st, TileSel sel) {
  if (st != nullptr && st->code != 0) return;
  if (prec_sel != nullptr && *prec_sel != FP32) return;
  __shared__ __align__(16) float As[BK][BM];
  __shared__ __align__(16) float Bs[BK][BM];
  int I, J;
  sel_tile(blockIdx.x, sel, ceil_div(m, BM), I, J);
  syrk_f32_tile(C, ldc, m, k, P, ldp, I, J, As, Bs, threadIdx.x, 0);
}

// Persistent: two independent 256-thread tile groups per CTA (one CTA per SM
// by its register use), each walking the selected tiles with stride
// 2 * gridDim.x.
__global__ void __launch_bounds__(2 * NTH, 1)
syrk_f32_persistent_kernel(float* __restrict__ C, int ldc, int m, int k,
                           const float* __restrict__ P, int ldp, const int* prec_sel,
                           DevStatus* st, TileSel sel) {
  if (st != nullptr && st->code != 0) return;
  if (prec_sel != nullptr && *prec_sel != FP32) return;
  __shared__ __align__(16) float As[2][BK][BM];
  __shared__ __align__(16) float Bs[2][BK][BM];
  const int group = threadIdx.x / NTH, tid = threadIdx.x % NTH;
  const int T = ceil_div(m, BM);
  const int ntiles = sel_tile_count(T, sel);
  for (int t = 2 * blockIdx.x + group; t < ntiles; t += 2 * gridDim.x) {
    int I, J;
    sel_tile(t, sel, T, I, J);
    syrk_f32_tile(C, ldc, m, k, P, ldp, I, J, As[group], Bs[group], tid, group);
  }
}

}  // namespace

cudaError_t launch_syrk_f32(float* C, int ldc, int m, int k, const float* P, int ldp,
                            const int* prec_sel, DevStatus* st, cudaStream_t stream, TileSel sel,
                            int max_sms) {
  if (m <= 0) return cudaSuccess;
  const int ntiles = sel_tile_count(ceil_div(m, BM), sel);
  if (ntiles <= 0) return cudaSuccess;
  if (max_sms > 0) {
    const int grid = std::min(max_sms, ceil_div(ntiles, 2));
    syrk_f32_persistent_kernel<<<grid, 2 * NTH, 0, stream>>>(C, ldc, m, k, P, ldp, prec_sel, st, sel);
  } else {
    syrk_f32_kernel<<<ntiles, NTH, 0, stream>>>(C, ldc, m, k, P, ldp, prec_sel, st, sel);
  }
  return cudaGetLastError();
}

}  // namespace mpchol
