// Tensor-core trailing update (tcgen05 + TMEM + TMA) for the low-precision
// steps of the factorization.
//
// Replaces the reference's cuBLASLt trailing updates LtHSgemm_fp16in_fp32out
// (src/switching_chol.cuh:170-197, src/fp8_utils.cuh:304-412), the per-tensor
// scaled FP8 CUTLASS GEMM (src/fp8Chol.cuh:236-275) and the WMMA SYRK
// (src/syrk_gemm.cuh:14-124).  C(m x m, lower tiles) -= s_i s_j (Q Q^T): Q is
// the K-major quantized panel (FP16 / E4M3 / E5M2), s the per-row power-of-two
// scales, accumulation in FP32 in tensor memory.  One CTA per 128 x 128 lower
// tile: thread 0 stages both 128-row strips of Q with TMA (128-byte swizzle,
// no multicast), issues the k/K_mma tcgen05.mma instructions into a 128-column
// TMEM accumulator and commits to an mbarrier; four warps then read their 32
// TMEM lanes and apply the scaled update to C in FP32 (coalesced along rows).
// Diagonal tiles load one strip and use it for both operands.
#include <cudaTypedefs.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace mpchol {
namespace {

constexpr int TM = 128;            // output tile (M = N = 128)
constexpr int BOX_BYTES = 128;     // inner TMA box = one 128-byte swizzle row
constexpr int STRIP_CHUNK = TM * BOX_BYTES;   // 16 KB per (strip, K chunk)

__device__ __forceinline__ void tile_of(int t, int& I, int& J) {
  int i = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (i * (i + 1) / 2 > t) --i;
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  I = i;
  J = t - i * (i + 1) / 2;
}

template <int FMT>
__global__ void __launch_bounds__(128, 1)
syrk_tc_kernel(const __grid_constant__ CUtensorMap tmap, float* __restrict__ C, int ldc, int m,
               int k, const int8_t* __restrict__ rowexp, const int* prec_sel, DevStatus* st) {
  if (st != nullptr && st->code != 0) return;
  if (prec_sel != nullptr && *prec_sel != FMT) return;
  constexpr int ESIZE = (FMT == FP16) ? 2 : 1;
  constexpr int ELEMS_PER_BOX = BOX_BYTES / ESIZE;
  constexpr uint32_t IDESC = (FMT == FP16) ? tc::make_idesc(0, 0, TM, TM)
                             : (FMT == E5M2) ? tc::make_idesc(1, 1, TM, TM)
                                             : tc::make_idesc(0, 0, TM, TM);
  constexpr int KSTEP_BYTES = 32;   // K per MMA: 16 x 2 B (f16) or 32 x 1 B (f8f6f4)

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nbox = (k * ESIZE) / BOX_BYTES;
  uint8_t* sA = smem;
  uint8_t* sB = smem + (size_t)nbox * STRIP_CHUNK;
  __shared__ __align__(8) uint64_t bar_tma;
  __shared__ __align__(8) uint64_t bar_mma;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int ok_sh;
  __shared__ float s_scale_j[TM];

  int I, J;
  tile_of(blockIdx.x, I, J);
  const bool diag = (I == J);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    tc::prefetch_tmap(&tmap);
    tc::mbar_init(&bar_tma, 1);
    tc::mbar_init(&bar_mma, 1);
    tc::fence_mbar_init();
    ok_sh = 1;
  }
  if (warp == 0) tc::tmem_alloc(&tmem_base_sh, TM);
  {
    const int j = J * TM + threadIdx.x;
    s_scale_j[threadIdx.x] = (j < m) ? pow2f(rowexp[j]) : 0.0f;
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (threadIdx.x == 0) {
    const uint32_t bytes = (uint32_t)((diag ? 1 : 2) * nbox * STRIP_CHUNK);
    tc::mbar_expect_tx(&bar_tma, bytes);
    for (int b = 0; b < nbox; ++b) {
      tc::tma_load_2d(sA + (size_t)b * STRIP_CHUNK, &tmap, &bar_tma, b * ELEMS_PER_BOX, I * TM);
      if (!diag)
        tc::tma_load_2d(sB + (size_t)b * STRIP_CHUNK, &tmap, &bar_tma, b * ELEMS_PER_BOX, J * TM);
    }
    if (tc::mbar_wait(&bar_tma, 0)) {
      tc::tc_fence_after();
      const uint8_t* sBop = diag ? sA : sB;
      uint32_t accumulate = 0;
      for (int b = 0; b < nbox; ++b) {
        const uint32_t a0 = tc::smem_u32(sA + (size_t)b * STRIP_CHUNK);
        const uint32_t b0 = tc::smem_u32(sBop + (size_t)b * STRIP_CHUNK);
#pragma unroll
        for (int kk = 0; kk < BOX_BYTES / KSTEP_BYTES; ++kk) {
          const uint64_t ad = tc::make_desc_sw128(a0 + kk * KSTEP_BYTES);
          const uint64_t bd = tc::make_desc_sw128(b0 + kk * KSTEP_BYTES);
          if (FMT == FP16) tc::mma_f16(tmem, ad, bd, IDESC, accumulate);
          else tc::mma_f8f6f4(tmem, ad, bd, IDESC, accumulate);
          accumulate = 1;
        }
      }
      tc::mma_commit(&bar_mma);
    } else {
      ok_sh = 0;
      if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, blockIdx.x);
      tc::mbar_wait(&bar_tma, 0);   // give in-flight copies one more bounded chance to land
    }
  }
  __syncthreads();
  if (ok_sh) {
    if (!tc::mbar_wait(&bar_mma, 0)) {
      if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, blockIdx.x);
    } else {
      tc::tc_fence_after();
      const int i = I * TM + warp * 32 + lane;
      const float si = (i < m) ? pow2f(rowexp[i]) : 0.0f;
#pragma unroll 1
      for (int c0 = 0; c0 < TM; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        if (i < m) {
#pragma unroll
          for (int t = 0; t < 32; ++t) {
            const int j = J * TM + c0 + t;
            if (j < m && i >= j) C[(size_t)j * ldc + i] -= (v[t] * si) * s_scale_j[c0 + t];
          }
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, TM);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (fn == nullptr) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

bool syrk_tc_supported(int fmt, int k) {
  if (fmt == FP16) return k > 0 && (k * 2) % BOX_BYTES == 0 && k <= 256;
  if (fmt == E4M3 || fmt == E5M2) return k > 0 && k % BOX_BYTES == 0 && k <= 256;
  return false;
}

cudaError_t launch_syrk_tc(float* C, int ldc, int m, int k, int fmt, const void* q, int ldq,
                           const int8_t* rowexp, const uint8_t* mxexp, int ldmx,
                           const int* prec_sel, DevStatus* st, cudaStream_t stream) {
  (void)mxexp; (void)ldmx;
  if (m <= 0) return cudaSuccess;
  if (!syrk_tc_supported(fmt, k)) return cudaErrorInvalidValue;
  auto encode = get_encode_fn();
  if (encode == nullptr) return cudaErrorNotSupported;
  const int esize = (fmt == FP16) ? 2 : 1;
  CUtensorMap map;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)m};
  cuuint64_t strides[1] = {(cuuint64_t)ldq * esize};
  cuuint32_t box[2] = {(cuuint32_t)(BOX_BYTES / esize), (cuuint32_t)TM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(&map, esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8,
                      2, const_cast<void*>(q), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const int nbox = (k * esize) / BOX_BYTES;
  const size_t smem = (size_t)2 * nbox * STRIP_CHUNK + 1024;
  const int T = ceil_div(m, TM);
  const int grid = T * (T + 1) / 2;
  cudaError_t e;
  switch (fmt) {
    case FP16:
      e = cudaFuncSetAttribute(syrk_tc_kernel<FP16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      syrk_tc_kernel<FP16><<<grid, 128, smem, stream>>>(map, C, ldc, m, k, rowexp, prec_sel, st);
      break;
    case E4M3:
      e = cudaFuncSetAttribute(syrk_tc_kernel<E4M3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      syrk_tc_kernel<E4M3><<<grid, 128, smem, stream>>>(map, C, ldc, m, k, rowexp, prec_sel, st);
      break;
    case E5M2:
      e = cudaFuncSetAttribute(syrk_tc_kernel<E5M2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      syrk_tc_kernel<E5M2><<<grid, 128, smem, stream>>>(map, C, ldc, m, k, rowexp, prec_sel, st);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace mpchol
