// Step-precision decision and panel quantization.
//
// Replaces the reference's can_switch decision + host read of the result
// (src/kernels_macros.cuh:191-211, src/switching_chol.cuh:117-124) and its
// panel conversions convert_fp32_to_mxe4m3 / convert_transpose_fp32_to_mxe4m3
// (src/fp8_utils.cuh:27-130) and convertFloatToHalf (src/kernels_macros.cuh:115-124).
// The decision never leaves the device: the fused panel solve (trsm.cu)
// resolves it from its own statistics after a grid barrier and quantizes the
// panel with the tile routine of quant.cuh; this file keeps the stand-alone
// and batched quantizers.  The quantized panel is written K-major
// (row-major m x k) so TMA can stage it for the tensor-core update.
#include "common.cuh"
#include "kernels.cuh"
#include "quant.cuh"

namespace mpchol {
namespace {

__global__ void __launch_bounds__(QTHR)
quantize_rows_kernel(const float* __restrict__ P, int ldp, int m, int k, int fmt, void* q, int ldq,
                     int8_t* rowexp, uint8_t* mxexp, int ldmx) {
  extern __shared__ __align__(16) float qtile[];
  quantize_tile(P, ldp, m, k, fmt, q, ldq, rowexp, mxexp, ldmx, qtile, m, blockIdx.x * QROWS);
}

// Batched: blockIdx.y = system; its panel goes to rows q_row0.. of the
// panel arena (qrows rows per FP16X2 half), scales alongside.
__global__ void __launch_bounds__(QTHR)
quantize_batched_kernel(BatchSys* __restrict__ sys, const BatchStep* __restrict__ steps, int s,
                        int b, int fmt, void* q, int qrows, int8_t* rowexp, uint8_t* mxexp,
                        int diag_pert) {
  const BatchSys& S = sys[blockIdx.y];
  const BatchStep& T = steps[blockIdx.y];
  const int m = T.m;
  if (m <= 0 || (int)blockIdx.x * QROWS >= m || S.st->code != 0) return;
  extern __shared__ __align__(16) float qtile[];
  const int bs = b;                       // a step with rows below is a full block
  const float* P = S.A + (size_t)s * S.ld + s + bs;
  if (diag_pert) {
    const float u = unit_roundoff(fmt);
    for (int r = threadIdx.x; r < QROWS; r += QTHR) {
      const int gi = blockIdx.x * QROWS + r;
      if (gi < m) S.sh[s + bs + gi] = __fmaf_rn(u, S.rowsq[s + bs + gi], S.sh[s + bs + gi]);
    }
  }
  const size_t esz = (fmt == FP16 || fmt == FP16X2) ? 2 : 1;
  void* qs = reinterpret_cast<uint8_t*>(q) + (size_t)T.q_row0 * bs * esz;
  quantize_tile(P, S.ld, m, bs, fmt, qs, bs, rowexp + T.q_row0,
                mxexp ? mxexp + (size_t)T.q_row0 * (bs / 32) : nullptr, bs / 32, qtile, qrows, blockIdx.x * QROWS);
}

__global__ void quantize_elems_kernel(const float* __restrict__ x, void* q, long long count, int fmt) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i];
    if (fmt == FP16) reinterpret_cast<uint16_t*>(q)[i] = f32_to_f16(v);
    else if (fmt == E5M2) reinterpret_cast<uint8_t*>(q)[i] = f32_to_e5m2(v);
    else reinterpret_cast<uint8_t*>(q)[i] = f32_to_e4m3(v);
  }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long h, unsigned long long v) {
  return h ^ (v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2));
}

// One warp per chunk of raw bit patterns: lanes convert 32 consecutive
// patterns at a time, lane 0 folds them in order (the hash is sequential).
__global__ void quantize_hash_kernel(unsigned long long first, unsigned long long count,
                                     unsigned long long chunk, int fmt, unsigned long long* hashes) {
  const int lane = threadIdx.x & 31;
  const long long nch = (long long)((count + chunk - 1) / chunk);
  const long long warp_g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long c = warp_g; c < nch; c += nwarps) {
    const unsigned long long lo = first + (unsigned long long)c * chunk;
    unsigned long long hi = lo + chunk;
    if (hi > first + count) hi = first + count;
    unsigned long long h = 0;
    for (unsigned long long b0 = lo; b0 < hi; b0 += 32) {
      const unsigned long long b = b0 + lane;
      unsigned int qv = 0;
      if (b < hi) {
        const float x = __uint_as_float((unsigned int)b);
        if (fmt == FP16) qv = f32_to_f16(x);
        else if (fmt == E5M2) qv = f32_to_e5m2(x);
        else qv = f32_to_e4m3(x);
        if (isnan(x)) qv = 0xffffu;
        else if (isinf(x)) qv = 0xfffeu;
      }
      const int nvalid = (int)min(32ull, hi - b0);
      for (int l = 0; l < nvalid; ++l) {
        const unsigned int ql = __shfl_sync(0xffffffffu, qv, l);
        h = mix64(h, ql);
      }
    }
    if (lane == 0) hashes[c] = h;
  }
}

size_t qtile_smem(int k) { return (size_t)k * (QROWS + 1) * sizeof(float); }

}  // namespace

cudaError_t launch_quantize_rows(const float* P, int ldp, int m, int k, int fmt, void* q, int ldq,
                                 int8_t* rowexp, uint8_t* mxexp, int ldmx, cudaStream_t stream) {
  if (m <= 0) return cudaSuccess;
  const size_t smem = qtile_smem(k);
  cudaError_t e = cudaFuncSetAttribute(quantize_rows_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  quantize_rows_kernel<<<ceil_div(m, QROWS), QTHR, smem, stream>>>(P, ldp, m, k, fmt, q, ldq, rowexp,
                                                                   mxexp, ldmx);
  return cudaGetLastError();
}

cudaError_t launch_quantize_elems(const float* x, void* q, long long count, int fmt,
                                  cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  long long blocks = (count + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  quantize_elems_kernel<<<(int)blocks, 256, 0, stream>>>(x, q, count, fmt);
  return cudaGetLastError();
}

cudaError_t launch_quantize_hash(unsigned long long first, unsigned long long count,
                                 unsigned long long chunk, int fmt, unsigned long long* hashes,
                                 cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  const long long nch = (long long)((count + chunk - 1) / chunk);
  long long blocks = (nch * 32 + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  quantize_hash_kernel<<<(int)blocks, 256, 0, stream>>>(first, count, chunk, fmt, hashes);
  return cudaGetLastError();
}

cudaError_t launch_quantize_batched(BatchSys* sys, const BatchStep* steps, int nact, int s, int b,
                                    int max_m, int fmt, void* q, int qrows, int8_t* rowexp,
                                    uint8_t* mxexp, int diag_pert, cudaStream_t stream) {
  if (nact <= 0 || max_m <= 0) return cudaSuccess;
  const size_t smem = qtile_smem(b);
  cudaError_t e = cudaFuncSetAttribute(quantize_batched_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  quantize_batched_kernel<<<dim3(ceil_div(max_m, QROWS), nact), QTHR, smem, stream>>>(
      sys, steps, s, b, fmt, q, qrows, rowexp, mxexp, diag_pert);
  return cudaGetLastError();
}

}  // namespace mpchol
