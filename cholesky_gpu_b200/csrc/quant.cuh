// Step-precision resolution and the panel quantizer shared by the quantize
// kernels (quant.cu) and the fused panel solve (trsm.cu).
#pragma once
#include "common.cuh"
#include "kernels.cuh"

namespace mpchol {

constexpr int QROWS = 32;    // rows per CTA
constexpr int QTHR = 256;

__device__ __forceinline__ int resolve_precision(const StepState* step, const DecisionParams& dp) {
  if (dp.policy != SWITCHING) return dp.policy;
  if (dp.switch_mode == 1) {
    const int code = step->literal_code;            // 2 - min choice index
    const int choice = 2 - code;
    return choice == 0 ? FP32 : (choice == 1 ? FP16 : E4M3);
  }
  const float ratio = __uint_as_float(step->max_ratio_bits);
  const float coh = dp.coherence ? __uint_as_float(step->coh_bits) : 0.0f;
  for (int k = 0; k < dp.ladder_len; ++k) {
    const int p = dp.ladder[k];
    const float u = unit_roundoff(p);
    if (u * ratio <= dp.eps_prime && u * coh <= dp.eps_coh) return p;
  }
  // no entry meets the bound: the ladder's most precise (last) entry
  return dp.ladder_len > 0 ? dp.ladder[dp.ladder_len - 1] : FP32;
}

// Quantize one tile of QROWS rows (starting at row0) x k columns with QTHR
// threads.  Lane l of a warp owns the
// contiguous columns [l*c, (l+1)*c), c = k/32 (k is a multiple of 32, <= 256).
// lo_rows: rows from a row of the FP16X2 hi panel to the same row of the lo
// panel (m for a single panel; the arena height for batched panels).
__device__ inline void quantize_tile(const float* __restrict__ P, int ldp, int m, int k, int fmt,
                                     void* q, int ldq, int8_t* rowexp, uint8_t* mxexp, int ldmx,
                                     float* tile, int lo_rows, int row0) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nr = min(QROWS, m - row0);
  // stage the rows (coalesced column reads, 16 loads in flight per thread
  // before their shared-memory stores), padded stride QROWS+1
  constexpr int B = 16;
  for (int e0 = tid; e0 < k * QROWS; e0 += B * QTHR) {
    float vv[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int e = e0 + u * QTHR;
      const int c = e / QROWS, r = e % QROWS;
      vv[u] = (e < k * QROWS && r < nr) ? P[(size_t)c * ldp + row0 + r] : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int e = e0 + u * QTHR;
      if (e < k * QROWS) tile[(e / QROWS) * (QROWS + 1) + e % QROWS] = vv[u];
    }
  }
  __syncthreads();
  const int cpl = k / 32;                   // columns per lane
  for (int r = warp; r < nr; r += QTHR / 32) {
    const int gi = row0 + r;
    float v[8];
    float amax = 0.0f;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      v[t] = (t < cpl) ? tile[(lane * cpl + t) * (QROWS + 1) + r] : 0.0f;
      amax = fmaxf(amax, fabsf(v[t]));
    }
    if (is_mx(fmt)) {
      // one E8M0 scale per 32 consecutive columns = 32/cpl lanes
      const int lpb = 32 / cpl;
      float bmax = amax;
      for (int o = 1; o < lpb; o <<= 1) bmax = fmaxf(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
      const int e = mx_scale_exp(bmax, fmt);
      const float inv = pow2f(-e);
      uint8_t* qr = reinterpret_cast<uint8_t*>(q) + (size_t)gi * ldq + lane * cpl;
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < cpl) qr[t] = (uint8_t)mx_code_x2(v[t] * inv, 0.0f, fmt);
      if ((lane % lpb) == 0) mxexp[(size_t)gi * ldmx + lane / lpb] = (uint8_t)(e + 127);
    } else {
      const float rmax = warp_max(amax);
      const int e = row_scale_exp(rmax, fmt);
      const float inv = pow2f(-e);
      if (fmt == FP16) {
        uint16_t* qr = reinterpret_cast<uint16_t*>(q) + (size_t)gi * ldq + lane * cpl;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (t < cpl) qr[t] = f32_to_f16(v[t] * inv);
      } else if (fmt == FP16X2) {
        // hi = fp16(x), lo = fp16(x - hi); x - hi is exact in FP32.  The lo
        // panel follows the hi panel (lo_rows rows further on).
        uint16_t* qh = reinterpret_cast<uint16_t*>(q) + (size_t)gi * ldq + lane * cpl;
        uint16_t* ql = qh + (size_t)lo_rows * ldq;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (t < cpl) {
            const float xs = v[t] * inv;
            const __half h = __float2half_rn(xs);
            qh[t] = __half_as_ushort(h);
            ql[t] = f32_to_f16(xs - __half2float(h));
          }
      } else {
        uint8_t* qr = reinterpret_cast<uint8_t*>(q) + (size_t)gi * ldq + lane * cpl;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (t < cpl) qr[t] = (fmt == E4M3) ? f32_to_e4m3(v[t] * inv) : f32_to_e5m2(v[t] * inv);
      }
      if (lane == 0) rowexp[gi] = (int8_t)e;
    }
  }
}


}  // namespace mpchol
