// Shared device/host helpers for the mpchol sm_100a library.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <stdint.h>

#include "../../include/mpchol.h"

namespace mpchol {

// Storage format ids match MPCHOL_PREC_*.
enum Fmt : int {
  FP32 = 0, FP16 = 1, E4M3 = 2, E5M2 = 3, MXFP8 = 4, SWITCHING = 5, FP16X2 = 6,
  MXFP6E2M3 = 7, MXFP6E3M2 = 8, MXFP4 = 9
};
constexpr int kNumFmts = 10;

// The OCP MX family: E8M0 scales per 32 elements along K with E4M3, E2M3,
// E3M2 or E2M1 elements.  The FP6/FP4 element values are exactly
// representable in E4M3, so they are stored as E4M3 codes of the same value
// and multiplied by the block-scaled E4M3 MMA -- the products are those of a
// native FP6/FP4 MMA (FP32 accumulation), the storage and speed are FP8's.
__host__ __device__ __forceinline__ bool is_mx(int f) {
  return f == MXFP8 || f == MXFP6E2M3 || f == MXFP6E3M2 || f == MXFP4;
}
struct MxElem {
  int mbits;    // stored mantissa bits
  int emin;     // exponent of the smallest normal binade (subnormal spacing 2^(emin - mbits))
  int emax;     // exponent of the largest binade (the OCP MX scale is floor(log2 amax) - emax)
  float maxv;   // largest finite value (saturation)
};
__host__ __device__ __forceinline__ MxElem mx_elem(int f) {
  switch (f) {
    case MXFP6E2M3: return {3, 0, 2, 7.5f};
    case MXFP6E3M2: return {2, -2, 4, 28.0f};
    case MXFP4: return {1, 0, 2, 6.0f};
    default: return {3, -6, 8, 448.0f};      // E4M3
  }
}

// Device-side status block shared by every kernel of one factor/solve.  A
// kernel that detects a failure (non-SPD pivot, exhausted bounded wait, bad
// index) records it here and returns; it never traps.
struct DevStatus {
  int code;        // mpchol_status (0 = OK)
  int row;         // failing global row for NOT_SPD, or diagnostic index
  int perturbed;   // number of floored pivots (diag_pert)
  int pad;
};

__device__ __forceinline__ void set_status(DevStatus* st, int code, int row) {
  if (atomicCAS(&st->code, 0, code) == 0) st->row = row;
}

// Exact 2^e as a float for e in [-149, 127] (subnormal results included).
__host__ __device__ __forceinline__ float pow2f(int e) {
  uint32_t bits;
  if (e >= -126) bits = (uint32_t)(e + 127) << 23;
  else bits = 1u << (e + 149);
#ifdef __CUDA_ARCH__
  return __uint_as_float(bits);
#else
  float f; memcpy(&f, &bits, 4); return f;
#endif
}

// floor(log2(a)) for finite a > 0 (subnormals included).
__device__ __forceinline__ int ilog2f_dev(float a) {
  const uint32_t u = __float_as_uint(a) & 0x7fffffffu;
  const int fexp = (int)(u >> 23);
  if (fexp > 0) return fexp - 127;
  return -126 - (__clz(u & 0x7fffffu) - 8) - 1;
}

// Per-row power-of-two scale exponent for a non-MX format: the smallest e
// with amax * 2^-e <= the format's largest finite value (no saturation).
__device__ __forceinline__ int row_scale_exp(float amax, int fmt) {
  if (!(amax > 0.0f) || isinf(amax)) return 0;
  int emax; uint32_t mmax;
  if (fmt == E4M3) { emax = 8; mmax = 0x600000u; }
  else if (fmt == E5M2) { emax = 15; mmax = 0x600000u; }
  else { emax = 15; mmax = 0x7fe000u; }           // FP16: 65504
  const int E = ilog2f_dev(amax);
  uint32_t u = __float_as_uint(amax) & 0x7fffffu;
  if (((__float_as_uint(amax) >> 23) & 0xff) == 0) {
    u <<= (__clz(u) - 8);                          // normalise subnormal mantissa
    u &= 0x7fffffu;
  }
  int e = E - emax + (u > mmax ? 1 : 0);
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return e;
}

// OCP MX shared exponent: floor(log2 amax) - emax of the element format
// (8 for E4M3), clamped to [-127, 127]; amax == 0 gives -127 (E8M0 code 0).
__device__ __forceinline__ int mx_scale_exp(float amax, int fmt = MXFP8) {
  if (!(amax > 0.0f) || isinf(amax)) return -127;
  int e = ilog2f_dev(amax) - mx_elem(fmt).emax;
  return e < -127 ? -127 : (e > 127 ? 127 : e);
}

// Round-to-nearest-even onto an FP6/FP4 element grid (OCP: no Inf/NaN codes,
// saturating at the largest value; NaN stays NaN).  a / q = a * 2^(mbits - e)
// and r * q are exact: q is a power of two and a lies far inside the FP32
// range.
__device__ __forceinline__ float mx_round_elem(float x, const MxElem& m) {
  const float a = fabsf(x);
  if (!(a == a)) return x;
  if (a >= m.maxv) return copysignf(m.maxv, x);
  int e = (a > 0.0f) ? ilog2f_dev(a) : m.emin;
  if (e < m.emin) e = m.emin;
  return copysignf(fminf(rintf(a * pow2f(m.mbits - e)) * pow2f(e - m.mbits), m.maxv), x);
}

// Hardware RNE + satfinite conversions (cvt.rn.satfinite.{e4m3,e5m2}x2.f32).
__device__ __forceinline__ uint8_t f32_to_e4m3(float x) {
  return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}
__device__ __forceinline__ uint8_t f32_to_e5m2(float x) {
  return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E5M2);
}
__device__ __forceinline__ uint16_t f32_to_f16(float x) {
  return __half_as_ushort(__float2half_rn(x));
}
// Two elements per conversion (low half / byte = a), rounded as the scalar
// forms above.
__device__ __forceinline__ uint32_t f32x2_to_f16x2(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ uint16_t f32x2_to_e4m3x2(float a, float b) {
  return (uint16_t)__nv_cvt_float2_to_fp8x2(make_float2(a, b), __NV_SATFINITE, __NV_E4M3);
}
__device__ __forceinline__ uint16_t f32x2_to_e5m2x2(float a, float b) {
  return (uint16_t)__nv_cvt_float2_to_fp8x2(make_float2(a, b), __NV_SATFINITE, __NV_E5M2);
}
// An MX-family element as its E4M3 code (two at a time): E4M3 directly,
// FP6/FP4 rounded onto their grid first (the rounded value is exact in E4M3)
__device__ __forceinline__ uint16_t mx_code_x2(float a, float b, int fmt) {
  if (fmt != MXFP8) {
    const MxElem m = mx_elem(fmt);
    a = mx_round_elem(a, m);
    b = mx_round_elem(b, m);
  }
  return f32x2_to_e4m3x2(a, b);
}

// Unit roundoff of each storage format (used by the switching criterion).
__host__ __device__ __forceinline__ float unit_roundoff(int fmt) {
  switch (fmt) {
    case E4M3: case MXFP8: case MXFP6E2M3: return 0.0625f;
    case MXFP6E3M2: return 0.125f;
    case MXFP4: return 0.25f;
    case E5M2: return 0.125f;
    case FP16: return 4.8828125e-4f;
    case FP16X2: return 2.3841858e-7f;   // hi + lo: 22 significant bits
    default: return 5.9604645e-8f;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace mpchol

#define MPCHOL_CUDA_TRY(expr)                                   \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) {                                    \
      mpchol::record_cuda_error(_e, #expr, __FILE__, __LINE__); \
      return MPCHOL_ERR_CUDA;                                   \
    }                                                           \
  } while (0)

namespace mpchol {
void record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
}
