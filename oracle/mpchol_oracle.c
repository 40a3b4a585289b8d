/*
 * mpchol CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm for the mixed-precision
 * blocked Cholesky preconditioner (SudhanvaKulkarni123/Cholesky_GPU).  It is
 * the checker for the CUDA library: only tests/, the smoke check and the CPU
 * baseline leg of bench.py load it.  The shipped library never links it.
 *
 * Parity is pinned by tests/golden/ (vectors produced by the reference's own
 * lo_float.h, built by oracle/Makefile into oracle/_ref/) for the number
 * formats, and by an FP64 dense Cholesky solve for factor/solution quality.
 *
 * Reference anchors (paths inside the reference project):
 *   float -> 8-bit conversion   src/lo_float.h:1896-1910 (RNE bias add),
 *                               src/lo_float.h:1960-2120 (ConvertImpl::run)
 *   e4m3fn / e5m2 limits        src/lo_float.h:789-846, 962-1024
 *   MX E8M0 scale intent        src/fp8_utils.cuh:7-13, 27-66
 *   unblocked POTRF             src/micro_chol.hpp:14-44
 *   blocked right-looking order src/sChol.cuh:222-311 (potrf -> trsm RIGHT/LOWER/T -> C -= X X^T)
 *   diagonal tracker            src/kernels_macros.cuh:177-190 (update_diag)
 *   precision choice            src/kernels_macros.cuh:191-211 (can_switch),
 *                               src/switching_chol.cuh:5-15, 117-122
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Format ids shared with include/mpchol.h (MPCHOL_PREC_*). */
enum { ORC_FP32 = 0, ORC_FP16 = 1, ORC_E4M3 = 2, ORC_E5M2 = 3, ORC_MXFP8 = 4, ORC_SWITCHING = 5,
       ORC_FP16X2 = 6, ORC_MXFP6E2M3 = 7, ORC_MXFP6E3M2 = 8, ORC_MXFP4 = 9 };
static int orc_is_mx(int p) {
  return p == ORC_MXFP8 || p == ORC_MXFP6E2M3 || p == ORC_MXFP6E3M2 || p == ORC_MXFP4;
}

static inline uint32_t f2u(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static inline float u2f(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

/* Round-to-nearest-even by bias add before truncating `roundoff` low bits
 * (src/lo_float.h:1896-1910). */
static inline uint32_t rne_bias(uint32_t bits, int roundoff) {
  if (roundoff <= 0) return bits;
  uint32_t bias = ((bits >> roundoff) & 1u) + (1u << (roundoff - 1)) - 1u;
  return bits + bias;
}

/*
 * Float32 -> small float with `ebits` exponent bits, `mbits` mantissa bits,
 * exponent bias `bias`; `max_rep` is the code of the largest finite magnitude,
 * `inf_rep` the code lo_float returns for +-infinity, `nan_rep` its NaN code.
 * saturate != 0 clamps finite overflow to max_rep (lo_float kSaturate=true),
 * otherwise finite overflow gives inf_rep.
 * Follows the structure of ConvertImpl::run for a narrower target
 * (src/lo_float.h:1960-2120): specials, target-subnormal path with re-rounding
 * from the original bits, normal path with RNE, re-bias and overflow check.
 */
static uint32_t orc_f32_to_small(float x, int ebits, int mbits, int bias, uint32_t max_rep,
                                 uint32_t inf_rep, uint32_t nan_rep, int saturate) {
  const int total_bits = 1 + ebits + mbits;
  const uint32_t sign = f2u(x) >> 31;
  const uint32_t a = f2u(x) & 0x7fffffffu;
  const uint32_t sbit = sign << (total_bits - 1);
  if (a == 0x7f800000u) return sbit | inf_rep;         /* +-inf */
  if (a > 0x7f800000u) return nan_rep;                 /* NaN */
  if (a == 0) return sbit;                              /* +-0 */
  const int digit_shift = 23 - mbits;                   /* mantissa bits dropped */
  const int fexp = (int)(a >> 23);
  const int texp = fexp - 127 + bias;                   /* biased target exponent */
  if (texp <= 0) {
    /* target subnormal (or zero) */
    const uint32_t lead = fexp > 0 ? 1u : 0u;
    const int shift = digit_shift - texp + (int)lead;
    uint32_t mant = (a & 0x7fffffu) | (lead << 23);
    uint32_t bits = 0;
    if (shift <= 24) {
      mant = rne_bias(mant, shift);
      bits = mant >> shift;
    }
    return sbit | bits;
  }
  uint32_t r = rne_bias(a, digit_shift);
  r &= ~((1u << digit_shift) - 1u);
  r -= (uint32_t)(127 - bias) << 23;                    /* re-bias exponent */
  const uint32_t aligned_max = max_rep << digit_shift;
  if (r > aligned_max) return sbit | (saturate ? max_rep : inf_rep);
  return sbit | (r >> digit_shift);
}

/* E4M3 (fn): bias 7, max 448 = 0x7E; lo_float's "infinity" is 0x7F, NaN 0x80. */
uint8_t orc_f32_to_e4m3(float x, int saturate) {
  return (uint8_t)orc_f32_to_small(x, 4, 3, 7, 0x7e, 0x7f, 0x80, saturate);
}
/* E5M2: bias 15, max 57344 = 0x7B, inf 0x7C, quiet NaN 0x7E. */
uint8_t orc_f32_to_e5m2(float x, int saturate) {
  return (uint8_t)orc_f32_to_small(x, 5, 2, 15, 0x7b, 0x7c, 0x7e, saturate);
}
/* IEEE binary16 with RNE; overflow -> inf (the __float2half convention). */
uint16_t orc_f32_to_f16(float x) {
  return (uint16_t)orc_f32_to_small(x, 5, 10, 15, 0x7bff, 0x7c00, 0x7e00, 0);
}

/* Decode helpers (used by the oracle's own arithmetic). */
float orc_e4m3_to_f32(uint8_t c) {
  const int s = c >> 7, e = (c >> 3) & 0xf, m = c & 7;
  if (e == 0xf && m == 7) return NAN;
  float v = e == 0 ? ldexpf((float)m, -9) : ldexpf(1.0f + m / 8.0f, e - 7);
  return s ? -v : v;
}
float orc_e5m2_to_f32(uint8_t c) {
  const int s = c >> 7, e = (c >> 2) & 0x1f, m = c & 3;
  float v;
  if (e == 0x1f) v = m ? NAN : INFINITY;
  else v = e == 0 ? ldexpf((float)m, -16) : ldexpf(1.0f + m / 4.0f, e - 15);
  return s ? -v : v;
}
float orc_f16_to_f32(uint16_t c) {
  const int s = c >> 15, e = (c >> 10) & 0x1f, m = c & 0x3ff;
  float v;
  if (e == 0x1f) v = m ? NAN : INFINITY;
  else v = e == 0 ? ldexpf((float)m, -24) : ldexpf(1.0f + m / 1024.0f, e - 15);
  return s ? -v : v;
}

/* floor(log2(|x|)) for finite nonzero x, exact for subnormals. */
static int ilog2f(float x) {
  const uint32_t a = f2u(x) & 0x7fffffffu;
  const int fexp = (int)(a >> 23);
  if (fexp > 0) return fexp - 127;
  int lz = __builtin_clz(a & 0x7fffffu);               /* a != 0 */
  return -126 - (lz - 8) - 1;
}

/*
 * Power-of-two row scale for a non-MX format: the smallest integer e with
 * amax * 2^-e <= largest finite value of the format (so no element saturates),
 * clamped so 2^e and 2^-e stay normal floats.  amax == 0 gives e = 0.
 */
int orc_row_scale_exp(float amax, int fmt) {
  if (!(amax > 0.0f) || isinf(amax)) return 0;
  int emax; uint32_t mmax_bits;                         /* max finite = (1.m) * 2^emax */
  switch (fmt) {
    case ORC_E4M3: emax = 8; mmax_bits = 0x600000u; break;    /* 1.75 * 2^8  = 448   */
    case ORC_E5M2: emax = 15; mmax_bits = 0x600000u; break;   /* 1.75 * 2^15 = 57344 */
    case ORC_FP16: case ORC_FP16X2: emax = 15; mmax_bits = 0x7fe000u; break;   /* 65504 */
    default: return 0;
  }
  const int E = ilog2f(amax);
  uint32_t mant;
  if (((f2u(amax) >> 23) & 0xff) == 0) {
    /* subnormal amax: normalise mantissa */
    uint32_t a = f2u(amax) & 0x7fffffu;
    while (!(a & 0x800000u)) a <<= 1;
    mant = a & 0x7fffffu;
  } else {
    mant = f2u(amax) & 0x7fffffu;
  }
  int e = E - emax + (mant > mmax_bits ? 1 : 0);
  if (e < -126) e = -126;
  if (e > 127) e = 127;
  return e;
}

/*
 * OCP MX shared exponent for one 32-element block with E4M3 elements:
 * floor(log2(amax)) - 8, clamped to the E8M0 range [-127, 127]; amax == 0 gives
 * -127.  The reference's intent is src/fp8_utils.cuh:7-13 (frexp -> biased
 * exponent, clamp to [0,255]); the E8M0 code is exp + 127.
 */
int orc_mx_scale_exp(float amax) {
  if (!(amax > 0.0f) || isinf(amax)) return -127;
  int e = ilog2f(amax) - 8;
  if (e < -127) e = -127;
  if (e > 127) e = 127;
  return e;
}

static inline float pow2f(int e) {
  /* exact 2^e for e in [-149, 127] */
  return ldexpf(1.0f, e);
}

/* The OCP MX element formats with FP6/FP4 elements (OCP Microscaling
 * Formats spec v1.0, element types E2M3, E3M2, E2M1): stored mantissa bits,
 * smallest normal exponent, largest exponent (the block scale is
 * floor(log2 amax) - emax) and largest value. */
static void orc_mx_elem(int p, int* mbits, int* emin, int* emax, float* maxv) {
  switch (p) {
    case ORC_MXFP6E2M3: *mbits = 3; *emin = 0; *emax = 2; *maxv = 7.5f; break;
    case ORC_MXFP6E3M2: *mbits = 2; *emin = -2; *emax = 4; *maxv = 28.0f; break;
    case ORC_MXFP4: *mbits = 1; *emin = 0; *emax = 2; *maxv = 6.0f; break;
    default: *mbits = 3; *emin = -6; *emax = 8; *maxv = 448.0f; break;   /* E4M3 */
  }
}

/* MX shared exponent of a block for element format p. */
int orc_mx_scale_exp_fmt(float amax, int p) {
  int mb, en, ex; float mv;
  orc_mx_elem(p, &mb, &en, &ex, &mv);
  if (!(amax > 0.0f) || isinf(amax)) return -127;
  int e = ilog2f(amax) - ex;
  if (e < -127) e = -127;
  if (e > 127) e = 127;
  return e;
}

/* Round to nearest even onto an FP6/FP4 element grid, saturating at the
 * largest value; NaN stays NaN (the formats have no Inf/NaN codes: OCP).
 * The steps of lo_float's ConvertImpl (src/lo_float.h:1960-2120) restricted
 * to these targets: the quantum of x's binade (or of the subnormal range)
 * and RNE of x to a multiple of it.  E4M3 (p = MXFP8) goes through the
 * E4M3 conversion. */
float orc_mx_round(float x, int p) {
  if (p == ORC_MXFP8 || p == ORC_E4M3) return orc_e4m3_to_f32(orc_f32_to_e4m3(x, 1));
  int mb, en, ex; float mv;
  orc_mx_elem(p, &mb, &en, &ex, &mv);
  const float a = fabsf(x);
  if (a != a) return x;
  if (a >= mv) return copysignf(mv, x);
  int e = a > 0.0f ? ilog2f(a) : en;
  if (e < en) e = en;
  const float q = pow2f(e - mb);
  float r = rintf(a / q) * q;          /* exact: q is a power of two; rintf is RNE */
  if (r > mv) r = mv;
  return copysignf(r, x);
}

/* Quantize `count` floats (already scaled) to format `fmt`; used by tests. */
void orc_quantize(const float* x, void* out, long long count, int fmt) {
  for (long long i = 0; i < count; ++i) {
    if (fmt == ORC_E4M3) ((uint8_t*)out)[i] = orc_f32_to_e4m3(x[i], 1);
    else if (fmt == ORC_E5M2) ((uint8_t*)out)[i] = orc_f32_to_e5m2(x[i], 1);
    else if (fmt == ORC_FP16) ((uint16_t*)out)[i] = orc_f32_to_f16(x[i]);
  }
}

/* Same quantization over a contiguous range of raw bit patterns, folded into
 * a 64-bit hash per chunk of `chunk` inputs.  The GPU exhaustive sweep
 * computes the identical hash so 2^32 codes can be compared as 256 words. */
static inline uint64_t mix64(uint64_t h, uint64_t v) {
  h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  return h;
}
void orc_quantize_hash(uint64_t first, uint64_t count, uint64_t chunk, int fmt, uint64_t* hashes) {
  const long long nch = (long long)((count + chunk - 1) / chunk);
#pragma omp parallel for schedule(dynamic, 1)
  for (long long c = 0; c < nch; ++c) {
    uint64_t h = 0;
    const uint64_t lo = first + (uint64_t)c * chunk;
    uint64_t hi = lo + chunk;
    if (hi > first + count) hi = first + count;
    for (uint64_t b = lo; b < hi; ++b) {
      const float x = u2f((uint32_t)b);
      uint32_t q;
      if (fmt == ORC_E4M3) q = orc_f32_to_e4m3(x, 1);
      else if (fmt == ORC_E5M2) q = orc_f32_to_e5m2(x, 1);
      else q = orc_f32_to_f16(x);
      /* Non-finite inputs are compared by class only (lo_float returns its
       * own "infinity"/NaN codes, hardware satfinite returns +-max and the
       * OCP NaN): fold a fixed token per class. */
      if (isnan(x)) q = 0xffffu;
      else if (isinf(x)) q = 0xfffeu;
      h = mix64(h, q);
    }
    hashes[c] = h;
  }
}

/* ------------------------------------------------------------------------ */
/* Blocked mixed-precision Cholesky restatement                              */
/* ------------------------------------------------------------------------ */

typedef struct {
  int block_size;
  int precision;        /* ORC_* policy */
  float eps_prime;
  float floor_ratio;    /* near-indefinite threshold on dtilde/d (flags FP64 diag) */
  int diag_pert;        /* 1: shift pivots by pert * rounding estimate, floor them */
  float pert;           /* shift multiplier */
  float pivot_floor;    /* with diag_pert: pivots <= pivot_floor * d_i are raised to it */
  int switch_mode;      /* 0: build criterion, 1: reference-literal can_switch */
  int ladder_len;       /* switching ladder, lowest precision first */
  int ladder[4];
  const int* force_prec;   /* nullable: per-step precision override */
  const int* force_fp64;   /* nullable: per-step FP64 diag override */
  int coherence;        /* switch_mode 0: also require u_p * coh <= eps_coh */
  int equilibrate;      /* 1: factor D A D, D = diag(2^-e_i), then unscale L's rows */
  float eps_coherence;  /* the coherence threshold; 0: eps' */
} orc_chol_opts;

typedef struct {
  int status;           /* 0 ok, 2 not SPD */
  int fail_row;
  int n_perturbed;
  int nsteps;
} orc_chol_info;

float orc_unit_roundoff(int fmt) {
  switch (fmt) {
    case ORC_E4M3: case ORC_MXFP8: case ORC_MXFP6E2M3: return 0.0625f;    /* 2^-4 */
    case ORC_MXFP6E3M2: return 0.125f;                 /* 2^-3 */
    case ORC_MXFP4: return 0.25f;                      /* 2^-2 */
    case ORC_E5M2: return 0.125f;                     /* 2^-3 */
    case ORC_FP16: return 4.8828125e-4f;               /* 2^-11 */
    case ORC_FP16X2: return 2.3841858e-7f;             /* 2^-22: hi + lo */
    default: return 5.9604645e-8f;                    /* 2^-24 */
  }
}

/* Machine epsilons the reference compares against (src/switching_chol.cuh:5-8). */
static float ref_mach_eps(int fmt) {
  switch (fmt) {
    case ORC_E4M3: case ORC_MXFP8: return 0.125f;
    case ORC_FP16: return 0.0009765625f;
    default: return 1.1920929e-7f;
  }
}

/*
 * Step precision choice.  mode 0 (build criterion): the first ladder entry p
 * (lowest precision first) with u_p * max_i d_i / dtilde_i <= eps_prime over
 * the trailing rows -- and, with the coherence rule, u_p * coh <= eps_prime,
 * coh = (||P^T 1||^2 / m) / min_i dtilde_i (orc_coherence_ratio) -- the last
 * (most precise) entry if none.  mode 1 (reference-literal): per row, the
 * first entry of the reference list {FP32, FP16, E4M3} with
 * mach_eps_p * dtilde_i >= eps_prime * d_i (src/kernels_macros.cuh:191-211);
 * rows with no match choose FP32; the step takes the most precise row choice.
 */
/* Coherence ratio of a solved panel P (m x bs, column-major, ld lda) with
 * the Schur diagonal dt after the step: (||P^T 1||^2 / m) / min_i dt_i, +inf
 * when some dt_i <= 0.  The column sums are formed as the GPU forms them: a
 * float sum per 32-row slab, column c's rows taken from row c % 32 on, and the
 * slab sums added in double. */
float orc_coherence_ratio(const float* P, int lda, int m, int bs, const float* dt) {
  if (m <= 0) return 0.0f;
  float mind = INFINITY;
  for (int i = 0; i < m; ++i) mind = dt[i] > 0.0f ? (dt[i] < mind ? dt[i] : mind) : 0.0f;
  double c2 = 0.0;
  for (int c = 0; c < bs; ++c) {
    double cs = 0.0;
    for (int r0 = 0; r0 < m; r0 += 32) {
      const int nr = m - r0 < 32 ? m - r0 : 32;
      float part = 0.0f;
      for (int q = 0; q < 32; ++q) {
        const int r = (q + c) & 31;
        part += r < nr ? P[(size_t)c * lda + r0 + r] : 0.0f;
      }
      cs += (double)part;
    }
    c2 += cs * cs;
  }
  if (!(mind > 0.0f)) return INFINITY;
  const float coh = (float)((c2 / (double)m) / (double)mind);
  return coh != coh ? INFINITY : coh;
}

int orc_choose_precision(const float* d, const float* dt, int m, float coh, const orc_chol_opts* o) {
  if (m <= 0) return ORC_FP32;
  if (o->switch_mode == 1) {
    const int list[3] = {ORC_FP32, ORC_FP16, ORC_E4M3};
    int best = 2;
    for (int i = 0; i < m; ++i) {
      int pick = 0;
      for (int p = 0; p < 3; ++p) {
        if (ref_mach_eps(list[p]) * dt[i] >= o->eps_prime * d[i]) { pick = p; break; }
      }
      if (pick < best) best = pick;
    }
    return list[best];
  }
  float ratio = 0.0f;
  for (int i = 0; i < m; ++i) {
    float r = dt[i] > 0.0f ? d[i] / dt[i] : INFINITY;
    if (!(r <= ratio)) ratio = r;
  }
  for (int k = 0; k < o->ladder_len; ++k) {
    const int p = o->ladder[k];
    const float u = orc_unit_roundoff(p);
    const float ec = o->eps_coherence > 0.0f ? o->eps_coherence : o->eps_prime;
    if (u * ratio <= o->eps_prime && (!o->coherence || u * coh <= ec)) return p;
  }
  return o->ladder_len > 0 ? o->ladder[o->ladder_len - 1] : ORC_FP32;
}

/* Unblocked right-looking POTRF of an nb x nb column-major block (lower),
 * src/micro_chol.hpp:23-40, in float or double.  Returns -1 on success or the
 * failing local row.  With pivmin != NULL, pivots at or below pivmin[j] are
 * replaced by pivmin[j] (diagonal perturbation) and counted. */
#define DEFINE_POTRF(NAME, T, SQRT)                                                   \
  static int NAME(T* a, int nb, int ld, const T* shift, const T* pivmin, int* nperturbed) { \
    for (int k = 0; k < nb; ++k) {                                                    \
      T piv = a[k + (size_t)k * ld];                                                  \
      if (shift) piv += shift[k];                                                     \
      if (!(piv - piv == 0)) return k; /* NaN / inf: overflowed, not repairable */    \
      if (pivmin) {                                                                   \
        if (!(piv > pivmin[k])) { /* max(|piv|, floor): fixDiag, src/kernels_macros.cuh:90-99 */ \
          const T ap = piv < 0 ? -piv : piv;                                          \
          piv = (ap > pivmin[k]) ? ap : pivmin[k];                                    \
          ++*nperturbed;                                                              \
        }                                                                             \
      } else if (!(piv > 0)) {                                                        \
        return k;                                                                     \
      }                                                                               \
      const T lkk = SQRT(piv);                                                        \
      a[k + (size_t)k * ld] = lkk;                                                    \
      for (int i = k + 1; i < nb; ++i) a[i + (size_t)k * ld] /= lkk;                  \
      for (int j = k + 1; j < nb; ++j) {                                              \
        const T ljk = a[j + (size_t)k * ld];                                          \
        for (int i = j; i < nb; ++i) a[i + (size_t)j * ld] -= a[i + (size_t)k * ld] * ljk; \
      }                                                                               \
    }                                                                                 \
    return -1;                                                                        \
  }
DEFINE_POTRF(potrf_f32, float, sqrtf)
DEFINE_POTRF(potrf_f64, double, sqrt)

/* The reference's CPU path restated (src/micro_chol.hpp:14-44): unblocked,
 * single thread, column-major lower.  Returns 0, or 1 + failing row. */
int orc_micro_cholesky(float* A, int n, int ld) {
  int k = potrf_f32(A, n, ld, NULL, NULL, NULL);
  return k < 0 ? 0 : k + 1;
}

/* Quantize one panel row (length bs, stride ld) in format p with a per-row
 * (or, for MXFP8, per-32-block) power-of-two scale; returns dequantized
 * values (exact products of code value and scale) in out[]. */
static void quant_row(const float* row, int ld, int bs, int p, float* out) {
  if (orc_is_mx(p)) {
    for (int kb = 0; kb < bs; kb += 32) {
      const int ke = kb + 32 < bs ? kb + 32 : bs;
      float amax = 0.0f;
      for (int k = kb; k < ke; ++k) { float v = fabsf(row[(size_t)k * ld]); if (v > amax) amax = v; }
      const int e = orc_mx_scale_exp_fmt(amax, p);
      const float inv = pow2f(-e), sc = pow2f(e);
      for (int k = kb; k < ke; ++k) out[k] = orc_mx_round(row[(size_t)k * ld] * inv, p) * sc;
    }
    return;
  }
  float amax = 0.0f;
  for (int k = 0; k < bs; ++k) { float v = fabsf(row[(size_t)k * ld]); if (v > amax) amax = v; }
  const int e = orc_row_scale_exp(amax, p);
  const float inv = pow2f(-e), sc = pow2f(e);
  for (int k = 0; k < bs; ++k) {
    const float v = row[(size_t)k * ld] * inv;
    float q;
    if (p == ORC_E4M3) q = orc_e4m3_to_f32(orc_f32_to_e4m3(v, 1));
    else if (p == ORC_E5M2) q = orc_e5m2_to_f32(orc_f32_to_e5m2(v, 1));
    else if (p == ORC_FP16X2) {
      /* two-term split: hi = fp16(v), lo = fp16(v - hi); the update uses
       * hi hi^T + hi lo^T + lo hi^T, i.e. (hi+lo)(hi+lo)^T - lo lo^T; the
       * dropped lo lo^T term is below the FP32 accumulation error, so the
       * oracle uses hi + lo */
      const float hi = orc_f16_to_f32(orc_f32_to_f16(v));
      const float lo = orc_f16_to_f32(orc_f32_to_f16(v - hi));
      q = hi + lo;
    }
    else q = orc_f16_to_f32(orc_f32_to_f16(v));
    out[k] = q * sc;
  }
}

/*
 * Blocked right-looking factorisation, in place on the lower triangle of the
 * column-major n x n matrix A (ld = lda).  d[] holds the original diagonal,
 * dt[] the running Schur-complement diagonal (initialised to d by the caller);
 * sh[] (nullable) accumulates the per-row rounding-shift estimate.
 * step_prec / step_fp64 (length ceil(n/b), nullable) receive the per-step
 * choices.  Structure per step follows src/sChol.cuh:222-311 with the
 * switching additions of src/switching_chol.cuh:76-221.
 */
int orc_blocked_chol(float* A, int n, int lda, const float* d, float* dt, float* sh,
                     const orc_chol_opts* o, int* step_prec, int* step_fp64, orc_chol_info* info) {
  const int b = o->block_size;
  const int nsteps = (n + b - 1) / b;
  info->status = 0; info->fail_row = -1; info->n_perturbed = 0; info->nsteps = nsteps;
  int next_fp64 = 0;
  float* qbuf = (float*)malloc(sizeof(float) * (size_t)b * (size_t)(n > 0 ? n : 1));
  double* blk64 = (double*)malloc(sizeof(double) * (size_t)b * b);
  float* shiftf = (float*)malloc(sizeof(float) * b);
  float* pminf = (float*)malloc(sizeof(float) * b);
  double* shiftd = (double*)malloc(sizeof(double) * b);
  double* pmind = (double*)malloc(sizeof(double) * b);
  for (int k = 0; k < nsteps; ++k) {
    const int s = k * b;
    const int bs = n - s < b ? n - s : b;
    const int m = n - s - bs;
    float* D = A + s + (size_t)s * lda;
    /* 1. diagonal block POTRF (FP64 when flagged near-indefinite) */
    int use64 = o->force_fp64 ? o->force_fp64[k] : next_fp64;
    if (step_fp64) step_fp64[k] = use64;
    for (int j = 0; j < bs; ++j) {
      shiftf[j] = (o->diag_pert && sh) ? o->pert * sh[s + j] : 0.0f;
      pminf[j] = o->pivot_floor * d[s + j];
      shiftd[j] = shiftf[j];
      pmind[j] = pminf[j];
    }
    int fail;
    if (use64) {
      for (int j = 0; j < bs; ++j)
        for (int i = j; i < bs; ++i) blk64[i + (size_t)j * bs] = D[i + (size_t)j * lda];
      fail = potrf_f64(blk64, bs, bs, o->diag_pert ? shiftd : NULL, o->diag_pert ? pmind : NULL,
                       &info->n_perturbed);
      for (int j = 0; j < bs; ++j)
        for (int i = j; i < bs; ++i) D[i + (size_t)j * lda] = (float)blk64[i + (size_t)j * bs];
    } else {
      fail = potrf_f32(D, bs, lda, o->diag_pert ? shiftf : NULL, o->diag_pert ? pminf : NULL,
                       &info->n_perturbed);
    }
    if (fail >= 0) { info->status = 2; info->fail_row = s + fail; break; }
    if (m == 0) { if (step_prec) step_prec[k] = ORC_FP32; break; }
    /* 2. panel TRSM: X = A21 * L11^-T (RIGHT, LOWER, TRANS, NON_UNIT) */
    float* P = A + s + bs + (size_t)s * lda;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m; ++i) {
      for (int j = 0; j < bs; ++j) {
        float acc = P[i + (size_t)j * lda];
        for (int l = 0; l < j; ++l) acc -= P[i + (size_t)l * lda] * D[j + (size_t)l * lda];
        P[i + (size_t)j * lda] = acc / D[j + (size_t)j * lda];
      }
    }
    /* 3. Schur-complement diagonal tracker (src/kernels_macros.cuh:177-190) */
    float* dtt = dt + s + bs;
    for (int i = 0; i < m; ++i) {
      float acc = 0.0f;
      for (int j = 0; j < bs; ++j) acc += P[i + (size_t)j * lda] * P[i + (size_t)j * lda];
      dtt[i] -= acc;
    }
    /* 4. precision for this step's trailing update */
    int p;
    if (o->force_prec) p = o->force_prec[k];
    else if (o->precision == ORC_SWITCHING) {
      const float coh = (o->switch_mode == 0 && o->coherence)
                            ? orc_coherence_ratio(P, lda, m, bs, dtt) : 0.0f;
      p = orc_choose_precision(d + s + bs, dtt, m, coh, o);
    }
    else p = o->precision;
    if (step_prec) step_prec[k] = p;
    /* near-indefinite flag for the next diagonal block */
    next_fp64 = 0;
    {
      const int nb = m < b ? m : b;
      for (int i = 0; i < nb; ++i)
        if (o->floor_ratio > 0.0f && dtt[i] <= o->floor_ratio * d[s + bs + i]) next_fp64 = 1;
    }
    /* rounding-shift estimate: u_p * sum_j L_ij^2 for low-precision steps */
    if (sh && p != ORC_FP32) {
      const float u = orc_unit_roundoff(p);
      for (int i = 0; i < m; ++i) {
        float acc = 0.0f;
        for (int j = 0; j < bs; ++j) acc += P[i + (size_t)j * lda] * P[i + (size_t)j * lda];
        sh[s + bs + i] += u * acc;
      }
    }
    /* 5. quantize the panel (row-major copy qbuf[i*bs + j]) */
    for (int i = 0; i < m; ++i) {
      if (p == ORC_FP32) {
        for (int j = 0; j < bs; ++j) qbuf[(size_t)i * bs + j] = P[i + (size_t)j * lda];
      } else {
        quant_row(P + i, lda, bs, p, qbuf + (size_t)i * bs);
      }
    }
    /* 6. trailing update C -= Q Q^T, lower triangle, FP64 accumulate of the
     *    exactly-representable dequantized products, one rounding to FP32. */
    float* C = A + s + bs + (size_t)(s + bs) * lda;
#pragma omp parallel for schedule(dynamic, 16)
    for (int j = 0; j < m; ++j) {
      const float* qj = qbuf + (size_t)j * bs;
      for (int i = j; i < m; ++i) {
        const float* qi = qbuf + (size_t)i * bs;
        double acc = 0.0;
        for (int l = 0; l < bs; ++l) acc += (double)qi[l] * (double)qj[l];
        C[i + (size_t)j * lda] = (float)((double)C[i + (size_t)j * lda] - acc);
      }
    }
  }
  free(qbuf); free(blk64); free(shiftf); free(pminf); free(shiftd); free(pmind);
  return info->status;
}

/* OpenMP blocked FP32 restatement of the reference's uniform-precision factor
 * (src/sChol.cuh:222-311): the all-core CPU baseline.  Returns 0 or 1+row. */
int orc_chol_fp32_omp(float* A, int n, int lda, int b) {
  for (int s = 0; s < n; s += b) {
    const int bs = n - s < b ? n - s : b;
    const int m = n - s - bs;
    float* D = A + s + (size_t)s * lda;
    int f = potrf_f32(D, bs, lda, NULL, NULL, NULL);
    if (f >= 0) return s + f + 1;
    if (m == 0) break;
    float* P = A + s + bs + (size_t)s * lda;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < bs; ++j) {
        float acc = P[i + (size_t)j * lda];
        for (int l = 0; l < j; ++l) acc -= P[i + (size_t)l * lda] * D[j + (size_t)l * lda];
        P[i + (size_t)j * lda] = acc / D[j + (size_t)j * lda];
      }
    float* C = A + s + bs + (size_t)(s + bs) * lda;
#pragma omp parallel for schedule(dynamic, 8)
    for (int j = 0; j < m; ++j)
      for (int l = 0; l < bs; ++l) {
        const float pjl = P[j + (size_t)l * lda];
        const float* pl = P + (size_t)l * lda;
        float* cj = C + (size_t)j * lda;
        for (int i = j; i < m; ++i) cj[i] -= pl[i] * pjl;
      }
  }
  return 0;
}

/* Dense FP32-matrix x FP64-vector product with FP64 accumulation (CPU
 * baseline PCG operator; column-major, ld). */
void orc_gemv_f32_f64(const float* A, int n, int ld, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) y[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    const double xj = x[j];
    const float* a = A + (size_t)j * ld;
    for (int i = 0; i < n; ++i) y[i] += (double)a[i] * xj;
  }
}

/* Forward then backward substitution with the FP32 lower factor, FP64
 * vectors: z = L^-T L^-1 r (the reference's Dpotrs, src/mixed_cholesky.cu:204-206). */
void orc_potrs_f32_f64(const float* L, int n, int ld, const double* r, double* z) {
  for (int i = 0; i < n; ++i) z[i] = r[i];
  for (int j = 0; j < n; ++j) {
    z[j] /= (double)L[j + (size_t)j * ld];
    const double zj = z[j];
    const float* c = L + (size_t)j * ld;
    for (int i = j + 1; i < n; ++i) z[i] -= (double)c[i] * zj;
  }
  for (int j = n - 1; j >= 0; --j) {
    const float* c = L + (size_t)j * ld;
    double acc = z[j];
    for (int i = j + 1; i < n; ++i) acc -= (double)c[i] * z[i];
    z[j] = acc / (double)L[j + (size_t)j * ld];
  }
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
