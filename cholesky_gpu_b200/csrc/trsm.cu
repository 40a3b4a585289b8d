// Panel TRSM with the fused switching epilogue.
//
// Replaces the reference's cublasStrsm of the panel (src/switching_chol.cuh:98-110,
// correct form RIGHT/LOWER/TRANS at src/sChol.cuh:273-280), its update_diag
// kernel (src/kernels_macros.cuh:177-190) and the per-row part of can_switch
// (src/kernels_macros.cuh:191-211).
//
// X * L11^T = A21 for the m rows below the diagonal block.  Rows are
// independent, so one CTA owns a 32-row slab.  TMA stages the slab (one 2-D
// box) and streams L11 one 32-row tile row at a time (the strictly-lower
// tiles L_{J,<J} as 2-D boxes and the inverse of the diagonal tile L_JJ, which
// the POTRF kernel wrote, as a 1-D bulk copy) two rows ahead of its use, so a
// CTA needs about 108 KB of shared memory and two CTAs share an SM.  The CTA
// walks the 32-column tiles J: X_J -= X_{<J} L_{J,<J}^T (register-tiled,
// K split over four thread groups), X_J = X_J L_JJ^-T, writes the slab back
// and, in the epilogue, folds each row's sum of squares into the
// Schur-diagonal tracker dtilde, reduces the switching statistics
// (max d/dtilde, reference-literal choice) and the near-indefinite flag of
// the next diagonal block, and writes the slab's codes in every candidate
// format.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "quant.cuh"
#include "tc_ptx.cuh"

namespace mpchol {
namespace {

constexpr int TR = 32;       // rows per CTA
constexpr int NTHR = 256;    // 8 warps
constexpr int TSZ = 32 * 32; // dense 32 x 32 tile
constexpr int XLD = TR;      // X staged column-major, rows contiguous
constexpr int KG = 4;        // groups the update's K dimension is split over
constexpr int KPG = 32 / KG; // K values of each L tile per group
static_assert(NTHR == KG * (TR / 4) * 8, "a group maps 4 x 4 outputs to each of its threads");

__device__ __forceinline__ int tl(int I, int M) { return I * (I - 1) / 2 + M; }  // I > M

// Shared memory of the streaming panel kernel: the slab, two buffers of one
// tile row of L11 (up to NT - 1 tiles) and of one tile inverse, the partial
// sums of the split update.
size_t trsm_smem_floats(int bs) {
  const int NT = bs / 32;
  return (size_t)bs * XLD + 2 * (size_t)(NT - 1) * TSZ + 2 * (size_t)TSZ + (size_t)(KG - 1) * TR * 32;
}
// Shared memory of the batched kernel: the slab, all of L11's tiles and
// inverses, the partial sums.
size_t trsm_batched_smem_floats(int bs) {
  const int NT = bs / 32;
  return (size_t)bs * XLD + (size_t)(NT * (NT - 1) / 2) * TSZ + (size_t)NT * TSZ +
         (size_t)(KG - 1) * TR * 32;
}

// Step J of the slab solve: X_J -= X_{<J} L_{J,<J}^T, then X_J = X_J L_JJ^-T.
// LJ: the tiles L_{J,0..J-1} (column-major 32 x 32, contiguous); WJ: L_JJ^-1.
// The update splits K over four groups of 64 threads: a thread keeps 4 rows x
// 4 columns of X_J in registers and does 16 FMAs per 16-byte load of X and of
// L; groups 1-3 hand their partial sums to group 0 through red, which adds
// them in group order.  Every output's operations, and so its rounding, are
// fixed by this split.
__device__ void trsm_step(float* Xs, const float* LJ, const float* WJ, float* red, int J, int tid) {
  const int g = tid / 64, t = tid % 64;
  const int r4 = t % (TR / 4), c4 = t / (TR / 4);   // rows 4*r4.., columns 4*c4.. of X_J
  const int kend = 32 * J;
  if (J > 0) {
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float4 v = (g == 0) ? *reinterpret_cast<const float4*>(&Xs[(kend + 4 * c4 + j) * XLD + 4 * r4])
                                : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      acc[0][j] = v.x; acc[1][j] = v.y; acc[2][j] = v.z; acc[3][j] = v.w;
    }
    for (int kt = 0; kt < J; ++kt) {
      const float* lt = LJ + kt * TSZ + 4 * c4 + KPG * g * 32;
      const float* xt = Xs + (32 * kt + KPG * g) * XLD + 4 * r4;
#pragma unroll
      for (int kk = 0; kk < KPG; ++kk) {
        const float4 xv = *reinterpret_cast<const float4*>(xt + kk * XLD);
        const float4 lv = *reinterpret_cast<const float4*>(lt + kk * 32);
        const float xr[4] = {xv.x, xv.y, xv.z, xv.w};
        const float lr[4] = {lv.x, lv.y, lv.z, lv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] -= xr[i] * lr[j];
      }
    }
    if (g > 0) {
      float* rg = red + (g - 1) * TR * 32;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        *reinterpret_cast<float4*>(&rg[(4 * c4 + j) * TR + 4 * r4]) =
            make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
    }
    __syncthreads();
    if (g == 0) {
#pragma unroll
      for (int q = 0; q < KG - 1; ++q) {
        const float* rg = red + q * TR * 32;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float4 pv = *reinterpret_cast<const float4*>(&rg[(4 * c4 + j) * TR + 4 * r4]);
          acc[0][j] += pv.x; acc[1][j] += pv.y; acc[2][j] += pv.z; acc[3][j] += pv.w;
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        *reinterpret_cast<float4*>(&Xs[(kend + 4 * c4 + j) * XLD + 4 * r4]) =
            make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
    }
    __syncthreads();
  }
  // X_J = X_J * L_JJ^-T :  x[r][c] = sum_{m<=c} a[r][m] * (L^-1)[c][m]
  const int tr = tid % (TR / 4), tc_ = tid / (TR / 4);   // rows 4*tr.., column tc_
  float out[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 8
  for (int m = 0; m < 32; ++m) {
    const float4 av = *reinterpret_cast<const float4*>(&Xs[(kend + m) * XLD + 4 * tr]);
    const float wv = WJ[m * 32 + tc_];
    out[0] += av.x * wv; out[1] += av.y * wv; out[2] += av.z * wv; out[3] += av.w * wv;
  }
  __syncthreads();
  *reinterpret_cast<float4*>(&Xs[(kend + tc_) * XLD + 4 * tr]) = make_float4(out[0], out[1], out[2], out[3]);
  __syncthreads();
}

// Per-row sum of squares and max |x| of the solved slab, by all threads:
// thread (r, part) = (tid % TR, tid / TR) covers row r's 32 columns `part`
// (sums of squares as a chain of FMAs in column order), leaving the partials
// in s_sq / s_amax [part][r]; the row's sum is then the partials added in
// part order (row_sq).  One fixed order for the streaming and the batched
// kernel, so both give the same bits.
__device__ __forceinline__ void slab_row_partials(const float* Xs, int NT, float (*s_sq)[TR],
                                                  float (*s_amax)[TR], int tid) {
  const int r = tid % TR, part = tid / TR;
  float sq = 0.0f, amax = 0.0f;
  if (part < NT) {
#pragma unroll 8
    for (int c = part * 32; c < part * 32 + 32; ++c) {
      const float v = Xs[c * XLD + r];
      sq = __fmaf_rn(v, v, sq);
      amax = fmaxf(amax, fabsf(v));
    }
  }
  s_sq[part][r] = sq;
  if (s_amax != nullptr) s_amax[part][r] = amax;
}
__device__ __forceinline__ float row_sq(float (*s_sq)[TR], int NT, int r) {
  float sq = s_sq[0][r];
  for (int q = 1; q < NT; ++q) sq += s_sq[q][r];
  return sq;
}

// Codes of one solved slab in one format.  Xs: the slab (bs columns x TR
// rows, column-major, stride XLD).  Thread (r, part) = (tid % TR, tid / TR)
// converts row r's 32-column block `part` (for MXFP8 with its own scale)
// into packed words of a shared staging panel (row stride bs/4 + 1 words for
// 8-bit codes, bs/2 + 1 for 16-bit ones, so the column-wise writes of 32
// consecutive rows hit 32 banks); the CTA then copies the staged rows out as
// coalesced 4-byte words.
__device__ void quantize_slab(const float* Xs, int bs, int nrows, int gi0, int m, int fmt, float rmax,
                              const QuantAll& qa, uint32_t* stage, int tid) {
  const int r = tid % TR, part = tid / TR;
  const int cw = part < bs / 32 ? 32 : 0;      // columns of this thread
  const int c0 = part * 32;
  const int gi = gi0 + r;
  const bool live = r < nrows;
  if (fmt == FP16 || fmt == FP16X2) {
    const int sw = bs / 2 + 1;
    uint32_t* hi = stage;
    uint32_t* lo = stage + TR * sw;
    const int e = row_scale_exp(rmax, FP16);
    const float inv = pow2f(-e);
    if (cw == 32) {
#pragma unroll
      for (int c = c0; c < c0 + 32; c += 2) {
        const float x0 = Xs[c * XLD + r] * inv, x1 = Xs[(c + 1) * XLD + r] * inv;
        const __half2 h = __floats2half2_rn(x0, x1);
        hi[r * sw + c / 2] = *reinterpret_cast<const uint32_t*>(&h);
        if (fmt == FP16X2) {   // x - hi is exact in FP32
          const float2 hf = __half22float2(h);
          lo[r * sw + c / 2] = f32x2_to_f16x2(x0 - hf.x, x1 - hf.y);
        }
      }
    }
    if (live && part == 0) qa.rexp[2][gi] = (int8_t)e;
    __syncthreads();
    const int wpr = bs / 2;                    // words per row
#pragma unroll 4
    for (int q = tid; q < nrows * wpr; q += NTHR) {
      const int rr = q / wpr, w = q % wpr;
      reinterpret_cast<uint32_t*>(qa.q16 + (size_t)(gi0 + rr) * qa.ldq)[w] = hi[rr * sw + w];
      if (fmt == FP16X2)
        reinterpret_cast<uint32_t*>(qa.q16 + (size_t)(m + gi0 + rr) * qa.ldq)[w] = lo[rr * sw + w];
    }
  } else {
    const int sw = bs / 4 + 1;
    int e = 0;
    float inv = 1.0f;
    if (fmt != MXFP8) {
      e = row_scale_exp(rmax, fmt);
      inv = pow2f(-e);
      if (live && part == 0) qa.rexp[rexp_slot(fmt)][gi] = (int8_t)e;
    }
    for (int cb = c0; cb < c0 + cw; cb += 32) {
      if (fmt == MXFP8) {
        // one E8M0 scale per 32 consecutive columns (OCP MX)
        float bmax = 0.0f;
        for (int c = cb; c < cb + 32; ++c) bmax = fmaxf(bmax, fabsf(Xs[c * XLD + r]));
        const int eb = mx_scale_exp(bmax);
        inv = pow2f(-eb);
        if (live) qa.mxexp[(size_t)gi * qa.ldmx + cb / 32] = (uint8_t)(eb + 127);
      }
#pragma unroll
      for (int c = cb; c < cb + 32; c += 4) {
        float x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = Xs[(c + u) * XLD + r] * inv;
        const uint32_t w01 = (fmt == E5M2) ? f32x2_to_e5m2x2(x[0], x[1]) : f32x2_to_e4m3x2(x[0], x[1]);
        const uint32_t w23 = (fmt == E5M2) ? f32x2_to_e5m2x2(x[2], x[3]) : f32x2_to_e4m3x2(x[2], x[3]);
        stage[r * sw + c / 4] = w01 | (w23 << 16);
      }
    }
    __syncthreads();
    uint8_t* q = qa.q8[q8_slot(fmt)];
    const int wpr = bs / 4;
#pragma unroll 4
    for (int q4 = tid; q4 < nrows * wpr; q4 += NTHR) {
      const int rr = q4 / wpr, w = q4 % wpr;
      reinterpret_cast<uint32_t*>(q + (size_t)(gi0 + rr) * qa.ldq)[w] = stage[rr * sw + w];
    }
  }
  __syncthreads();                             // the staging panel is reused
}

// Panel solve with the quantization of the panel fused in; one 32-row slab
// per CTA, two CTAs per SM (the launch may exceed the resident CTAs: no CTA
// waits on another).  Each CTA stages its slab and streams L11's tile rows by
// TMA, solves the slab, writes it back, folds its rows into the diagonal
// tracker and the switching statistics, and writes the slab's codes in every
// candidate format (the step's precision is not known yet; the trailing
// update reads the panel of the one the step picks).  The CTA that finishes
// last (a ticket counter) resolves the step precision and adds the step's
// rounding shift u_p * sum_j L_ij^2 to sh.
__global__ void __launch_bounds__(NTHR, 2)
trsm_panel_kernel(const __grid_constant__ CUtensorMap tmapX, const __grid_constant__ CUtensorMap tmap32,
                  float* __restrict__ A, int lda, int n, int s, int bs, const float* __restrict__ winv,
                  const float* __restrict__ d, float* __restrict__ dtilde, float* __restrict__ rowsq,
                  StepState* step, StepState* next, int next_bs, DecisionParams dp, DevStatus* st,
                  QuantAll qa, const StepState* prev, double* __restrict__ colacc) {
  extern __shared__ __align__(128) float sm[];
  const int NT = bs / 32;
  float* Xs = sm;                                        // [bs][XLD]
  float* Lb = Xs + (size_t)bs * XLD;                     // 2 x (NT - 1) tiles: rows of L11
  float* Wb = Lb + 2 * (size_t)(NT - 1) * TSZ;           // 2 x 1 tile: inverses of L_JJ
  float* red = Wb + 2 * (size_t)TSZ;                     // partial sums of the split update
  uint32_t* stage = reinterpret_cast<uint32_t*>(Lb);     // code staging, once L11 is used
  __shared__ float red_max[NTHR / 32];
  __shared__ int red_lit[NTHR / 32];
  __shared__ float red_min[NTHR / 32];
  __shared__ double red_coh[NTHR / 32];
  __shared__ float s_rmax[NTHR / TR][TR];
  __shared__ float s_sq[NTHR / TR][TR];
  __shared__ __align__(8) uint64_t barx, barl[2];
  __shared__ int s_ok, s_last;

  const int tid = threadIdx.x;
  const int m = n - s - bs;
  const int slab = blockIdx.x;
  const int row0 = s + bs + slab * TR;                   // first global row of the slab
  const int nrows = min(TR, n - row0);
  // the previous step's rounding shift for the slab's rows, before this
  // step's sums of squares replace the previous ones in rowsq
  if (prev != nullptr && qa.sh != nullptr && tid < nrows) {
    const int pp = prev->prec;
    if (pp != FP32) {
      float* shp = qa.sh + slab * TR + tid;
      *shp = __fmaf_rn(unit_roundoff(pp), rowsq[row0 + tid], *shp);
    }
  }
  // tile row J of L11 (tiles L_{J,0..J-1} and L_JJ^-1) into buffer J % 2
  auto issue_row = [&](int J) {
    const int buf = J & 1;
    tc::mbar_expect_tx(&barl[buf], (uint32_t)((J + 1) * TSZ * sizeof(float)));
    for (int M = 0; M < J; ++M)
      tc::tma_load_2d(Lb + ((size_t)buf * (NT - 1) + M) * TSZ, &tmap32, &barl[buf], s + 32 * J, s + 32 * M);
    tc::bulk_load_1d(Wb + buf * TSZ, winv + J * TSZ, (uint32_t)(TSZ * sizeof(float)), &barl[buf]);
  };
  if (tid == 0) {
    s_ok = st->code == 0;
    tc::mbar_init(&barx, 1);
    tc::mbar_init(&barl[0], 1);
    tc::mbar_init(&barl[1], 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  int issued = 0, consumed = 0;   // tile rows issued / waited for (thread 0's counts)
  if (s_ok && tid == 0) {
    tc::mbar_expect_tx(&barx, (uint32_t)(bs * XLD * sizeof(float)));
    tc::tma_load_2d(Xs, &tmapX, &barx, row0, s);
    for (; issued < 2 && issued < NT; ++issued) issue_row(issued);
    if (!tc::mbar_wait(&barx, 0)) {
      s_ok = 0;
      set_status(st, MPCHOL_ERR_TIMEOUT, row0);
      tc::mbar_wait(&barx, 0);
    }
  }
  __syncthreads();
  float bm = 0.0f;   // this CTA's max d/dtilde, min dtilde and literal code
  float bmin = INFINITY;
  int bl = 0;
  if (s_ok) {
    for (int J = 0; J < NT; ++J) {
      if (tid == 0 && s_ok) {
        if (tc::mbar_wait(&barl[J & 1], (uint32_t)((J >> 1) & 1))) {
          consumed = J + 1;
        } else {
          s_ok = 0;
          set_status(st, MPCHOL_ERR_TIMEOUT, row0);
        }
      }
      __syncthreads();
      if (!s_ok) break;
      trsm_step(Xs, Lb + (size_t)(J & 1) * (NT - 1) * TSZ, Wb + (J & 1) * TSZ, red, J, tid);
      // trsm_step ends with a barrier: buffer J % 2 is free for row J + 2
      if (tid == 0 && issued < NT) issue_row(issued++);
    }
    if (tid == 0) {
      // rows still in flight after an abort (bounded waits): their copies
      // must land before the CTA's shared memory is released
      for (int J = consumed; J < issued; ++J) tc::mbar_wait(&barl[J & 1], (uint32_t)((J >> 1) & 1));
    }
  }
  __syncthreads();
  if (s_ok) {
    // ---- write the solved slab back (coalesced; rows past n skipped) -----
#pragma unroll 8
    for (int e = tid; e < bs * TR; e += NTHR) {
      const int c = e / TR, r = e % TR;
      if (r < nrows) A[(size_t)(s + c) * lda + row0 + r] = Xs[c * XLD + r];
    }
    // ---- Schur diagonal tracker and switching statistics of the slab -----
    slab_row_partials(Xs, NT, s_sq, s_rmax, tid);
    __syncthreads();
    if (tid < nrows) {
      const int gi = row0 + tid;
      const float sq = row_sq(s_sq, NT, tid);
      rowsq[gi] = sq;
      const float dt = dtilde[gi] - sq;
      dtilde[gi] = dt;
      const float di = d[gi];
      float ratio = dt > 0.0f ? di / dt : INFINITY;
      if (isnan(ratio)) ratio = INFINITY;
      bm = fmaxf(bm, ratio);
      bmin = dt > 0.0f ? fminf(bmin, dt) : 0.0f;
      // reference list {FP32, FP16, E4M3} with the reference's machine epsilons
      const float ref_eps[3] = {1.1920929e-7f, 0.0009765625f, 0.125f};
      int pick = 0;
      for (int p = 0; p < 3; ++p)
        if (ref_eps[p] * dt >= dp.eps_prime * di) { pick = p; break; }
      bl = max(bl, 2 - pick);
      if (next != nullptr && dp.floor_ratio > 0.0f && gi - (s + bs) < next_bs &&
          dt <= dp.floor_ratio * di)
        next->fp64_diag = 1;
    }
    // ---- column sums of the slab (coherence rule): thread c sums column c
    // over the slab's rows, starting at row c % 32 so that the 32 threads of
    // a warp read 32 different banks (a fixed order per column), and adds it
    // into colacc.  The sums reach colacc as FP64 atomics of FP32 partials,
    // which are exact while a column's partials span less than 2^20 in
    // magnitude; the order of the atomics then does not change the result
    if (colacc != nullptr) {
      if (tid < bs) {
        float cs = 0.0f;
#pragma unroll 8
        for (int q = 0; q < TR; ++q) {
          const int r = (q + tid) & (TR - 1);
          cs += (r < nrows) ? Xs[tid * XLD + r] : 0.0f;
        }
        atomicAdd(colacc + tid, (double)cs);
      }
      __threadfence();
    }
    // ---- the slab's codes in every candidate format -------------------------
    if (qa.cand != 0) {
      const int r = tid % TR;
      float rmax = 0.0f;
#pragma unroll
      for (int q = 0; q < NTHR / TR; ++q) rmax = fmaxf(rmax, s_rmax[q][r]);
      const int gi0 = slab * TR;                         // first trailing row of the slab
      const bool f16 = (qa.cand >> FP16) & 1u, f16x2 = (qa.cand >> FP16X2) & 1u;
      if (f16 || f16x2) quantize_slab(Xs, bs, nrows, gi0, m, f16x2 ? FP16X2 : FP16, rmax, qa, stage, tid);
      const int f8[3] = {E4M3, E5M2, MXFP8};
      for (int i = 0; i < 3; ++i)
        if ((qa.cand >> f8[i]) & 1u) quantize_slab(Xs, bs, nrows, gi0, m, f8[i], rmax, qa, stage, tid);
    }
  }
  // ---- statistics of the CTA; the last CTA resolves the step --------------
  bm = warp_max(bm);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bl = max(bl, __shfl_xor_sync(0xffffffffu, bl, o));
    bmin = fminf(bmin, __shfl_xor_sync(0xffffffffu, bmin, o));
  }
  if ((tid & 31) == 0) { red_max[tid >> 5] = bm; red_lit[tid >> 5] = bl; red_min[tid >> 5] = bmin; }
  __syncthreads();
  if (tid == 0) {
    float cm = 0.0f, cmin = INFINITY; int cl = 0;
    for (int w = 0; w < NTHR / 32; ++w) {
      cm = fmaxf(cm, red_max[w]);
      cl = max(cl, red_lit[w]);
      cmin = fminf(cmin, red_min[w]);
    }
    atomicMax(&step->max_ratio_bits, __float_as_uint(cm));
    atomicMax(&step->literal_code, cl);
    if (cmin < INFINITY) atomicMax(&step->not_min_dt_bits, ~__float_as_uint(fmaxf(cmin, 0.0f)));
    __threadfence();
    s_last = atomicAdd(&step->grid_bar, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();                                       // every CTA's statistics
  // coherence ratio (||P^T 1||^2 / m) / min dtilde: the column sums' squares
  // summed in a fixed order (warp butterflies, then warps in order)
  if (colacc != nullptr) {
    double c2 = 0.0;
    if (tid < bs) {
      const double cs = *reinterpret_cast<volatile double*>(colacc + tid);
      c2 = cs * cs;
    }
    c2 = warp_sum(c2);
    if ((tid & 31) == 0) red_coh[tid >> 5] = c2;
    __syncthreads();
  }
  if (tid != 0) return;
  if (*reinterpret_cast<volatile int*>(&st->code) != 0) return;
  StepState ss;
  ss.max_ratio_bits = *reinterpret_cast<volatile unsigned int*>(&step->max_ratio_bits);
  ss.literal_code = *reinterpret_cast<volatile int*>(&step->literal_code);
  float coh = 0.0f;
  if (colacc != nullptr) {
    double c2 = 0.0;
    for (int w = 0; w < NTHR / 32; ++w) c2 += red_coh[w];
    const float mind = __uint_as_float(~*reinterpret_cast<volatile unsigned int*>(&step->not_min_dt_bits));
    const double g = c2 / (double)m;
    coh = (mind > 0.0f) ? (float)(g / (double)mind) : INFINITY;
    if (isnan(coh)) coh = INFINITY;
    step->coh_bits = __float_as_uint(coh);
  }
  ss.coh_bits = __float_as_uint(coh);
  step->prec = resolve_precision(&ss, dp);
}

// Batched: blockIdx.y = system, blockIdx.x = 32-row slab.  Staging by
// plain coalesced loads (no per-system tensor maps); the epilogue keeps the
// row sums of squares (rounding-shift estimate) and the diagonal tracker.
__global__ void __launch_bounds__(NTHR)
trsm_batched_kernel(BatchSys* __restrict__ sys, int s, int b) {
  const BatchSys& S = sys[blockIdx.y];
  const int n = S.n;
  const int bs = min(b, n - s);
  const int row0 = s + bs + blockIdx.x * TR;
  const int nrows = min(TR, n - row0);
  if (bs <= 0 || nrows <= 0 || S.st->code != 0) return;
  extern __shared__ __align__(128) float sm[];
  const int NT = bs / 32;                     // bs == b: only the last block can be partial
  float* Xs = sm;
  float* Lt = Xs + (size_t)bs * XLD;
  float* Wt = Lt + (size_t)(NT * (NT - 1) / 2) * TSZ;
  float* red = Wt + (size_t)NT * TSZ;
  const int tid = threadIdx.x;
  const float* A = S.A;
  const int ld = S.ld;
  for (int e = tid; e < bs * TR; e += NTHR) {
    const int c = e / TR, r = e % TR;
    Xs[c * XLD + r] = (r < nrows) ? A[(size_t)(s + c) * ld + row0 + r] : 0.0f;
  }
  for (int I = 1; I < NT; ++I)
    for (int M = 0; M < I; ++M)
      for (int e = tid; e < TSZ; e += NTHR) {
        const int c = e / 32, r = e % 32;
        Lt[tl(I, M) * TSZ + e] = A[(size_t)(s + 32 * M + c) * ld + s + 32 * I + r];
      }
  for (int e = tid; e < NT * TSZ; e += NTHR) Wt[e] = S.winv[e];
  __syncthreads();
  for (int J = 0; J < NT; ++J) trsm_step(Xs, Lt + tl(J, 0) * TSZ, Wt + J * TSZ, red, J, tid);
  for (int e = tid; e < bs * TR; e += NTHR) {
    const int c = e / TR, r = e % TR;
    if (r < nrows) S.A[(size_t)(s + c) * ld + row0 + r] = Xs[c * XLD + r];
  }
  __shared__ float s_sq[NTHR / TR][TR];
  slab_row_partials(Xs, NT, s_sq, nullptr, tid);
  __syncthreads();
  if (tid < nrows) {
    const int gi = row0 + tid;
    const float sq = row_sq(s_sq, NT, tid);
    S.rowsq[gi] = sq;
    S.dtilde[gi] -= sq;
  }
}

}  // namespace

cudaError_t launch_trsm_panel(const CUtensorMap& tmapX, const CUtensorMap& tmap32, float* A,
                              int lda, int n, int s, int bs, const float* winv, const float* d,
                              float* dtilde, float* rowsq, StepState* step, StepState* next,
                              int next_bs, const DecisionParams& dp, const QuantAll& qa,
                              DevStatus* st, cudaStream_t stream, const StepState* prev,
                              double* colacc) {
  const int m = n - s - bs;
  if (m <= 0) return cudaSuccess;
  const size_t smem = trsm_smem_floats(bs) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(trsm_panel_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(trsm_smem_floats(256) * sizeof(float)));
  if (e != cudaSuccess) return e;
  trsm_panel_kernel<<<ceil_div(m, TR), NTHR, smem, stream>>>(tmapX, tmap32, A, lda, n, s, bs, winv, d,
                                                             dtilde, rowsq, step, next, next_bs, dp, st,
                                                             qa, prev, colacc);
  return cudaGetLastError();
}

cudaError_t launch_trsm_batched(BatchSys* sys, int nact, int s, int b, int max_m,
                                cudaStream_t stream) {
  if (nact <= 0 || max_m <= 0) return cudaSuccess;
  const size_t smem = trsm_batched_smem_floats(b) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(trsm_batched_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  trsm_batched_kernel<<<dim3(ceil_div(max_m, TR), nact), NTHR, smem, stream>>>(sys, s, b);
  return cudaGetLastError();
}

}  // namespace mpchol
