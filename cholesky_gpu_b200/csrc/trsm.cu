// Panel TRSM with the fused switching epilogue.
//
// Replaces the reference's cublasStrsm of the panel (src/switching_chol.cuh:98-110,
// correct form RIGHT/LOWER/TRANS at src/sChol.cuh:273-280), its update_diag
// kernel (src/kernels_macros.cuh:177-190) and the per-row part of can_switch
// (src/kernels_macros.cuh:191-211).
//
// X * L11^T = A21 for the m rows below the diagonal block.  Rows are
// independent, so one CTA of 16 warps owns a slab of 32 or 64 rows (64 while
// the panel has more 32-row slabs than the GPU has SMs).  TMA stages the slab
// and all of L11: the strictly-lower 32 x 32 tiles L_{J,M} as 2-D boxes and
// the inverses of the diagonal tiles L_JJ, which the POTRF kernel wrote, as
// 1-D bulk copies, one mbarrier per tile row.  The solve is a pipeline over
// the 32-column tiles J of the slab, a warp pair per tile (each thread a
// register block of 4 or 8 rows x 4 columns, so a k step reads two or three
// 16-byte vectors for 16 or 32 FMAs; the shared-memory return path, not the
// FMA rate, bounds these small products):
//   X_J = (A_J - sum_{K<J} X_K L_{J,K}^T) L_JJ^-T,
// where the pair of tile J applies X_K as soon as the pair of tile K has
// published it (an mbarrier per tile, bounded waits), so the only chain is
// one tile update plus one diagonal multiply per tile column.  The epilogue
// writes the slab back (TMA stores), folds each row's sum of squares into the
// Schur-diagonal tracker dtilde, reduces the switching statistics (max
// d/dtilde, min dtilde, the reference-literal choice, the panel's column sums)
// and the near-indefinite flag of the next diagonal block, and writes the
// slab's codes in every candidate format.  The last CTA to finish (a ticket
// counter) resolves the step precision.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "quant.cuh"
#include "tc_ptx.cuh"

namespace mpchol {
namespace {

constexpr int NTHR = 512;    // 16 warps: two per 32-column tile of a 256-wide block
constexpr int TSZ = 32 * 32; // dense 32 x 32 tile
constexpr int MAXNT = 8;     // tiles per block column (b <= 256)

__device__ __forceinline__ int tl(int I, int M) { return I * (I - 1) / 2 + M; }  // I > M

// The slab in shared memory: 32-row halves, each column-major with its 32
// rows contiguous (the layout of a 32 x bs TMA box), so lane l reading row l
// (or l + 32) of one column touches 32 different banks.
__device__ __forceinline__ int xoff(int r, int c, int bs) {
  return (r >> 5) * bs * 32 + c * 32 + (r & 31);
}

// Code staging panel of the epilogue (32-bit words): FP16X2 hi + lo rows of
// bs / 2 + 1 words, or 8-bit code rows of bs / 4 + 1 words.
size_t stage_words(int tr, int bs) {
  return std::max((size_t)2 * tr * (bs / 2 + 1), (size_t)tr * (bs / 4 + 1));
}
// Shared memory of both panel kernels (floats): the slab, then L11's
// strictly-lower tiles and the inverses of its diagonal tiles (the code
// staging panel reuses that space once the solve is done).
size_t trsm_smem_floats(int tr, int bs) {
  const int NT = bs / 32;
  const size_t lw = (size_t)(NT * (NT - 1) / 2 + NT) * TSZ;
  return (size_t)bs * tr + std::max(lw, stage_words(tr, bs));
}

__device__ __forceinline__ void pair_sync(int J) {   // the two warps of tile column J
  asm volatile("bar.sync %0, 64;" ::"r"(J + 1) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// The slab solve.  The warp pair of tile column J (warps 2J, 2J + 1; w = 2J +
// h) computes the TR x 32 tile X_J: thread t of the pair (t = 32 h + lane)
// holds a block of 4 RPL rows x 4 columns in registers, rows 4 rg .. 4 rg + 3
// of each 32-row half (rg = t % 8) and columns 4 cg .. 4 cg + 3 (cg = t / 8),
// so every k step of the tile products reads 16-byte vectors of X (one per
// half) and of L (one), and a quarter-warp's eight X vectors are 128
// contiguous bytes.  Lt: L11's tiles L_{I,M} (I > M) at tl(I, M) * TSZ; Wt:
// the inverses W_JJ = L_JJ^-1, tile J at J * TSZ; both column-major (L(c, m)
// at m * 32 + c, W(c, m) zero for m > c).  lrow[J] (null: already staged)
// completes when tile row J has landed; ready[J] (64 arrivals) when X_J is
// final:
//   X_J = (A_J - sum_{K<J} X_K L_{J,K}^T) W_JJ^T.
// Each output is one fma chain in a fixed order: the update over K, then m;
// the diagonal multiply over m.  Returns false if a bounded wait gave up.
template <int RPL>
__device__ bool slab_solve(float* Xs, int bs, const float* Lt, const float* Wt, uint64_t* lrow,
                           uint64_t* ready, int tid) {
  const int NT = bs / 32;
  const int warp = tid >> 5, lane = tid & 31;
  const int J = warp >> 1, h = warp & 1;
  if (J >= NT) return true;
  const int XH = bs * 32;                              // floats per 32-row half
  const int t = 32 * h + lane;
  const int rg = t & 7, cg = t >> 3;
  const int r0 = 4 * rg;                               // rows r0.. of each half
  const int cl = 4 * cg;                               // columns cl.. of the tile
  bool ok = lrow == nullptr || tc::mbar_wait(&lrow[J], 0);
  float acc[RPL][4][4];                                // [half][row][column]
#pragma unroll
  for (int q = 0; q < RPL; ++q)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float4 v = *reinterpret_cast<const float4*>(Xs + q * XH + (32 * J + cl + j) * 32 + r0);
      acc[q][0][j] = v.x; acc[q][1][j] = v.y; acc[q][2][j] = v.z; acc[q][3][j] = v.w;
    }
#pragma unroll 1
  for (int K = 0; K < J; ++K) {
    ok = tc::mbar_wait(&ready[K], 0) && ok;
    const float* L = Lt + (size_t)tl(J, K) * TSZ + cl;
    const float* xk = Xs + 32 * K * 32 + r0;
#pragma unroll 8
    for (int m = 0; m < 32; ++m) {
      const float4 lv = *reinterpret_cast<const float4*>(L + m * 32);
      const float l[4] = {lv.x, lv.y, lv.z, lv.w};
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const float4 xv = *reinterpret_cast<const float4*>(xk + q * XH + m * 32);
        const float x[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[q][i][j] = fmaf(-x[i], l[j], acc[q][i][j]);
      }
    }
  }
  // the updated tile into the slab, then X_J = Y W_JJ^T
  float* xj = Xs + 32 * J * 32 + r0;
#pragma unroll
  for (int q = 0; q < RPL; ++q)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      *reinterpret_cast<float4*>(xj + q * XH + (cl + j) * 32) =
          make_float4(acc[q][0][j], acc[q][1][j], acc[q][2][j], acc[q][3][j]);
  pair_sync(J);
  const float* W = Wt + (size_t)J * TSZ + cl;
#pragma unroll
  for (int q = 0; q < RPL; ++q)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[q][i][j] = 0.0f;
  const int mend = 16 * h + 16;                        // W(c, m) = 0 for m > c (the warp's columns)
#pragma unroll 8
  for (int m = 0; m < mend; ++m) {
    const float4 wv = *reinterpret_cast<const float4*>(W + m * 32);
    const float w[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
      const float4 yv = *reinterpret_cast<const float4*>(xj + q * XH + m * 32);
      const float y[4] = {yv.x, yv.y, yv.z, yv.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[q][i][j] = fmaf(y[i], w[j], acc[q][i][j]);
    }
  }
  pair_sync(J);                                        // every read of Y is done
#pragma unroll
  for (int q = 0; q < RPL; ++q)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      *reinterpret_cast<float4*>(xj + q * XH + (cl + j) * 32) =
          make_float4(acc[q][0][j], acc[q][1][j], acc[q][2][j], acc[q][3][j]);
  mbar_arrive(&ready[J]);                              // release: X_J to the later tiles
  return ok;
}

// Per-row sum of squares and max |x| of the solved slab: thread (r, part) =
// (tid % TR, tid / TR) covers row r's 32 columns `part` (sums of squares as a
// chain of FMAs in column order), leaving the partials in s_sq / s_amax
// [part][r]; the row's sum is then the partials added in part order (row_sq).
// One fixed order for the streaming and the batched kernel, so both give the
// same bits.
template <int TR>
__device__ __forceinline__ void slab_row_partials(const float* Xs, int bs, float (*s_sq)[TR],
                                                  float (*s_amax)[TR], int tid) {
  const int NT = bs / 32;
  const int r = tid % TR, part = tid / TR;
  float sq = 0.0f, amax = 0.0f;
  if (part < NT) {
#pragma unroll 8
    for (int c = part * 32; c < part * 32 + 32; ++c) {
      const float v = Xs[xoff(r, c, bs)];
      sq = __fmaf_rn(v, v, sq);
      amax = fmaxf(amax, fabsf(v));
    }
  }
  s_sq[part][r] = sq;
  if (s_amax != nullptr) s_amax[part][r] = amax;
}
template <int TR>
__device__ __forceinline__ float row_sq(float (*s_sq)[TR], int NT, int r) {
  float sq = s_sq[0][r];
  for (int q = 1; q < NT; ++q) sq += s_sq[q][r];
  return sq;
}

// Two elements as 8-bit codes of format FMT (already scaled): E4M3 / E5M2
// by the hardware conversion; the FP6/FP4 MX elements rounded onto their
// grid first (the rounded value is exact in E4M3).
template <int FMT>
__device__ __forceinline__ uint32_t code8_x2(float a, float b) {
  if constexpr (FMT == E5M2) return f32x2_to_e5m2x2(a, b);
  else if constexpr (FMT == E4M3 || FMT == MXFP8) return f32x2_to_e4m3x2(a, b);
  else {
    const MxElem me = mx_elem(FMT);
    return f32x2_to_e4m3x2(mx_round_elem(a, me), mx_round_elem(b, me));
  }
}

// 8-bit codes of thread (r, part)'s 32-column block in format FMT into the
// staging panel (row stride bs/4 + 1 words): the block's values are read once
// into registers; an MX format takes the block's own E8M0 scale, the others
// the row's power-of-two scale (from the row maximum rmax).
template <int TR, int FMT>
__device__ __forceinline__ void stage_codes8(const float* Xs, int bs, int nrows, int gi0, float rmax,
                                             const QuantAll& qa, uint32_t* stage, int tid) {
  constexpr bool MX = FMT == MXFP8 || FMT == MXFP6E2M3 || FMT == MXFP6E3M2 || FMT == MXFP4;
  const int r = tid % TR, part = tid / TR;
  const int gi = gi0 + r;
  const bool live = r < nrows;
  if (part >= bs / 32) return;
  const int sw = bs / 4 + 1;
  const int cb = part * 32;
  float v[32];
#pragma unroll
  for (int u = 0; u < 32; ++u) v[u] = Xs[xoff(r, cb + u, bs)];
  float inv;
  if constexpr (MX) {
    float mx[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      mx[u] = fmaxf(fmaxf(fabsf(v[u]), fabsf(v[u + 8])), fmaxf(fabsf(v[u + 16]), fabsf(v[u + 24])));
    const float bmax = fmaxf(fmaxf(fmaxf(mx[0], mx[1]), fmaxf(mx[2], mx[3])),
                             fmaxf(fmaxf(mx[4], mx[5]), fmaxf(mx[6], mx[7])));
    const int eb = mx_scale_exp(bmax, FMT);
    inv = pow2f(-eb);
    if (live) qa.mxexp[(size_t)gi * qa.ldmx + part] = (uint8_t)(eb + 127);
  } else {
    const int e = row_scale_exp(rmax, FMT);
    inv = pow2f(-e);
    if (live && part == 0) qa.rexp[rexp_slot(FMT)][gi] = (int8_t)e;
  }
#pragma unroll
  for (int c = 0; c < 32; c += 4) {
    const uint32_t w01 = code8_x2<FMT>(v[c] * inv, v[c + 1] * inv);
    const uint32_t w23 = code8_x2<FMT>(v[c + 2] * inv, v[c + 3] * inv);
    stage[r * sw + (cb + c) / 4] = w01 | (w23 << 16);
  }
}

// Codes of one solved slab in one format.  Thread (r, part) = (tid % TR,
// tid / TR) converts row r's 32-column block `part` (for an MX format with
// its own scale) into packed words of a shared staging panel (row stride
// bs/4 + 1 words for 8-bit codes, bs/2 + 1 for 16-bit ones, so the
// column-wise writes of 32 consecutive rows hit 32 banks); the CTA then
// copies the staged rows out as coalesced 4-byte words.
template <int TR>
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
        const float x0 = Xs[xoff(r, c, bs)] * inv, x1 = Xs[xoff(r, c + 1, bs)] * inv;
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
    switch (fmt) {
      case E4M3: stage_codes8<TR, E4M3>(Xs, bs, nrows, gi0, rmax, qa, stage, tid); break;
      case E5M2: stage_codes8<TR, E5M2>(Xs, bs, nrows, gi0, rmax, qa, stage, tid); break;
      case MXFP8: stage_codes8<TR, MXFP8>(Xs, bs, nrows, gi0, rmax, qa, stage, tid); break;
      case MXFP6E2M3: stage_codes8<TR, MXFP6E2M3>(Xs, bs, nrows, gi0, rmax, qa, stage, tid); break;
      case MXFP6E3M2: stage_codes8<TR, MXFP6E3M2>(Xs, bs, nrows, gi0, rmax, qa, stage, tid); break;
      default: stage_codes8<TR, MXFP4>(Xs, bs, nrows, gi0, rmax, qa, stage, tid); break;
    }
    __syncthreads();
    uint8_t* q = qa.q8[q8_slot(fmt)];
    const int sw = bs / 4 + 1;
    const int wpr = bs / 4;
#pragma unroll 4
    for (int q4 = tid; q4 < nrows * wpr; q4 += NTHR) {
      const int rr = q4 / wpr, w = q4 % wpr;
      reinterpret_cast<uint32_t*>(q + (size_t)(gi0 + rr) * qa.ldq)[w] = stage[rr * sw + w];
    }
  }
  __syncthreads();                             // the staging panel is reused
}

// Panel solve with the quantization of the panel fused in; one slab of TR =
// 32 * RPL rows per CTA (the launch may exceed the resident CTAs: no CTA
// waits on another).  Each CTA stages its slab and L11 by TMA, solves the
// slab, writes it back, folds its rows into the diagonal tracker and the
// switching statistics, and writes the slab's codes in every candidate
// format (the step's precision is not known yet; the trailing update reads
// the panel of the one the step picks).  The CTA that finishes last (a
// ticket counter) resolves the step precision.
template <int RPL>
__global__ void __launch_bounds__(NTHR, 1)
trsm_panel_kernel(const __grid_constant__ CUtensorMap tmapX, const __grid_constant__ CUtensorMap tmap32,
                  float* __restrict__ A, int lda, int n, int s, int bs, const float* __restrict__ winv,
                  const float* __restrict__ d, float* __restrict__ dtilde, float* __restrict__ rowsq,
                  StepState* step, StepState* next, int next_bs, DecisionParams dp, DevStatus* st,
                  QuantAll qa, const StepState* prev, double* __restrict__ colacc) {
  constexpr int TR = 32 * RPL;
  extern __shared__ __align__(128) float sm[];
  const int NT = bs / 32;
  float* Xs = sm;                                        // the slab (xoff layout)
  float* Lt = Xs + (size_t)bs * TR;                      // L_{I,M}, I > M
  float* Wt = Lt + (size_t)(NT * (NT - 1) / 2) * TSZ;    // L_JJ^-1
  uint32_t* stage = reinterpret_cast<uint32_t*>(Lt);     // code staging, once L11 is used
  __shared__ float red_max[NTHR / 32];
  __shared__ int red_lit[NTHR / 32];
  __shared__ float red_min[NTHR / 32];
  __shared__ double red_coh[NTHR / 32];
  __shared__ float s_rmax[NTHR / TR][TR];
  __shared__ float s_sq[NTHR / TR][TR];
  __shared__ __align__(8) uint64_t barx, lrow[MAXNT], ready[MAXNT];
  __shared__ int s_ok, s_last;

  const int tid = threadIdx.x;
  const int m = n - s - bs;
  const int slab = blockIdx.x;
  const int row0 = s + bs + slab * TR;                   // first global row of the slab
  const int nrows = min(TR, n - row0);
  tc::grid_dep_wait();   // the POTRF (and the trailing update) before it are complete
  // the previous step's rounding shift for the slab's rows, before this
  // step's sums of squares replace the previous ones in rowsq
  if (prev != nullptr && qa.sh != nullptr && tid < nrows) {
    const int pp = prev->prec;
    if (pp != FP32) {
      float* shp = qa.sh + slab * TR + tid;
      *shp = __fmaf_rn(unit_roundoff(pp), rowsq[row0 + tid], *shp);
    }
  }
  if (tid == 0) {
    s_ok = st->code == 0;
    tc::mbar_init(&barx, 1);
    for (int J = 0; J < NT; ++J) {
      tc::mbar_init(&lrow[J], 1);
      tc::mbar_init(&ready[J], 64);
    }
    tc::fence_mbar_init();
  }
  __syncthreads();
  const bool issued = s_ok != 0;
  if (issued && tid == 0) {
    tc::mbar_expect_tx(&barx, (uint32_t)(RPL * bs * 32 * sizeof(float)));
    for (int q = 0; q < RPL; ++q) tc::tma_load_2d(Xs + q * bs * 32, &tmapX, &barx, row0 + 32 * q, s);
    for (int J = 0; J < NT; ++J) {
      tc::mbar_expect_tx(&lrow[J], (uint32_t)((J + 1) * TSZ * sizeof(float)));
      for (int M = 0; M < J; ++M)
        tc::tma_load_2d(Lt + (size_t)tl(J, M) * TSZ, &tmap32, &lrow[J], s + 32 * J, s + 32 * M);
      tc::bulk_load_1d(Wt + (size_t)J * TSZ, winv + (size_t)J * TSZ, (uint32_t)(TSZ * sizeof(float)),
                       &lrow[J]);
    }
    if (!tc::mbar_wait(&barx, 0)) {
      s_ok = 0;
      set_status(st, MPCHOL_ERR_TIMEOUT, row0);
      tc::mbar_wait(&barx, 0);
    }
  }
  __syncthreads();
  if (s_ok) {
    if (!slab_solve<RPL>(Xs, bs, Lt, Wt, lrow, ready, tid)) {
      s_ok = 0;
      set_status(st, MPCHOL_ERR_TIMEOUT, row0);
    }
  }
  // every copy into L11's space has landed before it is reused (bounded;
  // immediate once the solve has seen each tile row)
  if (issued && tid == 0)
    for (int J = 0; J < NT; ++J) tc::mbar_wait(&lrow[J], 0);
  __syncthreads();
  float bm = 0.0f;   // this CTA's max d/dtilde, min dtilde and literal code
  float bmin = INFINITY;
  int bl = 0;
  if (s_ok) {
    // ---- write the solved slab back (TMA stores; rows past n are clipped)
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      for (int q = 0; q < RPL; ++q)
        if (row0 + 32 * q < n) tc::tma_store_2d(&tmapX, Xs + q * bs * 32, row0 + 32 * q, s);
      tc::bulk_commit();
    }
    // ---- Schur diagonal tracker and switching statistics of the slab -----
    slab_row_partials<TR>(Xs, bs, s_sq, s_rmax, tid);
    __syncthreads();
    if (tid < nrows) {
      const int gi = row0 + tid;
      const float sq = row_sq<TR>(s_sq, NT, tid);
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
    // over the slab's rows, starting at row c % TR so that the 32 threads of
    // a warp read 32 different banks (a fixed order per column), and adds it
    // into copy slab % kColCopies of colacc (the copies spread the CTAs'
    // atomics over more L2 lines).  The sums reach colacc as FP64 atomics of
    // FP32 partials, which are exact while a column's partials span less than
    // 2^20 in magnitude; the order of the atomics then does not change the
    // result
    if (colacc != nullptr && tid < bs) {
      float cs = 0.0f;
#pragma unroll 8
      for (int q = 0; q < TR; ++q) {
        const int r = (q + tid) & (TR - 1);
        cs += (r < nrows) ? Xs[xoff(r, tid, bs)] : 0.0f;
      }
      atomicAdd(colacc + (size_t)(slab % kColCopies) * bs + tid, (double)cs);
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
      if (f16 || f16x2)
        quantize_slab<TR>(Xs, bs, nrows, gi0, m, f16x2 ? FP16X2 : FP16, rmax, qa, stage, tid);
      // E4M3, E5M2 and the MX-family member of the candidates (at most one:
      // they share the MX code slot and scales)
      const int f8[6] = {E4M3, E5M2, MXFP8, MXFP6E2M3, MXFP6E3M2, MXFP4};
      for (int i = 0; i < 6; ++i)
        if ((qa.cand >> f8[i]) & 1u) quantize_slab<TR>(Xs, bs, nrows, gi0, m, f8[i], rmax, qa, stage, tid);
    }
    if (tid == 0) tc::bulk_wait_read();   // the slab's stores are complete before the ticket
  }
  // the next kernel (the head of the trailing update) may be scheduled once
  // every CTA is past its solve; it waits for this grid before reading
  tc::grid_dep_trigger();
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
      double cs = 0.0;
      for (int q = 0; q < kColCopies; ++q)
        cs += *reinterpret_cast<volatile double*>(colacc + (size_t)q * bs + tid);
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
// plain coalesced loads (no per-system tensor maps), the same slab solve;
// the epilogue keeps the row sums of squares (rounding-shift estimate) and
// the diagonal tracker.
__global__ void __launch_bounds__(NTHR, 2)
trsm_batched_kernel(BatchSys* __restrict__ sys, int s, int b) {
  constexpr int TR = 32;
  const BatchSys& S = sys[blockIdx.y];
  const int n = S.n;
  const int bs = min(b, n - s);
  const int row0 = s + bs + blockIdx.x * TR;
  const int nrows = min(TR, n - row0);
  if (bs <= 0 || nrows <= 0 || S.st->code != 0) return;
  extern __shared__ __align__(128) float sm[];
  const int NT = bs / 32;                     // bs == b: only the last block can be partial
  float* Xs = sm;
  float* Lt = Xs + (size_t)bs * TR;
  float* Wt = Lt + (size_t)(NT * (NT - 1) / 2) * TSZ;
  __shared__ __align__(8) uint64_t ready[MAXNT];
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  const float* A = S.A;
  const int ld = S.ld;
  if (tid == 0) {
    s_ok = 1;
    for (int J = 0; J < NT; ++J) tc::mbar_init(&ready[J], 64);
    tc::fence_mbar_init();
  }
  for (int e = tid; e < bs * TR; e += NTHR) {
    const int c = e / TR, r = e % TR;
    Xs[xoff(r, c, bs)] = (r < nrows) ? A[(size_t)(s + c) * ld + row0 + r] : 0.0f;
  }
  for (int I = 1; I < NT; ++I)
    for (int M = 0; M < I; ++M)
      for (int e = tid; e < TSZ; e += NTHR) {
        const int c = e / 32, r = e % 32;
        Lt[tl(I, M) * TSZ + e] = A[(size_t)(s + 32 * M + c) * ld + s + 32 * I + r];
      }
  for (int e = tid; e < NT * TSZ; e += NTHR) Wt[e] = S.winv[e];
  __syncthreads();
  if (!slab_solve<1>(Xs, bs, Lt, Wt, nullptr, ready, tid)) {
    s_ok = 0;
    set_status(S.st, MPCHOL_ERR_TIMEOUT, row0);
  }
  __syncthreads();
  if (!s_ok) return;
  for (int e = tid; e < bs * TR; e += NTHR) {
    const int c = e / TR, r = e % TR;
    if (r < nrows) S.A[(size_t)(s + c) * ld + row0 + r] = Xs[xoff(r, c, bs)];
  }
  __shared__ float s_sq[NTHR / TR][TR];
  slab_row_partials<TR>(Xs, bs, s_sq, nullptr, tid);
  __syncthreads();
  if (tid < nrows) {
    const int gi = row0 + tid;
    const float sq = row_sq<TR>(s_sq, NT, tid);
    S.rowsq[gi] = sq;
    S.dtilde[gi] -= sq;
  }
}

int sm_count() {
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
      nsm = v;
    else
      return 148;
  }
  return nsm;
}

template <int RPL>
cudaError_t launch_panel(const CUtensorMap& tmapX, const CUtensorMap& tmap32, float* A, int lda,
                         int n, int s, int bs, const float* winv, const float* d, float* dtilde,
                         float* rowsq, StepState* step, StepState* next, int next_bs,
                         const DecisionParams& dp, const QuantAll& qa, DevStatus* st,
                         cudaStream_t stream, const StepState* prev, double* colacc) {
  constexpr int TR = 32 * RPL;
  const int m = n - s - bs;
  const size_t smem = trsm_smem_floats(TR, bs) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(trsm_panel_kernel<RPL>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(trsm_smem_floats(TR, 256) * sizeof(float)));
  if (e != cudaSuccess) return e;
  PdlLaunch L(dim3(ceil_div(m, TR)), dim3(NTHR), smem, stream);
  e = cudaLaunchKernelEx(&L.cfg, trsm_panel_kernel<RPL>, tmapX, tmap32, A, lda, n, s, bs, winv, d,
                         dtilde, rowsq, step, next, next_bs, dp, st, qa, prev, colacc);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
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
  if (bs % 32 != 0 || bs > 32 * MAXNT) return cudaErrorInvalidValue;
  // 64-row slabs while the panel has more 32-row slabs than the GPU has SMs
  // (throughput: L11 staged once per 64 rows); 32-row slabs otherwise
  // (latency: the per-CTA chain is half as long)
  if (ceil_div(m, 32) > sm_count())
    return launch_panel<2>(tmapX, tmap32, A, lda, n, s, bs, winv, d, dtilde, rowsq, step, next,
                           next_bs, dp, qa, st, stream, prev, colacc);
  return launch_panel<1>(tmapX, tmap32, A, lda, n, s, bs, winv, d, dtilde, rowsq, step, next,
                         next_bs, dp, qa, st, stream, prev, colacc);
}

cudaError_t launch_trsm_batched(BatchSys* sys, int nact, int s, int b, int max_m,
                                cudaStream_t stream) {
  if (nact <= 0 || max_m <= 0) return cudaSuccess;
  if (b % 32 != 0 || b > 32 * MAXNT) return cudaErrorInvalidValue;
  const size_t smem = trsm_smem_floats(32, b) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(trsm_batched_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  trsm_batched_kernel<<<dim3(ceil_div(max_m, 32), nact), NTHR, smem, stream>>>(sys, s, b);
  return cudaGetLastError();
}

}  // namespace mpchol
