// Panel TRSM with the fused switching epilogue.
//
// Replaces the reference's cublasStrsm of the panel (src/switching_chol.cuh:98-110,
// correct form RIGHT/LOWER/TRANS at src/sChol.cuh:273-280), its update_diag
// kernel (src/kernels_macros.cuh:177-190) and the per-row part of can_switch
// (src/kernels_macros.cuh:191-211).
//
// X * L11^T = A21 for the m rows below the diagonal block.  Rows are
// independent, so one CTA owns 64 rows for the whole solve.  One thread stages
// everything the CTA needs with TMA in a single round: its 64 x b slab of the
// panel (one 2-D box), the strictly-lower 32 x 32 tiles of L11 (2-D boxes) and
// the inverses of L11's diagonal tiles (a 1-D bulk copy of what the POTRF
// kernel wrote).  The CTA then walks the 32-column tiles J:
// X_J -= X_{<J} L_{J,<J}^T (register-tiled), X_J = X_J L_JJ^-T, writes the
// slab back with one TMA store and, in the epilogue, folds each row's sum of
// squares into the Schur-diagonal tracker dtilde and reduces the switching
// statistics (max d/dtilde, reference-literal choice) and the near-indefinite
// flag of the next diagonal block.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "quant.cuh"
#include "tc_ptx.cuh"

namespace mpchol {
namespace {

constexpr int TR = 64;       // rows per CTA
constexpr int NTHR = 256;    // 8 warps: 4 rows x 2 columns of each tile per thread
constexpr int CPT = 32 / (NTHR / 16);   // tile columns per thread
constexpr int TSZ = 32 * 32; // dense 32 x 32 tile
constexpr int XLD = TR;      // X staged column-major, rows contiguous

__device__ __forceinline__ int tl(int I, int M) { return I * (I - 1) / 2 + M; }  // I > M

size_t trsm_smem_floats(int bs) {
  const int NT = bs / 32;
  return (size_t)bs * XLD + (size_t)(NT * (NT - 1) / 2) * TSZ + (size_t)NT * TSZ + (size_t)TR * 32;
}

// Solve the staged 64-row slab in place: for each 32-column tile J,
// X_J -= X_{<J} L_{J,<J}^T, then X_J = X_J L_JJ^-T.
// The update splits K between two 128-thread groups: a thread keeps 4 rows x
// 4 columns of X_J in registers and does 16 FMAs per 16-byte load of X and of
// L.  Group 1's partial sums reach group 0 through red (64 x 32).
__device__ void trsm_slab(float* Xs, const float* Lt, const float* Wt, float* red, int NT, int tid) {
  const int g = tid / 128, t = tid % 128;
  const int r4 = t % 16, c4 = t / 16;        // update: rows 4*r4.., columns 4*c4.. of X_J
  const int tr = tid % 16, tc_ = tid / 16;   // inverse: rows 4*tr.., columns CPT*tc_..
  for (int J = 0; J < NT; ++J) {
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
        const float* lt = Lt + tl(J, kt) * TSZ + 4 * c4 + 16 * g * 32;
        const float* xt = Xs + (32 * kt + 16 * g) * XLD + 4 * r4;
#pragma unroll 8
        for (int kk = 0; kk < 16; ++kk) {
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
      if (g == 1) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          *reinterpret_cast<float4*>(&red[(4 * c4 + j) * TR + 4 * r4]) =
              make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
      }
      __syncthreads();
      if (g == 0) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float4 p = *reinterpret_cast<const float4*>(&red[(4 * c4 + j) * TR + 4 * r4]);
          *reinterpret_cast<float4*>(&Xs[(kend + 4 * c4 + j) * XLD + 4 * r4]) =
              make_float4(acc[0][j] + p.x, acc[1][j] + p.y, acc[2][j] + p.z, acc[3][j] + p.w);
        }
      }
      __syncthreads();
    }
    // X_J = X_J * L_JJ^-T :  x[r][c] = sum_{m<=c} a[r][m] * (L^-1)[c][m]
    float out[4][CPT] = {};
    const float* W = Wt + J * TSZ + CPT * tc_;
#pragma unroll 8
    for (int m = 0; m < 32; ++m) {
      const float4 av = *reinterpret_cast<const float4*>(&Xs[(kend + m) * XLD + 4 * tr]);
      const float ar[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const float wv = W[m * 32 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i][j] += ar[i] * wv;
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < CPT; ++j) Xs[(kend + CPT * tc_ + j) * XLD + 4 * tr + i] = out[i][j];
    __syncthreads();
  }
}

constexpr long long kGridBarPolls = 1ll << 24;
static_assert(NTHR == QTHR, "the fused quantizer runs with the panel solve's threads");

// Persistent panel solve with the quantization of the panel fused in.
// Phase 1: CTA c solves the 64-row slabs c, c + grid, ... (L11's tiles and
// tile inverses are staged once per CTA by TMA, each slab by one 2-D box),
// writes them back, and folds their rows into the diagonal tracker and the
// switching statistics.  A grid barrier (the launch is cooperative, so all
// CTAs are resident; the wait is bounded) then makes the statistics and the
// solved panel complete.  Phase 2: every CTA resolves the same step
// precision and quantizes 32-row tiles of the panel (read back from L2) into
// the K-major codes the trailing update reads, adding the step's rounding
// shift u_p * sum_j L_ij^2 to sh.
__global__ void __launch_bounds__(NTHR, 1)
trsm_panel_kernel(const __grid_constant__ CUtensorMap tmapX, const __grid_constant__ CUtensorMap tmap32,
                  float* __restrict__ A, int lda, int n, int s, int bs, const float* __restrict__ winv,
                  const float* __restrict__ d, float* __restrict__ dtilde, float* __restrict__ rowsq,
                  StepState* step, StepState* next, int next_bs, DecisionParams dp, DevStatus* st,
                  QuantOut qo) {
  extern __shared__ __align__(128) float sm[];
  const int NT = bs / 32;
  float* Xs = sm;                                        // [bs][XLD]
  float* Lt = Xs + (size_t)bs * XLD;                     // strictly-lower tiles of L11
  float* Wt = Lt + (size_t)(NT * (NT - 1) / 2) * TSZ;    // inverses of the diagonal tiles
  float* red = Wt + (size_t)NT * TSZ;                    // partial sums of the split update
  __shared__ float red_max[NTHR / 32];
  __shared__ int red_lit[NTHR / 32];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;

  const int tid = threadIdx.x;
  const int m = n - s - bs;
  const int nslab = ceil_div(m, TR);
  if (tid == 0) {
    s_ok = st->code == 0;
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase = 0;
  float bm = 0.0f;   // this CTA's max d/dtilde and literal code over its slabs
  int bl = 0;
  for (int slab = blockIdx.x; slab < nslab && s_ok; slab += gridDim.x, phase ^= 1u) {
    const int row0 = s + bs + slab * TR;                 // first global row of the slab
    const int nrows = min(TR, n - row0);
    // ---- stage with TMA (rows past n arrive as zeros) ---------------------
    if (tid == 0) {
      const bool first = slab == (int)blockIdx.x;
      const int nlt = NT * (NT - 1) / 2;
      uint32_t bytes = (uint32_t)(bs * XLD * sizeof(float));
      if (first) bytes += (uint32_t)((nlt * TSZ + NT * TSZ) * sizeof(float));
      tc::mbar_expect_tx(&bar, bytes);
      tc::tma_load_2d(Xs, &tmapX, &bar, row0, s);
      if (first) {
        for (int I = 1; I < NT; ++I)
          for (int M = 0; M < I; ++M)
            tc::tma_load_2d(Lt + tl(I, M) * TSZ, &tmap32, &bar, s + 32 * I, s + 32 * M);
        tc::bulk_load_1d(Wt, winv, (uint32_t)(NT * TSZ * sizeof(float)), &bar);
      }
      if (!tc::mbar_wait(&bar, phase)) {
        s_ok = 0;
        set_status(st, MPCHOL_ERR_TIMEOUT, row0);
        tc::mbar_wait(&bar, phase);
      }
    }
    __syncthreads();
    if (!s_ok) break;
    trsm_slab(Xs, Lt, Wt, red, NT, tid);
    // ---- write the solved slab back (coalesced; rows past n skipped) -----
    for (int e = tid; e < bs * TR; e += NTHR) {
      const int c = e / TR, r = e % TR;
      if (r < nrows) A[(size_t)(s + c) * lda + row0 + r] = Xs[c * XLD + r];
    }
    // ---- Schur diagonal tracker and switching statistics of the slab -----
    if (tid < nrows) {
      const int gi = row0 + tid;
      float sq = 0.0f;
      for (int c = 0; c < bs; ++c) { const float v = Xs[c * XLD + tid]; sq += v * v; }
      rowsq[gi] = sq;
      const float dt = dtilde[gi] - sq;
      dtilde[gi] = dt;
      const float di = d[gi];
      float ratio = dt > 0.0f ? di / dt : INFINITY;
      if (isnan(ratio)) ratio = INFINITY;
      bm = fmaxf(bm, ratio);
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
    __syncthreads();                                     // Xs is restaged next
  }
  // ---- statistics of the CTA, then the grid barrier ----------------------
  bm = warp_max(bm);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bl = max(bl, __shfl_xor_sync(0xffffffffu, bl, o));
  if ((tid & 31) == 0) { red_max[tid >> 5] = bm; red_lit[tid >> 5] = bl; }
  __threadfence();                                       // this thread's panel writes
  __syncthreads();
  if (tid == 0) {
    float cm = 0.0f; int cl = 0;
    for (int w = 0; w < NTHR / 32; ++w) { cm = fmaxf(cm, red_max[w]); cl = max(cl, red_lit[w]); }
    atomicMax(&step->max_ratio_bits, __float_as_uint(cm));
    atomicMax(&step->literal_code, cl);
    __threadfence();
    atomicAdd(&step->grid_bar, 1);
    long long it = 0;
    while (*reinterpret_cast<volatile int*>(&step->grid_bar) < (int)gridDim.x) {
      if (++it > kGridBarPolls) {
        set_status(st, MPCHOL_ERR_TIMEOUT, s);
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
  if (*reinterpret_cast<volatile int*>(&st->code) != 0) return;
  // ---- phase 2: the step precision and the quantized panel ----------------
  StepState ss;
  ss.max_ratio_bits = *reinterpret_cast<volatile unsigned int*>(&step->max_ratio_bits);
  ss.literal_code = *reinterpret_cast<volatile int*>(&step->literal_code);
  const int p = resolve_precision(&ss, dp);
  if (blockIdx.x == 0 && tid == 0) step->prec = p;
  if (p == FP32) return;
  const float* P = A + (size_t)s * lda + s + bs;
  const float u = unit_roundoff(p);
  for (int t = blockIdx.x; t * QROWS < m; t += gridDim.x) {
    if (qo.sh != nullptr)
      for (int r = tid; r < QROWS; r += NTHR) {
        const int gi = t * QROWS + r;
        if (gi < m) qo.sh[gi] += u * rowsq[s + bs + gi];
      }
    quantize_tile(P, lda, m, bs, p, qo.q, qo.ldq, qo.rowexp, qo.mxexp, qo.ldmx, Xs, m, t * QROWS);
    __syncthreads();                                     // the staging tile is reused
  }
}

// Batched: blockIdx.y = system, blockIdx.x = 64-row slab.  Staging by
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
  trsm_slab(Xs, Lt, Wt, red, NT, tid);
  for (int e = tid; e < bs * TR; e += NTHR) {
    const int c = e / TR, r = e % TR;
    if (r < nrows) S.A[(size_t)(s + c) * ld + row0 + r] = Xs[c * XLD + r];
  }
  if (tid < nrows) {
    const int gi = row0 + tid;
    float sq = 0.0f;
    for (int c = 0; c < bs; ++c) { const float v = Xs[c * XLD + tid]; sq += v * v; }
    S.rowsq[gi] = sq;
    S.dtilde[gi] -= sq;
  }
}

}  // namespace

cudaError_t launch_trsm_panel(const CUtensorMap& tmapX, const CUtensorMap& tmap32, float* A,
                              int lda, int n, int s, int bs, const float* winv, const float* d,
                              float* dtilde, float* rowsq, StepState* step, StepState* next,
                              int next_bs, const DecisionParams& dp, const QuantOut& qo,
                              DevStatus* st, cudaStream_t stream) {
  const int m = n - s - bs;
  if (m <= 0) return cudaSuccess;
  const size_t smem = trsm_smem_floats(bs) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(trsm_panel_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(trsm_smem_floats(256) * sizeof(float)));
  if (e != cudaSuccess) return e;
  // one CTA per SM at most (shared memory), all resident: the launch is
  // cooperative because the CTAs meet at a grid barrier
  static int nsm_cache[64] = {};
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  int& nsm = nsm_cache[dev & 63];
  if (nsm == 0) {
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
             &per_sm, trsm_panel_kernel, NTHR, trsm_smem_floats(256) * sizeof(float))) != cudaSuccess)
      return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
      return e;
    nsm = std::max(1, per_sm) * sms;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(std::min(ceil_div(m, TR), nsm));
  cfg.blockDim = dim3(NTHR);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, trsm_panel_kernel, tmapX, tmap32, A, lda, n, s, bs, winv, d, dtilde,
                         rowsq, step, next, next_bs, dp, st, qo);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_trsm_batched(BatchSys* sys, int nact, int s, int b, int max_m,
                                cudaStream_t stream) {
  if (nact <= 0 || max_m <= 0) return cudaSuccess;
  const size_t smem = trsm_smem_floats(b) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(trsm_batched_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  trsm_batched_kernel<<<dim3(ceil_div(max_m, TR), nact), NTHR, smem, stream>>>(sys, s, b);
  return cudaGetLastError();
}

}  // namespace mpchol
