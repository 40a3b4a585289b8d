// Internal launch interfaces of the mpchol kernels (not part of the C ABI).
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace mpchol {

// Launch configuration with programmatic stream serialization: the kernel
// may be scheduled while the kernel ahead of it in the stream finishes, and
// waits on griddepcontrol.wait before its first dependent access.
struct PdlLaunch {
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  PdlLaunch(dim3 grid, dim3 block, size_t smem, cudaStream_t stream) {
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
};

struct PotrfParams {
  int diag_pert;
  float pert;
  float pivot_floor;
};

// Per-step device-side decision state (one slot per factor step).
struct StepState {
  unsigned int max_ratio_bits;  // max_i d_i / dtilde_i over trailing rows (float bits, >= 0)
  int literal_code;             // reference-literal: max over rows of (2 - choice index); choice index 0 FP32, 1 FP16, 2 E4M3
  int prec;                     // chosen trailing-update precision (Fmt)
  int fp64_diag;                // 1: factor this step's diagonal block in FP64
  int grid_bar;                 // arrivals at the panel solve's grid barrier
  unsigned int not_min_dt_bits; // ~(float bits of min_i dtilde_i) over trailing rows (atomicMax of
                                // the complement gives the minimum; a non-positive or NaN dtilde
                                // counts as 0)
  unsigned int coh_bits;        // coherence ratio (||P^T 1||^2 / m) / min_i dtilde_i (float bits;
                                // +inf when min dtilde <= 0), set by the resolving CTA
  int pad;
};

struct DecisionParams {
  int policy;          // Fmt or SWITCHING
  int switch_mode;     // 0 build criterion, 1 reference-literal
  float eps_prime;
  float floor_ratio;   // near-indefinite flag threshold
  int ladder_len;
  int ladder[4];
  int coherence;       // switch_mode 0: also bound u_p * coherence ratio
  float eps_coh;       // ... by eps_coh (eps_prime when not set)
};

// ---- POTRF of the diagonal block (one CTA) ------------------------------
size_t potrf_smem_bytes(int bs);
size_t potrf_scratch64_elems(int bs);
// Also writes the inverses of the 32x32 diagonal tiles of the factored block
// to winv (ceil(bs/32) tiles, column-major 32x32 each) for the panel solve.
// tmap32: TMA map over A (FP32, n x n, column stride lda) with 32 x 32 boxes.
// With diagonal perturbation, the block's rows first receive the previous
// step's rounding shift, sh += u(prev->prec) * rowsq (prev null: none).
// compact: the small-code variant, for a POTRF that runs beside a long
// trailing update (the fully unrolled one is faster on its own but slows
// down several times when its instructions are refetched through a busy L2).
cudaError_t launch_potrf(const CUtensorMap& tmap32, float* A, int lda, int n, int s, int bs,
                         const float* d, float* sh, const PotrfParams& p,
                         const int* fp64_flag, double* scratch64, float* winv, DevStatus* st,
                         bool may_fp64, cudaStream_t stream, const StepState* prev = nullptr,
                         const float* rowsq = nullptr, bool compact = false);

// ---- panel TRSM + fused diagonal tracker, decision and quantization ------
// Where the panel solve writes the quantized panel: one K-major code panel
// per format the step may pick (row i of a panel holds the codes of trailing
// row i, ldq elements apart), with its scales, and the rounding-shift
// accumulator of the trailing rows (nullable).  FP16X2 keeps its hi codes in
// the FP16 panel (same scale rule) and its lo codes m rows further on.
struct QuantAll {
  unsigned cand;        // bit f set: format f is a candidate of the step
  int ldq;
  uint8_t* q8[3];       // E4M3, E5M2, MX-family codes (slot q8_slot)
  uint16_t* q16;        // FP16 / FP16X2 hi codes, then FP16X2 lo codes
  int8_t* rexp[3];      // per-row pow-2 exponents: E4M3, E5M2, FP16 / FP16X2
  uint8_t* mxexp;       // MX-family E8M0 scales, ldmx per row
  int ldmx;
  float* sh;
};
__host__ __device__ inline int q8_slot(int fmt) { return fmt == E4M3 ? 0 : (fmt == E5M2 ? 1 : 2); }
__host__ __device__ inline int rexp_slot(int fmt) { return fmt == E4M3 ? 0 : (fmt == E5M2 ? 1 : 2); }
// Solves X * L11^T = A21 in place for rows [s+bs, n) of block column s, one
// slab of 32 or 64 rows per CTA; subtracts each row's sum of squares from dtilde,
// stores it in rowsq, folds the switching statistics into step (and the FP64
// flag of the next diagonal block into next), and writes the slab's codes in
// every candidate format.  The last CTA to finish resolves the step precision
// (step->prec).  Before its rows' sums of squares are overwritten, each CTA
// adds the previous step's rounding shift u(prev->prec) * rowsq to qa.sh for
// its rows (prev null: first step); the rows of the next diagonal block get
// theirs in its POTRF.  tmapX: TMA map over A with 32 x bs boxes; tmap32 as
// for launch_potrf.
// colacc (coherence rule, nullable otherwise): kColCopies x bs FP64
// accumulators, zeroed before the launch, that receive the panel's column
// sums (slab i adds into copy i % kColCopies).
constexpr int kColCopies = 8;
cudaError_t launch_trsm_panel(const CUtensorMap& tmapX, const CUtensorMap& tmap32, float* A,
                              int lda, int n, int s, int bs, const float* winv, const float* d,
                              float* dtilde, float* rowsq, StepState* step, StepState* next,
                              int next_bs, const DecisionParams& dp, const QuantAll& qa,
                              DevStatus* st, cudaStream_t stream, const StepState* prev = nullptr,
                              double* colacc = nullptr);

// ---- panel quantization ---------------------------------------------------
// Fixed-format variant (test entry point): no decision, no shift.
cudaError_t launch_quantize_rows(const float* P, int ldp, int m, int k, int fmt, void* q, int ldq,
                                 int8_t* rowexp, uint8_t* mxexp, int ldmx, cudaStream_t stream);
cudaError_t launch_quantize_elems(const float* x, void* q, long long count, int fmt,
                                  cudaStream_t stream);
cudaError_t launch_quantize_hash(unsigned long long first, unsigned long long count,
                                 unsigned long long chunk, int fmt, unsigned long long* hashes,
                                 cudaStream_t stream);

// ---- trailing update ----------------------------------------------------
// Which lower 128 x 128 tiles (I >= J) of the trailing block C a launch
// updates: all of them, only the tiles of the next diagonal block (I, J < jc:
// SEL_NEXT), or the rest (I >= jc: SEL_REST), which includes the next
// block's panel.  Splitting a step's update this way lets the next diagonal
// block be factored while the rest of the update runs (look-ahead).  The
// tiles are numbered along the rows of the lower triangle, so SEL_NEXT is
// the first jc(jc+1)/2 of them and SEL_REST the remainder.
// SEL_BAND picks the tiles of tile columns [jlo, jhi) with I >= max(J, ilo),
// numbered down each column: the columns of A that are on the device while
// the rest is still being copied (ilo = jc: the rest of a step's update over
// those columns), or the late columns' update by an earlier panel (ilo = 0).
enum TileSelMode { SEL_ALL = 0, SEL_NEXT = 1, SEL_REST = 2, SEL_BAND = 3 };
struct TileSel {
  int mode;
  int jc;
  int jlo = 0, jhi = 0, ilo = 0;   // SEL_BAND only
};
constexpr TileSel kAllTiles{SEL_ALL, 0};

__host__ __device__ inline int sel_tile_count(int T, TileSel s) {
  if (s.mode == SEL_BAND) {
    const int j1 = s.jhi < T ? s.jhi : T;
    int c = 0;
    for (int j = s.jlo < 0 ? 0 : s.jlo; j < j1; ++j) {
      const int i0 = j > s.ilo ? j : s.ilo;
      if (i0 < T) c += T - i0;
    }
    return c;
  }
  const int all = T * (T + 1) / 2;
  const int j = s.jc < T ? s.jc : T;
  const int head = j * (j + 1) / 2;
  if (s.mode == SEL_NEXT) return head;
  if (s.mode == SEL_REST) return all - head;
  return all;
}

// Tile t (< sel_tile_count) of the selection -> (I, J).
__host__ __device__ __forceinline__ void sel_tile(int t, TileSel s, int T, int& I, int& J) {
  if (s.mode == SEL_BAND) {
    const int j1 = s.jhi < T ? s.jhi : T;
    for (int j = s.jlo < 0 ? 0 : s.jlo; j < j1; ++j) {
      const int i0 = j > s.ilo ? j : s.ilo;
      const int cnt = T - i0 > 0 ? T - i0 : 0;
      if (t < cnt) { I = i0 + t; J = j; return; }
      t -= cnt;
    }
    I = J = 0;   // not reached for t < sel_tile_count(T, s)
    return;
  }
  if (s.mode == SEL_REST) {
    const int j = s.jc < T ? s.jc : T;
    t += j * (j + 1) / 2;
  }
  int i = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (i * (i + 1) / 2 > t) --i;
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  I = i;
  J = t - i * (i + 1) / 2;
}

// FP32 SIMT SYRK: C(m x m, lower) -= P P^T, P = m x k column-major (ldp),
// over the tiles `sel` picks.  Skips (returns immediately on device) unless
// *prec_sel == FP32 when prec_sel is non-null.  max_sms > 0: a persistent
// launch on at most that many SMs (one CTA of two 256-thread tile groups per
// SM), so the other SMs stay free.
cudaError_t launch_syrk_f32(float* C, int ldc, int m, int k, const float* P, int ldp,
                            const int* prec_sel, DevStatus* st, cudaStream_t stream,
                            TileSel sel = kAllTiles, int max_sms = 0);
// tcgen05 SYRK from the K-major quantized panel (FP16 / E4M3 / E5M2 / MXFP8 /
// FP16X2), one format per launch.
bool syrk_tc_supported(int fmt, int k);
cudaError_t launch_syrk_tc(float* C, int ldc, int m, int k, int fmt, const void* q, int ldq,
                           const int8_t* rowexp, const uint8_t* mxexp, int ldmx,
                           const int* prec_sel, DevStatus* st, cudaStream_t stream,
                           TileSel sel = kAllTiles, int max_sms = 0);
// The same with the format read on the device from *prec_sel (the step's
// resolved precision); fmt_mask (bit f for format f) lists the formats the
// step may pick.  The launch returns at once when the pick is not among
// them (FP32 steps go to launch_syrk_f32).  max_sms > 0 caps the grid.
// The panels and scales of each format are those of qa (the panel solve's
// outputs).
cudaError_t launch_syrk_tc_dispatch(float* C, int ldc, int m, int k, unsigned fmt_mask,
                                    const QuantAll& qa, const int* prec_sel, DevStatus* st,
                                    cudaStream_t stream, TileSel sel = kAllTiles, int max_sms = 0);

// ---- batched factorization and solve of many independent systems --------
// Systems are ordered by decreasing n, so the systems still active at a
// factor step are a prefix of the array.
struct BatchSys {
  float* A;            // factor storage (copy of the input), column-major, ld
  int ld;
  int n;
  float* d;            // original diagonal (pivot floors)
  float* dtilde;       // diagonal tracker (not used for decisions in batch mode)
  float* rowsq;        // per-row sum of squares of the latest panel
  float* sh;           // rounding-shift accumulator
  float* winv;         // inverses of the current diagonal block's 32-tiles
  float* wsup;         // super-block inverses for the solves
  DevStatus* st;
  // solve side
  const float* op;     // PCG operator (FP32, column-major, lda = op_ld)
  int op_ld;
  double* vec;         // 8 vector slots of n x nr (column-major), slot s at vec + s*n*nr
  double* part;        // partial sums: 4 groups x BATCH_VB x 8
  double* scal;        // 64 scalars (rho[2], alpha, bnorm2, misc)
  int* done;           // [0] converged (recursive residual), [1] iterations
  int sym_tile0;       // first unit of the system in the batched operator product
};
// Per system and factor step.
struct BatchStep {
  int m;               // trailing rows after this step's diagonal block (<= 0: none)
  int q_row0;          // first row of the system's panel in the panel arena (multiple of 128)
  int tile0;           // first tile of the system in this step's SYRK tile numbering
};
constexpr int BATCH_VB = 4;   // partial-sum blocks per system in the batched PCG reductions

cudaError_t launch_potrf_batched(BatchSys* sys, int nact, int s, int b, const PotrfParams& p,
                                 cudaStream_t stream);
cudaError_t launch_trsm_batched(BatchSys* sys, int nact, int s, int b, int max_m,
                                cudaStream_t stream);
cudaError_t launch_quantize_batched(BatchSys* sys, const BatchStep* steps, int nact, int s, int b,
                                    int max_m, int fmt, void* q, int qrows, int8_t* rowexp,
                                    uint8_t* mxexp, int diag_pert, cudaStream_t stream);
cudaError_t launch_syrk_tc_batched(BatchSys* sys, const BatchStep* steps, int nact, int ntiles,
                                   int s, int b, int fmt, const void* q, int qrows,
                                   const int8_t* rowexp, const uint8_t* mxexp,
                                   cudaStream_t stream);

// ---- PCG building blocks ------------------------------------------------
template <typename TA>
cudaError_t launch_symv(const TA* A, int lda, int n, const double* x, double* y, int nrhs,
                        cudaStream_t stream);

}  // namespace mpchol
