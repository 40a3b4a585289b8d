// Tensor-core trailing update (tcgen05 + TMEM + TMA) for the low-precision
// steps of the factorization.
//
// Replaces the reference's cuBLASLt trailing updates LtHSgemm_fp16in_fp32out
// (src/switching_chol.cuh:170-197, src/fp8_utils.cuh:304-412), the per-tensor
// scaled FP8 CUTLASS GEMM (src/fp8Chol.cuh:236-275) and the WMMA SYRK
// (src/syrk_gemm.cuh:14-124).
//
// C(m x m, lower 128 x 128 tiles) -= s_i s_j (Q Q^T), Q the K-major quantized
// panel with per-row power-of-two scales s, FP32 accumulation in tensor memory.
// FP16X2 carries each panel value as hi + lo (two FP16 terms) and accumulates
// hi hi^T + hi lo^T + lo hi^T, which is FP32-class accurate at FP16 tensor
// speed.
//
// Persistent and warp-specialized, one CTA per SM (320 threads):
//   warp 0  TMA producer: K chunks of 128 bytes per row (one 128-byte swizzle
//           row) of the A strip (rows of tile I) and the B strip (rows of tile
//           J; skipped on diagonal tiles) into a ring of NSTAGE stages;
//   warp 1  allocates the TMEM columns; one thread issues tcgen05.mma and
//           commits each stage back to the producer and each finished tile to
//           the epilogue;
//   warps 2-9 epilogue, two per 32-lane TMEM quarter (64 columns each):
//           tcgen05.ld of the accumulator and the scaled update of C in
//           32 x 32 boxes.  Each warp prefetches its boxes of C for the next
//           tile by TMA loads while it finishes the current one, subtracts
//           the update in shared memory and writes the boxes back by TMA
//           stores: C crosses DRAM once each way with the reads issued a tile
//           ahead.  (Adding the update by TMA reduce-adds instead leaves the
//           read of C to the L2, which fetches each line from DRAM when the
//           reduction arrives; at n = 16384 that ran DRAM at half its
//           bandwidth.  FP16X2, whose three operand sets leave no room for
//           the prefetch boxes, still adds by reduce-adds; batched launches,
//           whose C differs per system, use coalesced loads and stores.)
// The two TMEM accumulators let the epilogue of one tile overlap the MMAs of
// the next.  Every mbarrier wait is bounded.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_ptx.cuh"
#include "tmap.cuh"

namespace mpchol {
namespace {

constexpr int TM = 128;                    // output tile (M = N = 128)
constexpr int CHUNK = 128;                 // bytes of K per row per stage
constexpr int STRIP = TM * CHUNK;          // 16 KB: one operand strip chunk
constexpr int EPI_WARPS = 8;               // two per TMEM lane quarter, half the columns each
constexpr int NTHREADS = 64 + 32 * EPI_WARPS;

// NSTAGE: operand stages of batched launches (no epilogue boxes) and of the
// reduce-add epilogue (with EPI_BUFS boxes per epilogue warp); LDST_STAGES:
// operand stages beside the four C boxes per epilogue warp of the load /
// store epilogue (0: none), which a launch uses for K <= LDST_MAX_K.  Beyond
// that K the fewer stages starve the MMAs while C's traffic per flop falls
// (B200, m = 15360-16128: MXFP8 at K = 512 0.254 ms with load / store
// against 0.238 ms with reduce-adds, FP16 at K = 1024 0.414 against 0.361;
// E4M3 at K = 512 0.196 against 0.234).
template <int FMT> struct TcCfg;
template <> struct TcCfg<FP16> {
  static constexpr int ESIZE = 2, NSETS = 1, NSTAGE = 4, EPI_BUFS = 2, LDST_STAGES = 3, LDST_MAX_K = 256;
  static constexpr bool MX = false;
  static constexpr uint32_t IDESC = tc::make_idesc(0, 0, TM, TM);
};
template <> struct TcCfg<E4M3> {
  static constexpr int ESIZE = 1, NSETS = 1, NSTAGE = 4, EPI_BUFS = 2, LDST_STAGES = 3, LDST_MAX_K = 512;
  static constexpr bool MX = false;
  static constexpr uint32_t IDESC = tc::make_idesc(0, 0, TM, TM);
};
template <> struct TcCfg<E5M2> {
  static constexpr int ESIZE = 1, NSETS = 1, NSTAGE = 4, EPI_BUFS = 2, LDST_STAGES = 3, LDST_MAX_K = 512;
  static constexpr bool MX = false;
  static constexpr uint32_t IDESC = tc::make_idesc(1, 1, TM, TM);
};
template <> struct TcCfg<FP16X2> {
  static constexpr int ESIZE = 2, NSETS = 2, NSTAGE = 3, EPI_BUFS = 1, LDST_STAGES = 0, LDST_MAX_K = 0;
  static constexpr bool MX = false;
  static constexpr uint32_t IDESC = tc::make_idesc(0, 0, TM, TM);
};
// MXFP8: E4M3 codes with one E8M0 scale per 32 K-elements, applied by the
// block-scaled MMA (kind::mxf8f6f4) from scales staged in tensor memory.
// Two stages hold a whole K = 256 tile.
template <> struct TcCfg<MXFP8> {
  static constexpr int ESIZE = 1, NSETS = 1, NSTAGE = 4, EPI_BUFS = 2, LDST_STAGES = 2, LDST_MAX_K = 256;
  static constexpr bool MX = true;
  static constexpr uint32_t IDESC = tc::make_idesc_mx(0, 0, TM, TM);
};
// The epilogue of a launch: load / store (LDST), reduce-add (RED) or, for
// batched launches, neither (coalesced loads and stores of C).
template <int FMT, bool BATCH, bool WIDE> struct TcPlan {
  using Cfg = TcCfg<FMT>;
  static constexpr bool LDST = !BATCH && !WIDE && Cfg::LDST_STAGES > 0;
  static constexpr bool RED = !BATCH && !LDST;
  static constexpr int NSTAGE = LDST ? Cfg::LDST_STAGES : Cfg::NSTAGE;
  static constexpr int EPI_BOXES = BATCH ? 0 : (LDST ? 4 : Cfg::EPI_BUFS);   // per epilogue warp
};

// Scales of one stage (a 128-element K chunk = four 32-element blocks) for
// 128 rows, in the layout the 32x128b tensor-memory copy reads: 32 lines of
// 16 bytes; line l holds, in 32-bit word w, the four block scales of row
// 32 w + l (byte b = block b of the chunk).
constexpr int SF_BYTES = 512;

__device__ __forceinline__ void stage_scales(uint8_t* sf, const uint8_t* __restrict__ mxexp,
                                             int ldmx, int row0, int m, int kc, int lane) {
  uint32_t w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int row = row0 + 32 * q + lane;
    // rows past m multiply zero codes: give them a unit scale (code 127)
    w[q] = (row < m) ? *reinterpret_cast<const uint32_t*>(mxexp + (size_t)row * ldmx + 4 * kc)
                     : 0x7F7F7F7Fu;
  }
  *reinterpret_cast<uint4*>(sf + 16 * lane) = make_uint4(w[0], w[1], w[2], w[3]);
}

struct TcMaps {
  CUtensorMap hi;   // main (or hi) panel: rows m, K-major
  CUtensorMap lo;   // lo panel (FP16X2 only)
  CUtensorMap c;    // the trailing block C (FP32, m x m, 32 x 32 boxes)
};
constexpr int STAGE_C = 32 * 32 * 4;        // one 32 x 32 FP32 box of C

// Batched launches: the tiles of all active systems are numbered in one
// sequence (system i owns [steps[i].tile0, steps[i+1].tile0)); each system's
// panel sits at rows steps[i].q_row0.. of the shared panel arena.
struct TcBatch {
  BatchSys* sys;
  const BatchStep* steps;
  int nact;
  int s;
  int b;
};

// Where tile t of the launch writes: C (ld ldc, m x m lower), its tile
// coordinates and the first row of its panel in the panel arena.
struct TileCtx {
  int I, J;
  float* C;
  int ldc;
  int m;
  int row0;
};

template <bool BATCH>
__device__ __forceinline__ TileCtx tile_ctx(int t, const TcBatch& bt, float* C, int ldc, int m,
                                            TileSel sel) {
  TileCtx c;
  if (!BATCH) {
    sel_tile(t, sel, (m + TM - 1) / TM, c.I, c.J);
    c.C = C; c.ldc = ldc; c.m = m; c.row0 = 0;
    return c;
  }
  int lo = 0, hi = bt.nact - 1;           // last system with tile0 <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bt.steps[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const BatchSys& S = bt.sys[lo];
  const BatchStep& T = bt.steps[lo];
  sel_tile(t - T.tile0, kAllTiles, (T.m + TM - 1) / TM, c.I, c.J);
  c.C = S.A + (size_t)(bt.s + bt.b) * S.ld + bt.s + bt.b;
  c.ldc = S.ld;
  c.m = T.m;
  c.row0 = T.q_row0;
  return c;
}

// The kernel body for one format.  mhi / mlo / mc point at tensor maps in the
// launch's parameter space (TMA reads them from there).
template <int FMT, bool BATCH, bool WIDE>
__device__ __forceinline__ void
syrk_tc_body(const CUtensorMap* mhi, const CUtensorMap* mlo, const CUtensorMap* mc,
             float* __restrict__ C, int ldc, int m, int k, const int8_t* __restrict__ rowexp,
             const uint8_t* __restrict__ mxexp, int ldmx, DevStatus* st, const TcBatch& bt,
             int ntiles_b, TileSel sel) {
  using Cfg = TcCfg<FMT>;
  using Plan = TcPlan<FMT, BATCH, WIDE>;
  if (st != nullptr && st->code != 0) return;
  constexpr int NS = Plan::NSTAGE;
  constexpr int NSETS = Cfg::NSETS;
  constexpr bool MX = Cfg::MX;
  // A sets, B sets, then (MXFP8) the A and B scales of the chunk
  constexpr int STAGE_BYTES = 2 * NSETS * STRIP + (MX ? 2 * SF_BYTES : 0);
  constexpr uint32_t TMEM_COLS = MX ? 4 * TM : 2 * TM;  // accumulators (+ scales)
  constexpr bool RED = Plan::RED;
  constexpr bool LDST = Plan::LDST;
  constexpr int KSTEP = 32;                             // bytes of K per MMA
  constexpr int ELEMS_PER_CHUNK = CHUNK / Cfg::ESIZE;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[NS];
  __shared__ __align__(8) uint64_t empty_bar[NS];
  __shared__ __align__(8) uint64_t accf_bar[2];
  __shared__ __align__(8) uint64_t acce_bar[2];
  __shared__ __align__(8) uint64_t cld_bar[EPI_WARPS][2];   // LDST: each warp's C boxes landed
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int T = (m + TM - 1) / TM;
  const int ntiles = BATCH ? ntiles_b : sel_tile_count(T, sel);
  const int nchunks = (k * Cfg::ESIZE) / CHUNK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) { tc::mbar_init(&full_bar[s], 1); tc::mbar_init(&empty_bar[s], 1); }
    for (int b = 0; b < 2; ++b) { tc::mbar_init(&accf_bar[b], 1); tc::mbar_init(&acce_bar[b], EPI_WARPS); }
    if (LDST)
      for (int w = 0; w < EPI_WARPS; ++w) { tc::mbar_init(&cld_bar[w][0], 1); tc::mbar_init(&cld_bar[w][1], 1); }
    tc::fence_mbar_init();
    tc::prefetch_tmap(mhi);
    if (NSETS == 2) tc::prefetch_tmap(mlo);
    abort_sh = 0;
  }
  if (warp == 1) tc::tmem_alloc(&tmem_base_sh, TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    // lane 0 waits and issues the copies; for MXFP8 the whole warp stages the
    // chunk's scales into the stage first
    int c = 0;   // global chunk counter
    bool failed = false;
    for (int t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
      const TileCtx tc_ = tile_ctx<BATCH>(t, bt, C, ldc, m, sel);
      const int I = tc_.I, J = tc_.J;
      const bool diag = (I == J);
      const uint32_t bytes = (uint32_t)((diag ? 1 : 2) * NSETS * STRIP);
      for (int kc = 0; kc < nchunks; ++kc, ++c) {
        const int s = c % NS;
        const uint32_t pass = (uint32_t)(c / NS);
        int ok = 1;
        if (lane == 0) ok = (!abort_sh && tc::mbar_wait(&empty_bar[s], (pass & 1u) ^ 1u)) ? 1 : 0;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
          if (lane == 0) {
            abort_sh = 1;
            if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, t);
          }
          failed = true;
          break;
        }
        uint8_t* base = smem + (size_t)s * STAGE_BYTES;
        if (MX) {
          uint8_t* sf = base + 2 * NSETS * STRIP;
          const uint8_t* mx = mxexp + (size_t)tc_.row0 * ldmx;
          stage_scales(sf, mx, ldmx, I * TM, tc_.m, kc, lane);
          if (!diag) stage_scales(sf + SF_BYTES, mx, ldmx, J * TM, tc_.m, kc, lane);
          tc::fence_proxy_async_smem();    // generic writes -> async-proxy reader
          __syncwarp();
        }
        if (lane == 0) {
          tc::mbar_expect_tx(&full_bar[s], bytes);
          const int x = kc * ELEMS_PER_CHUNK;
          const int yi = tc_.row0 + I * TM, yj = tc_.row0 + J * TM;
          tc::tma_load_2d(base, mhi, &full_bar[s], x, yi);
          if (NSETS == 2) tc::tma_load_2d(base + STRIP, mlo, &full_bar[s], x, yi);
          if (!diag) {
            tc::tma_load_2d(base + NSETS * STRIP, mhi, &full_bar[s], x, yj);
            if (NSETS == 2)
              tc::tma_load_2d(base + (NSETS + 1) * STRIP, mlo, &full_bar[s], x, yj);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int c = 0, tcount = 0;
      for (int t = blockIdx.x; t < ntiles && !abort_sh; t += gridDim.x, ++tcount) {
        const TileCtx tc_ = tile_ctx<BATCH>(t, bt, C, ldc, m, sel);
        const bool diag = (tc_.I == tc_.J);
        const int buf = tcount & 1;
        const uint32_t use = (uint32_t)(tcount >> 1);
        if (!tc::mbar_wait(&acce_bar[buf], (use & 1u) ^ 1u)) {
          abort_sh = 1;
          if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, t);
          break;
        }
        tc::tc_fence_after();
        const uint32_t dacc = tmem + (uint32_t)(buf * TM);
        uint32_t accumulate = 0;
        bool ok = true;
        for (int kc = 0; kc < nchunks; ++kc, ++c) {
          const int s = c % NS;
          const uint32_t pass = (uint32_t)(c / NS);
          if (!tc::mbar_wait(&full_bar[s], pass & 1u)) {
            abort_sh = 1;
            if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, t);
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t a_hi = tc::smem_u32(smem + (size_t)s * STAGE_BYTES);
          const uint32_t a_lo = a_hi + STRIP;
          const uint32_t b_hi = diag ? a_hi : a_hi + NSETS * STRIP;
          const uint32_t b_lo = diag ? a_lo : a_hi + (NSETS + 1) * STRIP;
          // MXFP8: this chunk's scales -> TMEM columns 2*TM + buf*64 + kc*8
          // (A at +0, B at +4; kc < 8 for K <= 1024); chunks and accumulator
          // buffers use separate columns, so no copy overwrites scales an
          // unfinished MMA reads
          uint32_t sfa_t = 0, sfb_t = 0;
          if (MX) {
            const uint32_t sfa_s = a_hi + 2 * NSETS * STRIP;
            const uint32_t sfb_s = diag ? sfa_s : sfa_s + SF_BYTES;
            sfa_t = tmem + (uint32_t)(2 * TM + buf * 64 + kc * 8);
            sfb_t = sfa_t + 4;
            tc::utccp_32x128b_warpx4(sfa_t, tc::make_desc_plain(sfa_s, 128));
            tc::utccp_32x128b_warpx4(sfb_t, tc::make_desc_plain(sfb_s, 128));
          }
#pragma unroll
          for (int kk = 0; kk < CHUNK / KSTEP; ++kk) {
            const uint32_t off = kk * KSTEP;
            const uint64_t ad = tc::make_desc_sw128(a_hi + off);
            const uint64_t bd = tc::make_desc_sw128(b_hi + off);
            if (MX)
              tc::mma_mxf8f6f4(dacc, ad, bd, tc::idesc_sf_ids(Cfg::IDESC, kk, kk), accumulate,
                               sfa_t | ((uint32_t)kk << 30), sfb_t | ((uint32_t)kk << 30));
            else if (FMT == FP16 || FMT == FP16X2) tc::mma_f16(dacc, ad, bd, Cfg::IDESC, accumulate);
            else tc::mma_f8f6f4(dacc, ad, bd, Cfg::IDESC, accumulate);
            accumulate = 1;
            if (NSETS == 2) {
              tc::mma_f16(dacc, ad, tc::make_desc_sw128(b_lo + off), Cfg::IDESC, 1);
              tc::mma_f16(dacc, tc::make_desc_sw128(a_lo + off), bd, Cfg::IDESC, 1);
            }
          }
          tc::mma_commit(&empty_bar[s]);     // stage free once these MMAs finish
        }
        if (!ok) break;
        tc::mma_commit(&accf_bar[buf]);      // tile accumulated
      }
    }
  } else {
    // ---------------- epilogue (warps 2..5) ----------------
    const int q = warp & 3;                  // TMEM lane quarter this warp may access
    const int half = (warp - 2) >> 2;        // which 64 columns of the tile
    const int ew = warp - 2;
    // RED: EPI_BUFS staging boxes per warp, used in turn (with two, a box is
    // filled while the previous one is still being read by its reduce-add).
    // LDST: two sets of the warp's two boxes of C, one for the tile being
    // finished and one for the next tile's prefetch.
    constexpr int EB = Plan::EPI_BOXES;
    float* stg0 = reinterpret_cast<float*>(smem + (size_t)NS * STAGE_BYTES +
                                           (size_t)ew * STAGE_C * (EB > 0 ? EB : 1));
    // box hb (0, 1) of this warp in tile (I, J): rows I*TM + 32 q, columns
    // J*TM + 64 half + 32 hb; boxes wholly above the diagonal or past m are
    // skipped
    auto box_ok = [&](int I, int J, int mt, int hb) {
      const int i0 = I * TM + q * 32, j0 = J * TM + half * (TM / 2) + hb * 32;
      return i0 < mt && j0 < mt && !(I == J && j0 >= i0 + 32);
    };
    // LDST: TMA loads of tile t's boxes into set `set` (lane 0)
    auto load_boxes = [&](int t, int set) {
      const TileCtx x = tile_ctx<BATCH>(t, bt, C, ldc, m, sel);
      uint32_t bytes = 0;
      for (int hb = 0; hb < 2; ++hb) bytes += box_ok(x.I, x.J, x.m, hb) ? (uint32_t)STAGE_C : 0u;
      tc::mbar_expect_tx(&cld_bar[ew][set], bytes);
      for (int hb = 0; hb < 2; ++hb)
        if (box_ok(x.I, x.J, x.m, hb))
          tc::tma_load_2d(stg0 + (set * 2 + hb) * (STAGE_C / 4), mc, &cld_bar[ew][set],
                          x.I * TM + q * 32, x.J * TM + half * (TM / 2) + hb * 32);
    };
    int nbox = 0;
    int tcount = 0;
    // LDST: per set, the phase parity of loads issued and not yet waited for
    // (-1: none)
    int opar0 = -1, opar1 = -1;
    if (LDST && blockIdx.x < ntiles) {
      if (lane == 0) load_boxes(blockIdx.x, 0);
      opar0 = 0;
    }
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tcount) {
      const TileCtx tc_ = tile_ctx<BATCH>(t, bt, C, ldc, m, sel);
      const int I = tc_.I, J = tc_.J;
      float* Ct = tc_.C;
      const int ldct = tc_.ldc, mt = tc_.m;
      const int8_t* rexp = rowexp + tc_.row0;
      const int buf = tcount & 1;
      const uint32_t use = (uint32_t)(tcount >> 1);
      if (LDST && t + (int)gridDim.x < ntiles) {
        // prefetch the next tile's boxes into the other set, once the stores
        // of the tile that used it have read their boxes
        if (lane == 0) {
          tc::bulk_wait_smem_read();
          load_boxes(t + gridDim.x, buf ^ 1);
        }
        __syncwarp();
        const int par = (int)(((tcount + 1) >> 1) & 1);
        if (buf) opar0 = par; else opar1 = par;
      }
      if (!tc::mbar_wait(&accf_bar[buf], use & 1u)) {
        if (lane == 0) { abort_sh = 1; if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, t); }
        break;
      }
      if (LDST) {
        if (!tc::mbar_wait(&cld_bar[ew][buf], use & 1u)) {
          if (lane == 0) { abort_sh = 1; if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, t); }
          break;
        }
        if (buf) opar1 = -1; else opar0 = -1;
      }
      tc::tc_fence_after();
      const int i = I * TM + q * 32 + lane;
      const float si = (i < mt) ? (MX ? 1.0f : pow2f(__ldg(rexp + i))) : 0.0f;
      const uint32_t taddr = tmem + (uint32_t)(buf * TM) + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
      for (int c0 = half * (TM / 2); c0 < (half + 1) * (TM / 2); c0 += 32) {
        float v[32];
        tc::tmem_ld32(taddr + (uint32_t)c0, v);
        if (c0 + 32 >= (half + 1) * (TM / 2)) {
          // last read of this accumulator: hand it back to the MMA warp
          tc::tc_fence_before();
          __syncwarp();
          if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(&acce_bar[buf])) : "memory");
        }
        const int j0 = J * TM + c0;
        // column scales of the box: lane u loads s_{j0+u} once, the element
        // loops take it by shuffle
        const float sj_lane = (!MX && j0 + lane < mt) ? pow2f(__ldg(rexp + j0 + lane)) : 1.0f;
        if (LDST) {
          // C(rows i0.., cols j0..) -= s_i s_j acc in the prefetched box, then
          // one TMA store; entries above the diagonal keep their value
          const int i0 = I * TM + q * 32;
          const int hb = (c0 - half * (TM / 2)) / 32;
          if (box_ok(I, J, mt, hb)) {
            float* bx = stg0 + (buf * 2 + hb) * (STAGE_C / 4);
#pragma unroll
            for (int u = 0; u < 32; ++u) {
              const float sj = MX ? 1.0f : __shfl_sync(0xffffffffu, sj_lane, u);
              const float cv = bx[u * 32 + lane];
              bx[u * 32 + lane] = (I == J && j0 + u > i) ? cv : cv - (v[u] * si) * sj;
            }
            tc::fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
              tc::tma_store_2d(mc, bx, i0, j0);
              tc::bulk_commit();
            }
          }
        } else if (RED) {
          // C(rows i0.., cols j0..) += -(s_i s_j acc) as one 32 x 32 TMA
          // reduce-add; boxes wholly above the diagonal or past m are skipped,
          // and entries above the diagonal add -0.0, which leaves every value
          // (signed zeros included) as it was
          const int i0 = I * TM + q * 32;
          if (i0 < mt && j0 < mt && !(I == J && j0 >= i0 + 32)) {
            float* stg = stg0 + (EB > 0 ? nbox % EB : 0) * (STAGE_C / 4);
            ++nbox;
            // the box that last used this buffer has been read
            if (lane == 0) {
              if (EB == 2) tc::bulk_wait_smem_read_1();
              else tc::bulk_wait_smem_read();
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < 32; ++u) {
              const float sj = MX ? 1.0f : __shfl_sync(0xffffffffu, sj_lane, u);
              stg[u * 32 + lane] = (I == J && j0 + u > i) ? -0.0f : -((v[u] * si) * sj);
            }
            tc::fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
              tc::tma_reduce_add_2d(mc, stg, i0, j0);
              tc::bulk_commit();
            }
          }
        } else {
          // every lane takes part (the shuffles); rows past m only skip the stores
          const bool row_ok = i < mt;
          float cv[32];
#pragma unroll
          for (int u = 0; u < 32; ++u) {
            const int j = j0 + u;
            cv[u] = (row_ok && j < mt && i >= j) ? Ct[(size_t)j * ldct + i] : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < 32; ++u) {
            const int j = j0 + u;
            const float sj = MX ? 1.0f : __shfl_sync(0xffffffffu, sj_lane, u);
            if (row_ok && j < mt && i >= j) Ct[(size_t)j * ldct + i] = cv[u] - (v[u] * si) * sj;
          }
        }
      }
    }
    // a prefetch left behind by an aborted loop lands before the CTA exits
    if (LDST && lane == 0)
    {
      if (opar0 >= 0) tc::mbar_wait(&cld_bar[ew][0], (uint32_t)opar0);
      if (opar1 >= 0) tc::mbar_wait(&cld_bar[ew][1], (uint32_t)opar1);
    }
  }
  // reduce-adds and stores performed before exit
  if ((RED || LDST) && warp >= 2 && lane == 0) tc::bulk_wait_read();
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, TMEM_COLS);
  }
}

template <int FMT, bool BATCH, bool WIDE>
__global__ void __launch_bounds__(NTHREADS, 1)
syrk_tc_kernel(const __grid_constant__ TcMaps maps, float* __restrict__ C, int ldc, int m, int k,
               const int8_t* __restrict__ rowexp, const uint8_t* __restrict__ mxexp, int ldmx,
               const int* prec_sel, DevStatus* st, TcBatch bt, int ntiles_b, TileSel sel) {
  if (prec_sel != nullptr && *prec_sel != FMT) return;
  syrk_tc_body<FMT, BATCH, WIDE>(&maps.hi, &maps.lo, &maps.c, C, ldc, m, k, rowexp, mxexp, ldmx, st,
                                 bt, ntiles_b, sel);
}

// K beyond the format's load / store epilogue (see TcCfg)
template <int FMT> __host__ __device__ constexpr bool tc_wide(int k) {
  return k > TcCfg<FMT>::LDST_MAX_K;
}

// Maps for every format: the three 8-bit code panels (slot q8_slot), the
// FP16 hi and lo panels, C.
struct TcMapsAll {
  CUtensorMap h8[3];
  CUtensorMap h16;
  CUtensorMap l16;
  CUtensorMap c;
};
// One launch whatever the step picked: the format is read on the device.
__global__ void __launch_bounds__(NTHREADS, 1)
syrk_tc_dispatch_kernel(const __grid_constant__ TcMapsAll maps, float* __restrict__ C, int ldc,
                        int m, int k, const int8_t* __restrict__ rexp_e4m3,
                        const int8_t* __restrict__ rexp_e5m2, const int8_t* __restrict__ rexp_f16,
                        const uint8_t* __restrict__ mxexp, int ldmx, unsigned fmt_mask,
                        const int* prec_sel, DevStatus* st, TileSel sel) {
  tc::grid_dep_wait();      // the panel solve that resolved the step is complete
  tc::grid_dep_trigger();   // the POTRF after this (head) launch may be scheduled
  const int f = *prec_sel;
  if (f < 0 || f > 31 || ((fmt_mask >> f) & 1u) == 0) return;
  const TcBatch nb{};
  // one body per format and epilogue (the K test is uniform over the grid)
#define TC_BODY(F, MHI, MLO, REXP, MX, LDMX)                                                     \
  do {                                                                                        \
    if (tc_wide<F>(k))                                                                        \
      syrk_tc_body<F, false, true>(MHI, MLO, &maps.c, C, ldc, m, k, REXP, MX, LDMX, st, nb, 0, sel); \
    else                                                                                      \
      syrk_tc_body<F, false, false>(MHI, MLO, &maps.c, C, ldc, m, k, REXP, MX, LDMX, st, nb, 0, sel); \
  } while (0)
  switch (f) {
    case FP16:
      TC_BODY(FP16, &maps.h16, &maps.l16, rexp_f16, nullptr, 0);
      break;
    case FP16X2:   // reduce-add epilogue at every K
      syrk_tc_body<FP16X2, false, false>(&maps.h16, &maps.l16, &maps.c, C, ldc, m, k, rexp_f16,
                                         nullptr, 0, st, nb, 0, sel);
      break;
    case E4M3:
      TC_BODY(E4M3, &maps.h8[0], &maps.h8[0], rexp_e4m3, nullptr, 0);
      break;
    case E5M2:
      TC_BODY(E5M2, &maps.h8[1], &maps.h8[1], rexp_e5m2, nullptr, 0);
      break;
    case MXFP8:
    case MXFP6E2M3:    // FP6/FP4 element values stored as E4M3 codes: the same body
    case MXFP6E3M2:
    case MXFP4:
      TC_BODY(MXFP8, &maps.h8[2], &maps.h8[2], nullptr, mxexp, ldmx);
      break;
    default:
      break;
  }
#undef TC_BODY
}

template <int FMT, bool BATCH, bool WIDE = false>
size_t tc_smem() {
  using Cfg = TcCfg<FMT>;
  using Plan = TcPlan<FMT, BATCH, WIDE>;
  return (size_t)Plan::NSTAGE * (2 * Cfg::NSETS * STRIP + (Cfg::MX ? 2 * SF_BYTES : 0)) +
         (size_t)EPI_WARPS * STAGE_C * Plan::EPI_BOXES + 1024;
}

template <int FMT>
size_t tc_smem_k(int k) {
  return tc_wide<FMT>(k) ? tc_smem<FMT, false, true>() : tc_smem<FMT, false, false>();
}

int grid_for(int ntiles, int max_sms) {
  int nsm = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (max_sms > 0 && max_sms < nsm) nsm = max_sms;
  return ntiles < nsm ? ntiles : nsm;
}

template <int FMT, bool BATCH>
cudaError_t launch_fmt(const TcMaps& maps, float* C, int ldc, int m, int k, const int8_t* rowexp,
                       const uint8_t* mxexp, int ldmx, const int* prec_sel, DevStatus* st,
                       const TcBatch& bt, int ntiles_b, cudaStream_t stream,
                       TileSel sel = kAllTiles, int max_sms = 0) {
  const int ntiles = BATCH ? ntiles_b : sel_tile_count(ceil_div(m, TM), sel);
  if (ntiles <= 0) return cudaSuccess;
  const int grid = grid_for(ntiles, max_sms);
  auto go = [&](auto kernel, size_t smem) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kernel<<<grid, NTHREADS, smem, stream>>>(maps, C, ldc, m, k, rowexp, mxexp, ldmx, prec_sel, st,
                                             bt, ntiles_b, sel);
    return cudaGetLastError();
  };
  if constexpr (!BATCH)
    if (tc_wide<FMT>(k)) return go(syrk_tc_kernel<FMT, false, true>, tc_smem<FMT, false, true>());
  return go(syrk_tc_kernel<FMT, BATCH, false>, tc_smem<FMT, BATCH, false>());
}

}  // namespace

// K up to 1024 (the factor uses K = block size <= 256; the kernel-level entry
// point also takes the 512- and 1024-wide panels of larger-block schedules)
bool syrk_tc_supported(int fmt, int k) {
  if (fmt == FP16 || fmt == FP16X2) return k > 0 && (k * 2) % CHUNK == 0 && k <= 1024;
  if (fmt == E4M3 || fmt == E5M2 || is_mx(fmt)) return k > 0 && k % CHUNK == 0 && k <= 1024;
  return false;
}

cudaError_t launch_syrk_tc(float* C, int ldc, int m, int k, int fmt, const void* q, int ldq,
                           const int8_t* rowexp, const uint8_t* mxexp, int ldmx,
                           const int* prec_sel, DevStatus* st, cudaStream_t stream, TileSel sel,
                           int max_sms) {
  if (m <= 0) return cudaSuccess;
  if (is_mx(fmt)) fmt = MXFP8;    // the family shares the E4M3 block-scaled path
  if (fmt == MXFP8 && (mxexp == nullptr || ldmx < k / 32 ||
                       (reinterpret_cast<uintptr_t>(mxexp) & 3) != 0 || (ldmx & 3) != 0))
    return cudaErrorInvalidValue;
  if (!syrk_tc_supported(fmt, k)) return cudaErrorInvalidValue;
  const int esize = (fmt == FP16 || fmt == FP16X2) ? 2 : 1;
  const CUtensorMapDataType dt = esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  TcMaps maps;
  if (!encode_tmap_2d(&maps.hi, dt, esize, q, (uint64_t)k, (uint64_t)m, (uint64_t)ldq,
                      CHUNK / esize, TM, CU_TENSOR_MAP_SWIZZLE_128B))
    return cudaErrorInvalidValue;
  maps.lo = maps.hi;
  if (!encode_tmap_2d(&maps.c, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, (uint64_t)m, (uint64_t)m,
                      (uint64_t)ldc, 32, 32, CU_TENSOR_MAP_SWIZZLE_NONE))
    return cudaErrorInvalidValue;
  if (fmt == FP16X2) {
    const uint16_t* lo = reinterpret_cast<const uint16_t*>(q) + (size_t)m * ldq;
    if (!encode_tmap_2d(&maps.lo, dt, esize, lo, (uint64_t)k, (uint64_t)m, (uint64_t)ldq,
                        CHUNK / esize, TM, CU_TENSOR_MAP_SWIZZLE_128B))
      return cudaErrorInvalidValue;
  }
  switch (fmt) {
    case FP16: return launch_fmt<FP16, false>(maps, C, ldc, m, k, rowexp, mxexp, ldmx, prec_sel, st, TcBatch{}, 0, stream, sel, max_sms);
    case E4M3: return launch_fmt<E4M3, false>(maps, C, ldc, m, k, rowexp, mxexp, ldmx, prec_sel, st, TcBatch{}, 0, stream, sel, max_sms);
    case E5M2: return launch_fmt<E5M2, false>(maps, C, ldc, m, k, rowexp, mxexp, ldmx, prec_sel, st, TcBatch{}, 0, stream, sel, max_sms);
    case FP16X2: return launch_fmt<FP16X2, false>(maps, C, ldc, m, k, rowexp, mxexp, ldmx, prec_sel, st, TcBatch{}, 0, stream, sel, max_sms);
    case MXFP8: return launch_fmt<MXFP8, false>(maps, C, ldc, m, k, rowexp, mxexp, ldmx, prec_sel, st, TcBatch{}, 0, stream, sel, max_sms);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_syrk_tc_dispatch(float* C, int ldc, int m, int k, unsigned fmt_mask,
                                    const QuantAll& qa, const int* prec_sel, DevStatus* st,
                                    cudaStream_t stream, TileSel sel, int max_sms) {
  if (m <= 0) return cudaSuccess;
  if (prec_sel == nullptr) return cudaErrorInvalidValue;
  const int ntiles = sel_tile_count(ceil_div(m, TM), sel);
  if (ntiles <= 0) return cudaSuccess;
  for (int f : {FP16, E4M3, E5M2, FP16X2, MXFP8})
    if (((fmt_mask >> f) & 1u) && !syrk_tc_supported(f, k)) return cudaErrorInvalidValue;
  // an FP6/FP4 MX format takes the MXFP8 maps and shared memory (the kernel
  // still checks the step's own format against the full mask)
  const unsigned kMxFamily = (1u << MXFP6E2M3) | (1u << MXFP6E3M2) | (1u << MXFP4);
  const unsigned setup_mask = fmt_mask | ((fmt_mask & kMxFamily) ? (1u << MXFP8) : 0u);
  if (((setup_mask >> MXFP8) & 1u) &&
      (qa.mxexp == nullptr || qa.ldmx < k / 32 || (reinterpret_cast<uintptr_t>(qa.mxexp) & 3) != 0 ||
       (qa.ldmx & 3) != 0))
    return cudaErrorInvalidValue;
  TcMapsAll maps;
  if (!encode_tmap_2d(&maps.c, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, (uint64_t)m, (uint64_t)m,
                      (uint64_t)ldc, 32, 32, CU_TENSOR_MAP_SWIZZLE_NONE))
    return cudaErrorInvalidValue;
  maps.h8[0] = maps.h8[1] = maps.h8[2] = maps.h16 = maps.l16 = maps.c;   // unused slots
  for (int f : {E4M3, E5M2, MXFP8})
    if (((setup_mask >> f) & 1u) &&
        !encode_tmap_2d(&maps.h8[q8_slot(f)], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, qa.q8[q8_slot(f)],
                        (uint64_t)k, (uint64_t)m, (uint64_t)qa.ldq, CHUNK, TM,
                        CU_TENSOR_MAP_SWIZZLE_128B))
      return cudaErrorInvalidValue;
  if (setup_mask & ((1u << FP16) | (1u << FP16X2))) {
    if (!encode_tmap_2d(&maps.h16, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, qa.q16, (uint64_t)k,
                        (uint64_t)m, (uint64_t)qa.ldq, CHUNK / 2, TM, CU_TENSOR_MAP_SWIZZLE_128B))
      return cudaErrorInvalidValue;
    const uint16_t* lo = qa.q16 + (size_t)m * qa.ldq;
    if (!encode_tmap_2d(&maps.l16, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, lo, (uint64_t)k, (uint64_t)m,
                        (uint64_t)qa.ldq, CHUNK / 2, TM, CU_TENSOR_MAP_SWIZZLE_128B))
      return cudaErrorInvalidValue;
  }
  size_t smem = 0;
  if ((setup_mask >> FP16) & 1u) smem = std::max(smem, tc_smem_k<FP16>(k));
  if ((setup_mask >> E4M3) & 1u) smem = std::max(smem, tc_smem_k<E4M3>(k));
  if ((setup_mask >> E5M2) & 1u) smem = std::max(smem, tc_smem_k<E5M2>(k));
  if ((setup_mask >> FP16X2) & 1u) smem = std::max(smem, tc_smem<FP16X2, false>());
  if ((setup_mask >> MXFP8) & 1u) smem = std::max(smem, tc_smem_k<MXFP8>(k));
  if (smem == 0) return cudaSuccess;
  const size_t smem_all = std::max({tc_smem<FP16, false>(), tc_smem<E4M3, false>(),
                                    tc_smem<E5M2, false>(), tc_smem<FP16X2, false>(),
                                    tc_smem<MXFP8, false>(), tc_smem<FP16, false, true>(),
                                    tc_smem<E4M3, false, true>(), tc_smem<E5M2, false, true>(),
                                    tc_smem<MXFP8, false, true>()});
  cudaError_t e = cudaFuncSetAttribute(syrk_tc_dispatch_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_all);
  if (e != cudaSuccess) return e;
  const int grid = grid_for(ntiles, max_sms);
  PdlLaunch L(dim3(grid), dim3(NTHREADS), smem, stream);
  e = cudaLaunchKernelEx(&L.cfg, syrk_tc_dispatch_kernel, maps, C, ldc, m, k, qa.rexp[0],
                         qa.rexp[1], qa.rexp[2], qa.mxexp, qa.ldmx, fmt_mask, prec_sel, st, sel);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_syrk_tc_batched(BatchSys* sys, const BatchStep* steps, int nact, int ntiles,
                                   int s, int b, int fmt, const void* q, int qrows,
                                   const int8_t* rowexp, const uint8_t* mxexp,
                                   cudaStream_t stream) {
  if (nact <= 0 || ntiles <= 0) return cudaSuccess;
  if (!syrk_tc_supported(fmt, b)) return cudaErrorInvalidValue;
  const int esize = (fmt == FP16 || fmt == FP16X2) ? 2 : 1;
  const CUtensorMapDataType dt = esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  TcMaps maps;
  if (!encode_tmap_2d(&maps.hi, dt, esize, q, (uint64_t)b, (uint64_t)qrows, (uint64_t)b,
                      CHUNK / esize, TM, CU_TENSOR_MAP_SWIZZLE_128B))
    return cudaErrorInvalidValue;
  maps.lo = maps.hi;
  maps.c = maps.hi;            // unused: batched launches update C in place
  if (fmt == FP16X2) {
    const uint16_t* lo = reinterpret_cast<const uint16_t*>(q) + (size_t)qrows * b;
    if (!encode_tmap_2d(&maps.lo, dt, esize, lo, (uint64_t)b, (uint64_t)qrows, (uint64_t)b,
                        CHUNK / esize, TM, CU_TENSOR_MAP_SWIZZLE_128B))
      return cudaErrorInvalidValue;
  }
  const TcBatch bt{sys, steps, nact, s, b};
  const int ldmx = b / 32;
  switch (fmt) {
    case FP16: return launch_fmt<FP16, true>(maps, nullptr, 0, 0, b, rowexp, mxexp, ldmx, nullptr, nullptr, bt, ntiles, stream);
    case E4M3: return launch_fmt<E4M3, true>(maps, nullptr, 0, 0, b, rowexp, mxexp, ldmx, nullptr, nullptr, bt, ntiles, stream);
    case E5M2: return launch_fmt<E5M2, true>(maps, nullptr, 0, 0, b, rowexp, mxexp, ldmx, nullptr, nullptr, bt, ntiles, stream);
    case FP16X2: return launch_fmt<FP16X2, true>(maps, nullptr, 0, 0, b, rowexp, mxexp, ldmx, nullptr, nullptr, bt, ntiles, stream);
    case MXFP8: return launch_fmt<MXFP8, true>(maps, nullptr, 0, 0, b, rowexp, mxexp, ldmx, nullptr, nullptr, bt, ntiles, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mpchol
