// PCG operator and preconditioner: y = A x and z = (L L^T)^-1 r.
//
// Replaces the reference's per-iteration cublasDgemv on FP64 A
// (src/mixed_cholesky.cu:185-191) and cusolverDnDpotrs on an FP64 copy of L
// (src/mixed_cholesky.cu:141,204-206).  Both read the FP32 lower triangle once
// per application, in 128 x 128 tiles, with FP64 vectors and accumulation.
//
// Triangular solves.  A row-by-row (or 128-block-by-block) substitution is a
// chain of n/128 dependent steps and runs at a few GB/s on one B200.  Instead,
// once per factor, the inverses W_S of the 1024-row diagonal super-blocks
// L_SS are formed by recursive doubling (FP64 128-block inverses, FP32 GEMM
// tiles above that).  A
// forward solve is then n/1024 steps of two fully parallel kernels:
//     y_S  = W_S w_S                      (TRMV over the super-block's lower tiles)
//     w_T -= L_TS y_S   for T > S         (GEMV over the panel below)
// and the backward solve mirrors it with transposes.  The applied operator is
// (Lt Lt^T)^-1 with Lt = blockdiag(W_S^-1) + strictly-block-lower(L), which is
// symmetric positive definite whenever the W_S are nonsingular, so PCG stays
// well defined; it equals (L L^T)^-1 up to the FP32 rounding of the W_S.
// Partial sums are combined with FP64 atomics.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg.cuh"

namespace mpchol {
cudaError_t solve_set_attributes();
namespace {

constexpr int RB = 128;     // tile size
constexpr int NTH = 256;    // 8 warps: warp w owns tile columns 16w..16w+15
constexpr int RS = 1024;    // super-block rows

template <typename TA>
__device__ __forceinline__ void load4(const TA* p, int nvalid, float out[4]);
template <>
__device__ __forceinline__ void load4<float>(const float* p, int nvalid, float out[4]) {
  if (nvalid >= 4 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = (r < nvalid) ? __ldg(p + r) : 0.0f;
  }
}

// Tile loaded into registers: lane covers rows 4*lane..4*lane+3, warp covers
// CH consecutive columns starting at col0.  Elements outside (rows_valid,
// cols_valid) are zero.  Every load of the batch is issued before any use.
template <typename TA, int CH>
struct TileRegs {
  double v[CH][4];
};

// Tile values stay in the matrix's own type in registers (FP32 tiles take
// half the registers of a widened copy); they are widened at each use.
template <int CH>
__device__ __forceinline__ void load_cols(const float* T, int ld, int rloc, int rows_valid,
                                          int col0, int cols_valid, float (&v)[CH][4]) {
  const int nv = min(4, rows_valid - rloc);
#pragma unroll
  for (int cc = 0; cc < CH; ++cc) {
    const int c = col0 + cc;
    if (c < cols_valid && nv > 0) load4<float>(T + (size_t)c * ld + rloc, nv, v[cc]);
    else v[cc][0] = v[cc][1] = v[cc][2] = v[cc][3] = 0.0f;
  }
}

template <int CH>
__device__ __forceinline__ void load_cols(const double* T, int ld, int rloc, int rows_valid,
                                          int col0, int cols_valid, double (&v)[CH][4]) {
  const int nv = min(4, rows_valid - rloc);
#pragma unroll
  for (int cc = 0; cc < CH; ++cc) {
    const int c = col0 + cc;
#pragma unroll
    for (int r = 0; r < 4; ++r)
      v[cc][r] = (c < cols_valid && r < nv) ? __ldg(T + (size_t)c * ld + rloc + r) : 0.0;
  }
}

// Sum each of the W per-lane values w[i] (W = 8 or 16) over the 32 lanes of
// the warp: a butterfly that halves the values a lane keeps at each step
// (W/2 + W/4 + ... shuffles), then plain xor steps for the remaining lane
// bits.  Lane l ends with the sum of column col_of_lane<W>(l); the lanes
// that differ only in the low 5 - log2(W) bits hold the same sum.
template <int W>
__device__ __forceinline__ int col_of_lane(int lane) {
  int c = 0;
#pragma unroll
  for (int off = 16, h = W / 2; h >= 1; off >>= 1, h >>= 1) c += ((lane & off) ? h : 0);
  return c;
}
template <int W>
__device__ __forceinline__ double butterfly(double (&w)[W], int lane) {
  int off = 16;
#pragma unroll
  for (int h = W / 2; h >= 1; h >>= 1, off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const double send = upper ? w[i] : w[i + h];
      const double keep = upper ? w[i + h] : w[i];
      w[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  double v = w[0];
#pragma unroll
  for (; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Accumulate a 128 x 128 tile times a vector segment.
//   NOTRANS: part[r][k] += T[r][c] * vin[k][c]   (per-thread rows, summed over the warp's columns)
//   TRANS  : colsum[k][c] = sum_r T[r][c] * vin[k][r], the CH columns of a chunk reduced
//            over the warp together by one butterfly per rhs
// (staged vectors and column sums are k-major: [k * RB + index])
// `mask`: 0 none, 1 keep r >= c (lower incl. diagonal), 2 keep r > c.
template <typename TA, int NR, int CH>
__device__ __forceinline__ void tile_pass(const TA* T, int ld, int rows_valid, int cols_valid,
                                          const double* vin_cols, const double* vin_rows,
                                          double (&acc)[4][NR], double* colsum_smem, int mask_nt,
                                          int mask_t, bool do_nt, bool do_t) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rloc = 4 * lane;
  constexpr int LOWBITS = (CH == 16) ? 1 : 3;   // lanes holding the same column sum
#pragma unroll
  for (int cb = 0; cb < 16; cb += CH) {
    TA v[CH][4];
    load_cols<CH>(T, ld, rloc, rows_valid, warp * 16 + cb, cols_valid, v);
    if (do_nt) {
#pragma unroll
      for (int cc = 0; cc < CH; ++cc) {
        const int c = warp * 16 + cb + cc;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          const double xc = vin_cols[k * RB + c];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const bool keep = mask_nt == 0 || (mask_nt == 1 ? (rloc + r >= c) : (rloc + r > c));
            if (keep) acc[r][k] = fma((double)v[cc][r], xc, acc[r][k]);
          }
        }
      }
    }
    if (do_t) {
      // one rhs at a time (bounded register pressure for NR > 2)
#pragma unroll 1
      for (int k = 0; k < NR; ++k) {
        // this lane's four rows of the rhs, read once (two 16-byte loads)
        const double2 x01 = *reinterpret_cast<const double2*>(vin_rows + k * RB + rloc);
        const double2 x23 = *reinterpret_cast<const double2*>(vin_rows + k * RB + rloc + 2);
        const double xr[4] = {x01.x, x01.y, x23.x, x23.y};
        double w[CH];
#pragma unroll
        for (int cc = 0; cc < CH; ++cc) {
          const int c = warp * 16 + cb + cc;
          double sacc = 0.0;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const bool keep = mask_t == 0 || (mask_t == 1 ? (rloc + r >= c) : (rloc + r > c));
            if (keep) sacc = fma((double)v[cc][r], xr[r], sacc);
          }
          w[cc] = sacc;
        }
        const double sum = butterfly<CH>(w, lane);
        if ((lane & LOWBITS) == 0)
          colsum_smem[k * RB + warp * 16 + cb + col_of_lane<CH>(lane)] = sum;
      }
    }
  }
}

// Reduce the per-warp row partials of tile_pass(NOTRANS) and add sign * sum
// into out[row0 + r] (rows < nvalid) with FP64 atomics.
template <int NR>
__device__ __forceinline__ void flush_rows(double (&acc)[4][NR], double* red, double* out, int n,
                                           int row0, int nvalid, double sign) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < NR; ++k) red[(warp * NR + k) * RB + 4 * lane + r] = acc[r][k];
  __syncthreads();
  for (int e = threadIdx.x; e < RB * NR; e += NTH) {
    const int k = e / RB, r = e % RB;
    if (r < nvalid) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < NTH / 32; ++w) s += red[(w * NR + k) * RB + r];
      atomicAdd(&out[(size_t)k * n + row0 + r], sign * s);
    }
  }
}

// Vector segments are read from L2 (ld.global.cg): inside the persistent
// solve other CTAs produce them with atomics while this SM may hold older
// lines of the same arrays in L1.
template <int NR>
__device__ __forceinline__ void load_vec(const double* x, int n, int row0, int nvalid, double* s) {
  // k-major in shared memory (s[k * RB + r]): a lane's rows are contiguous
  for (int e = threadIdx.x; e < RB * NR; e += NTH) {
    const int k = e / RB, r = e % RB;
    s[e] = (r < nvalid) ? __ldcg(x + (size_t)k * n + row0 + r) : 0.0;
  }
}

__device__ __forceinline__ void tri_of(int t, int& i, int& j) {
  int a = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (a * (a + 1) / 2 > t) --a;
  while ((a + 1) * (a + 2) / 2 <= t) ++a;
  i = a;
  j = t - a * (a + 1) / 2;
}

template <typename TA> struct ChunkOf { static constexpr int value = 16; };
template <> struct ChunkOf<double> { static constexpr int value = 8; };

// ---- tiles staged in shared memory -------------------------------------------
// The streaming kernels (SYMV, the persistent triangular solve) copy each
// 128 x 128 FP32 tile into shared memory with cp.async, one or two tiles
// ahead of its use: the copies hold no registers, so an SM keeps 128-192 KB
// of HBM reads in flight while it computes on the current tile.
constexpr int TILE_ELEMS = RB * RB;   // 64 KB of FP32
constexpr int SCH = 8;                // columns per widened chunk

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Copy the rows_valid x cols_valid tile at T (column-major, leading dimension
// ld; T and ld keep 16-byte alignment) into a dense 128 x 128 column-major
// tile; everything outside the valid part is zero-filled by the copies.
// A warp copies one 512-byte column per instruction.
__device__ __forceinline__ void stage_tile(float* dst, const float* T, int ld, int rows_valid,
                                           int cols_valid) {
#pragma unroll 4
  for (int e = threadIdx.x; e < TILE_ELEMS / 4; e += NTH) {
    const int c = e / (RB / 4), r = 4 * (e % (RB / 4));
    const bool ok = c < cols_valid && r < rows_valid;
    cp_async16(dst + c * RB + r, ok ? T + (size_t)c * ld + r : T, ok ? 4 * min(4, rows_valid - r) : 0);
  }
}

// x[k * n + row0 + r] -> s[k * RB + r], zero for r >= nvalid (8-byte copies:
// n may be odd)
template <int NR>
__device__ __forceinline__ void stage_vec(const double* x, int n, int row0, int nvalid, double* s) {
  for (int e = threadIdx.x; e < RB * NR; e += NTH) {
    const int k = e / RB, r = e % RB;
    const bool ok = r < nvalid;
    cp_async8(s + e, ok ? x + (size_t)k * n + row0 + r : x, ok ? 8 : 0);
  }
}

// tile_pass on a staged tile.  Each lane widens its 4 x SCH chunk to FP64
// once and uses it for every rhs of both products.  DIAG: a diagonal tile of
// a symmetric operator stored lower -- NOTRANS keeps r >= c, TRANS r > c.
// FRO: also adds the tile's share of ||A||_F^2 to *fsq (the lower triangle,
// off-diagonal entries twice).
template <int NR, bool DIAG, bool FRO = false>
__device__ __forceinline__ void tile_pass_staged(const float* Ts, const double* vin_cols,
                                                 const double* vin_rows, double (&acc)[4][NR],
                                                 double* colsum_smem, bool do_nt, bool do_t,
                                                 double* fsq = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rloc = 4 * lane;
  constexpr int LOWBITS = 3;   // lanes holding the same column sum (SCH = 8)
#pragma unroll
  for (int cb = 0; cb < 16; cb += SCH) {
    double dv[SCH][4];
#pragma unroll
    for (int cc = 0; cc < SCH; ++cc) {
      const int c = warp * 16 + cb + cc;
      const float4 f = *reinterpret_cast<const float4*>(Ts + c * RB + rloc);
      dv[cc][0] = f.x; dv[cc][1] = f.y; dv[cc][2] = f.z; dv[cc][3] = f.w;
      if (DIAG) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (rloc + r < c) dv[cc][r] = 0.0;
      }
      if (FRO) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
          *fsq = fma((DIAG && rloc + r == c) ? dv[cc][r] : 2.0 * dv[cc][r], dv[cc][r], *fsq);
      }
    }
    if (do_nt) {
#pragma unroll
      for (int cc = 0; cc < SCH; cc += 2) {
        const int c = warp * 16 + cb + cc;
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          const double2 xc = *reinterpret_cast<const double2*>(vin_cols + k * RB + c);
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            acc[r][k] = fma(dv[cc][r], xc.x, acc[r][k]);
            acc[r][k] = fma(dv[cc + 1][r], xc.y, acc[r][k]);
          }
        }
      }
    }
    if (do_t) {
#pragma unroll 1
      for (int k = 0; k < NR; ++k) {
        const double2 x01 = *reinterpret_cast<const double2*>(vin_rows + k * RB + rloc);
        const double2 x23 = *reinterpret_cast<const double2*>(vin_rows + k * RB + rloc + 2);
        const double xr[4] = {x01.x, x01.y, x23.x, x23.y};
        double w[SCH];
#pragma unroll
        for (int cc = 0; cc < SCH; ++cc) {
          const int c = warp * 16 + cb + cc;
          double sacc = 0.0;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const double a = (DIAG && rloc + r == c) ? 0.0 : dv[cc][r];
            sacc = fma(a, xr[r], sacc);
          }
          w[cc] = sacc;
        }
        const double sum = butterfly<SCH>(w, lane);
        if ((lane & LOWBITS) == 0)
          colsum_smem[k * RB + warp * 16 + cb + col_of_lane<SCH>(lane)] = sum;
      }
    }
  }
}

// ---- eight right-hand sides on the FP64 tensor cores ---------------------
// With 8 rhs the tile passes are FP64-FMA bound (16 FMAs per tile element for
// the symmetric product), so they run as mma.sync m8n8k4 FP64 (DMMA): a warp
// owns 16 rows of the tile for the row sums and 16 columns for the column
// sums, and its accumulator fragments hold finished 8 x 8 (rows x rhs)
// blocks -- no butterflies and no cross-warp reduction.  Fragments follow the
// PTX ISA for m8n8k4.f64: a = A[lane / 4][lane % 4], b = B[lane % 4][lane / 4],
// d[i] = D[lane / 4][2 (lane % 4) + i].
//
// The tile is staged in a blocked layout in which both fragment patterns
// read 32 distinct banks: 4-row x 8-column blocks of 32 floats (column-major
// inside a block, so a 16-byte copy of 4 rows of one column lands contiguous),
// 16 blocks per 4-row group, and the groups 528 floats apart (16 banks of
// stagger between neighbouring groups).  Vector segments are staged k-major
// with a row of XS = 132 doubles per rhs.
constexpr int BL_RG = 16 * 32 + 16;          // floats per 4-row group
constexpr int BL_TILE = (RB / 4) * BL_RG;    // floats per blocked tile
constexpr int XS = RB + 4;                   // doubles per rhs in a staged segment

__device__ __forceinline__ int bl_off(int r, int c) {
  return (r >> 2) * BL_RG + (c >> 3) * 32 + (c & 7) * 4 + (r & 3);
}

__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// stage_tile into the blocked layout
__device__ __forceinline__ void stage_tile_bl(float* dst, const float* T, int ld, int rows_valid,
                                              int cols_valid) {
#pragma unroll 4
  for (int e = threadIdx.x; e < TILE_ELEMS / 4; e += NTH) {
    const int c = e / (RB / 4), r = 4 * (e % (RB / 4));
    const bool ok = c < cols_valid && r < rows_valid;
    cp_async16(dst + bl_off(r, c), ok ? T + (size_t)c * ld + r : T,
               ok ? 4 * min(4, rows_valid - r) : 0);
  }
}

// x[k * n + row0 + r] -> s[k * XS + r] (zero past nvalid), 8 rhs
__device__ __forceinline__ void stage_vec_x8(const double* x, int n, int row0, int nvalid, double* s) {
  for (int e = threadIdx.x; e < RB * 8; e += NTH) {
    const int k = e / RB, r = e % RB;
    const bool ok = r < nvalid;
    cp_async8(s + k * XS + r, ok ? x + (size_t)k * n + row0 + r : x, ok ? 8 : 0);
  }
}
// the same through L2 loads (the persistent solve's segments are produced by
// other CTAs' atomics)
__device__ __forceinline__ void load_vec_x8(const double* x, int n, int row0, int nvalid, double* s) {
  for (int e = threadIdx.x; e < RB * 8; e += NTH) {
    const int k = e / RB, r = e % RB;
    s[k * XS + r] = (r < nvalid) ? __ldcg(x + (size_t)k * n + row0 + r) : 0.0;
  }
}

// One blocked tile T (rows i0.., columns j0..) times 8 rhs on the DMMA pipe:
//   do_nt: y_rows[row0 + r] += sign * sum_c T[r][c] x_c[c]   (rows < nrows)
//   do_t : y_cols[col0 + c] += sign * sum_r T[r][c] x_r[r]   (columns < ncols)
// by FP64 atomics.  DIAG (a diagonal tile of a symmetric operator stored
// lower): the row sums keep r >= c, the column sums r > c.  FRO: adds the
// tile's share of ||A||_F^2 (off-diagonal entries twice) to *fsq.
// KC k-steps of fragments are loaded (and widened) per chunk and UNR chunks
// are unrolled, so the next chunk's loads overlap this chunk's DMMAs; ONLY
// fixes the product at compile time (1: row sums, 2: column sums, 0: by
// do_nt / do_t).  Both products: KC = 8, UNR = 2 (the 128 registers of two
// CTAs per SM allow no more); one product: KC = 4 fully unrolled.
template <bool DIAG, bool FRO, int KC = 8, int UNR = 2, int ONLY = 0>
__device__ __forceinline__ void tile_mma_x8(const float* Ts, const double* x_c, const double* x_r,
                                            double* y_rows, int row0, int nrows, double* y_cols,
                                            int col0, int ncols, int n, bool do_nt_rt, bool do_t_rt,
                                            double sign, double* fsq) {
  const bool do_nt = ONLY == 1 ? true : (ONLY == 2 ? false : do_nt_rt);
  const bool do_t = ONLY == 2 ? true : (ONLY == 1 ? false : do_t_rt);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int B0 = 16 * warp;
  // accumulators: [m-block][k-step parity] -- eight independent DMMA chains
  // per warp when both products run
  double dn[2][2][2] = {};
  double dt[2][2][2] = {};
  static_assert(KC % 2 == 0, "k-step parity picks the accumulator: chunks hold an even count");
#pragma unroll(UNR)
  for (int kb = 0; kb < RB; kb += 4 * KC) {
    // every fragment of the chunk is loaded (and widened) before its DMMAs
    float an[2][KC], at[2][KC];
    double bn[KC], bt[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      const int k0 = kb + 4 * j;
      if (do_nt) {
        bn[j] = x_c[g * XS + k0 + t];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          const int r = B0 + 8 * mb + g, c = k0 + t;
          const float v = Ts[bl_off(r, c)];
          an[mb][j] = (DIAG && r < c) ? 0.0f : v;
        }
      }
      if (do_t) {
        bt[j] = x_r[g * XS + k0 + t];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          const int c = B0 + 8 * mb + g, r = k0 + t;
          const float v = Ts[bl_off(r, c)];
          at[mb][j] = (DIAG && r <= c) ? 0.0f : v;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      if (do_nt) {
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          const double a = (double)an[mb][j];
          if (FRO) {
            const int r = B0 + 8 * mb + g, c = kb + 4 * j + t;
            *fsq = fma((DIAG && r == c) ? a : 2.0 * a, a, *fsq);
          }
          dmma_m8n8k4(dn[mb][j & 1], a, bn[j]);
        }
      }
      if (do_t) {
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) dmma_m8n8k4(dt[mb][j & 1], (double)at[mb][j], bt[j]);
      }
    }
  }
#pragma unroll
  for (int mb = 0; mb < 2; ++mb) {
    const int idx = B0 + 8 * mb + g;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int k = 2 * t + i;
      if (do_nt && idx < nrows)
        atomicAdd(&y_rows[(size_t)k * n + row0 + idx], sign * (dn[mb][0][i] + dn[mb][1][i]));
      if (do_t && idx < ncols)
        atomicAdd(&y_cols[(size_t)k * n + col0 + idx], sign * (dt[mb][0][i] + dt[mb][1][i]));
    }
  }
}

// Shared memory of the staged SYMV: STAGES x (tile + x_J + x_I) + column sums.
// 8 rhs: one 84 KB stage per CTA and two CTAs per SM (each CTA's load
// overlaps the other's tile pass; 16 warps hide the DMMA and shared-memory
// latencies better than one CTA with two stages: 306 vs 331 us at n = 16384)
template <int NR>
constexpr int symv_stages() { return NR >= 8 ? 1 : 3; }
template <int NR>
constexpr size_t symv_staged_smem() {
  if (NR == 8)   // blocked tiles and padded segments, no column-sum buffer
    return (size_t)symv_stages<NR>() * (BL_TILE * sizeof(float) + 2 * (size_t)XS * 8 * sizeof(double));
  return (size_t)symv_stages<NR>() * (TILE_ELEMS * sizeof(float) + 2 * RB * NR * sizeof(double)) +
         (size_t)RB * NR * sizeof(double);
}

// ---- y += A x, FP32 symmetric A (lower triangle), persistent over the tiles.
// CTA b takes tiles b, b + grid, ...; each tile is staged symv_stages - 1
// tiles ahead together with its two vector segments.  The row partials are
// reduced in the stage's own tile buffer once the tile has been used.
// fro != nullptr: CTA b also writes its share of ||A||_F^2 (lower triangle,
// off-diagonal entries twice) to fro[b] and zeroes fro[gridDim.x ..nfro).
template <int NR>
__global__ void __launch_bounds__(NTH, NR >= 8 ? 2 : 1)
symv_staged_kernel(const float* __restrict__ A, int lda, int n, const double* __restrict__ x,
                   double* __restrict__ y, const int* skip, double* fro, int nfro) {
  if (skip != nullptr && *skip) return;
  constexpr int STAGES = symv_stages<NR>();
  constexpr bool MMA = NR == 8;
  constexpr int TE = MMA ? BL_TILE : TILE_ELEMS;      // floats per staged tile
  constexpr int VEC = MMA ? XS * 8 : RB * NR;         // doubles per staged segment
  extern __shared__ __align__(16) unsigned char sm_raw[];
  float* tiles = reinterpret_cast<float*>(sm_raw);
  double* vecs = reinterpret_cast<double*>(tiles + STAGES * TE);   // [stage][xJ, xI]
  double* s_col = vecs + STAGES * 2 * VEC;
  const int T = ceil_div(n, RB);
  const int ntiles = T * (T + 1) / 2;
  auto issue = [&](int t, int stage) {
    int I, J;
    tri_of(t, I, J);
    const int i0 = I * RB, j0 = J * RB;
    const int ni = min(RB, n - i0), nj = min(RB, n - j0);
    if (MMA) {
      stage_tile_bl(tiles + stage * TE, A + (size_t)j0 * lda + i0, lda, ni, nj);
      stage_vec_x8(x, n, j0, nj, vecs + (2 * stage) * VEC);
      stage_vec_x8(x, n, i0, ni, vecs + (2 * stage + 1) * VEC);
    } else {
      stage_tile(tiles + stage * TE, A + (size_t)j0 * lda + i0, lda, ni, nj);
      stage_vec<NR>(x, n, j0, nj, vecs + (2 * stage) * VEC);
      stage_vec<NR>(x, n, i0, ni, vecs + (2 * stage + 1) * VEC);
    }
  };
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    const int t = blockIdx.x + s * gridDim.x;
    if (t < ntiles) issue(t, s);
    cp_async_commit();
  }
  int stage = 0;
  double fsq = 0.0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    {
      const int tn = t + (STAGES - 1) * gridDim.x;
      if (tn < ntiles) issue(tn, (stage + STAGES - 1) % STAGES);
      cp_async_commit();
    }
    cp_async_wait<STAGES - 1>();
    __syncthreads();
    int I, J;
    tri_of(t, I, J);
    const int i0 = I * RB, j0 = J * RB;
    const int ni = min(RB, n - i0), nj = min(RB, n - j0);
    float* Ts = tiles + stage * TE;
    const double* xJ = vecs + (2 * stage) * VEC;
    const double* xI = xJ + VEC;
    if (MMA) {
      // row sums to y_I, column sums to y_J, straight from the fragments
      if (fro != nullptr) {
        if (I == J) tile_mma_x8<true, true>(Ts, xJ, xI, y, i0, ni, y, j0, nj, n, true, true, 1.0, &fsq);
        else tile_mma_x8<false, true>(Ts, xJ, xI, y, i0, ni, y, j0, nj, n, true, true, 1.0, &fsq);
      } else {
        if (I == J) tile_mma_x8<true, false>(Ts, xJ, xI, y, i0, ni, y, j0, nj, n, true, true, 1.0, nullptr);
        else tile_mma_x8<false, false>(Ts, xJ, xI, y, i0, ni, y, j0, nj, n, true, true, 1.0, nullptr);
      }
      __syncthreads();   // the stage is free again
      stage = (stage + 1) % STAGES;
      continue;
    }
    double acc[4][NR] = {};
    if (fro != nullptr) {
      if (I == J) tile_pass_staged<NR, true, true>(Ts, xJ, xI, acc, s_col, true, true, &fsq);
      else tile_pass_staged<NR, false, true>(Ts, xJ, xI, acc, s_col, true, true, &fsq);
    } else {
      if (I == J) tile_pass_staged<NR, true>(Ts, xJ, xI, acc, s_col, true, true);
      else tile_pass_staged<NR, false>(Ts, xJ, xI, acc, s_col, true, true);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < VEC; e += NTH) {
      const int k = e / RB, c = e % RB;
      if (c < nj) atomicAdd(&y[(size_t)k * n + j0 + c], s_col[e]);
    }
    flush_rows<NR>(acc, reinterpret_cast<double*>(Ts), y, n, i0, ni, 1.0);
    __syncthreads();   // the stage and s_col are free again
    stage = (stage + 1) % STAGES;
  }
  cp_async_wait<0>();
  if (fro != nullptr) {
    // block sum in a fixed order: warps, then the CTA's warps in turn
    double v = fsq;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    double* wsum = reinterpret_cast<double*>(tiles);   // the stages are free
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < NTH / 32; ++w) t += wsum[w];
      fro[blockIdx.x] = t;
    }
    for (int e = gridDim.x + blockIdx.x; e < nfro; e += gridDim.x)
      if (threadIdx.x == 0) fro[e] = 0.0;
  }
}

// ---- y += A x, symmetric A, lower triangle only (one CTA per lower tile) ----
template <typename TA, int NR>
__device__ __forceinline__ void
symv_body(const TA* __restrict__ A, int lda, int n, const double* __restrict__ x,
            double* __restrict__ y, const int* skip, uint3 bid) {
  if (skip != nullptr && *skip) return;
  __shared__ __align__(16) double s_xJ[RB * NR];
  __shared__ __align__(16) double s_xI[RB * NR];
  __shared__ double s_col[RB * NR];
  extern __shared__ double s_red[];
  int I, J;
  tri_of(bid.x, I, J);
  const int i0 = I * RB, j0 = J * RB;
  const int ni = min(RB, n - i0), nj = min(RB, n - j0);
  load_vec<NR>(x, n, j0, nj, s_xJ);
  load_vec<NR>(x, n, i0, ni, s_xI);
  __syncthreads();
  double acc[4][NR] = {};
  const bool diag = (I == J);
  tile_pass<TA, NR, ChunkOf<TA>::value>(A + (size_t)j0 * lda + i0, lda, ni, nj, s_xJ, s_xI, acc,
                                        s_col, diag ? 1 : 0, diag ? 2 : 0, true, true);
  __syncthreads();
  // column sums go to y_J
  for (int e = threadIdx.x; e < RB * NR; e += NTH) {
    const int k = e / RB, c = e % RB;
    if (c < nj) atomicAdd(&y[(size_t)k * n + j0 + c], s_col[e]);
  }
  flush_rows<NR>(acc, s_red, y, n, i0, ni, 1.0);
}

template <typename TA, int NR>
__global__ void __launch_bounds__(NTH)
symv_kernel(const TA* __restrict__ A, int lda, int n, const double* __restrict__ x,
            double* __restrict__ y, const int* skip) {
  symv_body<TA, NR>(A, lda, n, x, y, skip, blockIdx);
}

// ---- setup: super-block inverses by recursive doubling ---------------------
// For a lower-triangular [A 0; B C], inv = [A^-1 0; X C^-1] with
// X = -C^-1 (B A^-1).  The inverses W_S of the RS-row diagonal super-blocks
// are built bottom-up: the 128-row diagonal blocks in FP64 inside one CTA each
// (32-row tiles, then the 32 -> 64 -> 128 doublings), then the 128 -> 1024
// doublings as 128 x 128 FP32 GEMM tiles over all super-blocks at once.
// Storage: W_S is RS x RS column-major at wsup + S*RS*RS.  Its lower 128-tiles
// hold the inverse (diagonal tiles with a zero upper part); the strictly
// upper 128-tiles are scratch for the doubling products T = B A^-1 and are
// never read by the solves.

constexpr int BLD = RB + 1;     // padded column stride of the shared tiles

// One 128-row diagonal block per CTA (256 threads), FP64 in shared memory;
// the FP32 result goes to its diagonal tile of W_S.  Rows and columns past n
// are identity.
__device__ __forceinline__ void
block_inverse_body(const float* __restrict__ L, int ldl, int n, float* __restrict__ wsup, uint3 bid) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double* W = reinterpret_cast<double*>(sm_raw);            // [RB][BLD], column-major
  float* Ls = reinterpret_cast<float*>(W + RB * BLD);        // [RB][BLD], column-major
  const int g = bid.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i0 = g * RB;
  const int nb = min(RB, n - i0);
  // 16 loads in flight per thread before their shared-memory stores
  constexpr int LB = 16;
  for (int e0 = tid; e0 < RB * RB; e0 += LB * NTH) {
    float v[LB];
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int e = e0 + u * NTH;
      const int col = e / RB, row = e % RB;
      if (row < nb && col < nb) v[u] = (row >= col) ? L[(size_t)(i0 + col) * ldl + i0 + row] : 0.0f;
      else v[u] = (row == col) ? 1.0f : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < LB; ++u) {
      const int e = e0 + u * NTH;
      const int col = e / RB, row = e % RB;
      Ls[col * BLD + row] = v[u];
      W[col * BLD + row] = 0.0;
    }
  }
  __syncthreads();
  // 32-row diagonal tiles: warp t, lane j solves L_tt w = e_j (right-looking,
  // the column held in registers)
  if (warp < RB / 32) {
    const int t0 = warp * 32;
    double w[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) w[i] = (i == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      w[k] = w[k] / (double)Ls[(t0 + k) * BLD + t0 + k];
#pragma unroll
      for (int i = k + 1; i < 32; ++i) w[i] -= (double)Ls[(t0 + k) * BLD + t0 + i] * w[k];
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) W[(t0 + lane) * BLD + t0 + i] = w[i];
  }
  __syncthreads();
  // doublings h = 32 (two pairs) and h = 64 (one pair) inside the block;
  // output e of a level: row r = e % h, column c = (e / h) % h of pair e / h^2
  // Every output of a doubling runs over the whole k range of its pair: the
  // inverses stored in W are zero above their diagonals, so the extra terms
  // add zeros, and a thread's outputs advance together (independent
  // accumulators instead of one dependent chain after another).
  for (int h = 32; h < RB; h *= 2) {
    const int per = (RB / (2 * h)) * h * h / NTH;    // outputs per thread: 8 or 16
    int pa[16], pb[16];                               // per output: operand bases
    double acc[16];
    // T = B A^-1 -> the pair's upper-right block (scratch):
    // T[r][c] = sum_k L[a0+h+r][a0+k] * Ainv[k][c]
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = tid + NTH * q;
      const int r = e % h, c = (e / h) % h, a0 = (e / (h * h)) * 2 * h;
      pa[q] = a0 * BLD + a0 + h + r;                  // Ls[(a0 + k) * BLD + a0 + h + r]
      pb[q] = (a0 + c) * BLD + a0;                    // W[(a0 + c) * BLD + a0 + k]
      acc[q] = 0.0;
    }
    for (int k = 0; k < h; ++k) {
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (q < per) acc[q] += (double)Ls[pa[q] + k * BLD] * W[pb[q] + k];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q)
      if (q < per) {
        const int e = tid + NTH * q;
        const int r = e % h, c = (e / h) % h, a0 = (e / (h * h)) * 2 * h;
        W[(a0 + h + c) * BLD + a0 + r] = acc[q];
      }
    __syncthreads();
    // X = -C^-1 T -> the pair's lower-left block; the scratch is cleared:
    // X[r][c] = -sum_k Cinv[r][k] * T[k][c]
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = tid + NTH * q;
      const int r = e % h, c = (e / h) % h, a0 = (e / (h * h)) * 2 * h;
      pa[q] = (a0 + h) * BLD + a0 + h + r;            // W[(a0 + h + k) * BLD + a0 + h + r]
      pb[q] = (a0 + h + c) * BLD + a0;                // W[(a0 + h + c) * BLD + a0 + k]
      acc[q] = 0.0;
    }
    for (int k = 0; k < h; ++k) {
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (q < per) acc[q] += W[pa[q] + k * BLD] * W[pb[q] + k];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 16; ++q)
      if (q < per) {
        const int e = tid + NTH * q;
        const int r = e % h, c = (e / h) % h, a0 = (e / (h * h)) * 2 * h;
        W[(a0 + c) * BLD + a0 + h + r] = -acc[q];
        W[(a0 + h + c) * BLD + a0 + r] = 0.0;
      }
    __syncthreads();
  }
  const int S = i0 / RS, t = (i0 % RS) / RB;
  float* out = wsup + (size_t)S * RS * RS + (size_t)(t * RB) * RS + t * RB;
  for (int e = tid; e < RB * RB; e += NTH) {
    const int col = e / RB, row = e % RB;
    out[(size_t)col * RS + row] = (float)W[col * BLD + row];
  }
}

__global__ void __launch_bounds__(NTH)
block_inverse_kernel(const float* __restrict__ L, int ldl, int n, float* __restrict__ wsup) {
  block_inverse_body(L, ldl, n, wsup, blockIdx);
}

// C(128x128) = A(128 x K) * B(K x 128), A and B column-major, FP32 FMA.
// 256 threads, 8 x 8 outputs each (rows tx*4+{0..3}, 64+tx*4+{0..3}).  K
// advances in chunks of GK (a multiple of GK): the next chunk is loaded into
// registers (coalesced: 128 consecutive rows of A, GK consecutive k of each B
// column) while the current one is multiplied from shared memory.
constexpr int GK = 32;
constexpr int GPT = GK * RB / NTH;   // elements of A (and of B) per thread per chunk
constexpr int BLDK = GK + 1;         // padded column stride of the staged B chunk

__device__ __forceinline__ int acc_col_of(int ty, int b) { return b < 4 ? ty * 4 + b : 64 + ty * 4 + (b - 4); }

__device__ __forceinline__ void gemm128_load(const float* A, int lda, int a_rows_valid,
                                             const float* B, int ldb, int k0, float (&ra)[GPT],
                                             float (&rb)[GPT]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < GPT; ++q) {
    const int e = tid + NTH * q;
    const int r = e % RB, kk = e / RB;          // A: rows fastest
    ra[q] = (r < a_rows_valid) ? A[(size_t)(k0 + kk) * lda + r] : 0.0f;
    const int k = e % GK, c = e / GK;           // B: k fastest within a column
    rb[q] = B[(size_t)c * ldb + k0 + k];
  }
}

__device__ void gemm128(const float* A, int lda, int a_rows_valid, const float* B, int ldb, int K,
                        float (&acc)[8][8], float* As, float* Bs) {
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  float ra[GPT], rb[GPT];
  gemm128_load(A, lda, a_rows_valid, B, ldb, 0, ra, rb);
  for (int k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
    for (int q = 0; q < GPT; ++q) {
      const int e = tid + NTH * q;
      As[(e / RB) * RB + e % RB] = ra[q];
      Bs[(e / GK) * BLDK + e % GK] = rb[q];      // B column-major in shared memory too
    }
    __syncthreads();
    if (k0 + GK < K) gemm128_load(A, lda, a_rows_valid, B, ldb, k0 + GK, ra, rb);
#pragma unroll 4
    for (int kk = 0; kk < GK; ++kk) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[kk * RB + tx * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[kk * RB + 64 + tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      float bv[8];
#pragma unroll
      for (int b = 0; b < 8; ++b) bv[b] = Bs[acc_col_of(ty, b) * BLDK + kk];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int acc_row(int a) { return a < 4 ? (threadIdx.x % 16) * 4 + a : 64 + (threadIdx.x % 16) * 4 + (a - 4); }
__device__ __forceinline__ int acc_col(int b) { return b < 4 ? (threadIdx.x / 16) * 4 + b : 64 + (threadIdx.x / 16) * 4 + (b - 4); }

// One doubling level of half-size h (a multiple of RB) for pair blockIdx.y of
// super-block blockIdx.z; blockIdx.x enumerates the (h/RB)^2 output tiles.
//   PHASE 0:  T(ti,tj) = sum_{kt >= tj} L(h + ti, kt) A^-1(kt, tj)  -> upper-right scratch
//   PHASE 1:  X(ti,tj) = -sum_{kt <= ti} C^-1(ti, kt) T(kt, tj)     -> lower-left block
// (128-tile indices relative to the pair's origin a0 = 2 h * pair).  Tiles
// whose rows start at or past n are skipped: the solves never read them.
template <int PHASE>
__device__ __forceinline__ void
superinv_gemm_body(const float* __restrict__ L, int ldl, int n, float* __restrict__ wsup, int h, uint3 bid) {
  __shared__ __align__(16) float As[GK * RB];
  __shared__ __align__(16) float Bs[RB * BLDK];
  const int tpr = h / RB;
  const int ti = bid.x / tpr, tj = bid.x % tpr;
  const int S = bid.z, s0 = S * RS, a0 = bid.y * 2 * h;
  const int grow = s0 + a0 + h + ti * RB;          // first global row of the output tile
  if (grow >= n) return;
  float* W = wsup + (size_t)S * RS * RS;
  float acc[8][8] = {};
  if (PHASE == 0) {
    gemm128(L + (size_t)(s0 + a0 + tj * RB) * ldl + grow, ldl, min(RB, n - grow),
            W + (size_t)(a0 + tj * RB) * RS + a0 + tj * RB, RS, h - tj * RB, acc, As, Bs);
    float* T = W + (size_t)(a0 + h + tj * RB) * RS + a0 + ti * RB;
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) T[(size_t)acc_col(b) * RS + acc_row(a)] = acc[a][b];
  } else {
    gemm128(W + (size_t)(a0 + h) * RS + a0 + h + ti * RB, RS, RB,
            W + (size_t)(a0 + h + tj * RB) * RS + a0, RS, (ti + 1) * RB, acc, As, Bs);
    float* X = W + (size_t)(a0 + tj * RB) * RS + a0 + h + ti * RB;
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) X[(size_t)acc_col(b) * RS + acc_row(a)] = -acc[a][b];
  }
}

template <int PHASE>
__global__ void __launch_bounds__(NTH)
superinv_gemm_kernel(const float* __restrict__ L, int ldl, int n, float* __restrict__ wsup, int h) {
  superinv_gemm_body<PHASE>(L, ldl, n, wsup, h, blockIdx);
}

// ---- y_S += W_S w_S (TRANS: z_S += W_S^T w_S) over the super-block's lower tiles
template <int NR, bool TRANS>
__device__ __forceinline__ void
trmv_super_body(const float* __restrict__ W, int n, int s0, int rs, const double* __restrict__ in,
                  double* __restrict__ out, const int* skip, uint3 bid) {
  if (skip != nullptr && *skip) return;
  __shared__ __align__(16) double s_v[RB * NR];
  __shared__ double s_col[RB * NR];
  extern __shared__ double s_red[];
  int i, j;
  tri_of(bid.x, i, j);
  const int ri0 = s0 + i * RB, rj0 = s0 + j * RB;
  const int ni = min(RB, s0 + rs - ri0), nj = min(RB, s0 + rs - rj0);
  if (!TRANS) load_vec<NR>(in, n, rj0, nj, s_v);
  else load_vec<NR>(in, n, ri0, ni, s_v);
  __syncthreads();
  double acc[4][NR] = {};
  const float* T = W + (size_t)(j * RB) * RS + i * RB;
  tile_pass<float, NR, 16>(T, RS, ni, nj, s_v, s_v, acc, s_col, 0, 0, !TRANS, TRANS);
  __syncthreads();
  if (!TRANS) {
    flush_rows<NR>(acc, s_red, out, n, ri0, ni, 1.0);
  } else {
    for (int e = threadIdx.x; e < RB * NR; e += NTH) {
      const int k = e / RB, c = e % RB;
      if (c < nj) atomicAdd(&out[(size_t)k * n + rj0 + c], s_col[e]);
    }
  }
}


// ---- panel updates ---------------------------------------------------------
// forward: w[rows below the super-block] -= L(rows, super-block cols) y_S
// backward: w[cols left of the super-block] -= L(super-block rows, cols)^T z_S
template <int NR, bool TRANS>
__device__ __forceinline__ void
panel_body(const float* __restrict__ L, int ldl, int n, int s0, int rs,
             const double* __restrict__ v, double* __restrict__ w, const int* skip, uint3 bid) {
  if (skip != nullptr && *skip) return;
  __shared__ __align__(16) double s_v[RB * NR];
  __shared__ double s_col[RB * NR];
  extern __shared__ double s_red[];
  int r0, c0, nr_, nc_;
  if (!TRANS) {
    r0 = s0 + rs + bid.x * RB;  c0 = s0 + bid.y * RB;
    nr_ = min(RB, n - r0);           nc_ = min(RB, s0 + rs - c0);
    load_vec<NR>(v, n, c0, nc_, s_v);
  } else {
    r0 = s0 + bid.y * RB;       c0 = bid.x * RB;
    nr_ = min(RB, s0 + rs - r0);     nc_ = min(RB, s0 - c0);
    load_vec<NR>(v, n, r0, nr_, s_v);
  }
  __syncthreads();
  double acc[4][NR] = {};
  tile_pass<float, NR, 16>(L + (size_t)c0 * ldl + r0, ldl, nr_, nc_, s_v, s_v, acc, s_col, 0, 0,
                           !TRANS, TRANS);
  __syncthreads();
  if (!TRANS) {
    flush_rows<NR>(acc, s_red, w, n, r0, nr_, -1.0);
  } else {
    for (int e = threadIdx.x; e < RB * NR; e += NTH) {
      const int k = e / RB, c = e % RB;
      if (c < nc_) atomicAdd(&w[(size_t)k * n + c0 + c], -s_col[e]);
    }
  }
}


// ---- persistent triangular solve -------------------------------------------
// One launch per solve.  The tiles of a solve form a dependency DAG: the
// TRMV tiles of W_S (which need every panel contribution to their input
// segment) and the panel tiles below (forward) or left of (backward) S (which
// need their segment of y_S / z_S complete).  Units are handed out by an
// atomic counter in a topological order (trsv_job: grouped by the
// super-block they feed), so a unit only ever waits on units already taken
// by running CTAs; the launch is cooperative, so all CTAs are resident and
// every wait ends.  Completion is
// counted per 128-row segment:
//   seg_in[g]   panel contributions received by segment g (global 128-tile g)
//   seg_out[g]  TRMV tiles finished that write segment g of the result
// Waits are bounded; a wait that runs out records MPCHOL_ERR_TIMEOUT and the
// unit proceeds (the result is then wrong, but no CTA waits forever).
constexpr long long kTrsvMaxPolls = 1ll << 24;

__device__ __forceinline__ void wait_count(const int* ctr, int need, DevStatus* st, int unit) {
  if (threadIdx.x == 0) {
    long long it = 0;
    while (*reinterpret_cast<const volatile int*>(ctr) < need) {
      if (++it > kTrsvMaxPolls) {
        if (st != nullptr) set_status(st, MPCHOL_ERR_TIMEOUT, unit);
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
}

__device__ __forceinline__ void signal_count(int* ctr) {
  __threadfence();                            // this thread's atomics visible device-wide
  __syncthreads();                            // ... for every thread of the unit
  if (threadIdx.x == 0) atomicAdd(ctr, 1);
}

// One unit of the solve: a tile, the vector segment it reads, where its
// result goes and the counters it waits on and signals.
struct TrsvJob {
  const float* T;       // tile origin (column-major)
  int ld, nrow, ncol;   // leading dimension, valid rows / columns
  int vin_row0, vin_n;  // input segment (of out for panels, of work for TRMV)
  int out_row0, out_n;  // output segment
  bool nt;              // NOTRANS (row sums) or TRANS (column sums)
  bool panel;           // L panel tile (reads out, writes work) or W_S tile
  const int* wait_ctr;
  int wait_need;
  int* sig_ctr;
};

// Decode unit u.  Units are grouped by the super-block B they feed, in solve
// order (forward: B = 0, 1, ..; backward: B = NS-1, NS-2, ..): group B holds
// the panel tiles that carry an earlier super-block's finished segment of the
// solution into B's input (sources in solve order, so the ones ready longest
// come first), then the TRMV tiles of W_B.  Every unit depends only on units
// of earlier groups or earlier in its own group, so the order is topological
// (the deadlock-freedom of the persistent loop needs that), and a CTA is
// never handed far-off panel work while the chain's next TRMV waits in the
// queue behind it.  Returns false past the last unit.
template <bool TRANS>
__device__ __forceinline__ bool trsv_job(int u, const float* L, int ldl, int n, const float* wsup,
                                         int* seg_in, int* seg_out, TrsvJob& jb) {
  const int ntiles = ceil_div(n, RB);
  const int NS = ceil_div(n, RS);
  constexpr int NSUB = RS / RB;              // segments of a full super-block
  for (int t = 0; t < NS; ++t) {
    const int B = TRANS ? NS - 1 - t : t;
    const int b0 = B * RS;
    const int rb = min(RS, n - b0);
    const int nsubB = ceil_div(rb, RB);
    const int gB = b0 / RB;                  // first global segment of B
    // panel tiles feeding B: forward from every T < B (NSUB columns of T x
    // nsubB rows of B); backward from every T > B (the rows of T x NSUB
    // columns of B)
    const int npan = TRANS ? (ntiles - gB - nsubB) * NSUB : B * NSUB * nsubB;
    if (u < npan) {
      jb.panel = true;
      jb.ld = ldl;
      if (!TRANS) {
        // w(rows r of B) -= L(r, T col c) y_T(c)
        const int T = u / (NSUB * nsubB), q = u % (NSUB * nsubB);
        const int r = q / NSUB, c = q % NSUB;
        const int r0 = b0 + r * RB, c0 = T * RS + c * RB;
        jb.T = L + (size_t)c0 * ldl + r0;
        jb.nrow = min(RB, n - r0); jb.ncol = RB;
        jb.nt = true;
        jb.vin_row0 = c0; jb.vin_n = RB;
        jb.out_row0 = r0; jb.out_n = jb.nrow;
        jb.wait_ctr = seg_out + T * NSUB + c; jb.wait_need = c + 1;
        jb.sig_ctr = seg_in + gB + r;
      } else {
        // w(col segment c of B) -= L(T row rt, c)^T z_T(rt); sources T from
        // the last super-block down
        int q = u, T = NS - 1;
        for (;; --T) {
          const int nsubT = ceil_div(min(RS, n - T * RS), RB);
          if (q < nsubT * NSUB) break;
          q -= nsubT * NSUB;
        }
        const int rt = q / NSUB, c = q % NSUB;
        const int t0 = T * RS;
        const int nsubT = ceil_div(min(RS, n - t0), RB);
        const int r0 = t0 + rt * RB, c0 = b0 + c * RB;
        jb.T = L + (size_t)c0 * ldl + r0;
        jb.nrow = min(RB, n - r0); jb.ncol = RB;
        jb.nt = false;
        jb.vin_row0 = r0; jb.vin_n = jb.nrow;
        jb.out_row0 = c0; jb.out_n = RB;
        jb.wait_ctr = seg_out + T * NSUB + rt; jb.wait_need = nsubT - rt;
        jb.sig_ctr = seg_in + gB + c;
      }
      return true;
    }
    u -= npan;
    const int ntr = nsubB * (nsubB + 1) / 2;
    if (u < ntr) {
      int i, j;
      tri_of(u, i, j);
      const int ri0 = b0 + i * RB, rj0 = b0 + j * RB;
      jb.T = wsup + (size_t)B * RS * RS + (size_t)(j * RB) * RS + i * RB;
      jb.ld = RS;
      jb.nrow = min(RB, b0 + rb - ri0);
      jb.ncol = min(RB, b0 + rb - rj0);
      jb.panel = false;
      if (!TRANS) {
        // y_B(i) += W(i,j) w_B(j): w_B(j) has all gB panel contributions
        jb.nt = true;
        jb.vin_row0 = rj0; jb.vin_n = jb.ncol;
        jb.out_row0 = ri0; jb.out_n = jb.nrow;
        jb.wait_ctr = seg_in + gB + j; jb.wait_need = gB;
        jb.sig_ctr = seg_out + gB + i;
      } else {
        // z_B(j) += W(i,j)^T w_B(i): w_B(i) has the contributions of every
        // segment below B
        jb.nt = false;
        jb.vin_row0 = ri0; jb.vin_n = jb.nrow;
        jb.out_row0 = rj0; jb.out_n = jb.ncol;
        jb.wait_ctr = seg_in + gB + i; jb.wait_need = ntiles - gB - nsubB;
        jb.sig_ctr = seg_out + gB + j;
      }
      return true;
    }
    u -= ntr;
  }
  return false;
}

template <int NR>
constexpr size_t trsv_staged_smem() {
  if (NR == 8) return (size_t)BL_TILE * sizeof(float) + (size_t)XS * 8 * sizeof(double);
  return (size_t)TILE_ELEMS * sizeof(float) + 2 * (size_t)RB * NR * sizeof(double);
}
size_t trsv_smem_bytes(int nrhs) {
  switch (nrhs) {
    case 1: return trsv_staged_smem<1>();
    case 2: return trsv_staged_smem<2>();
    case 4: return trsv_staged_smem<4>();
    default: return trsv_staged_smem<8>();
  }
}

// Two CTAs per SM, each with one tile stage: a unit's tile copy is issued
// as soon as the unit is taken and overlaps the wait for its input segment;
// while one CTA waits on L2 round trips (unit counter, dependency counter,
// vector segment, fence) the other computes.  The next unit number is taken
// one unit ahead.  A CTA holds at most two units and finishes the earlier
// one first; every unit depends only on earlier ones, so the earliest
// unfinished unit always belongs to a CTA that is working on it, and every
// wait ends.
template <int NR, bool TRANS>
__global__ void __launch_bounds__(NTH, 2)
trsv_persistent_kernel(const float* __restrict__ L, int ldl, int n, const float* __restrict__ wsup,
                       double* __restrict__ work, double* __restrict__ out, int* ctr,
                       const int* skip, DevStatus* st) {
  if (skip != nullptr && *skip) return;
  constexpr bool MMA = NR == 8;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  float* Ts = reinterpret_cast<float*>(sm_raw);                           // one stage
  double* s_v = reinterpret_cast<double*>(Ts + (MMA ? BL_TILE : TILE_ELEMS));   // RB x NR
  double* s_col = s_v + RB * NR;                                          // RB x NR
  __shared__ int s_unit[2];
  int* next = ctr;
  int* seg_in = ctr + 1;
  int* seg_out = seg_in + ceil_div(n, RB);
  if (threadIdx.x == 0) s_unit[0] = atomicAdd(next, 1);
  __syncthreads();
  int ucur = s_unit[0];
  TrsvJob cur;
  bool have = trsv_job<TRANS>(ucur, L, ldl, n, wsup, seg_in, seg_out, cur);
  for (int it = 1; have; ++it) {
    if (MMA) stage_tile_bl(Ts, cur.T, cur.ld, cur.nrow, cur.ncol);
    else stage_tile(Ts, cur.T, cur.ld, cur.nrow, cur.ncol);
    cp_async_commit();
    // the next unit number, taken by a thread of warp 1 so that its round
    // trip overlaps warp 0's dependency poll; read after this unit's
    // barriers (s_unit[it & 1] is not read again before its next write)
    if (threadIdx.x == 32) s_unit[it & 1] = atomicAdd(next, 1);
    wait_count(cur.wait_ctr, cur.wait_need, st, ucur);
    if (MMA) {
      load_vec_x8(cur.panel ? out : work, n, cur.vin_row0, cur.vin_n, s_v);
      cp_async_wait<0>();
      __syncthreads();
      double* dst = cur.panel ? work : out;
      if (cur.nt)
        tile_mma_x8<false, false, 4, RB / 16, 1>(Ts, s_v, s_v, dst, cur.out_row0, cur.out_n, dst,
                                                 cur.out_row0, cur.out_n, n, true, false,
                                                 cur.panel ? -1.0 : 1.0, nullptr);
      else
        tile_mma_x8<false, false, 4, RB / 16, 2>(Ts, s_v, s_v, dst, cur.out_row0, cur.out_n, dst,
                                                 cur.out_row0, cur.out_n, n, false, true,
                                                 cur.panel ? -1.0 : 1.0, nullptr);
      signal_count(cur.sig_ctr);   // its barrier also frees the stage and s_v
      ucur = s_unit[it & 1];
      have = trsv_job<TRANS>(ucur, L, ldl, n, wsup, seg_in, seg_out, cur);
      continue;
    }
    load_vec<NR>(cur.panel ? out : work, n, cur.vin_row0, cur.vin_n, s_v);
    cp_async_wait<0>();
    __syncthreads();
    double acc[4][NR] = {};
    tile_pass_staged<NR, false>(Ts, s_v, s_v, acc, s_col, cur.nt, !cur.nt);
    __syncthreads();
    double* dst = cur.panel ? work : out;
    const double sign = cur.panel ? -1.0 : 1.0;
    if (cur.nt) {
      flush_rows<NR>(acc, reinterpret_cast<double*>(Ts), dst, n, cur.out_row0, cur.out_n, sign);
    } else {
      for (int e = threadIdx.x; e < RB * NR; e += NTH) {
        const int k = e / RB, c = e % RB;
        if (c < cur.out_n) atomicAdd(&dst[(size_t)k * n + cur.out_row0 + c], sign * s_col[e]);
      }
    }
    signal_count(cur.sig_ctr);   // its barrier also frees the stage, s_v and s_col
    ucur = s_unit[it & 1];
    have = trsv_job<TRANS>(ucur, L, ldl, n, wsup, seg_in, seg_out, cur);
  }
}

// ---- batched variants: one launch serves every system of a batch --------
// blockIdx.y (or .z) selects the system; CTAs past a system's own extent
// return at once.  Vectors live in the system's slots (n x NR column-major).
__device__ __forceinline__ double* bslot(const BatchSys& S, int slot, int nr) {
  return S.vec + (size_t)slot * S.n * nr;
}

// A tile whose columns need not start on 16-byte boundaries, by 4-byte
// copies into the plain (BL = false) or blocked (BL = true) layout.
template <bool BL>
__device__ __forceinline__ void stage_tile_4b(float* dst, const float* T, int ld, int rows_valid,
                                              int cols_valid) {
#pragma unroll 4
  for (int e = threadIdx.x; e < TILE_ELEMS; e += NTH) {
    const int c = e / RB, r = e % RB;
    const bool ok = c < cols_valid && r < rows_valid;
    cp_async4(dst + (BL ? bl_off(r, c) : c * RB + r), ok ? T + (size_t)c * ld + r : T, ok ? 4 : 0);
  }
}

// One unit of the batched operator product: tile (I, J) of one system's
// lower triangle.  A == nullptr: the system has converged, nothing to do.
struct SymvUnit {
  const float* A;
  int lda, n, I, J;
  const double* x;
  double* y;
  int al16;             // columns start on 16-byte boundaries
};

// Unit t -> its system (binary search of the per-system first units; the
// systems are numbered in order of their first unit) and its tile.
template <int NR>
__device__ __forceinline__ SymvUnit symv_unit(const BatchSys* __restrict__ sys, int nsys, int t,
                                              int xslot, int yslot, int use_skip) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sys[mid].sym_tile0 <= t) lo = mid;
    else hi = mid - 1;
  }
  const BatchSys& S = sys[lo];
  SymvUnit u;
  tri_of(t - S.sym_tile0, u.I, u.J);
  u.A = (use_skip && S.done[0]) ? nullptr : S.op;
  u.lda = S.op_ld;
  u.n = S.n;
  u.x = bslot(S, xslot, NR);
  u.y = bslot(S, yslot, NR);
  u.al16 = (reinterpret_cast<uintptr_t>(S.op) & 15) == 0 && S.op_ld % 4 == 0;
  return u;
}

// y = A x for every system of a batch, persistent over the concatenated
// 128-tiles of all systems' lower triangles, with the unit's system found per
// tile.  Two single-stage CTAs per SM: each copies its next tile and vector
// segments into shared memory while the other runs its tile pass (both A x
// and A^T x from the one copy).  For 1-4 rhs this replaces three stages in
// one 190-register CTA per SM and caps the FP64 tile pass at 128 registers:
// the 512-system batch step (4 rhs, 10 products) took 54.8 against 57.5 ms.
// y slots are zeroed beforehand.
template <int NR>
constexpr size_t symv_batched_smem() {
  if (NR == 8)
    return (size_t)BL_TILE * sizeof(float) + 2 * (size_t)XS * 8 * sizeof(double);
  return (size_t)TILE_ELEMS * sizeof(float) + 3 * (size_t)RB * NR * sizeof(double);
}
template <int NR>
__global__ void __launch_bounds__(NTH, 2)
symv_staged_batched_kernel(const BatchSys* __restrict__ sys, int nsys, int ntiles, int xslot,
                           int yslot, int use_skip) {
  constexpr int STAGES = 1;
  constexpr bool MMA = NR == 8;
  constexpr int TE = MMA ? BL_TILE : TILE_ELEMS;
  constexpr int VEC = MMA ? XS * 8 : RB * NR;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  __shared__ SymvUnit s_unit[STAGES];
  float* tiles = reinterpret_cast<float*>(sm_raw);
  double* vecs = reinterpret_cast<double*>(tiles + STAGES * TE);
  double* s_col = vecs + STAGES * 2 * VEC;
  auto issue = [&](int t, int stage) {
    const SymvUnit u = symv_unit<NR>(sys, nsys, t, xslot, yslot, use_skip);
    if (threadIdx.x == 0) s_unit[stage] = u;
    if (u.A == nullptr) return;
    const int i0 = u.I * RB, j0 = u.J * RB;
    const int ni = min(RB, u.n - i0), nj = min(RB, u.n - j0);
    const float* T = u.A + (size_t)j0 * u.lda + i0;
    float* dst = tiles + stage * TE;
    if (MMA) {
      if (u.al16) stage_tile_bl(dst, T, u.lda, ni, nj);
      else stage_tile_4b<true>(dst, T, u.lda, ni, nj);
      stage_vec_x8(u.x, u.n, j0, nj, vecs + (2 * stage) * VEC);
      stage_vec_x8(u.x, u.n, i0, ni, vecs + (2 * stage + 1) * VEC);
    } else {
      if (u.al16) stage_tile(dst, T, u.lda, ni, nj);
      else stage_tile_4b<false>(dst, T, u.lda, ni, nj);
      stage_vec<NR>(u.x, u.n, j0, nj, vecs + (2 * stage) * VEC);
      stage_vec<NR>(u.x, u.n, i0, ni, vecs + (2 * stage + 1) * VEC);
    }
  };
#pragma unroll
  for (int st = 0; st < STAGES - 1; ++st) {
    const int t = blockIdx.x + st * gridDim.x;
    if (t < ntiles) issue(t, st);
    cp_async_commit();
  }
  int stage = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    {
      const int tn = t + (STAGES - 1) * gridDim.x;
      if (tn < ntiles) issue(tn, (stage + STAGES - 1) % STAGES);
      cp_async_commit();
    }
    cp_async_wait<STAGES - 1>();
    __syncthreads();
    const SymvUnit u = s_unit[stage];
    if (u.A != nullptr) {
      const int i0 = u.I * RB, j0 = u.J * RB;
      const int ni = min(RB, u.n - i0), nj = min(RB, u.n - j0);
      float* Ts = tiles + stage * TE;
      const double* xJ = vecs + (2 * stage) * VEC;
      const double* xI = xJ + VEC;
      if (MMA) {
        if (u.I == u.J)
          tile_mma_x8<true, false>(Ts, xJ, xI, u.y, i0, ni, u.y, j0, nj, u.n, true, true, 1.0, nullptr);
        else
          tile_mma_x8<false, false>(Ts, xJ, xI, u.y, i0, ni, u.y, j0, nj, u.n, true, true, 1.0, nullptr);
      } else {
        double acc[4][NR] = {};
        if (u.I == u.J) tile_pass_staged<NR, true>(Ts, xJ, xI, acc, s_col, true, true);
        else tile_pass_staged<NR, false>(Ts, xJ, xI, acc, s_col, true, true);
        __syncthreads();
        for (int e = threadIdx.x; e < VEC; e += NTH) {
          const int k = e / RB, c = e % RB;
          if (c < nj) atomicAdd(&u.y[(size_t)k * u.n + j0 + c], s_col[e]);
        }
        flush_rows<NR>(acc, reinterpret_cast<double*>(Ts), u.y, u.n, i0, ni, 1.0);
      }
    }
    __syncthreads();   // the stage, its unit record and s_col are free again
    stage = (stage + 1) % STAGES;
  }
  cp_async_wait<0>();
}

// dst slot = 0 (src < 0) or a copy of the src slot
__global__ void vec_slot_batched_kernel(const BatchSys* __restrict__ sys, int src, int dst, int nr,
                                        int use_skip) {
  const BatchSys& S = sys[blockIdx.y];
  if (use_skip && S.done[0]) return;
  const long long cnt = (long long)S.n * nr;
  double* d = bslot(S, dst, nr);
  const double* a = src >= 0 ? bslot(S, src, nr) : nullptr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = a ? a[i] : 0.0;
}

__global__ void __launch_bounds__(NTH)
block_inverse_batched_kernel(const BatchSys* __restrict__ sys) {
  const BatchSys& S = sys[blockIdx.y];
  if ((int)blockIdx.x * RB >= S.n) return;
  block_inverse_body(S.A, S.ld, S.n, S.wsup, make_uint3(blockIdx.x, 0, 0));
}

template <int PHASE>
__global__ void __launch_bounds__(NTH)
superinv_gemm_batched_kernel(const BatchSys* __restrict__ sys, int h, int max_super) {
  const BatchSys& S = sys[blockIdx.z / max_super];
  const int sup = blockIdx.z % max_super;
  if (sup * RS >= S.n) return;
  superinv_gemm_body<PHASE>(S.A, S.ld, S.n, S.wsup, h, make_uint3(blockIdx.x, blockIdx.y, sup));
}

template <int NR, bool TRANS>
__global__ void __launch_bounds__(NTH)
trmv_super_batched_kernel(const BatchSys* __restrict__ sys, int sup, int in_slot, int out_slot,
                          int use_skip) {
  const BatchSys& S = sys[blockIdx.y];
  const int s0 = sup * RS;
  if (s0 >= S.n) return;
  const int rs = min(RS, S.n - s0);
  const int nsub = ceil_div(rs, RB);
  if ((int)blockIdx.x >= nsub * (nsub + 1) / 2) return;
  trmv_super_body<NR, TRANS>(S.wsup + (size_t)sup * RS * RS, S.n, s0, rs, bslot(S, in_slot, NR),
                             bslot(S, out_slot, NR), use_skip ? S.done : nullptr,
                             make_uint3(blockIdx.x, 0, 0));
}

template <int NR, bool TRANS>
__global__ void __launch_bounds__(NTH)
panel_batched_kernel(const BatchSys* __restrict__ sys, int sup, int v_slot, int w_slot,
                     int use_skip) {
  const BatchSys& S = sys[blockIdx.z];
  const int s0 = sup * RS;
  if (s0 >= S.n) return;
  const int rs = min(RS, S.n - s0);
  const int nsub = ceil_div(rs, RB);
  const int span = TRANS ? s0 : S.n - s0 - rs;      // rows below (forward) / columns left (backward)
  if (span <= 0 || (int)blockIdx.x >= ceil_div(span, RB) || (int)blockIdx.y >= nsub) return;
  panel_body<NR, TRANS>(S.A, S.ld, S.n, s0, rs, bslot(S, v_slot, NR), bslot(S, w_slot, NR),
                        use_skip ? S.done : nullptr, make_uint3(blockIdx.x, blockIdx.y, 0));
}

// The persistent solve's inputs: work <- in, out <- 0 and its dependency
// counters cleared, in one launch.
__global__ void trsv_prep_kernel(const double* __restrict__ in, double* __restrict__ work,
                                 double* __restrict__ out, long long count, int* counters,
                                 int ncounters, const int* skip) {
  if (skip != nullptr && *skip) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long i = t0; i < count; i += stride) {
    work[i] = in[i];
    out[i] = 0.0;
  }
  for (long long i = t0; i < ncounters; i += stride) counters[i] = 0;
}

__global__ void zero_vec_kernel(double* __restrict__ a, long long count, const int* skip) {
  if (skip != nullptr && *skip) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = 0.0;
}

size_t red_bytes(int nr) { return (size_t)(NTH / 32) * RB * nr * sizeof(double); }

template <typename K>
cudaError_t set_dyn(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

#define NR_SWITCH(nrhs, CALL)                                 \
  switch (nrhs) {                                             \
    case 1: { constexpr int NRC = 1; CALL; } break;           \
    case 2: { constexpr int NRC = 2; CALL; } break;           \
    case 4: { constexpr int NRC = 4; CALL; } break;           \
    case 8: { constexpr int NRC = 8; CALL; } break;           \
    default: return cudaErrorInvalidValue;                    \
  }

int solve_super_rows() { return RS; }
size_t solve_wsup_elems(int n) {
  const int nbs = (n + RS - 1) / RS;
  return (size_t)nbs * RS * RS;
}

cudaError_t solve_init_attributes() {
  // once per device (kernel attributes are per device)
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  e = solve_set_attributes();
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

cudaError_t solve_set_attributes() {
  cudaError_t e;
  const size_t inv = (size_t)RB * BLD * (sizeof(double) + sizeof(float));
  if ((e = set_dyn(block_inverse_kernel, inv)) != cudaSuccess) return e;
#define SET_NR(NRC)                                                                         \
  if ((e = set_dyn(symv_kernel<float, NRC>, red_bytes(NRC))) != cudaSuccess) return e;      \
  if ((e = set_dyn(symv_kernel<double, NRC>, red_bytes(NRC))) != cudaSuccess) return e;
  SET_NR(1) SET_NR(2) SET_NR(4) SET_NR(8)
#undef SET_NR
#define SET_NRP(NRC)                                                                              \
  if ((e = set_dyn(trsv_persistent_kernel<NRC, false>, trsv_staged_smem<NRC>())) != cudaSuccess) return e; \
  if ((e = set_dyn(trsv_persistent_kernel<NRC, true>, trsv_staged_smem<NRC>())) != cudaSuccess) return e; \
  if ((e = set_dyn(symv_staged_kernel<NRC>, symv_staged_smem<NRC>())) != cudaSuccess) return e;
  SET_NRP(1) SET_NRP(2) SET_NRP(4) SET_NRP(8)
#undef SET_NRP
  if ((e = set_dyn(block_inverse_batched_kernel, inv)) != cudaSuccess) return e;
#define SET_NRB(NRC)                                                                              \
  if ((e = set_dyn(symv_staged_batched_kernel<NRC>, symv_batched_smem<NRC>())) != cudaSuccess) return e; \
  if ((e = set_dyn(trmv_super_batched_kernel<NRC, false>, red_bytes(NRC))) != cudaSuccess) return e; \
  if ((e = set_dyn(trmv_super_batched_kernel<NRC, true>, red_bytes(NRC))) != cudaSuccess) return e;  \
  if ((e = set_dyn(panel_batched_kernel<NRC, false>, red_bytes(NRC))) != cudaSuccess) return e;      \
  if ((e = set_dyn(panel_batched_kernel<NRC, true>, red_bytes(NRC))) != cudaSuccess) return e;
  SET_NRB(1) SET_NRB(2) SET_NRB(4) SET_NRB(8)
#undef SET_NRB
  return cudaSuccess;
}

int sm_count() {
  static int cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  int& c = cache[dev & 63];
  if (c == 0 && cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) c = 148;
  return c;
}

// FP32 operators whose columns start on 16-byte boundaries stream through
// the staged persistent kernel; others (and FP64 operators) take one CTA per
// tile with register loads.
template <typename TA>
bool symv_staged_ok(const TA* A, int lda) {
  return sizeof(TA) == 4 && (reinterpret_cast<uintptr_t>(A) & 15) == 0 && lda % 4 == 0;
}
template bool symv_staged_ok<float>(const float*, int);
template bool symv_staged_ok<double>(const double*, int);

template <typename TA>
cudaError_t launch_symv_skip(const TA* A, int lda, int n, const double* x, double* y, int nrhs,
                             const int* skip, cudaStream_t stream, double* fro, int nfro) {
  const long long cnt = (long long)n * nrhs;
  zero_vec_kernel<<<148, 256, 0, stream>>>(y, cnt, skip);
  const int T = ceil_div(n, RB);
  const int ntiles = T * (T + 1) / 2;
  if (symv_staged_ok(A, lda)) {
    int grid = std::min(ntiles, (nrhs >= 8 ? 2 : 1) * sm_count());
    if (fro != nullptr) grid = std::min(grid, nfro);   // one Frobenius partial per CTA
    const float* Af = reinterpret_cast<const float*>(A);
    NR_SWITCH(nrhs, (symv_staged_kernel<NRC><<<grid, NTH, symv_staged_smem<NRC>(), stream>>>(Af, lda, n, x, y, skip, fro, nfro)));
  } else {
    NR_SWITCH(nrhs, (symv_kernel<TA, NRC><<<ntiles, NTH, red_bytes(NRC), stream>>>(A, lda, n, x, y, skip)));
  }
  return cudaGetLastError();
}
template cudaError_t launch_symv_skip<float>(const float*, int, int, const double*, double*, int, const int*, cudaStream_t, double*, int);
template cudaError_t launch_symv_skip<double>(const double*, int, int, const double*, double*, int, const int*, cudaStream_t, double*, int);

cudaError_t launch_solve_setup(const float* L, int ldl, int n, float* wsup, cudaStream_t stream) {
  const size_t inv = (size_t)RB * BLD * (sizeof(double) + sizeof(float));
  block_inverse_kernel<<<ceil_div(n, RB), NTH, inv, stream>>>(L, ldl, n, wsup);
  const int nbs = ceil_div(n, RS);
  for (int h = RB; h < RS; h *= 2) {
    const dim3 grid((h / RB) * (h / RB), RS / (2 * h), nbs);
    superinv_gemm_kernel<0><<<grid, NTH, 0, stream>>>(L, ldl, n, wsup, h);
    superinv_gemm_kernel<1><<<grid, NTH, 0, stream>>>(L, ldl, n, wsup, h);
  }
  return cudaGetLastError();
}

int solve_setup_launches(int n) {
  (void)n;
  int k = 1;
  for (int h = RB; h < RS; h *= 2) k += 2;
  return k;
}

cudaError_t launch_vec_slot_batched(const BatchSys* sys, int nsys, int src, int dst, int nr,
                                    int use_skip, cudaStream_t stream) {
  vec_slot_batched_kernel<<<dim3(8, nsys), NTH, 0, stream>>>(sys, src, dst, nr, use_skip);
  return cudaGetLastError();
}

cudaError_t launch_symv_batched(const BatchSys* sys, int nsys, int ntiles, int xslot, int yslot,
                                int nr, int use_skip, cudaStream_t stream) {
  cudaError_t e = launch_vec_slot_batched(sys, nsys, -1, yslot, nr, use_skip, stream);
  if (e != cudaSuccess) return e;
  if (ntiles <= 0) return cudaSuccess;
  const int grid = std::min(ntiles, 2 * sm_count());
  NR_SWITCH(nr, (symv_staged_batched_kernel<NRC><<<grid, NTH, symv_batched_smem<NRC>(), stream>>>(sys, nsys, ntiles, xslot, yslot, use_skip)));
  return cudaGetLastError();
}

cudaError_t launch_solve_setup_batched(const BatchSys* sys, int nsys, int max_n,
                                       cudaStream_t stream) {
  const size_t inv = (size_t)RB * BLD * (sizeof(double) + sizeof(float));
  block_inverse_batched_kernel<<<dim3(ceil_div(max_n, RB), nsys), NTH, inv, stream>>>(sys);
  const int max_super = ceil_div(max_n, RS);
  for (int h = RB; h < RS; h *= 2) {
    const dim3 grid((h / RB) * (h / RB), RS / (2 * h), nsys * max_super);
    superinv_gemm_batched_kernel<0><<<grid, NTH, 0, stream>>>(sys, h, max_super);
    superinv_gemm_batched_kernel<1><<<grid, NTH, 0, stream>>>(sys, h, max_super);
  }
  return cudaGetLastError();
}

cudaError_t launch_trsv_batched(bool backward, const BatchSys* sys, int nsys, int max_n,
                                int in_slot, int out_slot, int work_slot, int nr, int use_skip,
                                cudaStream_t stream) {
  cudaError_t e = launch_vec_slot_batched(sys, nsys, in_slot, work_slot, nr, use_skip, stream);
  if (e == cudaSuccess) e = launch_vec_slot_batched(sys, nsys, -1, out_slot, nr, use_skip, stream);
  if (e != cudaSuccess) return e;
  const int max_super = ceil_div(max_n, RS);
  const int nsub_max = ceil_div(min(max_n, RS), RB);
  const int span_tiles = ceil_div(max_n, RB);
  for (int t = 0; t < max_super; ++t) {
    const int sup = backward ? max_super - 1 - t : t;
    const dim3 gt(nsub_max * (nsub_max + 1) / 2, nsys);
    const dim3 gp(span_tiles, nsub_max, nsys);
    if (!backward) {
      NR_SWITCH(nr, (trmv_super_batched_kernel<NRC, false><<<gt, NTH, red_bytes(NRC), stream>>>(sys, sup, work_slot, out_slot, use_skip)));
      NR_SWITCH(nr, (panel_batched_kernel<NRC, false><<<gp, NTH, red_bytes(NRC), stream>>>(sys, sup, out_slot, work_slot, use_skip)));
    } else {
      NR_SWITCH(nr, (trmv_super_batched_kernel<NRC, true><<<gt, NTH, red_bytes(NRC), stream>>>(sys, sup, work_slot, out_slot, use_skip)));
      NR_SWITCH(nr, (panel_batched_kernel<NRC, true><<<gp, NTH, red_bytes(NRC), stream>>>(sys, sup, out_slot, work_slot, use_skip)));
    }
  }
  return cudaGetLastError();
}

size_t trsv_counter_ints(int n) { return 1 + 2 * (size_t)ceil_div(n, RB); }

// The persistent solve: work <- in, out <- 0 and the counters
// (trsv_counter_ints(n) ints) cleared in one launch, then one cooperative
// launch over every resident CTA.
cudaError_t launch_trsv_persistent(bool backward, const float* L, int ldl, int n,
                                   const float* wsup, const double* in, double* out,
                                   double* work, int nrhs, int* counters, const int* skip,
                                   DevStatus* st, cudaStream_t stream) {
  const long long cnt = (long long)n * nrhs;
  cudaError_t e;
  trsv_prep_kernel<<<148, 256, 0, stream>>>(in, work, out, cnt, counters, (int)trsv_counter_ints(n),
                                            skip);
  static int grid_cache[64][2][4] = {};
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  const int nri = nrhs == 1 ? 0 : nrhs == 2 ? 1 : nrhs == 4 ? 2 : 3;
  int& grid = grid_cache[dev & 63][backward ? 1 : 0][nri];
  const size_t smem = trsv_smem_bytes(nrhs);
  auto launch = [&](auto kernel) -> cudaError_t {
    if (grid == 0) {
      int per_sm = 0, nsm = 0;
      cudaError_t ee = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NTH,
                                                                     smem);
      if (ee == cudaSuccess) ee = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (ee != cudaSuccess) return ee;
      grid = std::max(1, per_sm) * nsm;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NTH);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, L, ldl, n, wsup, work, out, counters, skip, st);
  };
  if (!backward) {
    NR_SWITCH(nrhs, (e = launch(trsv_persistent_kernel<NRC, false>)));
  } else {
    NR_SWITCH(nrhs, (e = launch(trsv_persistent_kernel<NRC, true>)));
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}


}  // namespace mpchol
