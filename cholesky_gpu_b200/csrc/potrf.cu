// Diagonal-block Cholesky (POTRF) for the blocked factorization.
//
// Replaces the reference's per-step cusolverDnSpotrf of the b x b diagonal
// block (src/switching_chol.cuh:86-95) and its CPU micro_cholesky variant
// (src/micro_chol.hpp:14-44, src/sChol.cuh:66-79).  One CTA factors a block of
// up to 256 x 256 as a blocked right-looking Cholesky on dense 32 x 32 tiles in
// shared memory (column-major, lane i of a warp always owns row i, so every
// shared access is either contiguous across lanes or a broadcast):
//   * the lower tiles are staged by TMA (one thread issues the 2-D copies,
//     an mbarrier counts the bytes) and written back by TMA stores;
//   * one warp factors each diagonal tile with the tile's rows held in
//     registers, one tile ahead of the trailing update of the other warps;
//   * warps solve the tiles below and update the trailing tiles;
//   * the inverses of the diagonal tiles are formed for the panel solve.
// Blocks flagged near-indefinite by the switching criterion are factored in
// FP64 by a second kernel on a global (L2-resident) scratch.
#include "common.cuh"
#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace mpchol {

namespace {

constexpr int TS = 32;          // tile size
constexpr int TSZ = TS * TS;    // elements per dense tile

__device__ __forceinline__ int tidx(int I, int J) { return I * (I + 1) / 2 + J; }

// 16-byte shared-memory vector load of 4 floats or 2 doubles.
__device__ __forceinline__ void load_vec16(const float* p, float (&v)[4]) {
  const float4 w = *reinterpret_cast<const float4*>(p);
  v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
}
__device__ __forceinline__ void load_vec16(const double* p, double (&v)[2]) {
  const double2 w = *reinterpret_cast<const double2*>(p);
  v[0] = w.x; v[1] = w.y;
}

template <typename T>
__device__ __forceinline__ T drsqrt(T x);
template <>
__device__ __forceinline__ float drsqrt<float>(float x) { return rsqrtf(x); }
template <>
__device__ __forceinline__ double drsqrt<double>(double x) { return rsqrt(x); }

// The pivot rule of column k, evaluated by every lane on its own candidate
// (no divergent branch on the chain; lane k's value is the pivot).
template <typename T>
struct Pivot {
  T piv, r;        // repaired pivot and 1/sqrt(piv)
  bool pert, bad;  // repaired by the floor; failed (non-positive without repair, or not finite)
};
template <typename T>
__device__ __forceinline__ Pivot<T> eval_pivot(T cand, bool real, T my_shift, T my_pmin,
                                               int diag_pert) {
  Pivot<T> p;
  T piv = real ? cand + my_shift : T(1);
  // a NaN or infinite pivot means the Schur complement has overflowed
  // (earlier pivots floored far below the rounding error of a low-precision
  // update): no repair makes that factor usable, so it fails as NOT_SPD
  const bool nonfin = real && !(piv - piv == T(0));
  p.pert = false;
  p.bad = nonfin;
  if (diag_pert) {
    // repair: max(|pivot|, floor), the reference's fixDiag rule
    // (src/kernels_macros.cuh:90-99)
    p.pert = real && !nonfin && !(piv > my_pmin);
    const T ap = piv < T(0) ? -piv : piv;
    piv = p.pert ? (ap > my_pmin ? ap : my_pmin) : piv;
  } else {
    p.bad = p.bad || (real && !(piv > T(0)));
  }
  p.piv = p.bad ? T(1) : piv;   // keep the arithmetic finite; the caller discards the result
  // one SFU reciprocal square root on the dependency chain:
  // r = 1/sqrt(piv), L(k,k) = piv * r
  p.r = drsqrt<T>(p.piv);
  return p;
}

// Factor the 32 x 32 tile t in place (lower triangle).  inv[k] receives
// 1 / L(k,k).  Returns false on a non-positive pivot when pivot flooring is
// off (first failing local row in *fail_row).
//
// Lane i holds row i of the tile in registers (a[j], j relative to the
// current block of CB columns): per column lane k's pivot is repaired, one
// shuffle broadcasts 1/sqrt(pivot), and the rank-1 update reads the column's
// multipliers from the 32-entry shared buffer col as 16-byte broadcasts.  The
// columns run as a loop over blocks of CB whose body is unrolled: after a
// block its finished columns are stored and the registers shift down by CB,
// so register indices stay compile-time constants while the kernel's code
// stays small (its instructions must stay cache-resident while the trailing
// update saturates L2 beside it).  The pivot of column k + 1 is lane k + 1's
// candidate a[k+1] - L(k+1,k)^2 (the same fma the rank-1 update applies to
// a[k+1]); it is evaluated, square-rooted and broadcast before column k's
// multipliers go through shared memory, so the pivot chain and the update's
// round trip overlap.  Registers past the tile's last column are updated
// with junk and never stored.
template <typename T, int CB>
__device__ bool factor_diag_tile(T* t, T* inv, int lane, int nreal, const T* shift, const T* pmin,
                                 int diag_pert, int* nperturbed, int* fail_row, T* col) {
  constexpr int V = 16 / sizeof(T);
  T a[TS];
#pragma unroll
  for (int j = 0; j < TS; ++j) a[j] = t[j * TS + lane];
  const T my_shift = (lane < nreal) ? shift[lane] : T(0);
  const T my_pmin = pmin[lane];
  bool failed = false, perturbed = false;
  T my_inv = T(1);
  Pivot<T> pv = eval_pivot<T>(a[0], 0 < nreal, my_shift, my_pmin, diag_pert);
  T rk = __shfl_sync(0xffffffffu, pv.r, 0);
#pragma unroll 1
  for (int c0 = 0; c0 < TS; c0 += CB) {
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      const int k = c0 + c;
      const bool mine = lane == k;
      perturbed = perturbed || (mine && pv.pert);
      failed = failed || (mine && pv.bad);
      my_inv = mine ? pv.r : my_inv;
      const T lik = (lane > k) ? a[c] * rk : T(0);
      a[c] = mine ? pv.piv * pv.r : ((lane > k) ? lik : a[c]);
      if (k + 1 < TS) {
        pv = eval_pivot<T>(fma(-lik, lik, a[c + 1]), k + 1 < nreal, my_shift, my_pmin, diag_pert);
        rk = __shfl_sync(0xffffffffu, pv.r, k + 1);
      }
      // two multiplier buffers used in turn: the next column's write cannot
      // overtake a lane still reading this one, so one warp barrier suffices
      T* cb = col + (k & 1) * TS;
      cb[lane] = lik;
      __syncwarp();
#pragma unroll
      for (int q = (c + 1) / V; q < TS / V; ++q) {
        if (c0 + V * q < TS) {
          T l[V];
          load_vec16(cb + c0 + V * q, l);
#pragma unroll
          for (int e = 0; e < V; ++e) {
            const int j = V * q + e;
            if (j > c) a[j] = fma(-lik, l[e], a[j]);
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CB; ++c)
      if (c0 + c <= lane) t[(c0 + c) * TS + lane] = a[c];
#pragma unroll
    for (int j = 0; j < TS - CB; ++j) a[j] = a[j + CB];
  }
  inv[lane] = my_inv;
  const unsigned fm = __ballot_sync(0xffffffffu, failed);
  const unsigned pm = __ballot_sync(0xffffffffu, perturbed);
  if (fm) *fail_row = __ffs(fm) - 1;
  if (lane == 0) *nperturbed += __popc(pm);
  __syncwarp();
  return fm == 0;
}

// X L^T = B for one tile (B in x, overwritten); lane i owns row i.
// Right-looking: once x(i, m) is final it is applied to the later columns,
// whose multipliers L(m+1.., m) are contiguous in the column-major tile l and
// arrive as 16-byte broadcasts.  Blocks of CB columns with register rotation,
// as in factor_diag_tile.
template <typename T, int CB>
__device__ void trsm_tile(T* x, const T* l, const T* inv, int lane) {
  constexpr int V = 16 / sizeof(T);
  T b[TS];
#pragma unroll
  for (int m = 0; m < TS; ++m) b[m] = x[m * TS + lane];
#pragma unroll 1
  for (int m0 = 0; m0 < TS; m0 += CB) {
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      const int m = m0 + c;
      b[c] *= inv[m];
#pragma unroll
      for (int q = (c + 1) / V; q < TS / V; ++q) {
        if (m0 + V * q < TS) {
          T lv[V];
          load_vec16(l + m * TS + m0 + V * q, lv);
#pragma unroll
          for (int e = 0; e < V; ++e)
            if (V * q + e > c) b[V * q + e] = fma(-b[c], lv[e], b[V * q + e]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CB; ++c) x[(m0 + c) * TS + lane] = b[c];
#pragma unroll
    for (int j = 0; j < TS - CB; ++j) b[j] = b[j + CB];
  }
}

// N contiguous elements of a shared tile (16-byte vectors, an 8-byte
// remainder; p aligned to the access size).
template <int N, typename T>
__device__ __forceinline__ void load_n(const T* p, T (&v)[N]) {
  constexpr int V = 16 / sizeof(T);
#pragma unroll
  for (int q = 0; q < N / V; ++q) {
    T w[V];
    load_vec16(p + V * q, w);
#pragma unroll
    for (int e = 0; e < V; ++e) v[V * q + e] = w[e];
  }
  if constexpr (N % V != 0) {
    static_assert(sizeof(T) == 4 && N % V == 2, "8-byte remainder of a float block");
    const float2 w = *reinterpret_cast<const float2*>(p + N - 2);
    v[N - 2] = w.x;
    v[N - 1] = w.y;
  }
}

// C(r0 .. r0+RR-1, c0 .. c0+CC-1) -= A B^T over the tiles' 32 k (32 x 32
// tiles, column-major).  The thread keeps its RR x CC block in registers and
// reads, per k, RR values of A's column and CC of B's as vectors, so a warp's
// shared-memory traffic per FMA is (RR + CC) / (RR CC) of a value (the
// return path of shared memory, not the FMA pipe, bounds these updates).
// Each output is the same fma chain in k order as a row-by-row update.
template <typename T, int RR, int CC>
__device__ __forceinline__ void syrk_block(T* c, const T* a, const T* b, int r0, int c0) {
  T acc[RR][CC];
#pragma unroll
  for (int j = 0; j < CC; ++j)
#pragma unroll
    for (int i = 0; i < RR; ++i) acc[i][j] = c[(c0 + j) * TS + r0 + i];
#pragma unroll 4
  for (int k = 0; k < TS; ++k) {
    T av[RR], bv[CC];
    load_n<RR>(a + k * TS + r0, av);
    load_n<CC>(b + k * TS + c0, bv);
#pragma unroll
    for (int i = 0; i < RR; ++i)
#pragma unroll
      for (int j = 0; j < CC; ++j) acc[i][j] = fma(-av[i], bv[j], acc[i][j]);
  }
#pragma unroll
  for (int j = 0; j < CC; ++j)
#pragma unroll
    for (int i = 0; i < RR; ++i) c[(c0 + j) * TS + r0 + i] = acc[i][j];
}

// A whole 32 x 32 tile C -= A B^T by one warp: lane (rg, cg) = (lane % 4,
// lane / 4) owns rows 8 rg .. and columns 4 cg .. (a quarter-warp reads four
// distinct 32-byte row groups and two column groups: no bank conflict).
template <typename T>
__device__ __forceinline__ void syrk_tile(T* c, const T* a, const T* b, int lane) {
  syrk_block<T, 8, 4>(c, a, b, 8 * (lane & 3), 4 * (lane >> 2));
}

// Inverse of the lower-triangular tile l into out (32 x 32 column-major,
// FP32).  Lane j solves L w = e_j for column j of L^-1, right-looking with the
// column held in registers; the column of L used at each step arrives as
// 16-byte broadcasts.  Blocks of CB steps with register rotation, as in
// factor_diag_tile; each block's finished entries go out as 16-byte vectors.
template <typename T, int CB>
__device__ void invert_tile(const T* l, const T* inv, float* out, int lane) {
  constexpr int V = 16 / sizeof(T);
  T w[TS];
#pragma unroll
  for (int i = 0; i < TS; ++i) w[i] = (i == lane) ? T(1) : T(0);
#pragma unroll 1
  for (int k0 = 0; k0 < TS; k0 += CB) {
#pragma unroll
    for (int c = 0; c < CB; ++c) {
      const int k = k0 + c;
      w[c] *= inv[k];
#pragma unroll
      for (int q = (c + 1) / V; q < TS / V; ++q) {
        if (k0 + V * q < TS) {
          T lv[V];
          load_vec16(l + k * TS + k0 + V * q, lv);
#pragma unroll
          for (int e = 0; e < V; ++e)
            if (V * q + e > c) w[V * q + e] = fma(-lv[e], w[c], w[V * q + e]);
        }
      }
    }
    // the finished entries k0 .. k0 + CB - 1 of column lane
    float4* o = reinterpret_cast<float4*>(out + lane * TS + k0);
#pragma unroll
    for (int q = 0; q < CB / 4; ++q)
      o[q] = make_float4((float)w[4 * q], (float)w[4 * q + 1], (float)w[4 * q + 2], (float)w[4 * q + 3]);
#pragma unroll
    for (int j = 0; j < TS - CB; ++j) w[j] = w[j + CB];
  }
}

template <typename T, bool TMA, int CB>
__device__ void potrf_block(const CUtensorMap* tmap, T* tiles, float* A, int lda, int n, int s,
                            int bs, const float* d, float* sh, const PotrfParams& p,
                            float* winv, DevStatus* st, const StepState* prev = nullptr,
                            const float* rowsq = nullptr) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int NT = (bs + TS - 1) / TS;
  const int ntiles = NT * (NT + 1) / 2;
  __shared__ T s_shift[256];
  __shared__ T s_pmin[256];
  __shared__ T s_inv[256];
  __shared__ __align__(16) T s_col[2 * TS];
  __shared__ int s_fail, s_pert, s_ok;
  __shared__ __align__(8) uint64_t bar;
  if (tid == 0) { s_fail = -1; s_pert = 0; s_ok = 1; }
  const int prev_prec = (prev != nullptr && p.diag_pert && sh) ? prev->prec : FP32;
  for (int i = tid; i < NT * TS; i += blockDim.x) {
    T shv = T(0), pm = T(0);
    if (i < bs) {
      if (p.diag_pert && sh) {
        float shf = sh[s + i];
        if (prev_prec != FP32) {   // the previous step's shift for this row
          shf = __fmaf_rn(unit_roundoff(prev_prec), rowsq[s + i], shf);
          sh[s + i] = shf;
        }
        shv = T(p.pert) * T(shf);
      }
      pm = T(p.pivot_floor) * T(d[s + i]);
    }
    s_shift[i] = shv;
    s_pmin[i] = pm;
  }
  if (TMA) {
    // stage the lower tiles with TMA (the lanes of warp 0 issue the copies);
    // rows/columns past n arrive as zeros
    if (warp == 0) {
      if (lane == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
        tc::mbar_expect_tx(&bar, (uint32_t)(ntiles * TSZ * sizeof(float)));
      }
      __syncwarp();
      for (int t = lane; t < ntiles; t += 32) {
        int I = 0;
        while ((I + 1) * (I + 2) / 2 <= t) ++I;
        const int J = t - I * (I + 1) / 2;
        tc::tma_load_2d(tiles + t * TSZ, tmap, &bar, s + I * TS, s + J * TS);
      }
      if (lane == 0 && !tc::mbar_wait(&bar, 0)) {
        s_ok = 0;
        set_status(st, MPCHOL_ERR_TIMEOUT, s);
        tc::mbar_wait(&bar, 0);
      }
    }
    __syncthreads();
    if (!s_ok) return;
    // identity padding past the block (only the last block can be partial)
    for (int i = bs + tid; i < NT * TS; i += blockDim.x)
      tiles[tidx(i / TS, i / TS) * TSZ + (i % TS) * TS + (i % TS)] = T(1);
  } else {
    // FP64 path: batched loads from the FP32 matrix
    const int total = NT * NT * TSZ;
    for (int base = 0; base < total; base += 8 * blockDim.x) {
      float v[8];
      int dst[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int e = base + q * blockDim.x + tid;
        dst[q] = -1;
        v[q] = 0.0f;
        if (e < total) {
          const int T2 = e / TSZ, rc = e % TSZ;
          const int I = T2 % NT, J = T2 / NT, c = rc / TS, r = rc % TS;
          if (I >= J) {
            const int gr = I * TS + r, gc = J * TS + c;
            dst[q] = tidx(I, J) * TSZ + c * TS + r;
            if (gr < bs && gc < bs) v[q] = A[(size_t)(s + gc) * lda + (s + gr)];
            else v[q] = (gr == gc) ? 1.0f : 0.0f;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (dst[q] >= 0) tiles[dst[q]] = T(v[q]);
    }
  }
  __syncthreads();
  // Step J: (A) the tiles below diagonal tile J are solved, one per warp;
  // (B) warps 0-3 apply column J to diagonal tile J+1 (8 columns each, one
  // warp per SM sub-partition) and warp 0 factors it at once, while warps
  // 1.. update the other trailing tiles, one tile per warp with 2-D register
  // blocks.  The factor of the next diagonal tile thus overlaps the trailing
  // update (look-ahead).
  auto factor_tile = [&](int J) {
    int nreal = bs - J * TS;
    nreal = nreal > TS ? TS : nreal;
    int fail = -1, npert = 0;
    const bool ok = factor_diag_tile<T, CB>(tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane, nreal,
                                        s_shift + J * TS, s_pmin + J * TS, p.diag_pert, &npert,
                                        &fail, s_col);
    if (lane == 0) {
      if (!ok) s_fail = J * TS + fail;
      s_pert += npert;
    }
  };
  // J = -1 factors diagonal tile 0 alone; the factor has one call site, so
  // its code is in the kernel once.  Warp 0 carries the chain (the solve of
  // tile (J+1, J) and the factor of diagonal tile J+1) and has its SM
  // sub-partition to itself: the other warps of that sub-partition (warp %
  // 4 == 0) stay idle, and the helper warps (warp % 4 != 0) take the other
  // tile solves and the trailing updates.
  const int helper = (warp & 3) ? warp - (warp >> 2) - 1 : -1;
  const int nhelp = nwarps - nwarps / 4;
  for (int J = -1; J < NT - 1; ++J) {
    if (J >= 0) {
      if (s_fail >= 0) break;
      // warp 0 solves tile (J+1, J), the one the next diagonal tile waits
      // on; the helpers take the others
      if (warp == 0 && J + 1 < NT)
        trsm_tile<T, CB>(tiles + tidx(J + 1, J) * TSZ, tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane);
      if (helper >= 0)
        for (int I = J + 2 + helper; I < NT; I += nhelp)
          trsm_tile<T, CB>(tiles + tidx(I, J) * TSZ, tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane);
      __syncthreads();
    }
    if (warp < 4) {
      if (J >= 0) {
        // columns 8 warp .. +7 of diagonal tile J+1: lane (rg, cg) = (lane %
        // 8, lane / 8) owns rows 4 rg .. and columns 8 warp + 2 cg ..
        T* dt = tiles + tidx(J + 1, J + 1) * TSZ;
        const T* pj = tiles + tidx(J + 1, J) * TSZ;
        syrk_block<T, 4, 2>(dt, pj, pj, 4 * (lane & 7), 8 * warp + 2 * (lane >> 3));
        asm volatile("bar.sync 1, 128;" ::: "memory");   // warps 0-3
      }
      if (warp == 0) factor_tile(J + 1);
    }
    if (J >= 0 && helper >= 0) {
      // work items: the trailing tiles (I, K), J < K <= I, diagonal tile J+1
      // excluded, numbered down each tile column; one helper warp per tile
      int item = 0;
      for (int K = J + 1; K < NT; ++K) {
        const int i0 = (K == J + 1) ? K + 1 : K;
        for (int I = i0; I < NT; ++I, ++item) {
          if (item % nhelp != helper) continue;
          syrk_tile<T>(tiles + tidx(I, K) * TSZ, tiles + tidx(I, J) * TSZ,
                       tiles + tidx(K, J) * TSZ, lane);
        }
      }
    }
    __syncthreads();
  }
  if (s_fail >= 0) {
    if (tid == 0) set_status(st, MPCHOL_ERR_NOT_SPD, s + s_fail);
    return;
  }
  // write back: TMA stores of the lower tiles (FP32 path), or a coalesced loop
  // that rounds the FP64 tiles to FP32.  The strictly upper part of a
  // diagonal tile is written back as it was staged; it is never read as data.
  if (TMA) {
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (warp == 0) {   // the lanes of warp 0 issue the stores
      for (int t = lane; t < ntiles; t += 32) {
        int I = 0;
        while ((I + 1) * (I + 2) / 2 <= t) ++I;
        const int J = t - I * (I + 1) / 2;
        tc::tma_store_2d(tmap, tiles + t * TSZ, s + I * TS, s + J * TS);
      }
      tc::bulk_commit();
    }
  } else {
    for (int c = warp; c < bs; c += nwarps) {
      const int J = c / TS, cc = c % TS;
      for (int r = c + lane; r < bs; r += TS) {
        const int I = r / TS, rr = r % TS;
        A[(size_t)(s + c) * lda + (s + r)] = (float)tiles[tidx(I, J) * TSZ + cc * TS + rr];
      }
    }
  }
  // inverses of the diagonal tiles, used by the panel solve
  for (int J = warp; J < NT; J += nwarps)
    invert_tile<T, CB>(tiles + tidx(J, J) * TSZ, s_inv + J * TS, winv + J * TS * TS, lane);
  if (tid == 0 && s_pert) atomicAdd(&st->perturbed, s_pert);
  if (TMA && warp == 0) tc::bulk_wait_read();   // smem must outlive the stores' reads
  (void)n;
}

// FP32 blocks: tiles in shared memory, staged by TMA.  Separate kernels for
// the two precisions keep the FP64 register footprint out of the FP32 path.
// CB = TS unrolls the tile loops fully (fastest on its own); CB = 4 keeps the
// kernel's code about a quarter of that size, so it stays cache-resident and
// fast while a trailing update saturates L2 beside it.
template <int CB>
__global__ void __launch_bounds__(512, 1)
potrf_f32_kernel(const __grid_constant__ CUtensorMap tmap, float* A, int lda, int n, int s, int bs,
                 const float* d, float* sh, PotrfParams p, const int* fp64_flag, float* winv,
                 DevStatus* st, const StepState* prev, const float* rowsq) {
  tc::grid_dep_wait();      // the block's update and the step state are final
  tc::grid_dep_trigger();   // the next kernel may be scheduled (it waits too)
  if (st->code != 0) return;
  if (fp64_flag != nullptr && *fp64_flag != 0) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  potrf_block<float, true, CB>(&tmap, reinterpret_cast<float*>(smem_raw), A, lda, n, s, bs, d, sh, p,
                           winv, st, prev, rowsq);
}

// Batched: CTA i factors the current diagonal block of system i (tiles in
// shared memory, staged with plain coalesced loads: one tensor map per
// system would not fit the launch).
__global__ void __launch_bounds__(512, 1)
potrf_batched_kernel(BatchSys* __restrict__ sys, int s, int b, PotrfParams p) {
  const BatchSys& S = sys[blockIdx.x];
  const int bs = min(b, S.n - s);
  if (bs <= 0 || S.st->code != 0) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  potrf_block<float, false, TS>(nullptr, reinterpret_cast<float*>(smem_raw), S.A, S.ld, S.n, s, bs,
                            S.d, S.sh, p, S.winv, S.st);
}

// FP64 blocks (flagged near-indefinite): tiles in a global scratch.
__global__ void __launch_bounds__(256, 1)
potrf_f64_kernel(float* A, int lda, int n, int s, int bs, const float* d, float* sh,
                 PotrfParams p, const int* fp64_flag, double* scratch64, float* winv, DevStatus* st,
                 const StepState* prev, const float* rowsq) {
  if (st->code != 0) return;
  if (fp64_flag == nullptr || *fp64_flag == 0) return;
  potrf_block<double, false, 8>(nullptr, scratch64, A, lda, n, s, bs, d, sh, p, winv, st, prev, rowsq);
}

}  // namespace

// the lower tiles of the block
size_t potrf_scratch64_elems(int bs) {
  const int NT = (bs + TS - 1) / TS;
  return (size_t)NT * (NT + 1) / 2 * TSZ;
}
size_t potrf_smem_bytes(int bs) { return potrf_scratch64_elems(bs) * sizeof(float); }

cudaError_t launch_potrf(const CUtensorMap& tmap32, float* A, int lda, int n, int s, int bs,
                         const float* d, float* sh, const PotrfParams& p,
                         const int* fp64_flag, double* scratch64, float* winv, DevStatus* st,
                         bool may_fp64, cudaStream_t stream, const StepState* prev,
                         const float* rowsq, bool compact) {
  const size_t smem = potrf_smem_bytes(256);
  cudaError_t e = cudaFuncSetAttribute(potrf_f32_kernel<4>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(potrf_f32_kernel<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
  if (e != cudaSuccess) return e;
  PdlLaunch L(dim3(1), dim3(512), smem, stream);
  const int* flag = may_fp64 ? fp64_flag : nullptr;
  e = compact ? cudaLaunchKernelEx(&L.cfg, potrf_f32_kernel<4>, tmap32, A, lda, n, s, bs, d, sh, p,
                                   flag, winv, st, prev, rowsq)
              : cudaLaunchKernelEx(&L.cfg, potrf_f32_kernel<TS>, tmap32, A, lda, n, s, bs, d, sh, p,
                                   flag, winv, st, prev, rowsq);
  if (e != cudaSuccess) return e;
  if (may_fp64)
    potrf_f64_kernel<<<1, 256, 0, stream>>>(A, lda, n, s, bs, d, sh, p, fp64_flag, scratch64, winv, st,
                                            prev, rowsq);
  return cudaGetLastError();
}

cudaError_t launch_potrf_batched(BatchSys* sys, int nact, int s, int b, const PotrfParams& p,
                                 cudaStream_t stream) {
  if (nact <= 0) return cudaSuccess;
  const size_t smem = potrf_smem_bytes(b);
  cudaError_t e = cudaFuncSetAttribute(potrf_batched_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  potrf_batched_kernel<<<nact, 512, smem, stream>>>(sys, s, b, p);
  return cudaGetLastError();
}

}  // namespace mpchol
