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
// Lane i holds row i of the tile in registers for the whole factorization (the
// column loop is unrolled so every register index is a constant): per column
// lane k's pivot is repaired, one shuffle broadcasts 1/sqrt(pivot),
// and the rank-1 update reads the column's multipliers from the 32-entry
// shared buffer col as 16-byte broadcasts.  The tile itself is read once and
// its lower triangle written once.
template <typename T>
__device__ bool factor_diag_tile(T* t, T* inv, int lane, int nreal, const T* shift, const T* pmin,
                                 int diag_pert, int* nperturbed, int* fail_row, T* col) {
  T a[TS];
#pragma unroll
  for (int j = 0; j < TS; ++j) a[j] = t[j * TS + lane];
  const T my_shift = (lane < nreal) ? shift[lane] : T(0);
  const T my_pmin = pmin[lane];
  bool failed = false, perturbed = false;
  T my_inv = T(1);
  // The pivot of column k + 1 is lane k + 1's candidate a[k+1] - L(k+1,k)^2
  // (the same fma the rank-1 update applies to a[k+1]); it is evaluated,
  // square-rooted and broadcast before column k's multipliers go through
  // shared memory, so the pivot chain and the update's round trip overlap.
  Pivot<T> pv = eval_pivot<T>(a[0], 0 < nreal, my_shift, my_pmin, diag_pert);
  T rk = __shfl_sync(0xffffffffu, pv.r, 0);
#pragma unroll
  for (int k = 0; k < TS; ++k) {
    const bool mine = lane == k;
    perturbed = perturbed || (mine && pv.pert);
    failed = failed || (mine && pv.bad);
    my_inv = mine ? pv.r : my_inv;
    const T lik = (lane > k) ? a[k] * rk : T(0);
    a[k] = mine ? pv.piv * pv.r : ((lane > k) ? lik : a[k]);
    if (k + 1 < TS) {
      pv = eval_pivot<T>(fma(-lik, lik, a[k + 1]), k + 1 < nreal, my_shift, my_pmin, diag_pert);
      rk = __shfl_sync(0xffffffffu, pv.r, k + 1);
    }
    // two multiplier buffers used in turn: the next column's write cannot
    // overtake a lane still reading this one, so one warp barrier suffices
    T* cb = col + (k & 1) * TS;
    cb[lane] = lik;
    __syncwarp();
    constexpr int V = 16 / sizeof(T);
#pragma unroll
    for (int q = 0; q < TS / V; ++q) {
      if (V * q + V - 1 <= k) continue;
      T l[V];
      load_vec16(cb + V * q, l);
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const int j = V * q + e;
        if (j > k) a[j] = fma(-lik, l[e], a[j]);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < TS; ++j)
    if (j <= lane) t[j * TS + lane] = a[j];
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
// arrive as 16-byte broadcasts.
template <typename T>
__device__ void trsm_tile(T* x, const T* l, const T* inv, int lane) {
  constexpr int V = 16 / sizeof(T);
  T b[TS];
#pragma unroll
  for (int m = 0; m < TS; ++m) b[m] = x[m * TS + lane];
#pragma unroll
  for (int m = 0; m < TS; ++m) {
    b[m] *= inv[m];
#pragma unroll
    for (int q = (m + 1) / V; q < TS / V; ++q) {
      T lv[V];
      load_vec16(l + m * TS + V * q, lv);
#pragma unroll
      for (int e = 0; e < V; ++e)
        if (V * q + e > m) b[V * q + e] = fma(-b[m], lv[e], b[V * q + e]);
    }
  }
#pragma unroll
  for (int m = 0; m < TS; ++m) x[m * TS + lane] = b[m];
}

// Columns c0..c0+7 of C -= A B^T for 32 x 32 tiles; lane i owns row i of C
// and holds row i of A in ar.  B's column values arrive as 16-byte
// broadcasts; with TWO, a second tile of the same tile column
// (C2 -= A2 B^T, A2's row in ar2) shares every broadcast.
template <typename T, bool TWO>
__device__ __forceinline__ void syrk_cols8(T* c, T* c2, const T (&ar)[TS], const T (&ar2)[TS],
                                           const T* b, int lane, int c0) {
  constexpr int V = 16 / sizeof(T);
  T acc[8], acc2[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    acc[u] = c[(c0 + u) * TS + lane];
    acc2[u] = TWO ? c2[(c0 + u) * TS + lane] : T(0);
  }
#pragma unroll
  for (int m = 0; m < TS; ++m) {
#pragma unroll
    for (int q = 0; q < 8 / V; ++q) {
      T bv[V];
      load_vec16(b + m * TS + c0 + V * q, bv);
#pragma unroll
      for (int e = 0; e < V; ++e) {
        acc[V * q + e] = fma(-ar[m], bv[e], acc[V * q + e]);
        if (TWO) acc2[V * q + e] = fma(-ar2[m], bv[e], acc2[V * q + e]);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    c[(c0 + u) * TS + lane] = acc[u];
    if (TWO) c2[(c0 + u) * TS + lane] = acc2[u];
  }
}

// C -= A B^T over columns [c_begin, c_end) (multiples of 8), and C2 -= A2 B^T
// over the same columns when c2 is set.
template <typename T>
__device__ void syrk_tiles(T* c, const T* a, T* c2, const T* a2, const T* b, int lane,
                           int c_begin = 0, int c_end = TS) {
  T ar[TS], ar2[TS];
#pragma unroll
  for (int m = 0; m < TS; ++m) ar[m] = a[m * TS + lane];
  if (c2 != nullptr) {
#pragma unroll
    for (int m = 0; m < TS; ++m) ar2[m] = a2[m * TS + lane];
#pragma unroll 1
    for (int c0 = c_begin; c0 < c_end; c0 += 8) syrk_cols8<T, true>(c, c2, ar, ar2, b, lane, c0);
  } else {
#pragma unroll 1
    for (int c0 = c_begin; c0 < c_end; c0 += 8) syrk_cols8<T, false>(c, nullptr, ar, ar, b, lane, c0);
  }
}

// Inverse of the lower-triangular tile l into out (32 x 32 column-major,
// FP32).  Lane j solves L w = e_j for column j of L^-1, right-looking with the
// column held in registers; the column of L used at each step is a shared
// broadcast.  Each lane then stores its column as 16-byte vectors.
template <typename T>
__device__ void invert_tile(const T* l, const T* inv, float* out, int lane) {
  T w[TS];
#pragma unroll
  for (int i = 0; i < TS; ++i) w[i] = (i == lane) ? T(1) : T(0);
#pragma unroll
  for (int k = 0; k < TS; ++k) {
    w[k] *= inv[k];
#pragma unroll
    for (int i = k + 1; i < TS; ++i) w[i] -= l[k * TS + i] * w[k];
  }
  float4* o = reinterpret_cast<float4*>(out + lane * TS);
#pragma unroll
  for (int q = 0; q < TS / 4; ++q)
    o[q] = make_float4((float)w[4 * q], (float)w[4 * q + 1], (float)w[4 * q + 2], (float)w[4 * q + 3]);
}

template <typename T, bool TMA>
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
  // 1.. update the other trailing tiles, two tiles of a tile column at a time
  // so that each broadcast of column J's values feeds both.  The factor of
  // the next diagonal tile thus overlaps the trailing update (look-ahead).
  auto factor_tile = [&](int J) {
    int nreal = bs - J * TS;
    nreal = nreal > TS ? TS : nreal;
    int fail = -1, npert = 0;
    const bool ok = factor_diag_tile<T>(tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane, nreal,
                                        s_shift + J * TS, s_pmin + J * TS, p.diag_pert, &npert,
                                        &fail, s_col);
    if (lane == 0) {
      if (!ok) s_fail = J * TS + fail;
      s_pert += npert;
    }
  };
  if (warp == 0) factor_tile(0);
  __syncthreads();
  for (int J = 0; J < NT; ++J) {
    if (s_fail >= 0) break;
    for (int I = J + 1 + warp; I < NT; I += nwarps)
      trsm_tile<T>(tiles + tidx(I, J) * TSZ, tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane);
    __syncthreads();
    if (J + 1 < NT) {
      if (warp < 4) {
        T* dt = tiles + tidx(J + 1, J + 1) * TSZ;
        const T* pj = tiles + tidx(J + 1, J) * TSZ;
        syrk_tiles<T>(dt, pj, nullptr, nullptr, pj, lane, 8 * warp, 8 * warp + 8);
        asm volatile("bar.sync 1, 128;" ::: "memory");   // warps 0-3
        if (warp == 0) factor_tile(J + 1);
      }
      if (warp >= 1) {
        // work items: pairs of vertically adjacent tiles (I, K), (I+1, K) of
        // each trailing tile column K, J < K <= I, diagonal tile J+1 excluded
        int item = 0;
        for (int K = J + 1; K < NT; ++K) {
          const int i0 = (K == J + 1) ? K + 1 : K;
          for (int I = i0; I < NT; I += 2, ++item) {
            if (item % (nwarps - 1) != warp - 1) continue;
            const bool two = I + 1 < NT;
            syrk_tiles<T>(tiles + tidx(I, K) * TSZ, tiles + tidx(I, J) * TSZ,
                          two ? tiles + tidx(I + 1, K) * TSZ : nullptr,
                          two ? tiles + tidx(I + 1, J) * TSZ : nullptr,
                          tiles + tidx(K, J) * TSZ, lane);
          }
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
    invert_tile<T>(tiles + tidx(J, J) * TSZ, s_inv + J * TS, winv + J * TS * TS, lane);
  if (tid == 0 && s_pert) atomicAdd(&st->perturbed, s_pert);
  if (TMA && warp == 0) tc::bulk_wait_read();   // smem must outlive the stores' reads
  (void)n;
}

// FP32 blocks: tiles in shared memory, staged by TMA.  Separate kernels for
// the two precisions keep the FP64 register footprint out of the FP32 path.
__global__ void __launch_bounds__(512, 1)
potrf_f32_kernel(const __grid_constant__ CUtensorMap tmap, float* A, int lda, int n, int s, int bs,
                 const float* d, float* sh, PotrfParams p, const int* fp64_flag, float* winv,
                 DevStatus* st, const StepState* prev, const float* rowsq) {
  if (st->code != 0) return;
  if (fp64_flag != nullptr && *fp64_flag != 0) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  potrf_block<float, true>(&tmap, reinterpret_cast<float*>(smem_raw), A, lda, n, s, bs, d, sh, p,
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
  potrf_block<float, false>(nullptr, reinterpret_cast<float*>(smem_raw), S.A, S.ld, S.n, s, bs,
                            S.d, S.sh, p, S.winv, S.st);
}

// FP64 blocks (flagged near-indefinite): tiles in a global scratch.
__global__ void __launch_bounds__(256, 1)
potrf_f64_kernel(float* A, int lda, int n, int s, int bs, const float* d, float* sh,
                 PotrfParams p, const int* fp64_flag, double* scratch64, float* winv, DevStatus* st,
                 const StepState* prev, const float* rowsq) {
  if (st->code != 0) return;
  if (fp64_flag == nullptr || *fp64_flag == 0) return;
  potrf_block<double, false>(nullptr, scratch64, A, lda, n, s, bs, d, sh, p, winv, st, prev, rowsq);
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
                         const float* rowsq) {
  const size_t smem = potrf_smem_bytes(256);
  cudaError_t e = cudaFuncSetAttribute(potrf_f32_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  potrf_f32_kernel<<<1, 512, smem, stream>>>(tmap32, A, lda, n, s, bs, d, sh, p,
                                             may_fp64 ? fp64_flag : nullptr, winv, st, prev, rowsq);
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
