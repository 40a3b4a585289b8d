// Diagonal-block Cholesky (POTRF) for the blocked factorization.
//
// Replaces the reference's per-step cusolverDnSpotrf of the b x b diagonal
// block (src/switching_chol.cuh:86-95) and its CPU micro_cholesky variant
// (src/micro_chol.hpp:14-44, src/sChol.cuh:66-79).  One CTA factors a block of
// up to 256 x 256 as a blocked right-looking Cholesky on 32 x 32 tiles held in
// shared memory: one warp factors the diagonal tile (lane i owns row i), warps
// solve the tiles below it, warps update the trailing tiles.  Blocks flagged
// near-indefinite by the switching criterion are factored in FP64 in a global
// scratch (L2-resident) by a separate kernel.
//
// The per-tile routines are rolled loops over shared memory: the same few
// hundred instructions run for every step, so they stay in the instruction
// cache (fully unrolled 32 x 32 code runs once per tile and is bound by
// instruction fetch).
#include "common.cuh"
#include "kernels.cuh"

namespace mpchol {

namespace {

constexpr int TS = 32;        // tile size
constexpr int TLD = 33;       // padded tile column stride (bank-conflict free)
constexpr int TSZ = TS * TLD; // elements per tile

__device__ __forceinline__ int tidx(int I, int J) { return I * (I + 1) / 2 + J; }

template <typename T>
__device__ __forceinline__ T dsqrt(T x);
template <>
__device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <>
__device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }

// Factor the 32 x 32 tile t in place (lower triangle); lane i owns row i.
// inv[k] receives 1 / L(k,k).  Returns false on a non-positive pivot when
// pivot flooring is off (first failing local row in *fail_row).
template <typename T>
__device__ bool factor_diag_tile(T* t, T* inv, int lane, int nreal, const T* shift, const T* pmin,
                                 int diag_pert, int* nperturbed, int* fail_row) {
  bool ok = true;
  int npert = 0;
#pragma unroll 1
  for (int k = 0; k < TS; ++k) {
    T piv = t[k * TLD + k];
    if (k < nreal) {
      piv += shift[k];
      if (diag_pert) {
        if (!(piv > pmin[k])) { piv = pmin[k]; ++npert; }
      } else if (!(piv > T(0))) {
        if (ok) *fail_row = k;
        ok = false;
        piv = T(1);   // keep the arithmetic finite; the caller discards the result
      }
    } else {
      piv = T(1);     // identity padding beyond the real block
    }
    const T lkk = dsqrt<T>(piv);
    const T rk = T(1) / lkk;
    __syncwarp();
    if (lane == k) { t[k * TLD + k] = lkk; inv[k] = rk; }
    else if (lane > k) t[k * TLD + lane] *= rk;
    __syncwarp();
    if (lane > k) {
      const T lik = t[k * TLD + lane];
#pragma unroll 4
      for (int j = k + 1; j <= lane; ++j) t[j * TLD + lane] -= lik * t[k * TLD + j];
    }
    __syncwarp();
  }
  if (lane == 0) *nperturbed += npert;
  return ok;
}

// X L^T = B for one tile (B in x, overwritten); lane i owns row i.
template <typename T>
__device__ void trsm_tile(T* x, const T* l, const T* inv, int lane) {
#pragma unroll 1
  for (int j = 0; j < TS; ++j) {
    T acc = x[j * TLD + lane];
#pragma unroll 4
    for (int m = 0; m < j; ++m) acc -= x[m * TLD + lane] * l[m * TLD + j];
    x[j * TLD + lane] = acc * inv[j];
  }
}

// C -= A B^T for 32 x 32 tiles; lane c owns column c of C.
template <typename T>
__device__ void syrk_tile(T* c, const T* a, const T* b, int lane) {
  T acc[TS];
#pragma unroll
  for (int r = 0; r < TS; ++r) acc[r] = c[lane * TLD + r];
#pragma unroll 2
  for (int m = 0; m < TS; ++m) {
    const T bv = b[m * TLD + lane];
#pragma unroll
    for (int r = 0; r < TS; ++r) acc[r] -= a[m * TLD + r] * bv;
  }
#pragma unroll
  for (int r = 0; r < TS; ++r) c[lane * TLD + r] = acc[r];
}

// Inverse of the lower-triangular tile l: lane c forms column c of L^-1 in the
// scratch tile w (column-major, stride TLD) and stores it to out (32 x 32,
// column-major, FP32).
template <typename T>
__device__ void invert_tile(const T* l, const T* inv, T* w, float* out, int lane) {
#pragma unroll 1
  for (int i = 0; i < TS; ++i) {
    T v = T(0);
    if (i >= lane) {
      T acc = (i == lane) ? T(1) : T(0);
#pragma unroll 4
      for (int k = lane; k < i; ++k) acc -= l[k * TLD + i] * w[lane * TLD + k];
      v = acc * inv[i];
    }
    w[lane * TLD + i] = v;
  }
  __syncwarp();
#pragma unroll 1
  for (int i = 0; i < TS; ++i) out[i * TS + lane] = (float)w[i * TLD + lane];
}

template <typename T>
__device__ void potrf_block(T* tiles, float* A, int lda, int s, int bs, const float* d,
                            const float* sh, const PotrfParams& p, float* winv, DevStatus* st) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int NT = (bs + TS - 1) / TS;
  const int ntiles = NT * (NT + 1) / 2;
  T* scratch = tiles + ntiles * TSZ;       // NT tiles for the inverses
  __shared__ T s_shift[256];
  __shared__ T s_pmin[256];
  __shared__ T s_inv[256];
  __shared__ int s_fail, s_pert;
  if (tid == 0) { s_fail = -1; s_pert = 0; }
  for (int i = tid; i < NT * TS; i += blockDim.x) {
    T shv = T(0), pm = T(0);
    if (i < bs) {
      if (p.diag_pert && sh) shv = T(p.pert) * T(sh[s + i]);
      pm = T(p.pivot_floor) * T(d[s + i]);
    }
    s_shift[i] = shv;
    s_pmin[i] = pm;
  }
  // load the lower tiles column by column (coalesced); padding is identity
  for (int c = warp; c < NT * TS; c += nwarps) {
    const int J = c / TS, cc = c % TS;
#pragma unroll 8
    for (int r = J * TS + lane; r < NT * TS; r += TS) {
      const int I = r / TS, rr = r % TS;
      T v;
      if (r < bs && c < bs) v = T(A[(size_t)(s + c) * lda + (s + r)]);
      else v = (r == c) ? T(1) : T(0);
      tiles[tidx(I, J) * TSZ + cc * TLD + rr] = v;
    }
  }
  __syncthreads();
  for (int J = 0; J < NT; ++J) {
    if (warp == 0) {
      int nreal = bs - J * TS;
      nreal = nreal > TS ? TS : nreal;
      int fail = -1, npert = 0;
      bool ok = factor_diag_tile<T>(tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane, nreal,
                                    s_shift + J * TS, s_pmin + J * TS, p.diag_pert, &npert, &fail);
      if (lane == 0) {
        if (!ok) s_fail = J * TS + fail;
        s_pert += npert;
      }
    }
    __syncthreads();
    if (s_fail >= 0) break;
    for (int I = J + 1 + warp; I < NT; I += nwarps)
      trsm_tile<T>(tiles + tidx(I, J) * TSZ, tiles + tidx(J, J) * TSZ, s_inv + J * TS, lane);
    __syncthreads();
    // trailing tiles (I, K), J < K <= I < NT
    const int T_ = NT - J - 1;
    const int nupd = T_ * (T_ + 1) / 2;
    for (int u = warp; u < nupd; u += nwarps) {
      int i = 0;
      while ((i + 1) * (i + 2) / 2 <= u) ++i;
      const int k = u - i * (i + 1) / 2;
      const int I = J + 1 + i, K = J + 1 + k;
      syrk_tile<T>(tiles + tidx(I, K) * TSZ, tiles + tidx(I, J) * TSZ, tiles + tidx(K, J) * TSZ,
                   lane);
    }
    __syncthreads();
  }
  if (s_fail >= 0) {
    if (tid == 0) set_status(st, MPCHOL_ERR_NOT_SPD, s + s_fail);
    return;
  }
  // write back the lower triangle (rounded to FP32 for the FP64 path)
  for (int c = warp; c < bs; c += nwarps) {
    const int J = c / TS, cc = c % TS;
    for (int r = c + lane; r < bs; r += TS) {
      const int I = r / TS, rr = r % TS;
      A[(size_t)(s + c) * lda + (s + r)] = (float)tiles[tidx(I, J) * TSZ + cc * TLD + rr];
    }
  }
  // inverses of the diagonal tiles, used by the panel solve
  for (int J = warp; J < NT; J += nwarps)
    invert_tile<T>(tiles + tidx(J, J) * TSZ, s_inv + J * TS, scratch + J * TSZ,
                   winv + J * TS * TS, lane);
  if (tid == 0 && s_pert) atomicAdd(&st->perturbed, s_pert);
}

// FP32 blocks: tiles in shared memory.  Separate kernels for the two
// precisions keep the FP64 register footprint out of the FP32 path.
__global__ void __launch_bounds__(512, 1)
potrf_f32_kernel(float* A, int lda, int s, int bs, const float* d, const float* sh, PotrfParams p,
                 const int* fp64_flag, float* winv, DevStatus* st) {
  if (st->code != 0) return;
  if (fp64_flag != nullptr && *fp64_flag != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  potrf_block<float>(reinterpret_cast<float*>(smem_raw), A, lda, s, bs, d, sh, p, winv, st);
}

// FP64 blocks (flagged near-indefinite): tiles in a global scratch.
__global__ void __launch_bounds__(256, 1)
potrf_f64_kernel(float* A, int lda, int s, int bs, const float* d, const float* sh, PotrfParams p,
                 const int* fp64_flag, double* scratch64, float* winv, DevStatus* st) {
  if (st->code != 0) return;
  if (fp64_flag == nullptr || *fp64_flag == 0) return;
  potrf_block<double>(scratch64, A, lda, s, bs, d, sh, p, winv, st);
}

}  // namespace

size_t potrf_smem_bytes(int bs) {
  const int NT = (bs + TS - 1) / TS;
  return ((size_t)NT * (NT + 1) / 2 + NT) * TSZ * sizeof(float);
}
size_t potrf_scratch64_elems(int bs) {
  const int NT = (bs + TS - 1) / TS;
  return ((size_t)NT * (NT + 1) / 2 + NT) * TSZ;
}

cudaError_t launch_potrf(float* A, int lda, int s, int bs, const float* d, const float* sh,
                         const PotrfParams& p, const int* fp64_flag, double* scratch64,
                         float* winv, DevStatus* st, bool may_fp64, cudaStream_t stream) {
  const size_t smem = potrf_smem_bytes(256);
  cudaError_t e = cudaFuncSetAttribute(potrf_f32_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  potrf_f32_kernel<<<1, 512, smem, stream>>>(A, lda, s, bs, d, sh, p, fp64_flag, winv, st);
  if (may_fp64)
    potrf_f64_kernel<<<1, 256, 0, stream>>>(A, lda, s, bs, d, sh, p, fp64_flag, scratch64, winv, st);
  return cudaGetLastError();
}

}  // namespace mpchol
