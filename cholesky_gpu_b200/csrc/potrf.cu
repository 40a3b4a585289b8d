// Diagonal-block Cholesky (POTRF) for the blocked factorization.
//
// Replaces the reference's per-step cusolverDnSpotrf of the b x b diagonal
// block (src/switching_chol.cuh:86-95) and its CPU micro_cholesky variant
// (src/micro_chol.hpp:14-44, src/sChol.cuh:66-79).  One CTA
// factors a block of up to 256 x 256 as a blocked right-looking Cholesky on
// 32 x 32 tiles (16 warps): one warp factors the diagonal tile in registers, warps solve
// the tiles below it, warps update the trailing tiles.  FP32 blocks live in
// shared memory; blocks flagged near-indefinite by the switching criterion are
// factored in FP64 in a global scratch (L2-resident) instead.
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

// Factor tile (J,J) in registers: lane i holds row i.  Returns false (and
// records the failing local row in *fail_row) on a non-positive pivot when
// pivot flooring is off.
template <typename T>
__device__ bool factor_diag_tile(T* tile, int lane, int nreal, const T* shift, const T* pmin,
                                 int diag_pert, int* nperturbed, int* fail_row) {
  T a[TS];
#pragma unroll
  for (int j = 0; j < TS; ++j) a[j] = tile[j * TLD + lane];
  bool ok = true;
#pragma unroll
  for (int k = 0; k < TS; ++k) {
    T piv = __shfl_sync(0xffffffffu, a[k], k);
    if (k < nreal) {
      piv += shift[k];
      if (diag_pert) {
        if (!(piv > pmin[k])) {
          piv = pmin[k];
          if (lane == 0) ++*nperturbed;
        }
      } else if (!(piv > T(0))) {
        if (lane == 0 && ok) *fail_row = k;
        ok = false;
        piv = T(1);   // keep the arithmetic finite; the caller discards the result
      }
    } else {
      piv = T(1);     // identity padding beyond the real block
    }
    const T lkk = dsqrt<T>(piv);
    if (lane == k) a[k] = lkk;
    else if (lane > k) a[k] = a[k] / lkk;
#pragma unroll
    for (int j = k + 1; j < TS; ++j) {
      const T ljk = __shfl_sync(0xffffffffu, a[k], j);
      if (lane >= j) a[j] -= a[k] * ljk;
    }
  }
#pragma unroll
  for (int j = 0; j < TS; ++j) tile[j * TLD + lane] = a[j];
  return ok;
}

// X * Ljj^T = B for one 32 x 32 tile; lane i holds row i.
template <typename T>
__device__ void trsm_tile(T* tile, const T* ljj, int lane) {
  T x[TS];
#pragma unroll
  for (int j = 0; j < TS; ++j) x[j] = tile[j * TLD + lane];
#pragma unroll
  for (int j = 0; j < TS; ++j) {
    T acc = x[j];
#pragma unroll
    for (int m = 0; m < j; ++m) acc -= x[m] * ljj[m * TLD + j];
    x[j] = acc / ljj[j * TLD + j];
  }
#pragma unroll
  for (int j = 0; j < TS; ++j) tile[j * TLD + lane] = x[j];
}

// C -= A * B^T for 32 x 32 tiles; lane c holds column c of C.
template <typename T>
__device__ void syrk_tile(T* c, const T* a, const T* b, int lane) {
  T acc[TS];
#pragma unroll
  for (int r = 0; r < TS; ++r) acc[r] = c[lane * TLD + r];
#pragma unroll 4
  for (int m = 0; m < TS; ++m) {
    const T bv = b[m * TLD + lane];
#pragma unroll
    for (int r = 0; r < TS; ++r) acc[r] -= a[m * TLD + r] * bv;
  }
#pragma unroll
  for (int r = 0; r < TS; ++r) c[lane * TLD + r] = acc[r];
}

// Inverse of a lower-triangular 32 x 32 tile: lane c forms column c of L^-1
// by forward substitution and stores it column-major (32 x 32) to out.
template <typename T>
__device__ void invert_tile(const T* l, float* out, int lane) {
  T w[TS];
#pragma unroll
  for (int i = 0; i < TS; ++i) {
    T acc = (i == lane) ? T(1) : T(0);
#pragma unroll
    for (int k = 0; k < i; ++k) acc -= l[k * TLD + i] * w[k];
    w[i] = (i >= lane) ? acc / l[i * TLD + i] : T(0);
  }
#pragma unroll
  for (int i = 0; i < TS; ++i) out[lane * TS + i] = (float)w[i];
}

template <typename T>
__device__ void potrf_block(T* tiles, float* A, int lda, int s, int bs, const float* d,
                            const float* sh, const PotrfParams& p, float* winv, DevStatus* st) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int NT = (bs + TS - 1) / TS;
  __shared__ T s_shift[256];
  __shared__ T s_pmin[256];
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
  // load lower tiles; padding is identity
  const int ntiles = NT * (NT + 1) / 2;
  for (int e = tid; e < ntiles * TS * TS; e += blockDim.x) {
    const int t = e / (TS * TS), rc = e % (TS * TS);
    const int c = rc / TS, r = rc % TS;
    int I = 0;
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    const int J = t - I * (I + 1) / 2;
    const int gi = I * TS + r, gj = J * TS + c;
    T v;
    if (gi < bs && gj < bs) v = T(A[(size_t)(s + gj) * lda + (s + gi)]);
    else v = (gi == gj) ? T(1) : T(0);
    tiles[t * TSZ + c * TLD + r] = v;
  }
  __syncthreads();
  for (int J = 0; J < NT; ++J) {
    if (warp == 0) {
      int nreal = bs - J * TS; nreal = nreal > TS ? TS : nreal;
      int fail = -1, npert = 0;
      bool ok = factor_diag_tile<T>(tiles + tidx(J, J) * TSZ, lane, nreal, s_shift + J * TS,
                                    s_pmin + J * TS, p.diag_pert, &npert, &fail);
      if (lane == 0) {
        if (!ok) s_fail = J * TS + fail;
        s_pert += npert;
      }
    }
    __syncthreads();
    if (s_fail >= 0) break;
    for (int I = J + 1 + warp; I < NT; I += nwarps)
      trsm_tile<T>(tiles + tidx(I, J) * TSZ, tiles + tidx(J, J) * TSZ, lane);
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
  for (int e = tid; e < ntiles * TS * TS; e += blockDim.x) {
    const int t = e / (TS * TS), rc = e % (TS * TS);
    const int c = rc / TS, r = rc % TS;
    int I = 0;
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    const int J = t - I * (I + 1) / 2;
    const int gi = I * TS + r, gj = J * TS + c;
    if (gi < bs && gj < bs && gi >= gj)
      A[(size_t)(s + gj) * lda + (s + gi)] = (float)tiles[t * TSZ + c * TLD + r];
  }
  // inverses of the diagonal tiles, used by the panel solve
  for (int J = warp; J < NT; J += nwarps) invert_tile<T>(tiles + tidx(J, J) * TSZ, winv + J * TS * TS, lane);
  if (tid == 0 && s_pert) atomicAdd(&st->perturbed, s_pert);
}

// FP32 blocks: tiles in shared memory.  Separate kernels for the two
// precisions keep the FP64 register footprint out of the FP32 path.
__global__ void __launch_bounds__(256, 1)
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
  return (size_t)NT * (NT + 1) / 2 * TSZ * sizeof(float);
}
size_t potrf_scratch64_elems(int bs) {
  const int NT = (bs + TS - 1) / TS;
  return (size_t)NT * (NT + 1) / 2 * TSZ;
}

cudaError_t launch_potrf(float* A, int lda, int s, int bs, const float* d, const float* sh,
                         const PotrfParams& p, const int* fp64_flag, double* scratch64,
                         float* winv, DevStatus* st, bool may_fp64, cudaStream_t stream) {
  const size_t smem = potrf_smem_bytes(256);
  cudaError_t e = cudaFuncSetAttribute(potrf_f32_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  potrf_f32_kernel<<<1, 256, smem, stream>>>(A, lda, s, bs, d, sh, p, fp64_flag, winv, st);
  if (may_fp64)
    potrf_f64_kernel<<<1, 256, 0, stream>>>(A, lda, s, bs, d, sh, p, fp64_flag, scratch64, winv, st);
  return cudaGetLastError();
}

}  // namespace mpchol
