// Batched factor + PCG of many independent SPD systems of uneven size.
//
// No counterpart in the reference (its driver solves one system per call,
// src/mixed_cholesky.cu:76-229).  Every kernel launch serves all systems:
// the systems are ordered by decreasing n, so the ones still active at factor
// step k are a prefix; per-system pointers and sizes live in a device array
// of BatchSys, per-step panel placement in an array of BatchStep.  The whole
// factorization (input copy, diagonal blocks, panels, quantization, the
// tensor-core trailing updates of all systems in one persistent launch per
// step, solve setup) is one CUDA graph; PCG runs all systems in lockstep, two
// iterations per graph launch, converged systems skipping their work.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg.cuh"

using namespace mpchol;

namespace {

constexpr int kSlots = 8;
constexpr int kScal = 64;

// A_i <- the caller's matrix (column-major, ld ldsrc[i]); d = dtilde = diag,
// sh = 0.
__global__ void batch_load_kernel(const BatchSys* __restrict__ sys, const float* const* __restrict__ src,
                                  const int* __restrict__ ldsrc) {
  const BatchSys& S = sys[blockIdx.y];
  const float* a = src[blockIdx.y];
  const int lda = ldsrc[blockIdx.y];
  const int n = S.n;
  // CTA x copies columns x, x + gridDim.x, ..., its threads run down a column
  for (int c = blockIdx.x; c < n; c += gridDim.x) {
    const float* ac = a + (size_t)c * lda;
    float* dc = S.A + (size_t)c * S.ld;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const float v = ac[r];
      dc[r] = v;
      if (r == c) {
        S.d[r] = v;
        S.dtilde[r] = v;
        S.sh[r] = 0.0f;
      }
    }
  }
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

struct mpchol_batch {
  mpchol_opts opts{};
  int count = 0, nrhs = 1, nr = 1, b = 128, fmt = FP16;
  int max_n = 0, nsteps = 0, qrows = 0;
  int sym_tiles = 0;           // 128-tiles of every system's lower triangle
  std::vector<int> n;          // user order
  std::vector<int> order;      // internal index -> user index (decreasing n)
  std::vector<int> nact, maxm, ntiles;
  std::vector<BatchSys> h_sys;
  std::vector<BatchStep> h_steps;
  // device memory
  float* A = nullptr;
  float* fv = nullptr;         // d, dtilde, rowsq, sh
  float* winv = nullptr;
  float* wsup = nullptr;
  DevStatus* st = nullptr;
  double* vec = nullptr;
  double* part = nullptr;
  double* scal = nullptr;
  int* done = nullptr;
  void* q = nullptr;
  int8_t* rowexp = nullptr;
  uint8_t* mxexp = nullptr;
  BatchSys* d_sys = nullptr;
  BatchStep* d_steps = nullptr;
  void** d_ptrs = nullptr;     // uploaded pointer tables: count src/B + count X
  int* d_ld = nullptr;
  int* d_open = nullptr;
  // pinned host staging
  void** h_ptrs = nullptr;
  int* h_ld = nullptr;
  double* h_scal = nullptr;
  int* h_done = nullptr;
  DevStatus* h_st = nullptr;
  int* h_open = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t fgraph = nullptr;
  cudaGraphExec_t igraph = nullptr;
  double ig_tol2 = -1.0;
};

namespace {

void batch_free(mpchol_batch* B) {
  if (!B) return;
  void* dev[] = {B->A, B->fv, B->winv, B->wsup, B->st, B->vec, B->part, B->scal, B->done,
                 B->q, B->rowexp, B->mxexp, B->d_sys, B->d_steps, B->d_ptrs, B->d_ld, B->d_open};
  for (void* p : dev)
    if (p) cudaFree(p);
  void* host[] = {B->h_ptrs, B->h_ld, B->h_scal, B->h_done, B->h_st, B->h_open};
  for (void* p : host)
    if (p) cudaFreeHost(p);
  if (B->fgraph) cudaGraphExecDestroy(B->fgraph);
  if (B->igraph) cudaGraphExecDestroy(B->igraph);
  if (B->cap) cudaStreamDestroy(B->cap);
  delete B;
}

// The factor sequence for every system (captured once into B->fgraph).
mpchol_status enqueue_factor(mpchol_batch* B, cudaStream_t s) {
  const PotrfParams pp{B->opts.diag_pert, B->opts.pert, B->opts.pivot_floor};
  MPCHOL_CUDA_TRY(cudaMemsetAsync(B->st, 0, sizeof(DevStatus) * B->count, s));
  batch_load_kernel<<<dim3(64, B->count), 256, 0, s>>>(
      B->d_sys, reinterpret_cast<const float* const*>(B->d_ptrs), B->d_ld);
  MPCHOL_CUDA_TRY(cudaGetLastError());
  for (int k = 0; k < B->nsteps; ++k) {
    const int sk = k * B->b;
    const BatchStep* steps = B->d_steps + (size_t)k * B->count;
    MPCHOL_CUDA_TRY(launch_potrf_batched(B->d_sys, B->nact[k], sk, B->b, pp, s));
    if (B->maxm[k] <= 0) continue;
    MPCHOL_CUDA_TRY(launch_trsm_batched(B->d_sys, B->nact[k], sk, B->b, B->maxm[k], s));
    MPCHOL_CUDA_TRY(launch_quantize_batched(B->d_sys, steps, B->nact[k], sk, B->b, B->maxm[k],
                                            B->fmt, B->q, B->qrows, B->rowexp, B->mxexp,
                                            B->opts.diag_pert, s));
    MPCHOL_CUDA_TRY(launch_syrk_tc_batched(B->d_sys, steps, B->nact[k], B->ntiles[k], sk, B->b,
                                           B->fmt, B->q, B->qrows, B->rowexp, B->mxexp, s));
  }
  MPCHOL_CUDA_TRY(launch_solve_setup_batched(B->d_sys, B->count, B->max_n, s));
  return MPCHOL_OK;
}

// z = M^-1 r for every open system (slots: in -> out, TMP and WORK as scratch)
mpchol_status precond_all(mpchol_batch* B, int in, int out, int use_skip, cudaStream_t s) {
  MPCHOL_CUDA_TRY(launch_trsv_batched(false, B->d_sys, B->count, B->max_n, in, 6, 7, B->nr,
                                      use_skip, s));
  MPCHOL_CUDA_TRY(launch_trsv_batched(true, B->d_sys, B->count, B->max_n, 6, out, 7, B->nr,
                                      use_skip, s));
  return MPCHOL_OK;
}

// One PCG iteration of every open system; rho[cur] -> rho[cur ^ 1].
mpchol_status enqueue_iteration(mpchol_batch* B, int cur, double tol2, cudaStream_t s) {
  const int ns = B->count, nr = B->nr;
  MPCHOL_CUDA_TRY(launch_symv_batched(B->d_sys, ns, B->sym_tiles, 3, 4, nr, 1, s));
  MPCHOL_CUDA_TRY(launch_dot_batched(B->d_sys, ns, 3, 4, 0, nr, 1, s));
  MPCHOL_CUDA_TRY(launch_update_xr_batched(B->d_sys, ns, cur, nr, s));
  mpchol_status e = precond_all(B, 1, 2, 1, s);
  if (e != MPCHOL_OK) return e;
  MPCHOL_CUDA_TRY(launch_dot_batched(B->d_sys, ns, 1, 2, 2, nr, 1, s));
  MPCHOL_CUDA_TRY(launch_update_p_batched(B->d_sys, ns, cur, B->nrhs, nr, tol2, s));
  return MPCHOL_OK;
}

mpchol_status read_open(mpchol_batch* B, cudaStream_t s, int* open) {
  MPCHOL_CUDA_TRY(launch_count_open(B->d_sys, B->count, B->d_open, s));
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->h_open, B->d_open, sizeof(int), cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  *open = *B->h_open;
  return MPCHOL_OK;
}

}  // namespace

extern "C" {

mpchol_status mpchol_batch_create(const mpchol_opts* opts, int count, const int* ns, int nrhs,
                                  mpchol_batch_t** out) {
  if (out == nullptr || opts == nullptr || ns == nullptr || count < 1) return MPCHOL_ERR_BAD_ARG;
  *out = nullptr;
  if (nrhs < 1 || nrhs > 8) return MPCHOL_ERR_BAD_ARG;
  const int fmt = opts->precision;
  const int b = opts->block_size;
  if (fmt == MPCHOL_PREC_FP32 || fmt == MPCHOL_PREC_SWITCHING) return MPCHOL_ERR_NOT_SUPPORTED;
  if (fmt < 0 || fmt > MPCHOL_PREC_MXFP4) return MPCHOL_ERR_BAD_ARG;
  if (fmt > MPCHOL_PREC_FP16X2) return MPCHOL_ERR_NOT_SUPPORTED;   // FP6/FP4: single systems only
  if (b < 32 || b > 256 || b % 32 != 0) return MPCHOL_ERR_BAD_ARG;
  if (!syrk_tc_supported(fmt, b)) return MPCHOL_ERR_NOT_SUPPORTED;
  if (opts->left != 0 || opts->equilibrate != 0) return MPCHOL_ERR_NOT_SUPPORTED;
  if (opts->diag_pert && !(opts->pivot_floor > 0.0f)) return MPCHOL_ERR_BAD_ARG;
  for (int i = 0; i < count; ++i)
    if (ns[i] < 1) return MPCHOL_ERR_BAD_ARG;

  mpchol_batch* B = new mpchol_batch();
  B->opts = *opts;
  B->count = count;
  B->nrhs = nrhs;
  B->nr = pcg_padded_nrhs(nrhs);
  B->b = b;
  B->fmt = fmt;
  B->n.assign(ns, ns + count);
  B->order.resize(count);
  std::iota(B->order.begin(), B->order.end(), 0);
  std::stable_sort(B->order.begin(), B->order.end(), [&](int a, int c) { return ns[a] > ns[c]; });
  B->max_n = ns[B->order[0]];
  B->nsteps = (B->max_n + b - 1) / b;

  // placement
  std::vector<size_t> aoff(count), voff(count), woff(count);
  size_t atot = 0, vtot = 0, wtot = 0;
  for (int i = 0; i < count; ++i) {
    const int n = ns[B->order[i]];
    const int ld = (n + 31) / 32 * 32;
    aoff[i] = atot; atot += (size_t)ld * n;
    voff[i] = vtot; vtot += (size_t)n;
    woff[i] = wtot; wtot += solve_wsup_elems(n);
  }
  B->nact.assign(B->nsteps, 0);
  B->maxm.assign(B->nsteps, 0);
  B->ntiles.assign(B->nsteps, 0);
  B->h_steps.assign((size_t)B->nsteps * count, BatchStep{0, 0, 0});
  for (int k = 0; k < B->nsteps; ++k) {
    int qrow = 0, tile = 0;
    for (int i = 0; i < count; ++i) {
      const int n = ns[B->order[i]];
      const int s = k * b;
      if (n <= s) break;
      B->nact[k] = i + 1;
      const int m = n - s - std::min(b, n - s);
      BatchStep& T = B->h_steps[(size_t)k * count + i];
      T.m = m;
      T.q_row0 = qrow;
      T.tile0 = tile;
      if (m > 0) {
        const int t = (m + 127) / 128;
        qrow += t * 128;
        tile += t * (t + 1) / 2;
        B->maxm[k] = std::max(B->maxm[k], m);
      }
    }
    B->ntiles[k] = tile;
    B->qrows = std::max(B->qrows, qrow);
  }
  B->qrows = std::max(B->qrows, 128);

  const size_t nr = B->nr;
  bool ok = dalloc(&B->A, atot) == cudaSuccess && dalloc(&B->fv, 4 * vtot) == cudaSuccess &&
            dalloc(&B->winv, (size_t)count * 8 * 1024) == cudaSuccess &&
            dalloc(&B->wsup, wtot) == cudaSuccess && dalloc(&B->st, count) == cudaSuccess &&
            dalloc(&B->vec, kSlots * vtot * nr) == cudaSuccess &&
            dalloc(&B->part, (size_t)count * 4 * BATCH_VB * 8) == cudaSuccess &&
            dalloc(&B->scal, (size_t)count * kScal) == cudaSuccess &&
            dalloc(&B->done, (size_t)count * 2) == cudaSuccess &&
            dalloc(reinterpret_cast<uint8_t**>(&B->q), (size_t)B->qrows * b * 4) == cudaSuccess &&
            dalloc(&B->rowexp, (size_t)B->qrows) == cudaSuccess &&
            dalloc(&B->mxexp, (size_t)B->qrows * (b / 32)) == cudaSuccess &&
            dalloc(&B->d_sys, count) == cudaSuccess &&
            dalloc(&B->d_steps, (size_t)B->nsteps * count) == cudaSuccess &&
            dalloc(&B->d_ptrs, (size_t)2 * count) == cudaSuccess &&
            dalloc(&B->d_ld, count) == cudaSuccess && dalloc(&B->d_open, 1) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&B->h_ptrs), sizeof(void*) * 2 * count) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&B->h_ld), sizeof(int) * count) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&B->h_scal), sizeof(double) * kScal * count) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&B->h_done), sizeof(int) * 2 * count) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&B->h_st), sizeof(DevStatus) * count) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&B->h_open), sizeof(int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    batch_free(B);
    return MPCHOL_ERR_ALLOC;
  }
  // zero-initialised panel arena: rows past a system's panel hold finite codes
  if (cudaMemset(B->q, 0, (size_t)B->qrows * b * 4) != cudaSuccess ||
      cudaMemset(B->rowexp, 0, (size_t)B->qrows) != cudaSuccess ||
      cudaMemset(B->mxexp, 127, (size_t)B->qrows * (b / 32)) != cudaSuccess ||
      solve_init_attributes() != cudaSuccess) {
    batch_free(B);
    return MPCHOL_ERR_CUDA;
  }
  B->h_sys.resize(count);
  for (int i = 0; i < count; ++i) {
    const int n = ns[B->order[i]];
    BatchSys& S = B->h_sys[i];
    S.A = B->A + aoff[i];
    S.ld = (n + 31) / 32 * 32;
    S.n = n;
    S.d = B->fv + voff[i];
    S.dtilde = B->fv + vtot + voff[i];
    S.rowsq = B->fv + 2 * vtot + voff[i];
    S.sh = B->fv + 3 * vtot + voff[i];
    S.winv = B->winv + (size_t)i * 8 * 1024;
    S.wsup = B->wsup + woff[i];
    S.st = B->st + i;
    S.op = nullptr;
    S.op_ld = n;
    S.vec = B->vec + kSlots * voff[i] * nr;
    S.part = B->part + (size_t)i * 4 * BATCH_VB * 8;
    S.scal = B->scal + (size_t)i * kScal;
    S.done = B->done + (size_t)i * 2;
    const int t = (n + 127) / 128;
    S.sym_tile0 = B->sym_tiles;
    B->sym_tiles += t * (t + 1) / 2;
  }
  if (cudaMemcpy(B->d_sys, B->h_sys.data(), sizeof(BatchSys) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(B->d_steps, B->h_steps.data(), sizeof(BatchStep) * B->h_steps.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking) != cudaSuccess) {
    batch_free(B);
    return MPCHOL_ERR_CUDA;
  }
  *out = B;
  return MPCHOL_OK;
}

mpchol_status mpchol_batch_destroy(mpchol_batch_t* B) {
  batch_free(B);
  return MPCHOL_OK;
}

mpchol_status mpchol_batch_factor(mpchol_batch_t* B, const float* const* dA, const int* lda,
                                  mpchol_stream_t stream_) {
  if (B == nullptr || dA == nullptr || lda == nullptr) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_);
  for (int i = 0; i < B->count; ++i) {
    const int u = B->order[i];
    if (dA[u] == nullptr || lda[u] < B->n[u]) return MPCHOL_ERR_BAD_ARG;
    B->h_ptrs[i] = const_cast<float*>(dA[u]);
    B->h_ld[i] = lda[u];
  }
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->d_ptrs, B->h_ptrs, sizeof(void*) * B->count,
                                  cudaMemcpyHostToDevice, s));
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->d_ld, B->h_ld, sizeof(int) * B->count, cudaMemcpyHostToDevice, s));
  if (B->fgraph == nullptr) {
    cudaGraph_t g = nullptr;
    // relaxed: the launchers set kernel attributes (not stream work) as they go
    MPCHOL_CUDA_TRY(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeRelaxed));
    const mpchol_status e = enqueue_factor(B, B->cap);
    const cudaError_t ce = cudaStreamEndCapture(B->cap, &g);
    if (e != MPCHOL_OK) {
      if (g) cudaGraphDestroy(g);
      return e;
    }
    MPCHOL_CUDA_TRY(ce);
    const cudaError_t ie = cudaGraphInstantiate(&B->fgraph, g, 0);
    cudaGraphDestroy(g);
    MPCHOL_CUDA_TRY(ie);
  }
  MPCHOL_CUDA_TRY(cudaGraphLaunch(B->fgraph, s));
  // the host pointer tables are reused by the next call: finish reading them
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  return MPCHOL_OK;
}

mpchol_status mpchol_batch_lower(const mpchol_batch_t* B, int index, const float** dL, int* ldl,
                                 int* n) {
  if (B == nullptr || dL == nullptr || index < 0 || index >= B->count) return MPCHOL_ERR_BAD_ARG;
  const int i = (int)(std::find(B->order.begin(), B->order.end(), index) - B->order.begin());
  *dL = B->h_sys[i].A;
  if (ldl) *ldl = B->h_sys[i].ld;
  if (n) *n = B->h_sys[i].n;
  return MPCHOL_OK;
}

mpchol_status mpchol_batch_info(mpchol_batch_t* B, int* status, int* fail_row, int* n_perturbed,
                                mpchol_stream_t stream_) {
  if (B == nullptr || status == nullptr) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_);
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->h_st, B->st, sizeof(DevStatus) * B->count,
                                  cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  for (int i = 0; i < B->count; ++i) {
    const int u = B->order[i];
    status[u] = B->h_st[i].code;
    if (fail_row) fail_row[u] = B->h_st[i].row;
    if (n_perturbed) n_perturbed[u] = B->h_st[i].perturbed;
  }
  return MPCHOL_OK;
}

mpchol_status mpchol_batch_pcg(mpchol_batch_t* B, const float* const* dA, const int* lda,
                               const double* const* dB, double* const* dX,
                               const mpchol_pcg_opts* popts, mpchol_report* reports,
                               mpchol_stream_t stream_) {
  if (B == nullptr || dA == nullptr || lda == nullptr || dB == nullptr || dX == nullptr)
    return MPCHOL_ERR_BAD_ARG;
  mpchol_pcg_opts po;
  mpchol_pcg_opts_default(&po);
  if (popts) po = *popts;
  if (po.check_every < 2) po.check_every = 2;
  if (po.max_it < 0) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream_);
  const int ns = B->count, nr = B->nr;
  for (int i = 0; i < ns; ++i) {
    const int u = B->order[i];
    if (dA[u] == nullptr || dB[u] == nullptr || dX[u] == nullptr || lda[u] < B->n[u])
      return MPCHOL_ERR_BAD_ARG;
    B->h_sys[i].op = dA[u];
    B->h_sys[i].op_ld = lda[u];
    B->h_ptrs[i] = const_cast<double*>(dB[u]);
    B->h_ptrs[ns + i] = dX[u];
  }
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->d_sys, B->h_sys.data(), sizeof(BatchSys) * ns,
                                  cudaMemcpyHostToDevice, s));
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->d_ptrs, B->h_ptrs, sizeof(void*) * 2 * ns,
                                  cudaMemcpyHostToDevice, s));
  MPCHOL_CUDA_TRY(cudaMemsetAsync(B->done, 0, sizeof(int) * 2 * ns, s));
  const double tol2 = po.rel_tol * po.rel_tol;
  // b, ||b||^2, x0
  MPCHOL_CUDA_TRY(launch_load_rhs_batched(B->d_sys, ns, reinterpret_cast<const double* const*>(B->d_ptrs),
                                          B->nrhs, nr, s));
  MPCHOL_CUDA_TRY(launch_dot_batched(B->d_sys, ns, 5, 5, 3, nr, 0, s));
  MPCHOL_CUDA_TRY(launch_reduce_batched(B->d_sys, ns, 3, 24, nr, 0, s));
  if (po.x0_precond) {
    const mpchol_status e = precond_all(B, 5, 0, 0, s);
    if (e != MPCHOL_OK) return e;
  } else {
    MPCHOL_CUDA_TRY(launch_vec_slot_batched(B->d_sys, ns, -1, 0, nr, 0, s));
  }
  // the iteration pair graph (all systems, converged ones skip)
  if (B->igraph == nullptr || B->ig_tol2 != tol2) {
    if (B->igraph) cudaGraphExecDestroy(B->igraph);
    B->igraph = nullptr;
    cudaGraph_t g = nullptr;
    MPCHOL_CUDA_TRY(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
    mpchol_status e = enqueue_iteration(B, 0, tol2, B->cap);
    if (e == MPCHOL_OK) e = enqueue_iteration(B, 1, tol2, B->cap);
    const cudaError_t ce = cudaStreamEndCapture(B->cap, &g);
    if (e != MPCHOL_OK) {
      if (g) cudaGraphDestroy(g);
      return e;
    }
    MPCHOL_CUDA_TRY(ce);
    const cudaError_t ie = cudaGraphInstantiate(&B->igraph, g, 0);
    cudaGraphDestroy(g);
    MPCHOL_CUDA_TRY(ie);
    B->ig_tol2 = tol2;
  }
  int launched = 0;
  const int max_restarts = 3;
  for (int restart = 0;; ++restart) {
    // true residual r = b - A x; systems within tolerance are marked done
    MPCHOL_CUDA_TRY(launch_symv_batched(B->d_sys, ns, B->sym_tiles, 0, 4, nr, 0, s));
    MPCHOL_CUDA_TRY(launch_residual_batched(B->d_sys, ns, nr, s));
    MPCHOL_CUDA_TRY(launch_reduce_batched(B->d_sys, ns, 1, 32, nr, 0, s));
    MPCHOL_CUDA_TRY(launch_check_true_batched(B->d_sys, ns, B->nrhs, tol2, s));
    int open = 0;
    mpchol_status e = read_open(B, s, &open);
    if (e != MPCHOL_OK) return e;
    if (open == 0 || launched >= po.max_it || restart > max_restarts) break;
    // z = M^-1 r, p = z, rho = r^T z for the open systems
    e = precond_all(B, 1, 2, 1, s);
    if (e != MPCHOL_OK) return e;
    MPCHOL_CUDA_TRY(launch_vec_slot_batched(B->d_sys, ns, 2, 3, nr, 1, s));
    MPCHOL_CUDA_TRY(launch_dot_batched(B->d_sys, ns, 1, 2, 2, nr, 1, s));
    MPCHOL_CUDA_TRY(launch_reduce_batched(B->d_sys, ns, 2, 0, nr, 1, s));
    while (launched < po.max_it) {
      // the graph runs iteration pairs: an odd remainder runs one extra
      // iteration (counted on the device like every other)
      const int pairs = (std::min(po.check_every, po.max_it - launched) + 1) / 2;
      for (int c = 0; c < pairs; ++c) MPCHOL_CUDA_TRY(cudaGraphLaunch(B->igraph, s));
      launched += 2 * pairs;
      e = read_open(B, s, &open);
      if (e != MPCHOL_OK) return e;
      if (open == 0) break;
    }
  }
  // results and reports
  MPCHOL_CUDA_TRY(launch_store_x_batched(B->d_sys, ns, reinterpret_cast<double* const*>(B->d_ptrs) + ns,
                                         B->nrhs, nr, s));
  if (reports != nullptr) {
    MPCHOL_CUDA_TRY(launch_dot_batched(B->d_sys, ns, 0, 0, 3, nr, 0, s));
    MPCHOL_CUDA_TRY(launch_reduce_batched(B->d_sys, ns, 3, 40, nr, 0, s));
    MPCHOL_CUDA_TRY(launch_frob_batched(B->d_sys, ns, s));
    MPCHOL_CUDA_TRY(launch_reduce_batched(B->d_sys, ns, 3, 48, 1, 0, s));
    MPCHOL_CUDA_TRY(launch_dot_batched(B->d_sys, ns, 1, 2, 2, nr, 0, s));
    MPCHOL_CUDA_TRY(launch_reduce_batched(B->d_sys, ns, 2, 56, nr, 0, s));
  }
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->h_scal, B->scal, sizeof(double) * kScal * ns,
                                  cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->h_done, B->done, sizeof(int) * 2 * ns, cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(B->h_st, B->st, sizeof(DevStatus) * ns, cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  bool all_conv = true, breakdown = false;
  for (int i = 0; i < ns; ++i) {
    const double* sc = B->h_scal + (size_t)i * kScal;
    bool conv = true;
    double relmax = 0.0, bemax = 0.0, prmax = 0.0;
    const double frob = std::sqrt(sc[48]);
    for (int k = 0; k < B->nrhs; ++k) {
      const double rr = sc[32 + k], bb2 = sc[24 + k], xx = sc[40 + k];
      if (!(rr <= tol2 * bb2)) conv = false;
      relmax = std::max(relmax, bb2 > 0 ? std::sqrt(rr / bb2) : std::sqrt(rr));
      bemax = std::max(bemax, std::sqrt(rr) / (frob * std::sqrt(xx) + std::sqrt(bb2)));
      prmax = std::max(prmax, bb2 > 0 ? std::sqrt(std::fabs(sc[56 + k]) / bb2) : 0.0);
    }
    if (B->h_st[i].code == MPCHOL_PCG_BREAKDOWN) breakdown = true;
    all_conv = all_conv && conv;
    if (reports) {
      mpchol_report& r = reports[B->order[i]];
      r.iterations = B->h_done[2 * i + 1];
      r.converged = conv ? 1 : 0;
      r.rel_residual = relmax;
      r.backward_error = bemax;
      r.precond_residual = prmax;
    }
  }
  if (breakdown) return MPCHOL_PCG_BREAKDOWN;
  return all_conv ? MPCHOL_OK : MPCHOL_PCG_MAXIT;
}

}  // extern "C"
