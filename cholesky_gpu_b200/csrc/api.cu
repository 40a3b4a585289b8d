// C-ABI implementation: factor objects, the blocked factorization driver, the
// PCG driver and the reference-shaped entry points.
//
// The driver replaces switching_chol's host loop (src/switching_chol.cuh:76-224)
// and precond_CG (src/mixed_cholesky.cu:76-229).  Differences that matter to a
// caller are deliberate: nothing is allocated per step, the precision decision
// never leaves the device, the work is ordered on the caller's stream (the
// library's own streams wait on it and it waits on them), and no caller-owned
// handle or stream is ever destroyed.
#include <cstdio>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg.cuh"
#include "tmap.cuh"

using namespace mpchol;

namespace mpchol {
static std::mutex g_err_mu;
static std::string g_last_err;
void record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  char buf[512];
  snprintf(buf, sizeof(buf), "%s (%d) at %s:%d in %s", cudaGetErrorString(e), (int)e, file, line,
           what);
  g_last_err = buf;
}
}  // namespace mpchol

// ---- per-phase profiling (the reference's cudaEvent phase timers,
// src/hChol.cuh:22-31,112-117, src/sChol.cuh:150-154) and launch counting ----
namespace {
struct ProfRec {
  int phase;
  cudaEvent_t a, b;
};
struct Profiler {
  std::mutex mu;
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t next = 0;
  std::vector<ProfRec> recs;
};
Profiler g_prof;
long long g_launches[MPCHOL_NPHASES] = {};
std::mutex g_launch_mu;

cudaEvent_t prof_event() {
  if (g_prof.next >= g_prof.pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    g_prof.pool.push_back(e);
  }
  return g_prof.pool[g_prof.next++];
}

struct PhaseScope {
  int ph;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  PhaseScope(int phase, cudaStream_t stream, int nkernels) : ph(phase), s(stream) {
    {
      std::lock_guard<std::mutex> lk(g_launch_mu);
      g_launches[phase] += nkernels;
    }
    if (g_prof.on) {
      std::lock_guard<std::mutex> lk(g_prof.mu);
      a = prof_event();
      if (a) cudaEventRecord(a, s);
    }
  }
  ~PhaseScope() {
    if (a) {
      std::lock_guard<std::mutex> lk(g_prof.mu);
      cudaEvent_t b = prof_event();
      if (b) {
        cudaEventRecord(b, s);
        g_prof.recs.push_back({ph, a, b});
      }
    }
  }
};
bool profiling_on() {
  std::lock_guard<std::mutex> lk(g_prof.mu);
  return g_prof.on;
}
void launch_counts(long long (&out)[MPCHOL_NPHASES]) {
  std::lock_guard<std::mutex> lk(g_launch_mu);
  for (int i = 0; i < MPCHOL_NPHASES; ++i) out[i] = g_launches[i];
}
void add_launch_counts(const long long* nk, long long times) {
  std::lock_guard<std::mutex> lk(g_launch_mu);
  for (int i = 0; i < MPCHOL_NPHASES; ++i) g_launches[i] += nk[i] * times;
}

// How a host-buffer solve overlaps the copy of A with the factorization: A's
// block columns are copied in groups, group g = block columns [c0[g], c1[g]).
// Group 0 is on the device before step 0; group g > 0 joins the trailing
// updates at step join[g] (<= c0[g] - 1), after a catch-up that applies
// panels 0 .. join[g]-1 to its tiles in step order.  Every tile of C thus
// receives the same updates in the same order as in the one-group
// factorization, so the factor is the same bit for bit.
constexpr int kMaxGroups = 8;
struct CopyPlan {
  int ng = 1;
  int c0[kMaxGroups] = {}, c1[kMaxGroups] = {}, join[kMaxGroups] = {};
};

// The factorization captured as one CUDA graph (its copies included for a
// host-buffer solve with a copy plan) and what it was captured for.
struct FactorGraph {
  cudaGraphExec_t exec = nullptr;
  bool failed = false;        // the runtime refused the graph: the work is launched directly
  bool seen = false;          // the key below was that of the previous call
  bool streamed = false;
  CopyPlan plan;
  const float* hA = nullptr;
  const float* hA_dev = nullptr;
  int lda = 0;
  long long nk[MPCHOL_NPHASES] = {};
};

// The captured device-side PCG loop (a WHILE node whose body is one
// iteration) and what it was captured for; nk: kernels per iteration.
struct PcgGraph {
  cudaGraphExec_t exec = nullptr;
  bool failed = false;        // the runtime refused the graph: iterations are launched directly
  const void* A = nullptr;
  int lda = 0, nr = 0, elem = 0;
  double tol2 = 0.0;
  long long nk[MPCHOL_NPHASES] = {};
};
}  // namespace

// Run `expr` (which launches `nk` library kernels) as phase `ph`.
#define PHASE(ph, nk, stream, expr)                 \
  do {                                              \
    PhaseScope _scope((ph), (stream), (nk));        \
    MPCHOL_CUDA_TRY(expr);                          \
  } while (0)

struct mpchol_factor {
  mpchol_opts opts;
  int n = 0, ld = 0, b = 0, nsteps = 0;
  int device = 0;
  float* A = nullptr;         // n columns x ld rows, factor in the lower triangle
  float* d = nullptr;         // original diagonal
  float* dtilde = nullptr;    // Schur-complement diagonal tracker
  float* rowsq = nullptr;     // per-row sum of squares of the latest panel
  float* sh = nullptr;        // accumulated rounding-shift estimate
  float* winv = nullptr;      // inverses of the 32x32 diagonal tiles of one block
  double* scratch64 = nullptr;
  // the step's panel quantized in every format the step may pick (K-major,
  // row i = trailing row i): 8-bit codes (E4M3, E5M2, MXFP8; n x b each),
  // FP16 / FP16X2-hi codes then FP16X2-lo codes (n x b each), per-row
  // exponents (E4M3, E5M2, FP16; n each) and MXFP8 block scales
  uint8_t* q8 = nullptr;
  uint16_t* q16 = nullptr;
  int8_t* rexp = nullptr;
  uint8_t* mxexp = nullptr;
  StepState* steps = nullptr;
  DevStatus* status = nullptr;    // the factorization's status word
  DevStatus* pstatus = nullptr;   // the solves' status word (breakdown, timeouts)
  double* colacc = nullptr;       // coherence rule: each step's panel column sums (kColCopies x b per step)
  int8_t* eqexp = nullptr;        // equilibration exponents e_i (row i scaled by 2^-e_i)
  // solve side
  float* wsup = nullptr;      // inverses of the 1024-row diagonal super-blocks
  int* trsv_ctr = nullptr;    // dependency counters of the persistent triangular solve
  bool solve_ready = false;
  // PCG workspace (sized for 8 rhs)
  double* vec = nullptr;      // x, r, z, p, Ap, b, tmp, work : 8 * n * 8
  double* partials = nullptr; // 4 * VG * 8
  double* scal = nullptr;     // rho[2][8], alpha[8], bnorm2[8], misc
  int* done = nullptr;        // [0] converged flag, [1] iteration counter
  int* h_done = nullptr;      // pinned
  double* h_scal = nullptr;   // pinned
  PcgGraph graph;             // captured PCG loop (see run_pcg)
  FactorGraph fgraph;         // captured factorization (see launch_factor)
  int* loop_ctl = nullptr;    // its iteration count and budget
  cudaStream_t capture_stream = nullptr;   // private stream used only to capture graphs
  // look-ahead: the bulk of each step's trailing update runs on aux while
  // the next diagonal block is factored on the caller's stream
  // host-buffer solves: the operator's lower triangle and the rhs / solution
  float* op = nullptr;        // n columns x ld, lower triangle
  double* hb = nullptr;       // n x 8
  double* hx = nullptr;       // n x 8
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_next = nullptr;   // the next block's columns are updated
  cudaEvent_t ev_rest = nullptr;   // the rest of the step's update is done
  // host-buffer solves with the copy of A overlapped (see CopyPlan): the
  // copy stream, one event per arrived group, the pinned diagonal of A, and
  // the quantized panels of the steps that late groups catch up with
  cudaStream_t cp = nullptr;
  cudaEvent_t ev_grp[kMaxGroups] = {};
  cudaEvent_t ev_start = nullptr;  // prior work on the caller's stream is done
  cudaEvent_t ev_catch = nullptr;  // a step's catch-ups are done
  cudaEvent_t ev_diag = nullptr;   // the pinned diagonal has been copied
  float* h_diag = nullptr;
  uint8_t* hq8 = nullptr;
  uint16_t* hq16 = nullptr;
  int8_t* hrexp = nullptr;
  uint8_t* hmx = nullptr;
  int hist_steps = 0;              // steps the panel history holds
  int plan_mode = -1;              // -1: automatic, otherwise set by mpchol_set_copy_plan
  CopyPlan plan;
  int nsm = 0;
  CUtensorMap tmap32;         // TMA map over A, 32 x 32 boxes
  CUtensorMap tmapX;          // TMA map over A, 32 x b boxes (panel slabs)
};

namespace {

mpchol_status validate_opts(const mpchol_opts* o, int n) {
  if (o == nullptr || n <= 0) return MPCHOL_ERR_BAD_ARG;
  if (o->block_size < 32 || o->block_size > 256 || o->block_size % 32 != 0) return MPCHOL_ERR_BAD_ARG;
  if (o->precision < 0 || o->precision > MPCHOL_PREC_MXFP4) return MPCHOL_ERR_BAD_ARG;
  if (o->left != 0 && o->left != 1) return MPCHOL_ERR_BAD_ARG;
  if (o->diag_pert && !(o->pivot_floor > 0.0f)) return MPCHOL_ERR_BAD_ARG;
  if (o->switch_mode != 0 && o->switch_mode != 1) return MPCHOL_ERR_BAD_ARG;
  if ((o->coherence != 0 && o->coherence != 1) || (o->equilibrate != 0 && o->equilibrate != 1))
    return MPCHOL_ERR_BAD_ARG;
  if (!(o->eps_coherence >= 0.0f)) return MPCHOL_ERR_BAD_ARG;
  if (o->ladder_len < 0 || o->ladder_len > 4) return MPCHOL_ERR_BAD_ARG;
  auto tc_ok = [&](int fmt) { return fmt == MPCHOL_PREC_FP32 || syrk_tc_supported(fmt, o->block_size); };
  if (o->precision != MPCHOL_PREC_SWITCHING && !tc_ok(o->precision)) return MPCHOL_ERR_NOT_SUPPORTED;
  if (o->precision == MPCHOL_PREC_SWITCHING) {
    if (o->switch_mode == 1) {
      if (!tc_ok(MPCHOL_PREC_FP16) || !tc_ok(MPCHOL_PREC_E4M3)) return MPCHOL_ERR_NOT_SUPPORTED;
    } else {
      for (int i = 0; i < o->ladder_len; ++i) {
        const int p = o->ladder[i];
        if (p < 0 || p > MPCHOL_PREC_MXFP4 || p == MPCHOL_PREC_SWITCHING) return MPCHOL_ERR_BAD_ARG;
        if (!tc_ok(p)) return MPCHOL_ERR_NOT_SUPPORTED;
      }
      // the MX formats share one code slot and scale buffer
      int nmx = 0;
      for (int i = 0; i < o->ladder_len; ++i) nmx += is_mx(o->ladder[i]) ? 1 : 0;
      if (nmx > 1) return MPCHOL_ERR_NOT_SUPPORTED;
    }
  }
  return MPCHOL_OK;
}

template <typename T>
cudaError_t dmalloc(T** p, size_t count) {
  return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T) + 256);
}

void free_factor(mpchol_factor_t* f) {
  if (f == nullptr) return;
  void* ptrs[] = {f->A, f->d, f->dtilde, f->rowsq, f->sh, f->winv, f->scratch64, f->q8,
                  f->q16, f->rexp, f->mxexp, f->steps, f->status, f->pstatus, f->colacc,
                  f->eqexp, f->wsup, f->trsv_ctr,
                  f->vec, f->partials, f->scal, f->done, f->loop_ctl, f->op, f->hb, f->hx,
                  f->hq8, f->hq16, f->hrexp, f->hmx};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (f->graph.exec) cudaGraphExecDestroy(f->graph.exec);
  if (f->fgraph.exec) cudaGraphExecDestroy(f->fgraph.exec);
  if (f->capture_stream) cudaStreamDestroy(f->capture_stream);
  if (f->aux) cudaStreamDestroy(f->aux);
  if (f->ev_next) cudaEventDestroy(f->ev_next);
  if (f->ev_rest) cudaEventDestroy(f->ev_rest);
  if (f->cp) cudaStreamDestroy(f->cp);
  for (cudaEvent_t e : f->ev_grp)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {f->ev_start, f->ev_catch, f->ev_diag})
    if (e) cudaEventDestroy(e);
  if (f->h_diag) cudaFreeHost(f->h_diag);
  if (f->h_done) cudaFreeHost(f->h_done);
  if (f->h_scal) cudaFreeHost(f->h_scal);
  delete f;
}

DecisionParams make_dp(const mpchol_opts& o) {
  DecisionParams dp;
  dp.policy = o.precision;
  dp.switch_mode = o.switch_mode;
  dp.eps_prime = o.eps_prime;
  dp.floor_ratio = o.floor;
  dp.ladder_len = o.ladder_len;
  for (int i = 0; i < 4; ++i) dp.ladder[i] = o.ladder[i];
  dp.coherence = (o.precision == MPCHOL_PREC_SWITCHING && o.switch_mode == 0 && o.coherence) ? 1 : 0;
  dp.eps_coh = o.eps_coherence > 0.0f ? o.eps_coherence : o.eps_prime;
  return dp;
}

// The lower triangle of an n x n column-major matrix, block column by block
// column (rows from the block's diagonal down): one 2-D copy per block
// column, about half of the matrix's bytes.  The factorization and the
// operator products read nothing above the diagonal.
// Block columns [j0, j1) only: copy_lower_cols.
cudaError_t copy_lower_cols(float* dst, int ldd, const float* src, int lds, int n, int b, int j0,
                            int j1, cudaMemcpyKind kind, cudaStream_t s) {
  for (int c = j0 * b; c < n && c < j1 * b; c += b) {
    const int w = std::min(b, n - c);
    cudaError_t e = cudaMemcpy2DAsync(dst + (size_t)c * ldd + c, sizeof(float) * ldd,
                                      src + (size_t)c * lds + c, sizeof(float) * lds,
                                      sizeof(float) * (n - c), w, kind, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
cudaError_t copy_lower_blocks(float* dst, int ldd, const float* src, int lds, int n, int b,
                              cudaMemcpyKind kind, cudaStream_t s) {
  return copy_lower_cols(dst, ldd, src, lds, n, b, 0, ceil_div(n, b), kind, s);
}

bool valid_copy_plan(const CopyPlan& p, int nb);

// Timeline model of a copy-overlap plan, in microseconds: the lower block
// columns cross PCIe at 50 GB/s in group order; on the caller's stream each
// step runs the panel solve ((25 + 22 m / 8192) b / 256), the head update
// (8) and the next POTRF (0.28 per column), the panel solve waiting for the
// previous step's second-stream work; on the second stream a group's
// catch-up (one launch per earlier panel) and each step's rest update cost
// 6 + (C elements * 8 B) / (3 TB/s) per launch.  The constants are B200
// measurements of the kernels at n = 8192, b = 256.
double model_copy_plan(int n, int b, const CopyPlan& p) {
  const int nb = ceil_div(n, b);
  std::vector<double> el(nb + 1, 0.0);   // prefix sums of lower block-column elements
  for (int j = 0; j < nb; ++j)
    el[j + 1] = el[j] + (double)(n - j * b) * std::min(b, n - j * b);
  auto cols = [&](int j0, int j1) { return el[std::min(j1, nb)] - el[std::min(j0, nb)]; };
  auto syrk_us = [](double e) { return 6.0 + e * 8.0 / 3.0e6; };
  std::vector<double> arr(p.ng);
  double t = 0.0;
  for (int g = 0; g < p.ng; ++g) {
    t += cols(p.c0[g], p.c1[g]) * 4.0 / 50.0e3;
    arr[g] = t;
  }
  double main_t = arr[0] + 0.28 * std::min(b, n), aux = 0.0, rest_done = 0.0;
  int joined = 1;
  for (int k = 0; k + 1 < nb; ++k) {
    double catch_end = -1.0;
    int first_new = -1;
    while (joined < p.ng && p.join[joined] == k) {
      aux = std::max(aux, arr[joined]);
      for (int s = 0; s < k; ++s) aux += syrk_us(cols(p.c0[joined], p.c1[joined]));
      catch_end = aux;
      if (first_new < 0) first_new = joined;
      ++joined;
    }
    const double m = n - (double)(k + 1) * b;
    main_t = std::max(main_t, rest_done) + (25.0 + 22.0 * m / 8192.0) * b / 256.0;
    if (first_new >= 0 && k + 1 >= p.c0[first_new]) main_t = std::max(main_t, catch_end);
    main_t += 8.0;
    aux = std::max(aux, main_t) + syrk_us(cols(k + 1, p.c1[joined - 1]));
    rest_done = aux;
    main_t += 0.28 * std::min(b, n - (k + 1) * b);
  }
  return std::max(main_t, rest_done);
}

// Eight groups cut at these fractions of the block columns, each joining
// the trailing updates two steps before its first block column is solved:
// the copy is the longer process, so the first group is small (the
// factorization starts early) and the later ones grow while the
// factorization's steps shorten.  Measured on a B200 against the plans of
// the model below and other cut rules: 23.2 against 24.3 ms end to end at
// n = 16384 (RBF matrix, 8 rhs) and 6.70 against 6.98 ms at n = 8192 (b = 256).
constexpr double kCutFrac[kMaxGroups - 1] = {0.04, 0.11, 0.19, 0.28, 0.38, 0.50, 0.66};
constexpr int kJoinLag = 2;
constexpr int kRuleMinBlocks = 32;

// The plan: the cut rule above when there are at least 32 block columns,
// else the one with the least modelled time among up to 5 groups (cuts among
// at most 16 block-column positions, each group joining 1-3 steps before its
// first block column is solved).  One group (copy everything, then factor)
// unless the 128-row tiles of the trailing update align with block columns
// (b a multiple of 128) and, for the model, overlap saves at least 2 %.
CopyPlan choose_copy_plan(int n, int b) {
  const int nb = ceil_div(n, b);
  CopyPlan best;
  best.ng = 1;
  best.c0[0] = 0;
  best.c1[0] = nb;
  if (b % 128 != 0 || nb < 4) return best;
  if (nb >= kRuleMinBlocks) {
    CopyPlan p;
    p.c0[0] = 0;
    int prev = 0, g = 0;
    for (double fr : kCutFrac) {
      const int c = std::max(prev + 1, (int)std::lround(fr * nb));
      if (c >= nb - 1) break;
      p.c1[g] = c;
      p.c0[g + 1] = c;
      p.join[g + 1] = std::max(p.join[g], std::max(0, c - kJoinLag));
      ++g;
      prev = c;
    }
    p.ng = g + 1;
    p.c1[g] = nb;
    if (valid_copy_plan(p, nb)) return p;
  }
  const double t1 = model_copy_plan(n, b, best);
  double tbest = t1;
  std::vector<int> pos;
  const int npos = nb - 2;   // candidate cuts 1 .. nb-2
  for (int i = 0; i < std::min(npos, 16); ++i)
    pos.push_back(1 + (int)((long long)i * npos / std::min(npos, 16)));
  pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
  std::vector<int> idx;
  CopyPlan p;
  // enumerate increasing index tuples of length ncut over pos
  auto rec = [&](auto&& self, int start, int ncut) -> void {
    if ((int)idx.size() == ncut) {
      p.ng = ncut + 1;
      p.c0[0] = 0;
      for (int g = 0; g < ncut; ++g) {
        p.c1[g] = pos[idx[g]];
        p.c0[g + 1] = pos[idx[g]];
      }
      p.c1[ncut] = nb;
      for (int lag = 1; lag <= 3; ++lag) {
        p.join[0] = 0;
        for (int g = 1; g < p.ng; ++g) p.join[g] = std::max(p.join[g - 1], std::max(0, p.c0[g] - lag));
        bool ok = true;
        for (int g = 1; g < p.ng; ++g) ok = ok && p.join[g] <= p.c0[g] - 1;
        if (!ok) continue;
        const double tp = model_copy_plan(n, b, p);
        if (tp < tbest) {
          tbest = tp;
          best = p;
        }
      }
      return;
    }
    for (int i = start; i < (int)pos.size(); ++i) {
      idx.push_back(i);
      self(self, i + 1, ncut);
      idx.pop_back();
    }
  };
  for (int ncut = 1; ncut <= 4; ++ncut) rec(rec, 0, ncut);
  if (tbest > 0.98 * t1) {
    best = CopyPlan{};
    best.c1[0] = nb;
  }
  return best;
}

// Checks a plan given by cuts (block columns) and join steps.
bool valid_copy_plan(const CopyPlan& p, int nb) {
  if (p.ng < 1 || p.ng > kMaxGroups || p.c0[0] != 0 || p.c1[p.ng - 1] != nb) return false;
  for (int g = 0; g < p.ng; ++g) {
    if (p.c1[g] <= p.c0[g]) return false;
    if (g > 0 && (p.c0[g] != p.c1[g - 1] || p.join[g] < 0 || p.join[g] > p.c0[g] - 1 ||
                  p.join[g] < p.join[g - 1]))
      return false;
  }
  return true;
}

// The second stream of the look-ahead and its events (created once, outside
// any stream capture).
mpchol_status ensure_factor_streams(mpchol_factor_t* f) {
  if (f->aux != nullptr) return MPCHOL_OK;
  MPCHOL_CUDA_TRY(cudaStreamCreateWithFlags(&f->aux, cudaStreamNonBlocking));
  MPCHOL_CUDA_TRY(cudaEventCreateWithFlags(&f->ev_next, cudaEventDisableTiming));
  MPCHOL_CUDA_TRY(cudaEventCreateWithFlags(&f->ev_rest, cudaEventDisableTiming));
  MPCHOL_CUDA_TRY(cudaEventCreateWithFlags(&f->ev_catch, cudaEventDisableTiming));
  MPCHOL_CUDA_TRY(cudaDeviceGetAttribute(&f->nsm, cudaDevAttrMultiProcessorCount, f->device));
  return MPCHOL_OK;
}

// One factorization of f->A in place, on `stream`, right-looking with a
// look-ahead of one block.  Step k: the panel solve (with the step decision
// and the panel quantization), then the trailing update of the tiles of
// diagonal block k+1 (SEL_NEXT), then -- on the caller's stream -- the POTRF
// of block k+1, while the rest of step k's update (block k+1's panel
// included) runs on the aux stream on all SMs but one.  The panel solve of step k+1 waits for that
// rest.  Every C tile receives the same updates in the same order as
// without the split, so the factor is unchanged by it.
//
// With a copy plan (host-buffer solves), A's block columns are still being
// copied on f->cp while the factorization runs: f->d / f->dtilde were filled
// by the caller, step 0 waits for group 0, the rest updates cover only the
// groups that have joined, and a joining group first receives the earlier
// panels' updates (one SEL_BAND launch per panel, in step order, from the
// panel history) on the aux stream.
// Trailing rows from which a step's concurrent update outlasts the POTRF
// beside it (B200, b = 256: about 80 us of update at 7168 rows).
constexpr int kCompactPotrfRows = 7168;

mpchol_status run_factor(mpchol_factor_t* f, cudaStream_t stream, const CopyPlan* plan = nullptr) {
  const mpchol_opts& o = f->opts;
  const int n = f->n, ld = f->ld, b = f->b;
  PotrfParams pp{o.diag_pert, o.pert, o.pivot_floor};
  const DecisionParams dp = make_dp(o);
  mpchol_status es = ensure_factor_streams(f);
  if (es != MPCHOL_OK) return es;
  const bool streamed = plan != nullptr && plan->ng > 1;
  const int cap = f->nsm > 1 ? f->nsm - 1 : 1;   // SMs for the concurrent part of the update
  MPCHOL_CUDA_TRY(cudaMemsetAsync(f->status, 0, sizeof(DevStatus), stream));
  MPCHOL_CUDA_TRY(cudaMemsetAsync(f->steps, 0, sizeof(StepState) * (f->nsteps + 1), stream));
  MPCHOL_CUDA_TRY(cudaMemsetAsync(f->sh, 0, sizeof(float) * n, stream));
  if (dp.coherence)
    MPCHOL_CUDA_TRY(cudaMemsetAsync(f->colacc, 0, sizeof(double) * (size_t)f->nsteps * kColCopies * b,
                                    stream));
  if (streamed) {
    MPCHOL_CUDA_TRY(cudaStreamWaitEvent(stream, f->ev_grp[0], 0));
  } else {
    if (o.equilibrate) {
      // D A D with D = diag(2^-e_i): exponents from A's diagonal, then the
      // lower triangle scaled in place (exact powers of two)
      PHASE(MPCHOL_PH_SETUP, 2, stream, launch_equil_exps(f->A, ld, n, f->eqexp, stream));
      MPCHOL_CUDA_TRY(launch_equil_scale(f->A, ld, n, f->eqexp, 0, n, false, stream));
    }
    PHASE(MPCHOL_PH_SETUP, 1, stream, launch_extract_diag(f->A, ld, n, f->d, f->dtilde, stream));
  }
  const bool fixed = o.precision != MPCHOL_PREC_SWITCHING;
  unsigned tc_mask = 0;   // tensor-core formats a switching step may pick
  bool f32_possible = fixed || o.switch_mode == 1 || o.ladder_len == 0;
  if (!fixed) {
    if (o.switch_mode == 1) tc_mask = (1u << FP16) | (1u << E4M3);
    else
      for (int i = 0; i < o.ladder_len; ++i) {
        if (o.ladder[i] != FP32) tc_mask |= 1u << o.ladder[i];
        else f32_possible = true;
      }
  }
  // beside: the POTRF of block k runs beside the rest of step k-1's trailing
  // update; with at least kCompactPotrfRows trailing rows that update lasts
  // longer than the POTRF itself, and the small-code POTRF variant is used
  auto potrf = [&](int k, bool beside) -> mpchol_status {
    const int s = k * b;
    const bool compact = beside && n - s >= kCompactPotrfRows;
    PHASE(MPCHOL_PH_POTRF, o.floor > 0.0f ? 2 : 1, stream,
          launch_potrf(f->tmap32, f->A, ld, n, s, std::min(b, n - s), f->d, f->sh, pp,
                       &f->steps[k].fp64_diag, f->scratch64, f->winv, f->status, o.floor > 0.0f,
                       stream, k > 0 ? &f->steps[k - 1] : nullptr, f->rowsq, compact));
    return MPCHOL_OK;
  };
  // where the panel solve of step k writes the codes of each candidate
  // format: the shared buffers, or the panel history for steps that a late
  // group catches up with
  const size_t nbq = (size_t)n * b;
  auto qa_for = [&](int k) -> QuantAll {
    QuantAll q{};
    q.cand = fixed ? (o.precision != FP32 ? 1u << o.precision : 0u) : tc_mask;
    q.ldq = b;
    q.ldmx = b / 32;
    const bool hist = (streamed || o.left) && k < f->hist_steps;
    uint8_t* q8 = hist ? f->hq8 + (size_t)k * 3 * nbq : f->q8;
    int8_t* rexp = hist ? f->hrexp + (size_t)k * 3 * n : f->rexp;
    for (int i = 0; i < 3; ++i) {
      q.q8[i] = q8 + (size_t)i * nbq;
      q.rexp[i] = rexp + (size_t)i * n;
    }
    q.q16 = hist ? f->hq16 + (size_t)k * 2 * nbq : f->q16;
    q.mxexp = hist ? f->hmx + (size_t)k * (nbq / 32) : f->mxexp;
    q.sh = o.diag_pert ? f->sh + k * b + std::min(b, n - k * b) : nullptr;
    return q;
  };
  // step k's trailing update over the tiles `sel` picks, on stream `ss`
  auto syrk = [&](int k, TileSel sel, int max_sms, cudaStream_t ss) -> mpchol_status {
    const int s = k * b;
    const int bs = std::min(b, n - s);
    const int m = n - s - bs;
    float* P = f->A + (size_t)s * ld + s + bs;
    float* C = f->A + (size_t)(s + bs) * ld + s + bs;
    const QuantAll qa = qa_for(k);
    if (fixed) {
      if (o.precision == FP32)
        PHASE(MPCHOL_PH_SYRK_F32, 1, ss,
              launch_syrk_f32(C, ld, m, bs, P, ld, nullptr, f->status, ss, sel, max_sms));
      else
        PHASE(MPCHOL_PH_SYRK_TC, 1, ss,
              launch_syrk_tc(C, ld, m, bs, o.precision,
                             (o.precision == FP16 || o.precision == FP16X2)
                                 ? static_cast<const void*>(qa.q16)
                                 : static_cast<const void*>(qa.q8[q8_slot(o.precision)]),
                             bs, qa.rexp[rexp_slot(o.precision)], qa.mxexp, bs / 32, nullptr,
                             f->status, ss, sel, max_sms));
      return MPCHOL_OK;
    }
    const int* pick = &f->steps[k].prec;
    if (f32_possible)
      PHASE(MPCHOL_PH_SYRK_F32, 1, ss,
            launch_syrk_f32(C, ld, m, bs, P, ld, pick, f->status, ss, sel, max_sms));
    if (tc_mask != 0)
      PHASE(MPCHOL_PH_SYRK_TC, 1, ss,
            launch_syrk_tc_dispatch(C, ld, m, bs, tc_mask, qa, pick, f->status, ss, sel, max_sms));
    return MPCHOL_OK;
  };
  // 128-tile column of step k's trailing matrix where block column j starts
  auto tcol = [&](int k, int j) { return ceil_div(std::min(j * b, n) - (k + 1) * b, 128); };
  if (o.left) {
    // Left-looking (settings.json "left"): block column k receives the
    // updates of panels 0 .. k-1 just before it is factored -- one band
    // launch per earlier panel, in step order, from the panels' quantized
    // codes kept in the panel history -- then its diagonal block is factored
    // and its panel solved.  Every tile receives the same FP32 updates in the
    // same order as in the right-looking schedule, so the factor is the same
    // bit for bit; the trailing matrix beyond block column k is never touched
    // before its turn.
    for (int k = 0; k < f->nsteps; ++k) {
      for (int p = 0; p < k; ++p) {
        TileSel band{SEL_BAND, 0, tcol(p, k), tcol(p, k + 1), 0};
        mpchol_status rs = syrk(p, band, 0, stream);
        if (rs != MPCHOL_OK) return rs;
      }
      mpchol_status rs = potrf(k, false);
      if (rs != MPCHOL_OK) return rs;
      const int s = k * b;
      const int bs = std::min(b, n - s);
      const int m = n - s - bs;
      if (m <= 0) break;
      const QuantAll qa = qa_for(k);
      PHASE(MPCHOL_PH_TRSM, 1, stream,
            launch_trsm_panel(f->tmapX, f->tmap32, f->A, ld, n, s, bs, f->winv, f->d, f->dtilde,
                              f->rowsq, &f->steps[k], &f->steps[k + 1], std::min(b, m), dp, qa,
                              f->status, stream, k > 0 ? &f->steps[k - 1] : nullptr,
                              dp.coherence ? f->colacc + (size_t)k * kColCopies * b : nullptr));
    }
    if (o.equilibrate)
      PHASE(MPCHOL_PH_SETUP, 1, stream, launch_equil_scale(f->A, ld, n, f->eqexp, 0, n, true, stream));
    f->solve_ready = false;
    return MPCHOL_OK;
  }
  mpchol_status rs = potrf(0, false);
  if (rs != MPCHOL_OK) return rs;
  bool rest_pending = false;
  int joined = 1;                                  // groups in the trailing updates
  int joined_end = streamed ? plan->c1[0] : f->nsteps;   // block columns on the device
  for (int k = 0; k < f->nsteps; ++k) {
    const int s = k * b;
    const int bs = std::min(b, n - s);
    const int m = n - s - bs;
    if (m <= 0) break;
    if (rest_pending) {
      MPCHOL_CUDA_TRY(cudaStreamWaitEvent(stream, f->ev_rest, 0));
      rest_pending = false;
    }
    const int next_bs = std::min(b, m);
    // panel solve, step decision and panel quantization in one launch
    const QuantAll qa = qa_for(k);
    PHASE(MPCHOL_PH_TRSM, 1, stream,
          launch_trsm_panel(f->tmapX, f->tmap32, f->A, ld, n, s, bs, f->winv, f->d, f->dtilde,
                            f->rowsq, &f->steps[k], &f->steps[k + 1], next_bs, dp, qa, f->status,
                            stream, k > 0 ? &f->steps[k - 1] : nullptr,
                            dp.coherence ? f->colacc + (size_t)k * kColCopies * b : nullptr));
    // groups joining at this step catch up with panels 0 .. k-1 (aux is
    // already ordered after those panels and after the previous rest)
    bool caught = false, head_waits = false;
    while (streamed && joined < plan->ng && plan->join[joined] == k) {
      const int g = joined;
      MPCHOL_CUDA_TRY(cudaStreamWaitEvent(f->aux, f->ev_grp[g], 0));
      for (int p = 0; p < k; ++p) {
        TileSel band{SEL_BAND, 0, tcol(p, plan->c0[g]), tcol(p, plan->c1[g]), 0};
        if ((rs = syrk(p, band, cap, f->aux)) != MPCHOL_OK) return rs;
      }
      caught = true;
      head_waits = head_waits || k + 1 >= plan->c0[g];
      joined_end = plan->c1[g];
      ++joined;
    }
    if (caught) {
      MPCHOL_CUDA_TRY(cudaEventRecord(f->ev_catch, f->aux));
      if (head_waits) MPCHOL_CUDA_TRY(cudaStreamWaitEvent(stream, f->ev_catch, 0));
    }
    const int jc = ceil_div(next_bs, 128);   // 128-tile columns of block k+1
    if ((rs = syrk(k, TileSel{SEL_NEXT, jc}, 0, stream)) != MPCHOL_OK) return rs;
    // the rest of the update, over the block columns on the device
    const int T = ceil_div(m, 128);
    const int jend = tcol(k, joined_end);
    const TileSel rest = jend >= T ? TileSel{SEL_REST, jc} : TileSel{SEL_BAND, jc, 0, jend, jc};
    if (sel_tile_count(T, rest) > 0) {
      MPCHOL_CUDA_TRY(cudaEventRecord(f->ev_next, stream));
      MPCHOL_CUDA_TRY(cudaStreamWaitEvent(f->aux, f->ev_next, 0));
      if ((rs = syrk(k, rest, cap, f->aux)) != MPCHOL_OK) return rs;
      MPCHOL_CUDA_TRY(cudaEventRecord(f->ev_rest, f->aux));
      rest_pending = true;
    } else if (caught) {
      MPCHOL_CUDA_TRY(cudaStreamWaitEvent(stream, f->ev_catch, 0));
    }
    if ((rs = potrf(k + 1, rest_pending)) != MPCHOL_OK) return rs;
  }
  if (rest_pending) MPCHOL_CUDA_TRY(cudaStreamWaitEvent(stream, f->ev_rest, 0));
  if (streamed) MPCHOL_CUDA_TRY(cudaStreamWaitEvent(stream, f->ev_grp[plan->ng - 1], 0));
  // equilibrated: L of A is D^-1 times the factor of D A D (rows times 2^e_i)
  if (o.equilibrate && !streamed)
    PHASE(MPCHOL_PH_SETUP, 1, stream, launch_equil_scale(f->A, ld, n, f->eqexp, 0, n, true, stream));
  f->solve_ready = false;
  return MPCHOL_OK;
}

bool same_plan(const CopyPlan& a, const CopyPlan& b) {
  if (a.ng != b.ng) return false;
  for (int g = 0; g < a.ng; ++g)
    if (a.c0[g] != b.c0[g] || a.c1[g] != b.c1[g] || a.join[g] != b.join[g]) return false;
  return true;
}

// Everything one factorization enqueues on `stream`.  With a copy plan: the
// copy stream forks from `stream` and copies A's lower block columns group by
// group (into the operator buffer, then device to device into the factor's
// storage); the diagonal of A comes straight from the caller's page-locked
// buffer (hA_dev, its device-side address) or, for pageable memory, from
// f->h_diag, which the caller filled.
mpchol_status enqueue_factor(mpchol_factor_t* f, cudaStream_t stream, const CopyPlan* plan,
                             const float* hA, int lda, const float* hA_dev) {
  if (plan == nullptr || plan->ng <= 1) return run_factor(f, stream);
  const int n = f->n, b = f->b;
  MPCHOL_CUDA_TRY(cudaEventRecord(f->ev_start, stream));
  MPCHOL_CUDA_TRY(cudaStreamWaitEvent(f->cp, f->ev_start, 0));
  for (int g = 0; g < plan->ng; ++g) {
    MPCHOL_CUDA_TRY(copy_lower_cols(f->op, f->ld, hA, lda, n, b, plan->c0[g], plan->c1[g],
                                    cudaMemcpyHostToDevice, f->cp));
    MPCHOL_CUDA_TRY(copy_lower_cols(f->A, f->ld, f->op, f->ld, n, b, plan->c0[g], plan->c1[g],
                                    cudaMemcpyDeviceToDevice, f->cp));
    MPCHOL_CUDA_TRY(cudaEventRecord(f->ev_grp[g], f->cp));
  }
  // the switching statistics of step 0 read the whole diagonal
  if (hA_dev != nullptr) {
    PHASE(MPCHOL_PH_SETUP, 1, stream, launch_extract_diag(hA_dev, lda, n, f->d, f->dtilde, stream));
  } else {
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->d, f->h_diag, sizeof(float) * n, cudaMemcpyHostToDevice, stream));
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->dtilde, f->d, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream));
  }
  return run_factor(f, stream, plan);
}

// One factorization as a CUDA graph, relaunched while the copy plan and the
// host buffer stay the same, which removes most of the launch gaps between
// the dependent kernels of the critical path (panel solve -> head update ->
// POTRF -> next panel solve).  The graph is captured on the second
// consecutive call with the same key: a factor object used once, or a
// caller that passes a new host buffer every time, pays no capture.
// Profiling runs, and runtimes that refuse the graph, enqueue directly.
mpchol_status launch_factor(mpchol_factor_t* f, cudaStream_t stream, const CopyPlan* plan = nullptr,
                            const float* hA = nullptr, int lda = 0, const float* hA_dev = nullptr) {
  const bool streamed = plan != nullptr && plan->ng > 1;
  FactorGraph& g = f->fgraph;
  if (profiling_on() || g.failed) return enqueue_factor(f, stream, plan, hA, lda, hA_dev);
  const bool same_key = g.seen && g.streamed == streamed &&
                        (!streamed || (same_plan(g.plan, *plan) && g.hA == hA && g.lda == lda &&
                                       g.hA_dev == hA_dev));
  if (!same_key) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    g.seen = true;
    g.streamed = streamed;
    if (streamed) g.plan = *plan;
    g.hA = hA;
    g.lda = lda;
    g.hA_dev = hA_dev;
    return enqueue_factor(f, stream, plan, hA, lda, hA_dev);
  }
  if (g.exec == nullptr) {
    mpchol_status es = ensure_factor_streams(f);
    if (es != MPCHOL_OK) return es;
    if (f->capture_stream == nullptr)
      MPCHOL_CUDA_TRY(cudaStreamCreateWithFlags(&f->capture_stream, cudaStreamNonBlocking));
    long long before[MPCHOL_NPHASES];
    launch_counts(before);
    bool ok = cudaStreamBeginCapture(f->capture_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      const mpchol_status st = enqueue_factor(f, f->capture_stream, plan, hA, lda, hA_dev);
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(f->capture_stream, &graph);
      ok = st == MPCHOL_OK && ce == cudaSuccess && cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
    }
    long long after[MPCHOL_NPHASES];
    launch_counts(after);
    for (int i = 0; i < MPCHOL_NPHASES; ++i) g.nk[i] = after[i] - before[i];
    add_launch_counts(g.nk, -1);   // nothing ran during capture
    if (!ok) {
      cudaGetLastError();
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
      g.failed = true;
      return enqueue_factor(f, stream, plan, hA, lda, hA_dev);
    }
  }
  MPCHOL_CUDA_TRY(cudaGraphLaunch(g.exec, stream));
  add_launch_counts(g.nk, 1);
  f->solve_ready = false;
  return MPCHOL_OK;
}

mpchol_status ensure_solve(mpchol_factor_t* f, cudaStream_t stream) {
  if (f->solve_ready) return MPCHOL_OK;
  PHASE(MPCHOL_PH_SETUP, solve_setup_launches(f->n), stream,
        launch_solve_setup(f->A, f->ld, f->n, f->wsup, stream));
  f->solve_ready = true;
  return MPCHOL_OK;
}

// kernels per triangular solve: the input preparation, the persistent solve
int trsv_launch_count(int n) {
  (void)n;
  return 2;
}

// z = M^-1 r for NR-padded vectors (tmp, work: n x nr scratch)
mpchol_status apply_precond(mpchol_factor_t* f, const double* r, double* tmp, double* z, int nr,
                            const int* skip, cudaStream_t stream) {
  double* work = f->vec + 7 * (size_t)f->n * 8;
  const int nk = trsv_launch_count(f->n);
  PHASE(MPCHOL_PH_TRSV, nk, stream,
        launch_trsv_persistent(false, f->A, f->ld, f->n, f->wsup, r, tmp, work, nr, f->trsv_ctr,
                               skip, f->pstatus, stream));
  PHASE(MPCHOL_PH_TRSV, nk, stream,
        launch_trsv_persistent(true, f->A, f->ld, f->n, f->wsup, tmp, z, work, nr, f->trsv_ctr,
                               skip, f->pstatus, stream));
  return MPCHOL_OK;
}

int read_status(const DevStatus* src, cudaStream_t stream, DevStatus* out) {
  if (cudaMemcpyAsync(out, src, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
    return -1;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
  return 0;
}

template <typename TA>
mpchol_status run_pcg(mpchol_factor_t* f, const TA* dA, int lda, const double* dB, double* dX,
                      int nrhs, const mpchol_pcg_opts* popts, mpchol_report* rep,
                      cudaStream_t stream) {
  if (f == nullptr || dA == nullptr || dB == nullptr || dX == nullptr) return MPCHOL_ERR_BAD_ARG;
  if (nrhs < 1 || nrhs > 8 || lda < f->n) return MPCHOL_ERR_BAD_ARG;
  mpchol_pcg_opts po;
  mpchol_pcg_opts_default(&po);
  if (popts) po = *popts;
  if (po.check_every < 1) po.check_every = 1;
  if (po.max_it < 0) return MPCHOL_ERR_BAD_ARG;
  const int n = f->n;
  const int nr = pcg_padded_nrhs(nrhs);
  const size_t nv = (size_t)n * 8;
  double* x = f->vec;
  double* r = x + nv;
  double* z = r + nv;
  double* p = z + nv;
  double* Ap = p + nv;
  double* bb = Ap + nv;
  double* tmp = bb + nv;
  const int VG = pcg_vgrid();
  double* part_pAp = f->partials;
  double* part_rr = part_pAp + (size_t)VG * 8;
  double* part_rz = part_rr + (size_t)VG * 8;
  double* part_misc = part_rz + (size_t)VG * 8;
  // shares of ||A||_F^2 (for the backward error), filled by the first
  // operator product when it streams A through the staged kernel
  double* part_fro = part_misc + (size_t)VG * 8;
  const bool fro_fused = symv_staged_ok(dA, lda);
  double* rho[2] = {f->scal, f->scal + 8};
  double* alpha = f->scal + 16;
  double* bnorm2 = f->scal + 24;
  double* misc = f->scal + 32;   // [0..7] rr true, [8..15] xnorm2, [16] frob2
  mpchol_status ss = ensure_solve(f, stream);
  if (ss != MPCHOL_OK) return ss;
  MPCHOL_CUDA_TRY(cudaMemsetAsync(f->pstatus, 0, sizeof(DevStatus), stream));
  MPCHOL_CUDA_TRY(cudaMemsetAsync(f->done, 0, 2 * sizeof(int), stream));
  PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_pad_columns(dB, n, nrhs, bb, nr, stream));
  PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_dot(bb, bb, n, nr, part_misc, nullptr, stream));
  PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_misc, bnorm2, nr, stream));
  // x0
  if (po.x0_precond) {
    mpchol_status s0 = apply_precond(f, bb, tmp, x, nr, nullptr, stream);
    if (s0 != MPCHOL_OK) return s0;
  } else {
    MPCHOL_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)n * nr, stream));
  }
  const double tol2 = po.rel_tol * po.rel_tol;
  int it = 0;         // iterations executed on the device
  int launched = 0;   // iterations counted against max_it (the direct path also counts
                      // iterations enqueued past convergence, which return at once)
  bool converged = false;
  const int max_restarts = 3;
  for (int restart = 0;; ++restart) {
    // r = b - A x ; z = M^-1 r ; p = z ; rho = r^T z
    PHASE(MPCHOL_PH_SYMV, 1, stream, launch_symv_skip<TA>(dA, lda, n, x, Ap, nr, nullptr, stream,
                                                          fro_fused ? part_fro : nullptr, VG));
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_residual(bb, Ap, r, n, nr, part_rr, stream));
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_rr, misc, nr, stream));
    // convergence of the true residual
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_scal, misc, sizeof(double) * 8, cudaMemcpyDeviceToHost, stream));
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_scal + 8, bnorm2, sizeof(double) * 8, cudaMemcpyDeviceToHost, stream));
    // the factorization's status rides along with the first check: a failed
    // factor (NOT_SPD, TIMEOUT) is not iterated with
    if (restart == 0)
      MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_scal + 48, f->status, sizeof(DevStatus),
                                      cudaMemcpyDeviceToHost, stream));
    MPCHOL_CUDA_TRY(cudaStreamSynchronize(stream));
    if (restart == 0) {
      DevStatus fst;
      memcpy(&fst, f->h_scal + 48, sizeof(DevStatus));
      if (fst.code != 0) {
        if (rep != nullptr) memset(rep, 0, sizeof(*rep));
        return (mpchol_status)fst.code;
      }
    }
    converged = true;
    for (int k = 0; k < nrhs; ++k)
      if (!(f->h_scal[k] <= tol2 * f->h_scal[8 + k])) converged = false;
    if (converged || launched >= po.max_it || restart > max_restarts) break;
    mpchol_status s1 = apply_precond(f, r, tmp, z, nr, nullptr, stream);
    if (s1 != MPCHOL_OK) return s1;
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_copy(z, p, n, nr, stream));
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_dot(r, z, n, nr, part_rz, nullptr, stream));
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_rz, rho[0], nr, stream));
    MPCHOL_CUDA_TRY(cudaMemsetAsync(f->done, 0, sizeof(int), stream));
    // One PCG iteration; rho[cur] is the current r^T z, rho[cur^1] receives
    // the next one.  Every kernel returns at once after *done is set.
    auto iteration = [&](int cur, cudaStream_t s) -> mpchol_status {
      PHASE(MPCHOL_PH_SYMV, 2, s, launch_symv_skip<TA>(dA, lda, n, p, Ap, nr, f->done, s));
      PHASE(MPCHOL_PH_PCG_VEC, 1, s, launch_dot(p, Ap, n, nr, part_pAp, f->done, s));
      PHASE(MPCHOL_PH_PCG_VEC, 1, s, launch_update_xr(x, r, p, Ap, n, nr, part_pAp, rho[cur], alpha, part_rr,
                                  f->done, f->pstatus, s));
      mpchol_status s2 = apply_precond(f, r, tmp, z, nr, f->done, s);
      if (s2 != MPCHOL_OK) return s2;
      PHASE(MPCHOL_PH_PCG_VEC, 1, s, launch_dot(r, z, n, nr, part_rz, f->done, s));
      PHASE(MPCHOL_PH_PCG_VEC, 1, s, launch_update_p(p, z, n, nr, part_rz, rho[cur], rho[cur ^ 1], part_rr,
                                 bnorm2, tol2, f->done, f->done, f->done + 1, s));
      return MPCHOL_OK;
    };
    // The iterations run in a device-side loop: one launch of a CUDA graph
    // whose WHILE node repeats one iteration until the recursive residual
    // meets the tolerance, an error is recorded or the budget is spent, with
    // no host round trip in between.  Captured once per operator / rhs
    // count / tolerance.
    PcgGraph& g = f->graph;
    bool use_graph = !profiling_on() && !g.failed;
    if (use_graph && (g.exec == nullptr || g.A != (const void*)dA || g.lda != lda || g.nr != nr ||
                      g.elem != (int)sizeof(TA) || g.tol2 != tol2)) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
      // capture on a private stream (the caller's may be the legacy default
      // stream, which cannot be captured); the graph is launched into the
      // caller's stream
      if (f->capture_stream == nullptr)
        MPCHOL_CUDA_TRY(cudaStreamCreateWithFlags(&f->capture_stream, cudaStreamNonBlocking));
      long long before[MPCHOL_NPHASES];
      launch_counts(before);
      cudaGraph_t graph = nullptr;
      cudaGraphConditionalHandle handle = 0;
      cudaGraphNodeParams cp = {};
      cudaGraphNode_t node = nullptr;
      bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
                cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault) ==
                    cudaSuccess;
      if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
      }
      if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(f->capture_stream, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
          const mpchol_status s0 = iteration(0, f->capture_stream);
          const bool cond_ok =
              s0 == MPCHOL_OK && launch_pcg_loop_cond(handle, f->loop_ctl, f->done, f->pstatus,
                                                      f->scal, nr, f->capture_stream) == cudaSuccess;
          cudaGraph_t captured = nullptr;
          const cudaError_t ce = cudaStreamEndCapture(f->capture_stream, &captured);
          ok = cond_ok && ce == cudaSuccess && cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess;
        }
      }
      if (graph) cudaGraphDestroy(graph);
      long long after[MPCHOL_NPHASES];
      launch_counts(after);
      for (int i = 0; i < MPCHOL_NPHASES; ++i) g.nk[i] = after[i] - before[i];
      add_launch_counts(g.nk, -1);   // nothing ran during capture
      g.nk[MPCHOL_PH_PCG_VEC] += 1;  // the loop condition kernel
      if (!ok) {
        cudaGetLastError();            // the refusal is not an error of this call
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.failed = true;
        use_graph = false;
      } else {
        g.A = dA; g.lda = lda; g.nr = nr; g.elem = (int)sizeof(TA); g.tol2 = tol2;
      }
    }
    if (use_graph) {
      PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_pcg_loop_init(f->loop_ctl, po.max_it - launched, stream));
      MPCHOL_CUDA_TRY(cudaGraphLaunch(g.exec, stream));
      MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_done, f->done, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
      DevStatus st;
      MPCHOL_CUDA_TRY(cudaMemcpyAsync(&st, f->pstatus, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
      MPCHOL_CUDA_TRY(cudaStreamSynchronize(stream));
      if (st.code == MPCHOL_ERR_TIMEOUT) return MPCHOL_ERR_TIMEOUT;
      add_launch_counts(g.nk, f->h_done[1] - it);
      it = f->h_done[1];                // iterations actually executed on the device
      launched = it;
      continue;                         // the true residual decides (residual replacement restart)
    }
    int cur = 0;
    bool stop = false;
    while (launched < po.max_it && !stop) {
      const int chunk = std::min(po.check_every, po.max_it - launched);
      for (int c = 0; c < chunk; ++c) {
        mpchol_status s3 = iteration(cur, stream);
        if (s3 != MPCHOL_OK) return s3;
        cur ^= 1;
      }
      launched += chunk;
      MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_done, f->done, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
      DevStatus st;
      MPCHOL_CUDA_TRY(cudaMemcpyAsync(&st, f->pstatus, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
      MPCHOL_CUDA_TRY(cudaStreamSynchronize(stream));
      if (st.code == MPCHOL_ERR_TIMEOUT) return MPCHOL_ERR_TIMEOUT;
      it = f->h_done[1];                // iterations actually executed on the device
      if (f->h_done[0]) stop = true;    // recursive residual met the tolerance
      if (st.code == MPCHOL_PCG_BREAKDOWN) stop = true;
    }
    // the loop exits on max_it or when the recursive residual says done; the
    // next pass re-checks the true residual (residual replacement restart)
  }
  // report
  DevStatus st;
  if (read_status(f->pstatus, stream, &st) != 0) return MPCHOL_ERR_CUDA;
  MPCHOL_CUDA_TRY(cudaMemcpy2DAsync(dX, sizeof(double) * n, x, sizeof(double) * n,
                                    sizeof(double) * n, nrhs, cudaMemcpyDeviceToDevice, stream));
  if (rep != nullptr) {
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_dot(x, x, n, nr, part_misc, nullptr, stream));
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_misc, misc + 8, nr, stream));
    if (fro_fused) {
      PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_fro, misc + 16, 1, stream));
    } else {
      PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_frob_lower<TA>(dA, lda, n, part_misc, stream));
      PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_misc, misc + 16, 1, stream));
    }
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_dot(r, z, n, nr, part_rz, nullptr, stream));
    PHASE(MPCHOL_PH_PCG_VEC, 1, stream, launch_reduce_partials(part_rz, misc + 24, nr, stream));
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_scal, misc, sizeof(double) * 32, cudaMemcpyDeviceToHost, stream));
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->h_scal + 32, bnorm2, sizeof(double) * 8, cudaMemcpyDeviceToHost, stream));
    MPCHOL_CUDA_TRY(cudaStreamSynchronize(stream));
    double relmax = 0.0, bemax = 0.0, prmax = 0.0;
    const double frob = sqrt(f->h_scal[16]);
    for (int k = 0; k < nrhs; ++k) {
      const double rr = f->h_scal[k], xx = f->h_scal[8 + k], bb2 = f->h_scal[32 + k];
      const double rel = bb2 > 0 ? sqrt(rr / bb2) : sqrt(rr);
      const double be = sqrt(rr) / (frob * sqrt(xx) + sqrt(bb2));
      const double pr = bb2 > 0 ? sqrt(fabs(f->h_scal[24 + k]) / bb2) : 0.0;
      relmax = std::max(relmax, rel);
      bemax = std::max(bemax, be);
      prmax = std::max(prmax, pr);
    }
    rep->iterations = it;
    rep->converged = converged ? 1 : 0;
    rep->rel_residual = relmax;
    rep->backward_error = bemax;
    rep->precond_residual = prmax;
  }
  if (st.code == MPCHOL_PCG_BREAKDOWN) return MPCHOL_PCG_BREAKDOWN;
  if (st.code != 0) return (mpchol_status)st.code;
  return converged ? MPCHOL_OK : MPCHOL_PCG_MAXIT;
}

// ---- factor blobs (mpchol_factor_save / _load / _blob_check) --------------
struct FactorBlobHeader {
  char magic[8];               // "MPCHOLF1"
  uint32_t version;            // 1
  uint32_t header_bytes;       // sizeof(FactorBlobHeader)
  int32_t n, b, nsteps;
  uint32_t step_bytes;         // sizeof(StepState)
  uint64_t l_bytes;            // L's lower block columns, packed
  uint64_t total_bytes;        // header + payload
  uint64_t checksum;           // blob_hash of the payload
  uint64_t reserved;
};
static_assert(sizeof(FactorBlobHeader) == 64, "the blob header is 64 bytes");
constexpr char kBlobMagic[8] = {'M', 'P', 'C', 'H', 'O', 'L', 'F', '1'};

// Bytes of the lower block columns of an n x n matrix with block b: each
// block column from its diagonal down.
uint64_t blob_l_bytes(int n, int b) {
  uint64_t t = 0;
  for (int64_t c = 0; c < n; c += b) t += (uint64_t)(n - c) * std::min<int64_t>(b, n - c) * sizeof(float);
  return t;
}
uint64_t blob_total_bytes(int n, int b, int nsteps) {
  return sizeof(FactorBlobHeader) + blob_l_bytes(n, b) + (uint64_t)(nsteps + 1) * sizeof(StepState) +
         2 * (uint64_t)n * sizeof(float) + sizeof(DevStatus);
}
// 64-bit FNV-1a over little-endian 8-byte words (the tail zero-padded).
uint64_t blob_hash(const unsigned char* p, size_t len) {
  uint64_t h = 0xcbf29ce484222325ull;
  size_t i = 0;
  for (; i + 8 <= len; i += 8) {
    uint64_t w;
    memcpy(&w, p + i, 8);
    h = (h ^ w) * 0x100000001b3ull;
  }
  if (i < len) {
    uint64_t w = 0;
    memcpy(&w, p + i, len - i);
    h = (h ^ w) * 0x100000001b3ull;
  }
  return h;
}
// Host <-> device copies of a factor's state in blob order; `host` points
// just past the header.
cudaError_t blob_copy(mpchol_factor_t* f, unsigned char* host, bool to_host, cudaStream_t s) {
  const int n = f->n, b = f->b;
  const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
  unsigned char* p = host;
  for (int c = 0; c < n; c += b) {
    const int w = std::min(b, n - c);
    const size_t col = sizeof(float) * (n - c);
    float* dev = f->A + (size_t)c * f->ld + c;
    cudaError_t e = to_host
        ? cudaMemcpy2DAsync(p, col, dev, sizeof(float) * f->ld, col, w, kind, s)
        : cudaMemcpy2DAsync(dev, sizeof(float) * f->ld, p, col, col, w, kind, s);
    if (e != cudaSuccess) return e;
    p += col * w;
  }
  struct Part { void* dev; size_t bytes; };
  const Part parts[] = {{f->steps, sizeof(StepState) * (f->nsteps + 1)},
                        {f->d, sizeof(float) * n},
                        {f->dtilde, sizeof(float) * n},
                        {f->status, sizeof(DevStatus)}};
  for (const Part& q : parts) {
    cudaError_t e = to_host ? cudaMemcpyAsync(p, q.dev, q.bytes, kind, s)
                            : cudaMemcpyAsync(q.dev, p, q.bytes, kind, s);
    if (e != cudaSuccess) return e;
    p += q.bytes;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

const char* mpchol_status_str(int s) {
  switch (s) {
    case MPCHOL_OK: return "ok";
    case MPCHOL_ERR_BAD_ARG: return "bad argument";
    case MPCHOL_ERR_NOT_SPD: return "matrix not positive definite (non-positive pivot)";
    case MPCHOL_ERR_CUDA: return "CUDA runtime error";
    case MPCHOL_ERR_ALLOC: return "device allocation failed";
    case MPCHOL_PCG_MAXIT: return "PCG reached max_it without converging";
    case MPCHOL_PCG_BREAKDOWN: return "PCG breakdown (p^T A p <= 0 or not finite)";
    case MPCHOL_ERR_TIMEOUT: return "bounded device wait timed out";
    case MPCHOL_ERR_NOT_SUPPORTED: return "option combination not supported";
    default: return "unknown status";
  }
}

void mpchol_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_prof.mu);
  g_prof.on = on != 0;
}

mpchol_status mpchol_profile_read(mpchol_profile* out, int reset) {
  if (out == nullptr) return MPCHOL_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_prof.mu);
  memset(out, 0, sizeof(*out));
  for (const ProfRec& r : g_prof.recs) {
    if (cudaEventSynchronize(r.b) != cudaSuccess) return MPCHOL_ERR_CUDA;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) return MPCHOL_ERR_CUDA;
    out->ms[r.phase] += ms;
    out->calls[r.phase] += 1;
  }
  {
    std::lock_guard<std::mutex> lk2(g_launch_mu);
    for (int i = 0; i < MPCHOL_NPHASES; ++i) out->launches[i] = g_launches[i];
  }
  if (reset) {
    g_prof.recs.clear();
    g_prof.next = 0;
  }
  return MPCHOL_OK;
}

long long mpchol_kernel_launches(void) {
  std::lock_guard<std::mutex> lk(g_launch_mu);
  long long t = 0;
  for (int i = 0; i < MPCHOL_NPHASES; ++i) t += g_launches[i];
  return t;
}

const char* mpchol_last_error(void) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  static thread_local std::string copy;
  copy = g_last_err;
  return copy.c_str();
}

void mpchol_opts_default(mpchol_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->block_size = 256;
  o->precision = MPCHOL_PREC_SWITCHING;
  o->eps_prime = 0.5f;
  o->floor = 0.0f;
  o->diag_pert = 1;
  o->pert = 1.0f;
  o->pivot_floor = 1e-7f;
  o->switch_mode = 0;
  o->ladder_len = 3;
  o->ladder[0] = MPCHOL_PREC_E4M3;
  o->ladder[1] = MPCHOL_PREC_FP16;
  o->ladder[2] = MPCHOL_PREC_FP32;
  o->ladder[3] = MPCHOL_PREC_FP32;
  o->left = 0;
  o->coherence = 1;
  o->equilibrate = 0;
  o->eps_coherence = 0.0f;
}

void mpchol_pcg_opts_default(mpchol_pcg_opts* o) {
  if (!o) return;
  o->rel_tol = 1e-10;
  o->max_it = 200;
  o->x0_precond = 1;
  o->check_every = 4;
}

mpchol_status mpchol_factor_create(const mpchol_opts* opts, int n, mpchol_factor_t** out) {
  if (out == nullptr) return MPCHOL_ERR_BAD_ARG;
  *out = nullptr;
  mpchol_status v = validate_opts(opts, n);
  if (v != MPCHOL_OK) return v;
  mpchol_factor_t* f = new mpchol_factor_t();
  f->opts = *opts;
  f->n = n;
  f->ld = (n + 31) / 32 * 32;
  f->b = opts->block_size;
  f->nsteps = (n + f->b - 1) / f->b;
  cudaGetDevice(&f->device);
  const size_t nv = (size_t)n * 8;
  bool ok = dmalloc(&f->A, (size_t)f->ld * n) == cudaSuccess &&
            dmalloc(&f->d, n) == cudaSuccess && dmalloc(&f->dtilde, n) == cudaSuccess &&
            dmalloc(&f->rowsq, n) == cudaSuccess && dmalloc(&f->sh, n) == cudaSuccess &&
            dmalloc(&f->winv, (size_t)8 * 32 * 32) == cudaSuccess &&
            dmalloc(&f->scratch64, potrf_scratch64_elems(256)) == cudaSuccess &&
            dmalloc(&f->q8, (size_t)3 * n * f->b) == cudaSuccess &&
            dmalloc(&f->q16, (size_t)2 * n * f->b) == cudaSuccess &&
            dmalloc(&f->rexp, (size_t)3 * n) == cudaSuccess &&
            dmalloc(&f->mxexp, (size_t)n * (f->b / 32)) == cudaSuccess &&
            dmalloc(&f->steps, f->nsteps + 1) == cudaSuccess &&
            dmalloc(&f->status, 1) == cudaSuccess && dmalloc(&f->pstatus, 1) == cudaSuccess &&
            dmalloc(&f->colacc, (size_t)f->nsteps * kColCopies * f->b) == cudaSuccess &&
            dmalloc(&f->eqexp, n) == cudaSuccess &&
            dmalloc(&f->wsup, solve_wsup_elems(n)) == cudaSuccess &&
            dmalloc(&f->trsv_ctr, trsv_counter_ints(n)) == cudaSuccess &&
            dmalloc(&f->vec, 8 * nv) == cudaSuccess &&
            dmalloc(&f->partials, (size_t)5 * pcg_vgrid() * 8) == cudaSuccess &&
            dmalloc(&f->scal, 64) == cudaSuccess && dmalloc(&f->done, 2) == cudaSuccess &&
            dmalloc(&f->loop_ctl, 2) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&f->h_done), 2 * sizeof(int)) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&f->h_scal), sizeof(double) * 64) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_factor(f);
    return MPCHOL_ERR_ALLOC;
  }
  if (opts->left) {
    // the quantized panels of every step (the left-looking schedule applies
    // each panel to the later block columns one at a time)
    const size_t nbq = (size_t)n * f->b;
    const int hist = f->nsteps;
    if (dmalloc(&f->hq8, (size_t)hist * 3 * nbq) != cudaSuccess ||
        dmalloc(&f->hq16, (size_t)hist * 2 * nbq) != cudaSuccess ||
        dmalloc(&f->hrexp, (size_t)hist * 3 * n) != cudaSuccess ||
        dmalloc(&f->hmx, (size_t)hist * (nbq / 32)) != cudaSuccess) {
      cudaGetLastError();
      free_factor(f);
      return MPCHOL_ERR_ALLOC;
    }
    f->hist_steps = hist;
  }
  if (solve_init_attributes() != cudaSuccess) {
    free_factor(f);
    return MPCHOL_ERR_CUDA;
  }
  // TMA maps over the factor's own storage (rows past n read as zeros and are
  // never written)
  if (!encode_tmap_2d(&f->tmap32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, f->A, n, n, f->ld, 32, 32,
                      CU_TENSOR_MAP_SWIZZLE_NONE) ||
      !encode_tmap_2d(&f->tmapX, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, f->A, n, n, f->ld, 32,
                      f->b, CU_TENSOR_MAP_SWIZZLE_NONE)) {
    free_factor(f);
    return MPCHOL_ERR_CUDA;
  }
  *out = f;
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_compute(mpchol_factor_t* f, const float* dA, int lda,
                                    mpchol_stream_t stream) {
  if (f == nullptr || dA == nullptr || lda < f->n) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  MPCHOL_CUDA_TRY(copy_lower_blocks(f->A, f->ld, dA, lda, f->n, f->b, cudaMemcpyDeviceToDevice, s));
  return launch_factor(f, s);
}

mpchol_status mpchol_factor_codes(const mpchol_factor_t* f, int fmt, const void** dCodes,
                                  const void** dScales, int* ldq, int* rows, int* col0) {
  if (f == nullptr || dCodes == nullptr || dScales == nullptr || ldq == nullptr ||
      rows == nullptr || col0 == nullptr)
    return MPCHOL_ERR_BAD_ARG;
  if (f->nsteps < 2) return MPCHOL_ERR_BAD_ARG;          // no trailing update
  if (fmt != FP16 && fmt != FP16X2 && fmt != E4M3 && fmt != E5M2 && !is_mx(fmt))
    return MPCHOL_ERR_BAD_ARG;
  const int s = (f->nsteps - 2) * f->b;                   // the last step with trailing rows
  const size_t nb = (size_t)f->n * f->b;
  // the left-looking schedule keeps every step's codes in the panel history
  const int ks = f->nsteps - 2;
  const bool hist = f->opts.left && ks < f->hist_steps;
  const uint8_t* q8 = hist ? f->hq8 + (size_t)ks * 3 * nb : f->q8;
  const uint16_t* q16 = hist ? f->hq16 + (size_t)ks * 2 * nb : f->q16;
  const int8_t* rexp = hist ? f->hrexp + (size_t)ks * 3 * f->n : f->rexp;
  const uint8_t* mx = hist ? f->hmx + (size_t)ks * (nb / 32) : f->mxexp;
  if (fmt == FP16 || fmt == FP16X2) {
    *dCodes = q16;
    *dScales = rexp + 2 * (size_t)f->n;
  } else {
    *dCodes = q8 + q8_slot(fmt) * nb;
    *dScales = is_mx(fmt) ? static_cast<const void*>(mx)
                            : static_cast<const void*>(rexp + (size_t)rexp_slot(fmt) * f->n);
  }
  *ldq = f->b;
  *rows = f->n - s - f->b;
  *col0 = s;
  return MPCHOL_OK;
}

mpchol_status mpchol_solve_host(mpchol_factor_t* f, const float* hA, int lda, const double* hB,
                                double* hX, int nrhs, const mpchol_pcg_opts* opts,
                                mpchol_report* rep, mpchol_stream_t stream) {
  if (f == nullptr || hA == nullptr || hB == nullptr || hX == nullptr || lda < f->n ||
      nrhs < 1 || nrhs > 8)
    return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int n = f->n, b = f->b;
  if (f->op == nullptr) {
    MPCHOL_CUDA_TRY(dmalloc(&f->op, (size_t)f->ld * n));
    MPCHOL_CUDA_TRY(dmalloc(&f->hb, (size_t)n * 8));
    MPCHOL_CUDA_TRY(dmalloc(&f->hx, (size_t)n * 8));
  }
  if (f->plan_mode < 0 && f->plan.c1[0] == 0) {
    // equilibration scales A's lower triangle in one pass before step 0, and
    // the left-looking schedule has no trailing updates for late block
    // columns to join: the copy does not overlap the factorization then
    if (f->opts.equilibrate || f->opts.left) {
      f->plan = CopyPlan{};
      f->plan.c1[0] = f->nsteps;
    } else {
      f->plan = choose_copy_plan(n, b);
    }
  }
  const CopyPlan& plan = f->plan;
  if (plan.ng <= 1) {
    MPCHOL_CUDA_TRY(copy_lower_blocks(f->op, f->ld, hA, lda, n, b, cudaMemcpyHostToDevice, s));
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->hb, hB, sizeof(double) * n * nrhs, cudaMemcpyHostToDevice, s));
    MPCHOL_CUDA_TRY(copy_lower_blocks(f->A, f->ld, f->op, f->ld, n, b, cudaMemcpyDeviceToDevice, s));
    mpchol_status st = launch_factor(f, s);
    if (st != MPCHOL_OK) return st;
  } else {
    if (f->cp == nullptr) {
      MPCHOL_CUDA_TRY(cudaStreamCreateWithFlags(&f->cp, cudaStreamNonBlocking));
      for (cudaEvent_t& e : f->ev_grp) MPCHOL_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      MPCHOL_CUDA_TRY(cudaEventCreateWithFlags(&f->ev_start, cudaEventDisableTiming));
      MPCHOL_CUDA_TRY(cudaEventCreateWithFlags(&f->ev_diag, cudaEventDisableTiming));
      MPCHOL_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&f->h_diag), sizeof(float) * n));
    }
    // panel history for the steps that late groups catch up with
    const int hist = plan.join[plan.ng - 1];
    if (hist > f->hist_steps) {
      for (void* p : {(void*)f->hq8, (void*)f->hq16, (void*)f->hrexp, (void*)f->hmx})
        if (p) MPCHOL_CUDA_TRY(cudaFree(p));
      f->hq8 = nullptr; f->hq16 = nullptr; f->hrexp = nullptr; f->hmx = nullptr;
      f->hist_steps = 0;
      const size_t nbq = (size_t)n * b;
      MPCHOL_CUDA_TRY(dmalloc(&f->hq8, (size_t)hist * 3 * nbq));
      MPCHOL_CUDA_TRY(dmalloc(&f->hq16, (size_t)hist * 2 * nbq));
      MPCHOL_CUDA_TRY(dmalloc(&f->hrexp, (size_t)hist * 3 * n));
      MPCHOL_CUDA_TRY(dmalloc(&f->hmx, (size_t)hist * (nbq / 32)));
      f->hist_steps = hist;
    }
    // The copies wait for earlier work on the caller's stream (which may
    // still read the operator and the factor).  A page-locked A is read by
    // the device directly for its diagonal; for pageable memory the host
    // gathers it (after the previous call's copy of it has finished).
    const float* hA_dev = nullptr;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, hA) == cudaSuccess && pa.type == cudaMemoryTypeHost &&
        pa.devicePointer != nullptr)
      hA_dev = static_cast<const float*>(pa.devicePointer);
    cudaGetLastError();
    if (hA_dev == nullptr) {
      MPCHOL_CUDA_TRY(cudaEventSynchronize(f->ev_diag));
      for (int i = 0; i < n; ++i) f->h_diag[i] = hA[(size_t)i * lda + i];
    }
    MPCHOL_CUDA_TRY(cudaMemcpyAsync(f->hb, hB, sizeof(double) * n * nrhs, cudaMemcpyHostToDevice, s));
    mpchol_status st = launch_factor(f, s, &plan, hA, lda, hA_dev);
    if (st != MPCHOL_OK) return st;
    MPCHOL_CUDA_TRY(cudaEventRecord(f->ev_diag, s));
  }
  mpchol_status st = run_pcg<float>(f, f->op, f->ld, f->hb, f->hx, nrhs, opts, rep, s);
  if (st != MPCHOL_OK && st != MPCHOL_PCG_MAXIT) return st;
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(hX, f->hx, sizeof(double) * n * nrhs, cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  return st;
}

mpchol_status mpchol_set_copy_plan(mpchol_factor_t* f, int ngroups, const int* cuts,
                                   const int* join) {
  if (f == nullptr) return MPCHOL_ERR_BAD_ARG;
  if (ngroups <= 0) {           // automatic
    f->plan_mode = -1;
    f->plan = CopyPlan{};
    return MPCHOL_OK;
  }
  const int nb = f->nsteps;
  CopyPlan p;
  p.ng = ngroups;
  if (ngroups > kMaxGroups || (ngroups > 1 && (cuts == nullptr || join == nullptr)))
    return MPCHOL_ERR_BAD_ARG;
  if (ngroups > 1 && (f->b % 128 != 0 || f->opts.equilibrate || f->opts.left))
    return MPCHOL_ERR_NOT_SUPPORTED;
  p.c0[0] = 0;
  for (int g = 1; g < ngroups; ++g) {
    p.c1[g - 1] = cuts[g - 1];
    p.c0[g] = cuts[g - 1];
    p.join[g] = join[g - 1];
  }
  p.c1[ngroups - 1] = nb;
  if (!valid_copy_plan(p, nb)) return MPCHOL_ERR_BAD_ARG;
  f->plan = p;
  f->plan_mode = 1;
  return MPCHOL_OK;
}

int mpchol_copy_plan(int n, int block_size, int* cuts, int* join, int cap) {
  if (n <= 0 || block_size < 32 || block_size > 256 || block_size % 32 != 0) return 0;
  const CopyPlan p = choose_copy_plan(n, block_size);
  for (int g = 1; g < p.ng && g - 1 < cap; ++g) {
    if (cuts) cuts[g - 1] = p.c0[g];
    if (join) join[g - 1] = p.join[g];
  }
  return p.ng;
}

mpchol_status mpchol_factor(const mpchol_opts* opts, int n, const float* dA, int lda,
                            mpchol_factor_t** out, mpchol_stream_t stream) {
  mpchol_status s = mpchol_factor_create(opts, n, out);
  if (s != MPCHOL_OK) return s;
  s = mpchol_factor_compute(*out, dA, lda, stream);
  if (s != MPCHOL_OK) {
    free_factor(*out);
    *out = nullptr;
  }
  return s;
}

mpchol_status mpchol_factor_destroy(mpchol_factor_t* f) {
  if (f == nullptr) return MPCHOL_ERR_BAD_ARG;
  free_factor(f);
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_info_get(const mpchol_factor_t* fc, mpchol_factor_info* info,
                                     int* hStepPrec, int* hStepFp64, mpchol_stream_t stream) {
  mpchol_factor_t* f = const_cast<mpchol_factor_t*>(fc);
  if (f == nullptr || info == nullptr) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::vector<StepState> steps(f->nsteps + 1);
  DevStatus st;
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(steps.data(), f->steps, sizeof(StepState) * (f->nsteps + 1),
                                  cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaMemcpyAsync(&st, f->status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  memset(info, 0, sizeof(*info));
  info->status = st.code;
  info->fail_row = st.code == MPCHOL_ERR_NOT_SPD ? st.row : -1;
  info->n_perturbed = st.perturbed;
  info->nsteps = f->nsteps;
  for (int k = 0; k < f->nsteps; ++k) {
    const int m = f->n - k * f->b - std::min(f->b, f->n - k * f->b);
    const int p = m > 0 ? steps[k].prec : FP32;
    if (hStepPrec) hStepPrec[k] = p;
    if (hStepFp64) hStepFp64[k] = steps[k].fp64_diag;
    if (steps[k].fp64_diag) info->n_fp64_blocks++;
    if (m > 0 && p >= 0 && p < kNumFmts) info->steps_by_prec[p]++;
  }
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_lower(const mpchol_factor_t* f, const float** dL, int* ldl, int* n) {
  if (f == nullptr) return MPCHOL_ERR_BAD_ARG;
  if (dL) *dL = f->A;
  if (ldl) *ldl = f->ld;
  if (n) *n = f->n;
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_blob_check(const void* blob, size_t size, int* n, int* block_size) {
  if (blob == nullptr || size < sizeof(FactorBlobHeader)) return MPCHOL_ERR_BAD_ARG;
  FactorBlobHeader h;
  memcpy(&h, blob, sizeof(h));
  if (memcmp(h.magic, kBlobMagic, 8) != 0 || h.version != 1 ||
      h.header_bytes != sizeof(FactorBlobHeader) || h.step_bytes != sizeof(StepState))
    return MPCHOL_ERR_BAD_ARG;
  // bound n before any arithmetic on it (a hostile header must not overflow
  // the step count or make the size loop run away)
  if (h.n < 1 || h.n > MPCHOL_BLOB_MAX_N || h.b < 32 || h.b > 256 || h.b % 32 != 0 ||
      (int64_t)h.nsteps != ((int64_t)h.n + h.b - 1) / h.b)
    return MPCHOL_ERR_BAD_ARG;
  if (h.l_bytes != blob_l_bytes(h.n, h.b) || h.total_bytes != blob_total_bytes(h.n, h.b, h.nsteps) ||
      size < h.total_bytes)
    return MPCHOL_ERR_BAD_ARG;
  const unsigned char* p = static_cast<const unsigned char*>(blob);
  if (blob_hash(p + sizeof(h), h.total_bytes - sizeof(h)) != h.checksum) return MPCHOL_ERR_BAD_ARG;
  if (n) *n = h.n;
  if (block_size) *block_size = h.b;
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_save(const mpchol_factor_t* fc, void* blob, size_t cap, size_t* size,
                                 mpchol_stream_t stream) {
  mpchol_factor_t* f = const_cast<mpchol_factor_t*>(fc);
  if (f == nullptr || size == nullptr) return MPCHOL_ERR_BAD_ARG;
  const uint64_t total = blob_total_bytes(f->n, f->b, f->nsteps);
  *size = (size_t)total;
  if (blob == nullptr) return MPCHOL_OK;
  if (cap < total) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // a failed factorization is not saved
  DevStatus fst;
  if (read_status(f->status, s, &fst) != 0) return MPCHOL_ERR_CUDA;
  if (fst.code != 0) return (mpchol_status)fst.code;
  unsigned char* out = static_cast<unsigned char*>(blob);
  MPCHOL_CUDA_TRY(blob_copy(f, out + sizeof(FactorBlobHeader), true, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  FactorBlobHeader h{};
  memcpy(h.magic, kBlobMagic, 8);
  h.version = 1;
  h.header_bytes = sizeof(FactorBlobHeader);
  h.n = f->n;
  h.b = f->b;
  h.nsteps = f->nsteps;
  h.step_bytes = sizeof(StepState);
  h.l_bytes = blob_l_bytes(f->n, f->b);
  h.total_bytes = total;
  h.checksum = blob_hash(out + sizeof(h), total - sizeof(h));
  memcpy(out, &h, sizeof(h));
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_load(mpchol_factor_t* f, const void* blob, size_t size,
                                 mpchol_stream_t stream) {
  if (f == nullptr) return MPCHOL_ERR_BAD_ARG;
  int n = 0, b = 0;
  const mpchol_status st = mpchol_factor_blob_check(blob, size, &n, &b);
  if (st != MPCHOL_OK) return st;
  if (n != f->n || b != f->b) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned char* in = const_cast<unsigned char*>(static_cast<const unsigned char*>(blob));
  MPCHOL_CUDA_TRY(blob_copy(f, in + sizeof(FactorBlobHeader), false, s));
  MPCHOL_CUDA_TRY(cudaStreamSynchronize(s));
  f->solve_ready = false;
  // the saved status word is the blob's last field
  DevStatus fst;
  memcpy(&fst, in + sizeof(FactorBlobHeader) + (blob_total_bytes(n, b, f->nsteps) -
                                                sizeof(FactorBlobHeader) - sizeof(DevStatus)),
         sizeof(DevStatus));
  return (mpchol_status)fst.code;
}

mpchol_status mpchol_factor_diags(const mpchol_factor_t* f, const float** dD, const float** dDt) {
  if (f == nullptr) return MPCHOL_ERR_BAD_ARG;
  if (dD) *dD = f->d;
  if (dDt) *dDt = f->dtilde;
  return MPCHOL_OK;
}

mpchol_status mpchol_factor_prepare_solve(mpchol_factor_t* f, mpchol_stream_t stream) {
  if (f == nullptr) return MPCHOL_ERR_BAD_ARG;
  return ensure_solve(f, reinterpret_cast<cudaStream_t>(stream));
}

mpchol_status mpchol_pcg(mpchol_factor_t* f, const float* dA, int lda, const double* dB,
                         double* dX, int nrhs, const mpchol_pcg_opts* opts, mpchol_report* rep,
                         mpchol_stream_t stream) {
  return run_pcg<float>(f, dA, lda, dB, dX, nrhs, opts, rep, reinterpret_cast<cudaStream_t>(stream));
}

mpchol_status mpchol_pcg_f64(mpchol_factor_t* f, const double* dA, int lda, const double* dB,
                             double* dX, int nrhs, const mpchol_pcg_opts* opts,
                             mpchol_report* rep, mpchol_stream_t stream) {
  return run_pcg<double>(f, dA, lda, dB, dX, nrhs, opts, rep, reinterpret_cast<cudaStream_t>(stream));
}

mpchol_status mpchol_adjoint_solve(mpchol_factor_t* f, const double* dA, int lda,
                                   const double* dX, const double* dG, double* dLam, int nrhs,
                                   double* dGradA, int ldg, const mpchol_pcg_opts* opts,
                                   mpchol_report* rep, mpchol_stream_t stream) {
  if (f == nullptr || dA == nullptr || dX == nullptr || dG == nullptr || dLam == nullptr)
    return MPCHOL_ERR_BAD_ARG;
  if (nrhs < 1 || nrhs > 8 || lda < f->n || (dGradA != nullptr && ldg < f->n))
    return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // A symmetric: the adjoint system A^T lambda = g is the forward operator
  // with the cotangent as right-hand side, preconditioned by the same factor
  const mpchol_status st = run_pcg<double>(f, dA, lda, dG, dLam, nrhs, opts, rep, s);
  if (st != MPCHOL_OK && st != MPCHOL_PCG_MAXIT) return st;
  if (dGradA != nullptr)
    PHASE(MPCHOL_PH_PCG_VEC, 1, s, launch_sym_outer(dLam, dX, f->n, nrhs, dGradA, ldg, s));
  return st;
}

mpchol_status mpchol_apply_precond(mpchol_factor_t* f, const double* dR, double* dZ, int nrhs,
                                   mpchol_stream_t stream) {
  if (f == nullptr || dR == nullptr || dZ == nullptr || nrhs < 1 || nrhs > 8) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  mpchol_status ss = ensure_solve(f, s);
  if (ss != MPCHOL_OK) return ss;
  const int nr = pcg_padded_nrhs(nrhs);
  const size_t nv = (size_t)f->n * 8;
  double* rp = f->vec + 5 * nv;     // bb slot
  double* tmp = f->vec + 6 * nv;
  double* zp = f->vec + 2 * nv;     // z slot
  MPCHOL_CUDA_TRY(cudaMemsetAsync(f->pstatus, 0, sizeof(DevStatus), s));
  PHASE(MPCHOL_PH_PCG_VEC, 1, s, launch_pad_columns(dR, f->n, nrhs, rp, nr, s));
  ss = apply_precond(f, rp, tmp, zp, nr, nullptr, s);
  if (ss != MPCHOL_OK) return ss;
  MPCHOL_CUDA_TRY(cudaMemcpy2DAsync(dZ, sizeof(double) * f->n, zp, sizeof(double) * f->n,
                                    sizeof(double) * f->n, nrhs, cudaMemcpyDeviceToDevice, s));
  DevStatus st;
  if (read_status(f->pstatus, s, &st) != 0) return MPCHOL_ERR_CUDA;
  return (mpchol_status)st.code;
}

mpchol_status mpchol_symv(const float* dA, int lda, int n, const double* dX, double* dY, int nrhs,
                          mpchol_stream_t stream) {
  if (dA == nullptr || dX == nullptr || dY == nullptr || n <= 0 || lda < n) return MPCHOL_ERR_BAD_ARG;
  if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8) return MPCHOL_ERR_BAD_ARG;
  MPCHOL_CUDA_TRY(solve_init_attributes());
  PHASE(MPCHOL_PH_SYMV, 1, reinterpret_cast<cudaStream_t>(stream), launch_symv_skip<float>(dA, lda, n, dX, dY, nrhs, nullptr,
                                          reinterpret_cast<cudaStream_t>(stream)));
  return MPCHOL_OK;
}

int mpchol_precond_cg(double* dA, double* dX, double* dB, int n, int r, double normA,
                      float eps_prime, float flr, int perturb_diag, int microscal_size,
                      double rel_tol, int max_it, mpchol_stream_t stream) {
  (void)normA;
  (void)microscal_size;
  if (dA == nullptr || dX == nullptr || dB == nullptr || n <= 0) return -(100 + MPCHOL_ERR_BAD_ARG);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  mpchol_opts o;
  mpchol_opts_default(&o);
  o.block_size = r;
  o.eps_prime = eps_prime;
  o.floor = flr;
  o.diag_pert = perturb_diag ? 1 : 0;
  mpchol_factor_t* f = nullptr;
  mpchol_status st = mpchol_factor_create(&o, n, &f);
  if (st != MPCHOL_OK) return -(100 + st);
  // FP64 -> FP32 directly into the factor's storage (src/mixed_cholesky.cu:122)
  if (launch_f64_to_f32(dA, n, f->A, f->ld, n, s) != cudaSuccess) {
    free_factor(f);
    return -(100 + MPCHOL_ERR_CUDA);
  }
  st = run_factor(f, s);
  mpchol_factor_info info;
  if (st == MPCHOL_OK) st = mpchol_factor_info_get(f, &info, nullptr, nullptr, stream);
  if (st != MPCHOL_OK) { free_factor(f); return -(100 + st); }
  if (info.status == MPCHOL_ERR_NOT_SPD) { free_factor(f); return info.fail_row + 1; }
  if (info.status != MPCHOL_OK) { free_factor(f); return -(100 + info.status); }
  mpchol_pcg_opts po;
  mpchol_pcg_opts_default(&po);
  po.rel_tol = rel_tol;
  po.max_it = max_it;
  po.x0_precond = 1;
  st = run_pcg<double>(f, dA, n, dB, dX, 1, &po, nullptr, s);
  free_factor(f);
  if (st == MPCHOL_OK) return 0;
  if (st == MPCHOL_PCG_MAXIT) return -1;
  return -(100 + st);
}

int mpchol_switching_chol(float* dA, int n, int b, float* d_diagVals, float* updated_diag,
                          float eps_prime, int perturb_diag, int microscal_size,
                          mpchol_stream_t stream, uint8_t* scales) {
  (void)microscal_size;
  (void)scales;
  if (dA == nullptr || n <= 0) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  mpchol_opts o;
  mpchol_opts_default(&o);
  o.block_size = b;
  o.eps_prime = eps_prime;
  o.diag_pert = perturb_diag ? 1 : 0;
  mpchol_factor_t* f = nullptr;
  mpchol_status st = mpchol_factor(&o, n, dA, n, &f, stream);
  if (st != MPCHOL_OK) return st;
  mpchol_factor_info info;
  st = mpchol_factor_info_get(f, &info, nullptr, nullptr, stream);
  if (st == MPCHOL_OK) {
    if (cudaMemcpy2DAsync(dA, sizeof(float) * n, f->A, sizeof(float) * f->ld, sizeof(float) * n, n,
                          cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      st = MPCHOL_ERR_CUDA;
    if (d_diagVals && cudaMemcpyAsync(d_diagVals, f->d, sizeof(float) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      st = MPCHOL_ERR_CUDA;
    if (updated_diag && cudaMemcpyAsync(updated_diag, f->dtilde, sizeof(float) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      st = MPCHOL_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) st = MPCHOL_ERR_CUDA;
    if (st == MPCHOL_OK) st = (mpchol_status)info.status;
  }
  free_factor(f);
  return st;
}

mpchol_status mpchol_quantize(const float* dX, void* dQ, long long count, int fmt,
                              mpchol_stream_t stream) {
  if (count < 0 || (count > 0 && (dX == nullptr || dQ == nullptr))) return MPCHOL_ERR_BAD_ARG;
  if (fmt != FP16 && fmt != E4M3 && fmt != E5M2) return MPCHOL_ERR_BAD_ARG;
  PHASE(MPCHOL_PH_TEST, 1, reinterpret_cast<cudaStream_t>(stream), launch_quantize_elems(dX, dQ, count, fmt, reinterpret_cast<cudaStream_t>(stream)));
  return MPCHOL_OK;
}

mpchol_status mpchol_quantize_rows(const float* dP, int m, int k, int ldp, int fmt, void* dQ,
                                   void* dScale, mpchol_stream_t stream) {
  if (dP == nullptr || dQ == nullptr || dScale == nullptr || m < 0 || ldp < m) return MPCHOL_ERR_BAD_ARG;
  if (k < 32 || k > 256 || k % 32 != 0) return MPCHOL_ERR_BAD_ARG;
  if (fmt != FP16 && fmt != E4M3 && fmt != E5M2 && !is_mx(fmt) && fmt != FP16X2)
    return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (is_mx(fmt))
    PHASE(MPCHOL_PH_QUANT, 1, s, launch_quantize_rows(dP, ldp, m, k, fmt, dQ, k, nullptr,
                                         reinterpret_cast<uint8_t*>(dScale), k / 32, s));
  else
    PHASE(MPCHOL_PH_QUANT, 1, s, launch_quantize_rows(dP, ldp, m, k, fmt, dQ, k,
                                         reinterpret_cast<int8_t*>(dScale), nullptr, 0, s));
  return MPCHOL_OK;
}

mpchol_status mpchol_quantize_hash(unsigned long long first, unsigned long long count,
                                   unsigned long long chunk, int fmt, unsigned long long* dHash,
                                   mpchol_stream_t stream) {
  if (dHash == nullptr || chunk == 0 || first + count > (1ull << 32)) return MPCHOL_ERR_BAD_ARG;
  if (fmt != FP16 && fmt != E4M3 && fmt != E5M2) return MPCHOL_ERR_BAD_ARG;
  PHASE(MPCHOL_PH_TEST, 1, reinterpret_cast<cudaStream_t>(stream), launch_quantize_hash(first, count, chunk, fmt, dHash,
                                       reinterpret_cast<cudaStream_t>(stream)));
  return MPCHOL_OK;
}

mpchol_status mpchol_syrk_update(float* dC, int ldc, int m, int k, int fmt, const void* dQ,
                                 const void* dScale, const float* dP, int ldp,
                                 mpchol_stream_t stream) {
  if (dC == nullptr || m < 0 || ldc < m || k <= 0) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (fmt == FP32) {
    if (dP == nullptr || ldp < m) return MPCHOL_ERR_BAD_ARG;
    PHASE(MPCHOL_PH_SYRK_F32, 1, s, launch_syrk_f32(dC, ldc, m, k, dP, ldp, nullptr, nullptr, s));
    return MPCHOL_OK;
  }
  if (!syrk_tc_supported(fmt, k)) return MPCHOL_ERR_NOT_SUPPORTED;
  if (dQ == nullptr || dScale == nullptr) return MPCHOL_ERR_BAD_ARG;
  if (is_mx(fmt))
    PHASE(MPCHOL_PH_SYRK_TC, 1, s, launch_syrk_tc(dC, ldc, m, k, fmt, dQ, k, nullptr,
                                   reinterpret_cast<const uint8_t*>(dScale), k / 32, nullptr,
                                   nullptr, s));
  else
    PHASE(MPCHOL_PH_SYRK_TC, 1, s, launch_syrk_tc(dC, ldc, m, k, fmt, dQ, k,
                                   reinterpret_cast<const int8_t*>(dScale), nullptr, 0, nullptr,
                                   nullptr, s));
  return MPCHOL_OK;
}

mpchol_status mpchol_rbf_build(const float* dX, int n, int d, int ldx, double lengthscale,
                               double nugget, double* dK64, float* dK32, int ldk, int lower_only,
                               mpchol_stream_t stream) {
  if (dX == nullptr || (dK64 == nullptr && dK32 == nullptr)) return MPCHOL_ERR_BAD_ARG;
  if (n < 1 || d < 1 || ldx < d || ldk < n || !(lengthscale > 0.0) || !(nugget >= 0.0))
    return MPCHOL_ERR_BAD_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  PHASE(MPCHOL_PH_SETUP, 1, s, launch_rbf_build(dX, n, d, ldx, lengthscale, nugget, dK64, dK32, ldk,
                                                lower_only, s));
  return MPCHOL_OK;
}

int mpchol_rbf_grad_work_elems(int n) { return n > 0 ? rbf_grad_work_elems(n) : 0; }

mpchol_status mpchol_rbf_grad(const float* dX, int n, int d, int ldx, double lengthscale,
                              const double* dA, const double* dB, double* dP, double* dS,
                              double* dWork, mpchol_stream_t stream) {
  if (dX == nullptr || dA == nullptr || dB == nullptr || dP == nullptr || dS == nullptr ||
      dWork == nullptr)
    return MPCHOL_ERR_BAD_ARG;
  if (n < 1 || d < 1 || ldx < d || !(lengthscale > 0.0)) return MPCHOL_ERR_BAD_ARG;
  if (d > rbf_grad_max_features()) return MPCHOL_ERR_NOT_SUPPORTED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  PHASE(MPCHOL_PH_SETUP, 2, s, launch_rbf_grad(dX, n, d, ldx, lengthscale, dA, dB, dP, dS, dWork, s));
  return MPCHOL_OK;
}

}  // extern "C"
