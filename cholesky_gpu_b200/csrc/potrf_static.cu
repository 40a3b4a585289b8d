// mpchol_potrf_static: the diagonal-block POTRF of the factorization as a
// stand-alone call that allocates nothing.
//
// The factor objects own their workspaces (cudaMalloc'd at creation).  This
// entry point serves callers that cannot allocate device memory at the point
// of the call -- cudaMalloc and cudaFree synchronize the whole device, which
// stalls every other stream of a pipeline, and a process whose device memory
// is already handed to a caching allocator may have none left to give.  Its
// scratch is a file-scope static device array sized for the largest block the
// kernel factors (256 x 256): the original diagonal (pivot floors), the
// inverses of the eight 32 x 32 diagonal tiles, and the status word.  The
// kernel is the same one mpchol_factor_compute launches for a block, so the
// factor it returns equals that of mpchol_factor on the same input.
//
// One static scratch per device: calls that overlap in time on one device
// (different streams, different host threads) race on it; calls ordered on
// one stream do not.  The first call on each device looks up the scratch's
// address (one-time setup); the tensor-map encoder's driver entry point is
// also resolved on the library's first use.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg.cuh"
#include "tmap.cuh"

using namespace mpchol;

namespace {

constexpr int kMaxBlock = 256;              // MPCHOL_POTRF_STATIC_MAX in mpchol.h
constexpr int kMaxDevices = 64;

// Static scratch.  The status word must be zero when the kernel starts (the
// kernel records the first failure with a compare-and-swap against zero);
// every call clears it on its stream before the launch.
struct StaticScratch {
  DevStatus status;
  float diag[kMaxBlock];                    // original diagonal -> pivot floors
  float diag_copy[kMaxBlock];               // second output of the diagonal extraction
  float winv[kMaxBlock * 32];               // inverses of the 32 x 32 diagonal tiles
};
static __device__ __align__(256) StaticScratch g_scratch;

struct DeviceSlot {
  std::once_flag once;
  cudaError_t err = cudaSuccess;
  StaticScratch* addr = nullptr;
};
DeviceSlot g_slots[kMaxDevices];

__global__ void potrf_static_info_kernel(const DevStatus* st, int* info) {
  // cusolver-style devInfo: 0 on success, i + 1 when pivot i is not positive,
  // -1 for any other device-side error
  const int code = st->code;
  *info = code == 0 ? 0 : (code == MPCHOL_ERR_NOT_SPD ? st->row + 1 : -1);
}

}  // namespace

extern "C" MPCHOL_API mpchol_status mpchol_potrf_static(float* dA, int lda, int n,
                                                        float pivot_floor, int* dInfo,
                                                        mpchol_stream_t stream_) {
  // argument checks come before any CUDA call
  if (dA == nullptr || dInfo == nullptr) return MPCHOL_ERR_BAD_ARG;
  if (n < 1 || n > kMaxBlock || lda < n) return MPCHOL_ERR_BAD_ARG;
  if (!(pivot_floor >= 0.0f)) return MPCHOL_ERR_BAD_ARG;
  // TMA needs the matrix base and its column stride on 16-byte boundaries
  if ((reinterpret_cast<uintptr_t>(dA) & 15) != 0 || (lda % 4) != 0) return MPCHOL_ERR_BAD_ARG;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  int dev = 0;
  MPCHOL_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return MPCHOL_ERR_CUDA;
  DeviceSlot& slot = g_slots[dev];
  std::call_once(slot.once, [&slot]() {
    // runs with `dev` current: the symbol's address on this device
    void* p = nullptr;
    slot.err = cudaGetSymbolAddress(&p, g_scratch);
    if (slot.err == cudaSuccess) slot.addr = static_cast<StaticScratch*>(p);
  });
  if (slot.err != cudaSuccess) {
    record_cuda_error(slot.err, "mpchol_potrf_static setup", __FILE__, __LINE__);
    return MPCHOL_ERR_CUDA;
  }
  StaticScratch* sc = slot.addr;
  CUtensorMap tmap;
  if (!encode_tmap_2d(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, dA, n, n, lda, 32, 32,
                      CU_TENSOR_MAP_SWIZZLE_NONE))
    return MPCHOL_ERR_CUDA;
  MPCHOL_CUDA_TRY(cudaMemsetAsync(&sc->status, 0, sizeof(DevStatus), stream));
  MPCHOL_CUDA_TRY(launch_extract_diag(dA, lda, n, sc->diag, sc->diag_copy, stream));
  const PotrfParams pp{pivot_floor > 0.0f ? 1 : 0, 0.0f, pivot_floor};
  MPCHOL_CUDA_TRY(launch_potrf(tmap, dA, lda, n, 0, n, sc->diag, nullptr, pp, nullptr, nullptr,
                               sc->winv, &sc->status, false, stream));
  potrf_static_info_kernel<<<1, 1, 0, stream>>>(&sc->status, dInfo);
  MPCHOL_CUDA_TRY(cudaGetLastError());
  return MPCHOL_OK;
}
