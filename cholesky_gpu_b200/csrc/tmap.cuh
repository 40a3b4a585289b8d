// Host-side construction of TMA tensor maps (cuTensorMapEncodeTiled through
// the runtime's driver entry point, so the library does not link libcuda).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mpchol {

// 2-D map over a column-major matrix: `inner` rows (contiguous), `outer`
// columns, column stride `ld` elements; boxes of box_inner x box_outer.
// Returns false if the encoder is unavailable or rejects the arguments.
bool encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, int esize, const void* base,
                    uint64_t inner, uint64_t outer, uint64_t ld, uint32_t box_inner,
                    uint32_t box_outer, CUtensorMapSwizzle swizzle);

}  // namespace mpchol
