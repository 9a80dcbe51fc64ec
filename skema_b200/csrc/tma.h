// tma.h -- tensor-map construction shared by the kernels that use the
// tensor-memory accelerator (cuTensorMapEncodeTiled, taken from the driver
// through the runtime's entry-point query, so the library links only the
// static CUDA runtime).
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace skema {

// 2-D tiled map: dim0 contiguous (extent d0), dim1 extent d1 with byte
// stride st1, box {b0, b1}, out-of-range elements read as zero and clipped
// on store. Fails with SKEMA_EINVAL on a misaligned base or stride.
CUtensorMap tmap_2d(CUtensorMapDataType dtype, const void* base, uint64_t d0, uint64_t d1, uint64_t st1,
                    uint32_t b0, uint32_t b1, CUtensorMapSwizzle swizzle);

// 3-D tiled map {d0, d1, d2} with byte strides st1, st2 and box {b0, b1, b2}.
CUtensorMap tmap_3d(CUtensorMapDataType dtype, const void* base, uint64_t d0, uint64_t d1, uint64_t d2,
                    uint64_t st1, uint64_t st2, uint32_t b0, uint32_t b1, uint32_t b2,
                    CUtensorMapSwizzle swizzle);

}  // namespace skema
