// tma_encode.hpp -- the driver's tensor-map encoder, shared by the TMA-fed
// kernels (staged backprojection, tcgen05 convolutions).
#pragma once
#include <cuda.h>

namespace ctas {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point, looked up
// once; null when the driver does not provide it.
EncodeTiledFn tensor_map_encoder();

}  // namespace ctas
