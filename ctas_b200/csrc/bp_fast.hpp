// bp_fast.hpp -- launch interface of the staged backprojection kernel.
#pragma once
#include <cuda_runtime.h>

#include "fbp_kernels.hpp"

namespace ctas {
// True when the staged kernel handles this launch (float32 or reduced store,
// every sine of the angle table >= 0 -- checked by the caller).
bool bp_fast_supported(const BpLaunch &a);
cudaError_t launch_bp_fast(const BpLaunch &a, cudaStream_t st);
// Same kernel with every shared-memory gather checked against its window
// (violations set bit 8 of *a.err and read 0); for tests.
cudaError_t launch_bp_fast_checked(const BpLaunch &a, cudaStream_t st);
}  // namespace ctas
