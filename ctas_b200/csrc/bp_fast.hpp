// bp_fast.hpp -- launch interface of the staged backprojection kernel.
#pragma once
#include <cuda_runtime.h>

#include <functional>

#include "fbp_kernels.hpp"

namespace ctas {
// True when the staged kernel can serve this launch (for the truncation rule
// the caller also checks that every sine of the angle table is >= 0).
bool bp_fast_supported(const BpLaunch &a);
// Number of tile configurations (ids 0 .. count-1).
int bp_fast_tile_count();
// Details of the last failure on this thread ("" if none).
const char *bp_fast_error_detail();
// Tile search: every shape with the arithmetic variant that is usually
// fastest, then every other variant of the winning shape (all_variants =
// float32 truncation launches; otherwise variant 0 only).  time_ms(tile)
// runs one candidate and returns its time, < 0 if it failed; each candidate
// runs twice and the second time counts.  Returns -1 if every one failed.
int bp_fast_search(const std::function<float(int)> &time_ms, bool all_variants);
// Tile for this launch: `requested` if it is a valid id, else the
// CTAS_FBP_TILE environment override, else the autotuner's choice for
// (device, W, N, store, interp) -- the first launch of a shape runs
// bp_fast_search on one slice of that launch (synchronising the stream).
int bp_fast_choose_tile(const BpLaunch &a, cudaStream_t st, int requested);
cudaError_t launch_bp_fast(const BpLaunch &a, cudaStream_t st, int tile);
// Same kernel with every shared-memory gather checked against its window
// (violations set bit 8 of *a.err and read 0); for tests.
cudaError_t launch_bp_fast_checked(const BpLaunch &a, cudaStream_t st, int tile);
// Rows x columns of a tile id's pixel tile, and its window length (samples).
void bp_fast_tile_shape(int tile, int *ty, int *tx);
int bp_fast_tile_window(int tile);
// Persistent backprojection of an uneven batch (float32 store, truncation
// rule, every sine >= 0): resident CTAs take (sinogram, tile) items from
// b.counter, which must be 0 at launch.
cudaError_t launch_bp_batch(const BatchLaunch &b, int tile, cudaStream_t st);
}  // namespace ctas
