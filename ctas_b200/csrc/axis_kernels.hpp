// axis_kernels.hpp -- launch interface of the rotation-axis search kernels
// (plain pointers, asynchronous on the given stream).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ctas {

// Largest Gaussian tap count the fused measure kernel stages (shared memory).
constexpr int kAgMaxTaps = 157;

struct AgLaunch {
  const float *slices;            // S x W x W backprojected slices
  int S, W;
  const int *crop;                // per slice: ceil(|centre|), rows cropped top and bottom
  const double *g;                // K taps g1(a) = exp(-a^2 / (2 sigma^2)); K = 1, g = {1}: no blur
  int K;
  int count_all;                  // 1: count every pixel of the region (smoothing on)
  double *part_sum;               // S x ag_blocks_per_slice(W) scratch
  unsigned long long *part_cnt;   // same
  double *out_sum;                // S: sum of the gradient magnitude
  unsigned long long *out_cnt;    // S: number of positive magnitudes
};
size_t ag_smem_bytes(int K);
int64_t ag_blocks_per_slice(int W);
cudaError_t launch_ag_measure(const AgLaunch &a, cudaStream_t st);

// Projection pair of raxis(proj0, proj180, maxDev).
struct PairLaunch {
  const float *p0, *p180;         // rows x W each (row strides below)
  int64_t stride0, stride180;
  int rows, W;
  int add_one;                    // 1: use value + 1 (raxisQ, lct.cpp:1152-1155)
  float aver;                     // fill value of uncovered columns
  const int *shifts;              // trial shifts (truncated)
  double *out;                    // per shift: sum of squared differences
};
cudaError_t launch_pair_err(const PairLaunch &a, int n_shifts, cudaStream_t st);
// per column: sum over rows of |p0 - 1| + |p180 - 1| (float, row order)
cudaError_t launch_pair_profile(const PairLaunch &a, float *out, cudaStream_t st);
// per column: sum over rows (float, row order)
cudaError_t launch_column_sum(const float *x, int rows, int W, float *out, cudaStream_t st);

}  // namespace ctas
