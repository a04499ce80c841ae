// axis_kernels.cu -- device kernels of the rotation-axis search (ctas
// src/common/lct.cpp:792-1212, the `ctas axis` tool).
//
// ag_measure_kernel: AverageGradient::apply (lct.cpp:863-913) after the
// backprojection, for S slices at once:
//   * Gaussian smoothing.  The reference multiplies the slice's 2-D FFT by the
//     FFT of g(a, b) = exp(-(a^2 + b^2) / (2 sigma^2)), a, b = 0 .. W-1 (a kernel
//     anchored at the array corner, not centred, not normalised) and divides
//     the inverse transform by W^2: a circular convolution
//       B[y][x] = sum_{a,b} g(a, b) S[(y - a) mod W][(x - b) mod W].
//     Here it is evaluated directly and separably, g(a, b) = g1(a) g1(b), in
//     FP64 over the K taps where g1 is not negligible, and rounded to float.
//   * Crop of k rows top and bottom (CTrec::recCrop, ct.h:276-279: k is
//     ceil(abs(c)) with the C library's int abs(), i.e. |(int)c|),
//     Sobel derivatives of the cropped image with the reference's term order
//     and zero padding at the crop border (lct.cpp:879-902), magnitude
//     sqrt(h*h + v*v) rounded like the reference (no fused multiply-add).
//   * The magnitude is assigned from the full-size derivative arrays into the
//     cropped view (lct.cpp:905): both are traversed from their first element,
//     so cropped row y receives the derivative of full row y, which is the
//     derivative of cropped row y - k (and 0 for y < k).  This
//     kernel reproduces that: output row y of the R = W - 2k rows is
//     the Sobel magnitude at full row y, with the crop's borders.
//   * First/last row and column zeroed; sum (FP64) and count of positive values.
//     With smoothing, the reference's single-precision FFT leaves rounding
//     noise in every pixel, so every magnitude of the evaluated region is
//     positive there: the count is then the whole region (count_all).
// Per-block partial sums are reduced in a fixed order, so results do not
// depend on scheduling.
#include <cuda_runtime.h>

#include <cstdint>

#include "axis_kernels.hpp"

namespace ctas {
namespace {

constexpr int kAgTile = 32;  // output tile edge
constexpr int kAgThreads = 256;

__device__ __forceinline__ int wrap(int v, int W) {
  v %= W;
  return v < 0 ? v + W : v;
}

// Fixed-order block reduction of (double, unsigned long long) pairs.
__device__ void block_reduce(double &s, unsigned long long &n, double *ssum,
                             unsigned long long *scnt) {
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    n += __shfl_down_sync(0xffffffffu, n, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    ssum[warp] = s;
    scnt[warp] = n;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    s = lane < nw ? ssum[lane] : 0.0;
    n = lane < nw ? scnt[lane] : 0ull;
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_down_sync(0xffffffffu, s, o);
      n += __shfl_down_sync(0xffffffffu, n, o);
    }
  }
}

__global__ void __launch_bounds__(kAgThreads)
    ag_measure_kernel(AgLaunch a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int W = a.W, K = a.K;
  const int sl = blockIdx.z;
  const int cc = a.crop[sl];
  const int R = W - 2 * cc;  // rows of the cropped slice
  const int y0 = blockIdx.y * kAgTile, x0 = blockIdx.x * kAgTile;
  const int SR = kAgTile + K + 1;  // staged rows: y0-K .. y0+T
  const int SC = kAgTile + K + 1;  // staged cols: x0-K .. x0+T
  const int HC = kAgTile + 2;      // blurred cols: x0-1 .. x0+T
  float *st = reinterpret_cast<float *>(smem);
  double *hb = reinterpret_cast<double *>(smem + (((size_t)SR * SC * 4 + 15) / 16) * 16);
  float *bl = reinterpret_cast<float *>(hb + (size_t)SR * HC);  // (T+2) x (T+2)
  __shared__ double ssum[kAgThreads / 32];
  __shared__ unsigned long long scnt[kAgThreads / 32];

  const float *slice = a.slices + (int64_t)sl * W * W;
  double s = 0.0;
  unsigned long long n = 0;
  if (y0 < R) {
    // stage the slice tile with its halo (circular)
    for (int e = threadIdx.x; e < SR * SC; e += blockDim.x) {
      const int r = e / SC, c = e - r * SC;
      st[e] = slice[(int64_t)wrap(y0 - K + r, W) * W + wrap(x0 - K + c, W)];
    }
    __syncthreads();
    // horizontal pass: hb[r][c'] = sum_b g1[b] S[r][x - b], x = x0 - 1 + c'
    for (int e = threadIdx.x; e < SR * HC; e += blockDim.x) {
      const int r = e / HC, c = e - r * HC;
      const float *row = st + r * SC + (c + K - 1);  // column x0 - 1 + c
      double acc = 0.0;
      for (int b = 0; b < K; b++) acc = fma(a.g[b], (double)row[-b], acc);
      hb[e] = acc;
    }
    __syncthreads();
    // vertical pass: bl[r'][c'] = float(sum_a g1[a] hb[y - a][c']), y = y0 - 1 + r'
    for (int e = threadIdx.x; e < HC * HC; e += blockDim.x) {
      const int r = e / HC, c = e - r * HC;
      const double *col = hb + (size_t)(r + K - 1) * HC + c;  // row y0 - 1 + r
      double acc = 0.0;
      for (int q = 0; q < K; q++) acc = fma(a.g[q], col[-(int64_t)q * HC], acc);
      bl[e] = (float)acc;
    }
    __syncthreads();
    // Sobel magnitude of output rows y (cropped-view index) = full rows y
    for (int e = threadIdx.x; e < kAgTile * kAgTile; e += blockDim.x) {
      const int ty = e / kAgTile, tx = e - ty * kAgTile;
      const int y = y0 + ty, x = x0 + tx;
      if (y >= R || x >= W) continue;
      if (y < cc || y == 0 || y == R - 1 || x == 0 || x == W - 1) continue;  // zero
      // cropped image C[r][x] = B[cc + r][x], r in [0, R); here r = y - cc
      const int r = y - cc;
      const bool up = r - 1 >= 0, dn = r + 1 < R, lf = x - 1 >= 0, rt = x + 1 < W;
      auto B = [&](int dy, int dx) { return bl[(ty + 1 + dy) * HC + (tx + 1 + dx)]; };
      // derH (lct.cpp:880-885), terms in the reference's order
      float h = 0.0f;
      if (dn && rt) h = __fadd_rn(h, -B(1, 1));
      if (dn) h = __fadd_rn(h, __fmul_rn(-2.0f, B(1, 0)));
      if (dn && lf) h = __fadd_rn(h, -B(1, -1));
      if (up && rt) h = __fadd_rn(h, B(-1, 1));
      if (up) h = __fadd_rn(h, __fmul_rn(2.0f, B(-1, 0)));
      if (up && lf) h = __fadd_rn(h, B(-1, -1));
      // derV (lct.cpp:887-892)
      float v = 0.0f;
      if (dn && rt) v = __fadd_rn(v, -B(1, 1));
      if (rt) v = __fadd_rn(v, __fmul_rn(-2.0f, B(0, 1)));
      if (up && rt) v = __fadd_rn(v, -B(-1, 1));
      if (dn && lf) v = __fadd_rn(v, B(1, -1));
      if (lf) v = __fadd_rn(v, __fmul_rn(2.0f, B(0, -1)));
      if (up && lf) v = __fadd_rn(v, B(-1, -1));
      const float m = __fsqrt_rn(__fadd_rn(__fmul_rn(h, h), __fmul_rn(v, v)));
      s += (double)m;
      n += (a.count_all || m > 0.0f) ? 1ull : 0ull;
    }
  }
  block_reduce(s, n, ssum, scnt);
  if (threadIdx.x == 0) {
    const int64_t blk = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    const int64_t nblk = (int64_t)gridDim.x * gridDim.y;
    a.part_sum[(int64_t)sl * nblk + blk] = s;
    a.part_cnt[(int64_t)sl * nblk + blk] = n;
  }
}

// out[sl] = sum over the slice's partials, fixed order.
__global__ void __launch_bounds__(kAgThreads)
    partial_reduce_kernel(const double *ps, const unsigned long long *pc, int64_t nblk,
                          double *out_sum, unsigned long long *out_cnt) {
  __shared__ double ssum[kAgThreads / 32];
  __shared__ unsigned long long scnt[kAgThreads / 32];
  const int sl = blockIdx.x;
  double s = 0.0;
  unsigned long long n = 0;
  for (int64_t i = threadIdx.x; i < nblk; i += blockDim.x) {
    s += ps[(int64_t)sl * nblk + i];
    n += pc[(int64_t)sl * nblk + i];
  }
  block_reduce(s, n, ssum, scnt);
  if (threadIdx.x == 0) {
    out_sum[sl] = s;
    out_cnt[sl] = n;
  }
}

// raxis(proj0, proj180, maxDev), calcErr (lct.cpp:1246-1252): one block per
// trial shift xs; the sum over all elements of dlt^2, dlt = (shifted mirrored
// proj180 or aver) - proj0, each square rounded to float and summed in FP64.
__global__ void __launch_bounds__(kAgThreads)
    pair_err_kernel(PairLaunch a) {
  __shared__ double ssum[kAgThreads / 32];
  __shared__ unsigned long long scnt[kAgThreads / 32];
  const int W = a.W;
  const int xs = a.shifts[blockIdx.x];
  // destination columns [max(0, xs), W - 1 + min(0, xs)] receive proj180R[i - xs]
  const int lo = xs > 0 ? xs : 0, hi = W - 1 + (xs < 0 ? xs : 0);
  double s = 0.0;
  unsigned long long n = 0;
  const int64_t total = (int64_t)a.rows * W;
  for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
    const int j = (int)(e / W), i = (int)(e - (int64_t)j * W);
    float p0 = a.p0[(int64_t)j * a.stride0 + i];
    if (a.add_one) p0 = __fadd_rn(p0, 1.0f);
    float d = a.aver;
    if (i >= lo && i <= hi) {
      // proj180R(j, i - xs) = proj180(j, W - 1 - (i - xs))
      float p1 = a.p180[(int64_t)j * a.stride180 + (W - 1 - (i - xs))];
      if (a.add_one) p1 = __fadd_rn(p1, 1.0f);
      d = p1;
    }
    d = __fsub_rn(d, p0);
    s += (double)__fmul_rn(d, d);
  }
  block_reduce(s, n, ssum, scnt);
  if (threadIdx.x == 0) a.out[blockIdx.x] = s;
}

// Column sums in row order with float accumulation, out[i] = sum_j x[j][i]
// (projLine of raxis algorithm 3, lct.cpp:1164-1166).
__global__ void column_sum_kernel(const float *x, int rows, int W, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
  float acc = 0.0f;
  for (int j = 0; j < rows; j++) acc = __fadd_rn(acc, x[(int64_t)j * W + i]);
  out[i] = acc;
}

// proj of raxis(proj0, proj180, maxDev) (lct.cpp:1233-1235): per column, in
// row order, proj = float(proj + (|p0 - 1| + |p180 - 1|)) with the inner terms
// in double (blitz promotes float - 1.0 to double).
__global__ void pair_profile_kernel(PairLaunch a, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.W) return;
  float acc = 0.0f;
  for (int j = 0; j < a.rows; j++) {
    float p0 = a.p0[(int64_t)j * a.stride0 + i];
    float p1 = a.p180[(int64_t)j * a.stride180 + i];
    if (a.add_one) {
      p0 = __fadd_rn(p0, 1.0f);
      p1 = __fadd_rn(p1, 1.0f);
    }
    const double t = __dadd_rn(fabs(__dsub_rn((double)p0, 1.0)), fabs(__dsub_rn((double)p1, 1.0)));
    acc = (float)__dadd_rn((double)acc, t);
  }
  out[i] = acc;
}

}  // namespace

size_t ag_smem_bytes(int K) {
  const size_t SR = kAgTile + K + 1, SC = kAgTile + K + 1, HC = kAgTile + 2;
  return ((SR * SC * 4 + 15) / 16) * 16 + SR * HC * 8 + HC * HC * 4;
}

int64_t ag_blocks_per_slice(int W) {
  const int64_t t = (W + kAgTile - 1) / kAgTile;
  return t * t;
}

cudaError_t launch_ag_measure(const AgLaunch &a, cudaStream_t st) {
  const size_t smem = ag_smem_bytes(a.K);
  cudaError_t e = cudaFuncSetAttribute(ag_measure_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int t = (a.W + kAgTile - 1) / kAgTile;
  ag_measure_kernel<<<dim3(t, t, a.S), kAgThreads, smem, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  partial_reduce_kernel<<<a.S, kAgThreads, 0, st>>>(a.part_sum, a.part_cnt, (int64_t)t * t,
                                                     a.out_sum, a.out_cnt);
  return cudaGetLastError();
}

cudaError_t launch_pair_err(const PairLaunch &a, int n_shifts, cudaStream_t st) {
  pair_err_kernel<<<n_shifts, kAgThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_pair_profile(const PairLaunch &a, float *out, cudaStream_t st) {
  pair_profile_kernel<<<(a.W + 127) / 128, 128, 0, st>>>(a, out);
  return cudaGetLastError();
}

cudaError_t launch_column_sum(const float *x, int rows, int W, float *out, cudaStream_t st) {
  column_sum_kernel<<<(W + 127) / 128, 128, 0, st>>>(x, rows, W, out);
  return cudaGetLastError();
}

}  // namespace ctas
