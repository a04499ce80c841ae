// fbp_kernels.hpp -- launch interface of the device kernels (plain pointers,
// no torch types).  All launches are asynchronous on the given stream.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ctas {

// Layout of the filtered sinogram kept on the device ("padded rows"):
// row r of slice s starts at q + s*slice_stride + r*Wp; the W samples sit at
// columns [OFF, OFF+W); column OFF-1 repeats sample 0 of the same row and
// column OFF+W holds sample 0 of the next row of the same slice (0 after the
// last row) -- the "guard columns" of the reference index rule.  Every other
// column is 0.  With this layout both the reference's truncating index rule
// and its flat-buffer reads one past the row end (lct.cpp:711-713 indexes the
// N*W buffer without bounds) need no branches.  Rows start on 16-byte
// boundaries for every element size (TMA tile loads need it): OFF and Wp are
// multiples of 8 elements.  Linear interpolation keeps the guard columns 0.
constexpr int kRowOff = 8;
inline int64_t padded_pitch(int64_t W) { return ((W + kRowOff + 1 + 7) / 8) * 8 + 8; }

// "Wide" layout, for angle sets with negative sines (e.g. 360-degree arcs),
// where the reference's index reaches up to |2c| + 1 < W samples before or
// after a row and reads the neighbouring rows of its flat N*W buffer
// (lct.cpp:711-713): the W samples of row r sit at columns [off, off + W),
// off = wide_offset(W), and every other column holds the flat sample it
// stands for -- column off + k is sample k mod W of row r + floor(k / W), 0
// outside the slice (launch_halo writes them).  There is no repeated guard
// sample: the staged kernel truncates toward zero where indices can be
// negative.
inline int64_t wide_offset(int64_t W) { return ((W + 16 + 7) / 8) * 8; }
inline int64_t wide_pitch(int64_t W) { return wide_offset(W) + ((2 * W + 16 + 7) / 8) * 8; }

struct FilterLaunch {
  const float *x;            // S x N x W input rows
  int64_t x_slice_stride;    // elements between slices of x
  void *q;                   // S x N x Wp output (f32 / f16 / bf16)
  int64_t q_slice_stride;
  float *row_scale;          // S x N (f16/bf16 store), else null
  const float2 *tw;          // per-stage twiddle tables of fft_twiddles (2 P floats,
                             // 16-byte aligned)
  const float *gperm;        // window in the FFT's output order, divided by P
  const float2 *minmax;      // per slice (min, max) for ABS, else null
  int N, W, Wp, P, zs;
  int contrast;              // 0 ABS, 1 REF, 2 PHS, 3 FLT
  int store;                 // 0 f32, 1 f16, 2 bf16
  int nradix;
  int radix[8];
  int S;                     // slices
  int guard;                 // 1: write the guard columns; 0: leave them 0
  const float *ring;         // ring-filter correction per column (S x W), or null
  int periodic;              // 1: the transform holds the row extended periodically,
                             // element p < 2W = sample (p - zs) mod W, 0 beyond;
                             // with a window symmetric about 0 this is the row's
                             // circular convolution of length W (unpadded filter)
  int off;                   // column of sample 0 in the output rows; 0 = kRowOff
};
cudaError_t launch_filter(const FilterLaunch &a, cudaStream_t st);
// Uneven batch (float32 store, filtering contrasts): jobs_dev[k] describes
// sinogram k with S = 1; its row pairs are blocks pair_begin_dev[k] ...
cudaError_t launch_filter_batch(const FilterLaunch *jobs_dev, const int *pair_begin_dev, int n_jobs,
                                int n_pairs, int max_pad, cudaStream_t st);

// Per-slice (min, max) of S x N x W inputs, and the deAbs validity check
// (physical.world.cpp:89-94): err (nullable) |= 1 when some slice has min <= 0 and
// max/1e6 <= 0.  `partials` needs 2*S*kMinMaxBlocks floats.
constexpr int kMinMaxBlocks = 64;
cudaError_t launch_minmax(const float *x, int64_t x_slice_stride, int64_t count,
                          int S, float2 *partials, float2 *minmax, int *err,
                          cudaStream_t st, const float *ring = nullptr, int W = 1);

// limit<T> of the volume writer (src/common/external.world.cpp:69-90): S
// images of `pixels` floats -> samples of bpp bits (negative = signed).
// range: per-image (min, max), used where mincon == maxcon (may be null
// otherwise).  dst contiguous.
cudaError_t launch_quantize(const float *src, int64_t pixels, int S, int bpp, float mincon,
                            float maxcon, const float2 *range, void *dst, cudaStream_t st);
int quantize_sample_bytes(int bpp);

// RingFilter::apply (lct.cpp:295-327, no mask): per slice the column means
// over the projections and their box-smoothed difference, written to
// ring (S x W); the filter kernels add it to every projection on load.
// avg: S x W scratch.
cudaError_t launch_ring(const float *x, int64_t x_slice_stride, int N, int W, int S, int box,
                        float *avg, float *ring, cudaStream_t st);

// Copy padded filtered rows back to a dense S x N x W float array (samples
// at column off of each row).
cudaError_t launch_unpad(const void *q, int64_t q_slice_stride, const float *row_scale,
                         int store, int N, int W, int Wp, int S, float *out,
                         int64_t out_slice_stride, cudaStream_t st, int off = kRowOff);

// Fill the halo columns of the wide layout (float32 rows; see wide_offset)
// from the filtered samples of the neighbouring rows of each slice.
cudaError_t launch_halo(float *q, int64_t q_slice_stride, int N, int W, int Wp, int off, int S,
                        cudaStream_t st);

struct BpLaunch {
  const void *q;             // padded filtered rows (see above)
  int interp;                // 0 reference truncation, 1 linear interpolation
  int64_t q_slice_stride;    // 0: every output slice backprojects the same
                             // rows (one filtered sinogram, several centres)
  const float *row_scale;    // f16/bf16 store: S x N scales
  int store;
  int N, W, Wp;
  const float2 *tab;         // N x (sin, cos), float, as lct.cpp:512-517
  float center, rec_cof;
  const float *centers;      // device, per output slice; null: `center` for all
  float *out;                // S x rows x cols
  int64_t out_slice_stride;
  int S;
  // output geometry: pixel (j, i) of a rows x cols grid stands for the
  // reference coordinates (oj + p j, oi + p i); rows = cols = W, oj = oi = 0,
  // p = 1 is the reference's W x W grid
  int out_rows, out_cols;
  float geo_oj, geo_oi, geo_p;
  int *err;                  // device error word: |= 4 on a wait timeout,
                             // |= 8 on a failed window check (checked variant)
  const double2 *lin;        // linear interpolation: per projection (sin, cos) in FP64
  int rule;                  // rounding order of the index expression (ref_base)
  int off;                   // column of sample 0 in the rows of q; 0 = kRowOff
  int wide;                  // 1: q has the wide layout (negative sines allowed)
  uint32_t wait_limit;       // staged kernel: iterations of each bounded wait; 0 = default
  int test_stall;            // staged kernel, test aid: skip the first chunk's copies so
                             // that the bounded waits run out (error word bit 2)
};
// Reference index rule for any angle set (flat reads outside the row).
cudaError_t launch_bp_generic(const BpLaunch &a, cudaStream_t st);

// One sinogram of an uneven batch, as the persistent backprojection sees it.
struct BatchJob {
  int W, N;
  int row0;                  // first row in the batch's padded buffer
  int tiles_x, tiles_y;      // tile grid of this slice (for the chosen tile shape)
  int item_begin;            // first work item of this slice
  float c, rec_cof;
  const float2 *tab;         // angle table of this sinogram
  float *out;                // W x W slice
  int rule;                  // rounding order of the index expression (ref_base)
};
struct BatchLaunch {
  const BatchJob *jobs;      // device array, ordered by item_begin
  int n_jobs, n_items;
  int *counter;              // work counter, 0 before the launch
  int *err;
  const void *q;             // padded rows of every sinogram, pitch Wp
  int Wp, rows;
};

}  // namespace ctas
