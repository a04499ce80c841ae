// bp_generic.cu -- backprojection for any angle set, reference index rule.
//
// Per output pixel (j = row, i = column) this is the arithmetic of
// CTrec::reconstructOnCPU (ctas src/common/lct.cpp:688-729), identical to the
// reference's OpenCL kernel fbp (src/common/ct.cl:14-43):
//   masks on i and on the disc, then
//   tot = sum_n q[n][ (int) t_n ],
//   t_n = ((c + ((1 - s_n) - c_n) * hp) + s_n * (j - c)) + c_n * i   (float)
//   slice = (recCof != 0 ? tot * recCof : tot) / N.
// Every float operation is an explicitly rounded intrinsic (no contraction),
// the sum runs in projection order, so the result is bit-identical to the
// reference for float32 storage.  Indices outside [0, W] read the buffer
// flat, as the reference does (row n + floor(k/W)), and 0 outside the
// sinogram.  This kernel serves every geometry; bp_fast.cu takes the common
// case where all sines are >= 0.  With interp == 1 it interpolates linearly
// instead (an extension; sample k centred at k + 0.5, 0 outside [0, W)).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bp_common.cuh"
#include "fbp_kernels.hpp"

namespace ctas {
namespace {

constexpr int kTile = 16;
constexpr int kAngChunk = 512;

template <typename T, int MODE>
__global__ void __launch_bounds__(kTile *kTile) bp_generic_kernel(BpLaunch a) {
  __shared__ float4 ang[kAngChunk];
  const int i = blockIdx.x * kTile + threadIdx.x;
  const int j = blockIdx.y * kTile + threadIdx.y;
  const int sl = blockIdx.z;
  const int W = a.W, N = a.N, hp = W / 2, R = a.out_rows, Cc = a.out_cols;
  const float c = a.centers ? a.centers[sl] : a.center;
  const float jj = geo(a.geo_oj, a.geo_p, j), ii = geo(a.geo_oi, a.geo_p, i);
  const bool valid = i < Cc && j < R;
  const bool inside = valid && ref_mask_f(jj, ii, W, c);
  float *out = a.out + sl * a.out_slice_stride;
  if (!__syncthreads_or(inside)) {
    if (valid) out[(int64_t)j * Cc + i] = 0.f;
    return;
  }
  const T *q = reinterpret_cast<const T *>(a.q) + sl * a.q_slice_stride;
  const float *rs = a.row_scale ? a.row_scale + (a.q_slice_stride ? (int64_t)sl * N : 0) : nullptr;
  const float jc = __fsub_rn(jj, c), fi = ii;
  const int off = a.off ? a.off : kRowOff;  // column of sample 0
  const int tid = threadIdx.y * kTile + threadIdx.x;
  float acc = 0.f;
  for (int n0 = 0; n0 < N; n0 += kAngChunk) {
    const int cnt = min(kAngChunk, N - n0);
    __syncthreads();
    for (int k = tid; k < cnt; k += kTile * kTile) {
      if (MODE == 0) {
        const float2 sc = a.tab[n0 + k];
        ang[k] = make_float4(sc.x, sc.y, ref_base(sc.x, sc.y, hp, c, a.rule), rs ? rs[n0 + k] : 1.f);
      } else {
        // linear: u = t0 + sin j + cos i, t0 = (hp + c)(1 - sin) - cos hp - 0.5 in FP64
        const double2 g = a.lin[n0 + k];
        const double hc = (double)hp + (double)c;
        ang[k] = make_float4((float)g.x, (float)g.y,
                             (float)(hc * (1.0 - g.x) - g.y * (double)hp - 0.5),
                             rs ? rs[n0 + k] : 1.f);
      }
    }
    __syncthreads();
    if (inside && MODE == 0) {
      for (int k = 0; k < cnt; k++) {
        const float4 g = ang[k];
        const float t = __fadd_rn(__fadd_rn(g.z, __fmul_rn(g.x, jc)), __fmul_rn(g.y, fi));
        const int idx = __float2int_rz(t);
        const int n = n0 + k;
        float v;
        if ((unsigned)idx <= (unsigned)W) {
          v = load_sample(q + (int64_t)n * a.Wp + off + idx);
          if (rs) v *= g.w;
        } else {
          // flat read of the N*W buffer (lct.cpp:713 indexes without bounds)
          const int64_t o = (int64_t)n * W + idx;
          if (o < 0 || o >= (int64_t)N * W) {
            v = 0.f;
          } else {
            const int64_t nn = o / W, kk = o - nn * W;
            v = load_sample(q + nn * a.Wp + off + kk);
            if (rs) v *= rs[nn];
          }
        }
        acc = __fadd_rn(acc, v);
      }
    } else if (inside) {
      const float fj = jj;
      for (int k = 0; k < cnt; k++) {
        const float4 g = ang[k];
        const float u = fmaf(g.y, fi, fmaf(g.x, fj, g.z));
        const float fl = floorf(u);
        const float f = u - fl;
        const int idx = (int)fl;
        const T *row = q + (int64_t)(n0 + k) * a.Wp + off;
        // samples outside [0, W) are 0 (the guard columns are 0 in this mode)
        const float v0 = (idx >= 0 && idx < W) ? load_sample(row + idx) : 0.f;
        const float v1 = (idx + 1 >= 0 && idx + 1 < W) ? load_sample(row + idx + 1) : 0.f;
        acc += (v0 + f * (v1 - v0)) * g.w;
      }
    }
  }
  if (valid) out[(int64_t)j * Cc + i] = inside ? ref_finish(acc, a.rec_cof, N) : 0.f;
}

}  // namespace

cudaError_t launch_bp_generic(const BpLaunch &a, cudaStream_t st) {
  const dim3 grid((a.out_cols + kTile - 1) / kTile, (a.out_rows + kTile - 1) / kTile, a.S);
  const dim3 block(kTile, kTile);
  if (a.interp == 1) {
    if (a.store == 1) bp_generic_kernel<__half, 1><<<grid, block, 0, st>>>(a);
    else if (a.store == 2) bp_generic_kernel<__nv_bfloat16, 1><<<grid, block, 0, st>>>(a);
    else bp_generic_kernel<float, 1><<<grid, block, 0, st>>>(a);
  } else {
    if (a.store == 1) bp_generic_kernel<__half, 0><<<grid, block, 0, st>>>(a);
    else if (a.store == 2) bp_generic_kernel<__nv_bfloat16, 0><<<grid, block, 0, st>>>(a);
    else bp_generic_kernel<float, 0><<<grid, block, 0, st>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace ctas
