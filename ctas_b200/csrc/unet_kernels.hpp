// unet_kernels.hpp -- launch interface of the learned-stage kernels (NHWC
// BF16 activations, FP32 accumulation; plain pointers, asynchronous).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ctas {

// 3x3 convolution, zero padding, stride 1: y[p][co] = act(sum w[co][t][ci]
// x[p + d_t][ci] + bias[co]) for the cout channels of a CTA tile.  x, y and
// mask are channel slices (stride cs, offset co) of NHWC buffers.  H % 8 == 0,
// W % 16 == 0, cout % 32 == 0, cin % 32 == 0 or cin == 16, channel strides and
// offsets of x multiples of 8.
struct ConvArgs {
  const __nv_bfloat16 *x;
  int x_cs, x_co, cin;
  const __nv_bfloat16 *w;      // [cout][9][cin]
  const float *bias;           // cout, or null
  __nv_bfloat16 *y;
  int y_cs, y_co, cout;
  const __nv_bfloat16 *mask;   // optional: y = 0 where mask <= 0
  int m_cs, m_co;
  int B, H, W;
  int relu;
};
bool conv_shape_ok(const ConvArgs &a);
// Runs the tensor-core (tcgen05) kernel where conv_tc_ok holds, else the
// mma.sync kernel.
cudaError_t launch_conv3x3(const ConvArgs &a, cudaStream_t st);
// The mma.sync kernel alone (kept for shapes outside conv_tc_ok).
cudaError_t launch_conv3x3_mma(const ConvArgs &a, cudaStream_t st);
// tcgen05 / tensor-memory implicit GEMM (conv_tc.cu): additionally needs
// y and mask channel strides and offsets that are multiples of 8.
bool conv_tc_ok(const ConvArgs &a);
cudaError_t launch_conv3x3_tc(const ConvArgs &a, cudaStream_t st);
// Error word of the tcgen05 kernels (bit 0: a bounded wait ran out), kept in
// mapped host memory; read without a device synchronisation.
int conv_tc_error();
void conv_tc_clear_error();

// dw[co][t][ci] += sum_p dy[p][co] x[p + d_t][ci]  (FP32, atomically added);
// cin % 32 == 0 or cin == 16
struct WgradArgs {
  const __nv_bfloat16 *x;
  int x_cs, x_co, cin;
  const __nv_bfloat16 *dy;
  int dy_cs, dy_co, cout;
  float *dw;
  int B, H, W;
};
// Runs the tcgen05 kernel where wgrad_tc_ok holds, else the mma.sync kernel.
cudaError_t launch_conv3x3_wgrad(const WgradArgs &a, cudaStream_t st);
bool wgrad_tc_ok(const WgradArgs &a);
cudaError_t launch_conv3x3_wgrad_tc(const WgradArgs &a, cudaStream_t st);
// db[c] += sum_p dy[p][c]
cudaError_t launch_bias_grad(const __nv_bfloat16 *dy, int cs, int co, int C, int64_t npix,
                             float *db, cudaStream_t st);

// 2x2 max pooling / nearest 2x upsampling of C channels; H, W are the input's
struct PoolArgs {
  const __nv_bfloat16 *x;
  int x_cs, x_co;
  __nv_bfloat16 *y;
  int y_cs, y_co;
  int B, H, W, C;
};
cudaError_t launch_maxpool(const PoolArgs &a, cudaStream_t st);
// dx slice += gradient routed to the first maximum, then dx *= (x > 0)
cudaError_t launch_maxpool_bwd(const PoolArgs &a, const __nv_bfloat16 *dy, int dy_cs, int dy_co,
                               __nv_bfloat16 *dx, int dx_cs, int dx_co, cudaStream_t st);
cudaError_t launch_upsample(const PoolArgs &a, cudaStream_t st);
// dx = (sum of the 2x2 block of dy) * (x > 0)
cudaError_t launch_upsample_bwd(const PoolArgs &a, const __nv_bfloat16 *dy, int dy_cs, int dy_co,
                                __nv_bfloat16 *dx, int dx_cs, int dx_co, cudaStream_t st);

// input image (FP32, scaled) -> BF16 NHWC with cpad channels (channel 0 used)
cudaError_t launch_unet_input(const float *x, int64_t npix, float scale, __nv_bfloat16 *y,
                              int cpad, cudaStream_t st);

// 1x1 head with the input added back
struct HeadArgs {
  const __nv_bfloat16 *feat;   // npix x C
  int C;
  const float *w, *b;
  const float *x;
  float scale;
  float *out;                  // npix: (x * scale + w . feat + b) * out_scale
  float out_scale;             // 1 in training (loss in scaled units), 1/scale in inference
  int64_t npix;
};
cudaError_t launch_head(const HeadArgs &a, cudaStream_t st);
// L2 loss against target * scale: *loss += sum (out - t)^2; gradients of the
// head and dfeat = dL/dfeat * (feat > 0)
cudaError_t launch_head_bwd(const HeadArgs &a, const float *target, double *loss, float *dw,
                            float *db, __nv_bfloat16 *dfeat, cudaStream_t st);

cudaError_t launch_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float b1,
                        float b2, float eps, int step, __nv_bfloat16 *wb, cudaStream_t st);
// wt[ci][8 - t][co] = w[co][t][ci]
cudaError_t launch_flip_weights(const __nv_bfloat16 *w, int cout, int cin, __nv_bfloat16 *wt,
                                cudaStream_t st);
cudaError_t launch_to_bf16(const float *x, __nv_bfloat16 *y, int64_t n, cudaStream_t st);

}  // namespace ctas
