/*
 * ctas_learned.h -- the learned sparse-angle stage (extension; no counterpart
 * in the reference): a 4-level 2-D U-Net (32 base channels, two 3x3
 * convolutions with ReLU per level, 2x2 max pooling, nearest 2x upsampling
 * with skip concatenation, a 1x1 head added to the input) in BF16 with FP32
 * accumulation, trained and run by hand-written kernels on the tensor cores.
 * Its job is to turn a filtered backprojection from every k-th projection into
 * a slice of full-angle quality; the plain full-angle reconstruction
 * (ctas_fbp.h) remains the fallback and the judge of its error.
 *
 * Images are FP32 [B][H][W] on the device; H % 64 == 0 and W % 128 == 0 (the
 * three poolings keep the 8 x 16 convolution blocks whole).  The network works
 * on x * scale (set the scale so typical values are of order 1).  Statuses and
 * last-error message as in ctas_fbp.h.
 */
#ifndef CTAS_LEARNED_H
#define CTAS_LEARNED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctas_unet ctas_unet;

/* He-initialised weights from `seed` (the head starts at zero, so the network
 * starts as the identity); device: CUDA ordinal, -1 = current. */
int ctas_unet_create(ctas_unet **out, uint64_t seed, int32_t device);
int ctas_unet_destroy(ctas_unet *u);
/* Input scale (default 1). */
int ctas_unet_set_scale(ctas_unet *u, float scale);
/* y = x + net(x * scale) / scale for B images, asynchronous on `stream`. */
int ctas_unet_forward_dev(ctas_unet *u, const float *x_dev, float *y_dev, int64_t B, int64_t H,
                          int64_t W, void *stream);
/* One Adam step (learning rate lr, betas 0.9 / 0.999) on the mean squared
 * error, in scaled units, between the output and target_dev; *loss (nullable)
 * receives that error before the step.  Synchronous. */
int ctas_unet_train_step_dev(ctas_unet *u, const float *x_dev, const float *target_dev, int64_t B,
                             int64_t H, int64_t W, float lr, double *loss, void *stream);
/* All parameters as FP32: count, copy out, copy in (same order: per layer
 * w[cout][9][cin] then bias[cout]; then the head's 32 weights and bias). */
int64_t ctas_unet_param_count(const ctas_unet *u);
int ctas_unet_get_params(const ctas_unet *u, float *host);
int ctas_unet_set_params(ctas_unet *u, const float *host);
/* Multiply-adds of one forward pass per pixel of the full-resolution level. */
double ctas_unet_macs_per_pixel(void);

/* ---- layer entry points (the kernels the network is built from; BF16 NHWC
 * channel slices: channel stride cs, offset co) ---- */
/* y = act(conv3x3(x, w[cout][9][cin]) + bias); act: relu != 0 -> ReLU; mask
 * (nullable): y = 0 where mask <= 0.  H % 8 == 0, W % 16 == 0, cout % 32 == 0,
 * cin % 32 == 0 or cin == 16.  Runs as an implicit GEMM on the tcgen05 tensor
 * cores (TMA-fed operands, accumulators in tensor memory) when the y and mask
 * channel strides and offsets are multiples of 8, else on the mma.sync kernel.
 * A bounded device wait that ran out is reported by the next call on this
 * library's learned-stage entry points as CTAS_E_TIMEOUT. */
int ctas_nn_conv3x3_dev(const void *x, int32_t x_cs, int32_t x_co, int32_t cin, const void *w,
                        const float *bias, void *y, int32_t y_cs, int32_t y_co, int32_t cout,
                        const void *mask, int32_t m_cs, int32_t m_co, int64_t B, int64_t H,
                        int64_t W, int32_t relu, void *stream);
/* dw[cout][9][cin] (FP32) += weight gradient of that convolution: per tap a
 * tcgen05 GEMM over the pixels, split over CTAs, partial sums added with
 * atomics (cin, cout multiples of 16, dw 16-byte aligned; else mma.sync). */
int ctas_nn_conv3x3_wgrad_dev(const void *x, int32_t x_cs, int32_t x_co, int32_t cin,
                              const void *dy, int32_t dy_cs, int32_t dy_co, int32_t cout,
                              float *dw, int64_t B, int64_t H, int64_t W, void *stream);
/* wt[cin][8 - t][cout] = w[cout][t][cin]: the weights of the data gradient. */
int ctas_nn_flip_weights_dev(const void *w, int32_t cout, int32_t cin, void *wt, void *stream);

/* Test aid: while enabled (on the current device), every tcgen05 convolution
 * kernel leaves its first stage of copies out and gives each wait a short
 * bound, so its waits run out; it then drains, frees its tensor memory and
 * returns, and the next learned-stage call reports CTAS_E_TIMEOUT.  Disable
 * before real work. */
int ctas_nn_test_timeout(int32_t enable);

#ifdef __cplusplus
}
#endif

#endif /* CTAS_LEARNED_H */
