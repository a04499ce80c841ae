// unet.cpp -- the learned sparse-angle stage: a 4-level U-Net, its forward
// pass, backward pass and Adam step, scheduled on one stream from the kernels
// of unet_kernels.cu.
//
// Layers (cin -> cout, 3x3, ReLU), levels at H, H/2, H/4, H/8:
//   e1a 16->32, e1b 32->32 | e2a 32->64, e2b 64->64 | e3a 64->128, e3b 128->128
//   | ba 128->256, bb 256->256 | d3a 384->128, d3b 128->128 | d2a 192->64,
//   d2b 64->64 | d1a 96->32, d1b 32->32 | head 1x1 32->1 added to the input.
// The input has 16 channels (channel 0 the image) to fit the 16-channel
// convolution chunk.  Encoder outputs are written into the upper channels of
// the decoder inputs (dec1 96 = 64 up + 32 skip, dec2 192, dec3 384), so the
// concatenation costs nothing; pooling reads them from there.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "../../include/ctas_fbp.h"
#include "../../include/ctas_learned.h"
#include "fbp_host.hpp"
#include "unet_kernels.hpp"

namespace {

using bf16 = __nv_bfloat16;

struct Spec {
  int cin, cout;
};
enum { E1A, E1B, E2A, E2B, E3A, E3B, BA, BB, D3A, D3B, D2A, D2B, D1A, D1B, NL };
constexpr Spec kSpec[NL] = {{16, 32},  {32, 32},   {32, 64},   {64, 64},  {64, 128},
                            {128, 128}, {128, 256}, {256, 256}, {384, 128}, {128, 128},
                            {192, 64},  {64, 64},   {96, 32},   {32, 32}};
constexpr int kLevel[NL] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0};
constexpr int kHeadC = 32, kInC = 16;

template <class F> int guarded(F &&f) {
  try {
    return f();
  } catch (const ctas::Error &e) {
    ctas::set_last_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    ctas::set_last_error("host allocation failed");
    return CTAS_E_NOMEM;
  } catch (const std::exception &e) {
    ctas::set_last_error(e.what());
    return CTAS_E_ARG;
  }
}

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  int code = CTAS_E_CUDA;
  if (e == cudaErrorMemoryAllocation) code = CTAS_E_NOMEM;
  if (e == cudaErrorInvalidValue) code = CTAS_E_SHAPE;
  cudaGetLastError();
  ctas::fail(code, std::string("learned stage: ") + what + ": " + cudaGetErrorString(e));
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cuda_check(cudaGetDevice(&prev), "cudaGetDevice");
    if (dev != prev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DevGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
  void ensure(size_t n) {
    if (n <= bytes) return;
    release();
    cuda_check(cudaMalloc(&p, n), "cudaMalloc");
    bytes = n;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
  ~Buf() { release(); }
};

// activation / gradient tensors of one (B, H, W), carved from one allocation
struct Acts {
  int64_t B = 0, H = 0, W = 0;
  bool grads = false;
  Buf mem;
  float *out = nullptr;
  double *loss = nullptr;
  bf16 *in16, *t1, *dec1, *p1, *t2, *dec2, *p2, *t3, *dec3, *p3, *t4, *bott, *u3, *d3o, *u2, *d2o,
      *u1, *d1o;
  bf16 *g_d1o, *g_u1, *g_dec1, *g_d2o, *g_u2, *g_dec2, *g_d3o, *g_u3, *g_dec3, *g_bott, *g_t4,
      *g_p3, *g_t3, *g_p2, *g_t2, *g_p1, *g_t1;
};

}  // namespace

struct ctas_unet {
  int device = 0;
  float scale = 1.f;
  int step = 0;
  int64_t npar = 0;
  int64_t woff[NL], boff[NL], hw_off = 0, hb_off = 0, tof[NL];
  Buf par, grad, m, v, parb, flip;  // FP32 params, grads, Adam moments; BF16 mirror; flipped
  cudaStream_t stream = nullptr;
  Acts act;
  ~ctas_unet() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    act.mem.release();
    par.release();
    grad.release();
    m.release();
    v.release();
    parb.release();
    flip.release();
    if (stream) cudaStreamDestroy(stream);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

namespace {

void layout(ctas_unet *u) {
  int64_t o = 0, t = 0;
  for (int l = 0; l < NL; l++) {
    u->woff[l] = o;
    o += (int64_t)kSpec[l].cout * 9 * kSpec[l].cin;
    u->boff[l] = o;
    o += kSpec[l].cout;
    u->tof[l] = t;
    t += (int64_t)kSpec[l].cout * 9 * kSpec[l].cin;
  }
  u->hw_off = o;
  o += kHeadC;
  u->hb_off = o;
  o += 1;
  u->npar = o;
}

void refresh_bf16(ctas_unet *u, cudaStream_t st) {
  cuda_check(ctas::launch_to_bf16(u->par.as<float>(), u->parb.as<bf16>(), u->npar, st), "to bf16");
  for (int l = 0; l < NL; l++)
    cuda_check(ctas::launch_flip_weights(u->parb.as<bf16>() + u->woff[l], kSpec[l].cout,
                                         kSpec[l].cin, u->flip.as<bf16>() + u->tof[l], st),
               "flip weights");
}

// A tensor-core convolution whose bounded wait ran out (sticky until read).
void check_tc_error() {
  if (ctas::conv_tc_error()) {
    ctas::conv_tc_clear_error();
    ctas::fail(CTAS_E_TIMEOUT, "tensor-core convolution: a bounded device wait ran out");
  }
}

void check_shape(int64_t B, int64_t H, int64_t W) {
  if (B < 1 || H < 64 || W < 128 || H % 64 || W % 128)
    ctas::fail(CTAS_E_SHAPE, "learned stage: images must be at least 64 x 128 with H % 64 == 0 "
                             "and W % 128 == 0");
  if (B * H * W > ((int64_t)1 << 28)) ctas::fail(CTAS_E_SHAPE, "learned stage: batch too large");
}

void ensure_acts(ctas_unet *u, int64_t B, int64_t H, int64_t W, bool grads) {
  Acts &a = u->act;
  if (a.B == B && a.H == H && a.W == W && (a.grads || !grads)) return;
  const int64_t P0 = B * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  struct Item {
    bf16 **ptr;
    int64_t n;
  };
  std::vector<Item> items = {
      {&a.in16, P0 * kInC}, {&a.t1, P0 * 32},   {&a.dec1, P0 * 96}, {&a.p1, P1 * 32},
      {&a.t2, P1 * 64},     {&a.dec2, P1 * 192}, {&a.p2, P2 * 64},  {&a.t3, P2 * 128},
      {&a.dec3, P2 * 384},  {&a.p3, P3 * 128},  {&a.t4, P3 * 256},  {&a.bott, P3 * 256},
      {&a.u3, P2 * 128},    {&a.d3o, P2 * 128}, {&a.u2, P1 * 64},   {&a.d2o, P1 * 64},
      {&a.u1, P0 * 32},     {&a.d1o, P0 * 32}};
  if (grads) {
    std::vector<Item> g = {
        {&a.g_d1o, P0 * 32},   {&a.g_u1, P0 * 32},  {&a.g_dec1, P0 * 96}, {&a.g_d2o, P1 * 64},
        {&a.g_u2, P1 * 64},    {&a.g_dec2, P1 * 192}, {&a.g_d3o, P2 * 128}, {&a.g_u3, P2 * 128},
        {&a.g_dec3, P2 * 384}, {&a.g_bott, P3 * 256}, {&a.g_t4, P3 * 256}, {&a.g_p3, P3 * 128},
        {&a.g_t3, P2 * 128},   {&a.g_p2, P2 * 64},   {&a.g_t2, P1 * 64},  {&a.g_p1, P1 * 32},
        {&a.g_t1, P0 * 32}};
    items.insert(items.end(), g.begin(), g.end());
  }
  size_t total = 256 + ((size_t)P0 * sizeof(float) + 255) / 256 * 256;
  for (auto &it : items) total += ((size_t)it.n * sizeof(bf16) + 255) / 256 * 256;
  a.B = a.H = a.W = 0;
  a.mem.release();
  a.mem.ensure(total);
  char *p = a.mem.as<char>();
  a.loss = reinterpret_cast<double *>(p);
  p += 256;
  a.out = reinterpret_cast<float *>(p);
  p += ((size_t)P0 * sizeof(float) + 255) / 256 * 256;
  for (auto &it : items) {
    *it.ptr = reinterpret_cast<bf16 *>(p);
    p += ((size_t)it.n * sizeof(bf16) + 255) / 256 * 256;
  }
  a.B = B;
  a.H = H;
  a.W = W;
  a.grads = grads;
}

void conv(ctas_unet *u, int l, const bf16 *x, int xcs, int xco, bf16 *y, int ycs, int yco,
          int64_t B, int64_t H, int64_t W, cudaStream_t st) {
  ctas::ConvArgs c{};
  c.x = x;
  c.x_cs = xcs;
  c.x_co = xco;
  c.cin = kSpec[l].cin;
  c.w = u->parb.as<bf16>() + u->woff[l];
  c.bias = u->par.as<float>() + u->boff[l];
  c.y = y;
  c.y_cs = ycs;
  c.y_co = yco;
  c.cout = kSpec[l].cout;
  c.B = (int)B;
  c.H = (int)H;
  c.W = (int)W;
  c.relu = 1;
  cuda_check(ctas::launch_conv3x3(c, st), "convolution");
}

// data gradient of layer l's input: dx = conv(dy, flipped w) * (mask > 0)
void dgrad(ctas_unet *u, int l, const bf16 *dy, int dycs, int dyco, bf16 *dx, int dxcs, int dxco,
           const bf16 *mask, int mcs, int mco, int64_t B, int64_t H, int64_t W, cudaStream_t st) {
  ctas::ConvArgs c{};
  c.x = dy;
  c.x_cs = dycs;
  c.x_co = dyco;
  c.cin = kSpec[l].cout;
  c.w = u->flip.as<bf16>() + u->tof[l];
  c.bias = nullptr;
  c.y = dx;
  c.y_cs = dxcs;
  c.y_co = dxco;
  c.cout = kSpec[l].cin;
  c.mask = mask;
  c.m_cs = mcs;
  c.m_co = mco;
  c.B = (int)B;
  c.H = (int)H;
  c.W = (int)W;
  c.relu = 0;
  cuda_check(ctas::launch_conv3x3(c, st), "convolution data gradient");
}

void wgrad(ctas_unet *u, int l, const bf16 *x, int xcs, int xco, const bf16 *dy, int dycs, int dyco,
           int64_t B, int64_t H, int64_t W, cudaStream_t st) {
  ctas::WgradArgs g{};
  g.x = x;
  g.x_cs = xcs;
  g.x_co = xco;
  g.cin = kSpec[l].cin;
  g.dy = dy;
  g.dy_cs = dycs;
  g.dy_co = dyco;
  g.cout = kSpec[l].cout;
  g.dw = u->grad.as<float>() + u->woff[l];
  g.B = (int)B;
  g.H = (int)H;
  g.W = (int)W;
  cuda_check(ctas::launch_conv3x3_wgrad(g, st), "weight gradient");
  cuda_check(ctas::launch_bias_grad(dy, dycs, dyco, kSpec[l].cout, B * H * W,
                                    u->grad.as<float>() + u->boff[l], st),
             "bias gradient");
}

ctas::PoolArgs pool_args(const bf16 *x, int xcs, int xco, bf16 *y, int ycs, int yco, int64_t B,
                         int64_t H, int64_t W, int C) {
  ctas::PoolArgs p{};
  p.x = x;
  p.x_cs = xcs;
  p.x_co = xco;
  p.y = y;
  p.y_cs = ycs;
  p.y_co = yco;
  p.B = (int)B;
  p.H = (int)H;
  p.W = (int)W;
  p.C = C;
  return p;
}

ctas::HeadArgs head_args(ctas_unet *u, const float *x, int64_t npix, float out_scale) {
  ctas::HeadArgs h{};
  h.feat = u->act.d1o;
  h.C = kHeadC;
  h.w = u->par.as<float>() + u->hw_off;
  h.b = u->par.as<float>() + u->hb_off;
  h.x = x;
  h.scale = u->scale;
  h.out = u->act.out;
  h.out_scale = out_scale;
  h.npix = npix;
  return h;
}

void forward(ctas_unet *u, const float *x, int64_t B, int64_t H, int64_t W, float out_scale,
             cudaStream_t st) {
  Acts &a = u->act;
  const int64_t H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  cuda_check(ctas::launch_unet_input(x, B * H * W, u->scale, a.in16, kInC, st), "input");
  conv(u, E1A, a.in16, kInC, 0, a.t1, 32, 0, B, H, W, st);
  conv(u, E1B, a.t1, 32, 0, a.dec1, 96, 64, B, H, W, st);
  cuda_check(ctas::launch_maxpool(pool_args(a.dec1, 96, 64, a.p1, 32, 0, B, H, W, 32), st), "pool");
  conv(u, E2A, a.p1, 32, 0, a.t2, 64, 0, B, H1, W1, st);
  conv(u, E2B, a.t2, 64, 0, a.dec2, 192, 128, B, H1, W1, st);
  cuda_check(ctas::launch_maxpool(pool_args(a.dec2, 192, 128, a.p2, 64, 0, B, H1, W1, 64), st),
             "pool");
  conv(u, E3A, a.p2, 64, 0, a.t3, 128, 0, B, H2, W2, st);
  conv(u, E3B, a.t3, 128, 0, a.dec3, 384, 256, B, H2, W2, st);
  cuda_check(ctas::launch_maxpool(pool_args(a.dec3, 384, 256, a.p3, 128, 0, B, H2, W2, 128), st),
             "pool");
  conv(u, BA, a.p3, 128, 0, a.t4, 256, 0, B, H3, W3, st);
  conv(u, BB, a.t4, 256, 0, a.bott, 256, 0, B, H3, W3, st);
  cuda_check(ctas::launch_upsample(pool_args(a.bott, 256, 0, a.dec3, 384, 0, B, H3, W3, 256), st),
             "upsample");
  conv(u, D3A, a.dec3, 384, 0, a.u3, 128, 0, B, H2, W2, st);
  conv(u, D3B, a.u3, 128, 0, a.d3o, 128, 0, B, H2, W2, st);
  cuda_check(ctas::launch_upsample(pool_args(a.d3o, 128, 0, a.dec2, 192, 0, B, H2, W2, 128), st),
             "upsample");
  conv(u, D2A, a.dec2, 192, 0, a.u2, 64, 0, B, H1, W1, st);
  conv(u, D2B, a.u2, 64, 0, a.d2o, 64, 0, B, H1, W1, st);
  cuda_check(ctas::launch_upsample(pool_args(a.d2o, 64, 0, a.dec1, 96, 0, B, H1, W1, 64), st),
             "upsample");
  conv(u, D1A, a.dec1, 96, 0, a.u1, 32, 0, B, H, W, st);
  conv(u, D1B, a.u1, 32, 0, a.d1o, 32, 0, B, H, W, st);
  cuda_check(ctas::launch_head(head_args(u, x, B * H * W, out_scale), st), "head");
}

void backward(ctas_unet *u, const float *x, const float *target, int64_t B, int64_t H, int64_t W,
              cudaStream_t st) {
  Acts &a = u->act;
  const int64_t H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  float *g = u->grad.as<float>();
  cuda_check(cudaMemsetAsync(g, 0, sizeof(float) * (size_t)u->npar, st), "cudaMemsetAsync");
  cuda_check(cudaMemsetAsync(a.loss, 0, sizeof(double), st), "cudaMemsetAsync");
  cuda_check(ctas::launch_head_bwd(head_args(u, x, B * H * W, 1.f), target, a.loss, g + u->hw_off,
                                   g + u->hb_off, a.g_d1o, st),
             "head gradient");
  // level 1 decoder
  wgrad(u, D1B, a.u1, 32, 0, a.g_d1o, 32, 0, B, H, W, st);
  dgrad(u, D1B, a.g_d1o, 32, 0, a.g_u1, 32, 0, a.u1, 32, 0, B, H, W, st);
  wgrad(u, D1A, a.dec1, 96, 0, a.g_u1, 32, 0, B, H, W, st);
  dgrad(u, D1A, a.g_u1, 32, 0, a.g_dec1, 96, 0, nullptr, 0, 0, B, H, W, st);
  cuda_check(ctas::launch_upsample_bwd(pool_args(a.d2o, 64, 0, nullptr, 0, 0, B, H1, W1, 64),
                                       a.g_dec1, 96, 0, a.g_d2o, 64, 0, st),
             "upsample gradient");
  // level 2 decoder
  wgrad(u, D2B, a.u2, 64, 0, a.g_d2o, 64, 0, B, H1, W1, st);
  dgrad(u, D2B, a.g_d2o, 64, 0, a.g_u2, 64, 0, a.u2, 64, 0, B, H1, W1, st);
  wgrad(u, D2A, a.dec2, 192, 0, a.g_u2, 64, 0, B, H1, W1, st);
  dgrad(u, D2A, a.g_u2, 64, 0, a.g_dec2, 192, 0, nullptr, 0, 0, B, H1, W1, st);
  cuda_check(ctas::launch_upsample_bwd(pool_args(a.d3o, 128, 0, nullptr, 0, 0, B, H2, W2, 128),
                                       a.g_dec2, 192, 0, a.g_d3o, 128, 0, st),
             "upsample gradient");
  // level 3 decoder
  wgrad(u, D3B, a.u3, 128, 0, a.g_d3o, 128, 0, B, H2, W2, st);
  dgrad(u, D3B, a.g_d3o, 128, 0, a.g_u3, 128, 0, a.u3, 128, 0, B, H2, W2, st);
  wgrad(u, D3A, a.dec3, 384, 0, a.g_u3, 128, 0, B, H2, W2, st);
  dgrad(u, D3A, a.g_u3, 128, 0, a.g_dec3, 384, 0, nullptr, 0, 0, B, H2, W2, st);
  cuda_check(ctas::launch_upsample_bwd(pool_args(a.bott, 256, 0, nullptr, 0, 0, B, H3, W3, 256),
                                       a.g_dec3, 384, 0, a.g_bott, 256, 0, st),
             "upsample gradient");
  // bottom
  wgrad(u, BB, a.t4, 256, 0, a.g_bott, 256, 0, B, H3, W3, st);
  dgrad(u, BB, a.g_bott, 256, 0, a.g_t4, 256, 0, a.t4, 256, 0, B, H3, W3, st);
  wgrad(u, BA, a.p3, 128, 0, a.g_t4, 256, 0, B, H3, W3, st);
  dgrad(u, BA, a.g_t4, 256, 0, a.g_p3, 128, 0, nullptr, 0, 0, B, H3, W3, st);
  // level 3 encoder: skip gradient + pooled path, then the ReLU of e3b
  cuda_check(ctas::launch_maxpool_bwd(pool_args(a.dec3, 384, 256, nullptr, 0, 0, B, H2, W2, 128),
                                      a.g_p3, 128, 0, a.g_dec3, 384, 256, st),
             "pool gradient");
  wgrad(u, E3B, a.t3, 128, 0, a.g_dec3, 384, 256, B, H2, W2, st);
  dgrad(u, E3B, a.g_dec3, 384, 256, a.g_t3, 128, 0, a.t3, 128, 0, B, H2, W2, st);
  wgrad(u, E3A, a.p2, 64, 0, a.g_t3, 128, 0, B, H2, W2, st);
  dgrad(u, E3A, a.g_t3, 128, 0, a.g_p2, 64, 0, nullptr, 0, 0, B, H2, W2, st);
  cuda_check(ctas::launch_maxpool_bwd(pool_args(a.dec2, 192, 128, nullptr, 0, 0, B, H1, W1, 64),
                                      a.g_p2, 64, 0, a.g_dec2, 192, 128, st),
             "pool gradient");
  // level 2 encoder
  wgrad(u, E2B, a.t2, 64, 0, a.g_dec2, 192, 128, B, H1, W1, st);
  dgrad(u, E2B, a.g_dec2, 192, 128, a.g_t2, 64, 0, a.t2, 64, 0, B, H1, W1, st);
  wgrad(u, E2A, a.p1, 32, 0, a.g_t2, 64, 0, B, H1, W1, st);
  dgrad(u, E2A, a.g_t2, 64, 0, a.g_p1, 32, 0, nullptr, 0, 0, B, H1, W1, st);
  cuda_check(ctas::launch_maxpool_bwd(pool_args(a.dec1, 96, 64, nullptr, 0, 0, B, H, W, 32),
                                      a.g_p1, 32, 0, a.g_dec1, 96, 64, st),
             "pool gradient");
  // level 1 encoder
  wgrad(u, E1B, a.t1, 32, 0, a.g_dec1, 96, 64, B, H, W, st);
  dgrad(u, E1B, a.g_dec1, 96, 64, a.g_t1, 32, 0, a.t1, 32, 0, B, H, W, st);
  wgrad(u, E1A, a.in16, kInC, 0, a.g_t1, 32, 0, B, H, W, st);
}

void create(ctas_unet *u, uint64_t seed, int32_t device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    ctas::fail(CTAS_E_NODEVICE, "no CUDA device");
  }
  int dev = device;
  if (dev < 0) cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= n) ctas::fail(CTAS_E_ARG, "device ordinal out of range");
  u->device = dev;
  layout(u);
  std::vector<float> p((size_t)u->npar, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < NL; l++) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.0f / (9.0f * kSpec[l].cin)));
    for (int64_t i = 0; i < (int64_t)kSpec[l].cout * 9 * kSpec[l].cin; i++)
      p[(size_t)(u->woff[l] + i)] = nd(rng);
  }
  // head starts at zero: the network starts as the identity on its input
  DevGuard g(dev);
  cuda_check(cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  const size_t fb = sizeof(float) * (size_t)u->npar;
  u->par.ensure(fb);
  u->grad.ensure(fb);
  u->m.ensure(fb);
  u->v.ensure(fb);
  u->parb.ensure(sizeof(bf16) * (size_t)u->npar);
  u->flip.ensure(sizeof(bf16) * (size_t)u->npar);
  cuda_check(cudaMemcpy(u->par.p, p.data(), fb, cudaMemcpyHostToDevice), "cudaMemcpy");
  cuda_check(cudaMemset(u->m.p, 0, fb), "cudaMemset");
  cuda_check(cudaMemset(u->v.p, 0, fb), "cudaMemset");
  refresh_bf16(u, u->stream);
  cuda_check(cudaStreamSynchronize(u->stream), "cudaStreamSynchronize");
}

}  // namespace

extern "C" {

int ctas_unet_create(ctas_unet **out, uint64_t seed, int32_t device) {
  return guarded([&] {
    if (!out) ctas::fail(CTAS_E_ARG, "null output");
    *out = nullptr;
    ctas_unet *u = new ctas_unet();
    try {
      create(u, seed, device);
    } catch (...) {
      delete u;
      throw;
    }
    *out = u;
    return CTAS_OK;
  });
}

int ctas_unet_destroy(ctas_unet *u) {
  delete u;
  return CTAS_OK;
}

int ctas_unet_set_scale(ctas_unet *u, float scale) {
  return guarded([&] {
    if (!u) ctas::fail(CTAS_E_ARG, "null handle");
    if (!(scale > 0.f) || !std::isfinite(scale)) ctas::fail(CTAS_E_ARG, "scale must be positive");
    u->scale = scale;
    return CTAS_OK;
  });
}

int ctas_unet_forward_dev(ctas_unet *u, const float *x_dev, float *y_dev, int64_t B, int64_t H,
                          int64_t W, void *stream) {
  return guarded([&] {
    if (!u || !x_dev || !y_dev) ctas::fail(CTAS_E_ARG, "null argument");
    check_shape(B, H, W);
    check_tc_error();
    DevGuard g(u->device);
    const cudaStream_t st = (cudaStream_t)stream;
    ensure_acts(u, B, H, W, false);
    forward(u, x_dev, B, H, W, 1.f / u->scale, st);
    cuda_check(cudaMemcpyAsync(y_dev, u->act.out, sizeof(float) * (size_t)(B * H * W),
                               cudaMemcpyDeviceToDevice, st),
               "cudaMemcpyAsync");
    return CTAS_OK;
  });
}

int ctas_unet_train_step_dev(ctas_unet *u, const float *x_dev, const float *target_dev, int64_t B,
                             int64_t H, int64_t W, float lr, double *loss, void *stream) {
  return guarded([&] {
    if (!u || !x_dev || !target_dev) ctas::fail(CTAS_E_ARG, "null argument");
    check_shape(B, H, W);
    if (!(lr > 0.f)) ctas::fail(CTAS_E_ARG, "learning rate must be positive");
    DevGuard g(u->device);
    const cudaStream_t st = (cudaStream_t)stream;
    ensure_acts(u, B, H, W, true);
    forward(u, x_dev, B, H, W, 1.f, st);
    backward(u, x_dev, target_dev, B, H, W, st);
    double l = 0.0;
    cuda_check(cudaMemcpyAsync(&l, u->act.loss, sizeof(double), cudaMemcpyDeviceToHost, st),
               "cudaMemcpyAsync");
    u->step++;
    cuda_check(ctas::launch_adam(u->par.as<float>(), u->grad.as<float>(), u->m.as<float>(),
                                 u->v.as<float>(), u->npar, lr, 0.9f, 0.999f, 1e-8f, u->step,
                                 nullptr, st),
               "adam");
    refresh_bf16(u, st);
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    check_tc_error();
    if (loss) *loss = l / (double)(B * H * W);
    return CTAS_OK;
  });
}

int64_t ctas_unet_param_count(const ctas_unet *u) { return u ? u->npar : 0; }

int ctas_unet_get_params(const ctas_unet *u, float *host) {
  return guarded([&] {
    if (!u || !host) ctas::fail(CTAS_E_ARG, "null argument");
    DevGuard g(u->device);
    cuda_check(cudaMemcpy(host, u->par.p, sizeof(float) * (size_t)u->npar, cudaMemcpyDeviceToHost),
               "cudaMemcpy");
    return CTAS_OK;
  });
}

int ctas_unet_set_params(ctas_unet *u, const float *host) {
  return guarded([&] {
    if (!u || !host) ctas::fail(CTAS_E_ARG, "null argument");
    DevGuard g(u->device);
    cuda_check(cudaMemcpy(u->par.p, host, sizeof(float) * (size_t)u->npar, cudaMemcpyHostToDevice),
               "cudaMemcpy");
    refresh_bf16(u, u->stream);
    cuda_check(cudaStreamSynchronize(u->stream), "cudaStreamSynchronize");
    return CTAS_OK;
  });
}

double ctas_unet_macs_per_pixel(void) {
  // level l holds 4^-l of the pixels
  double s = 0.0;
  for (int l = 0; l < NL; l++) s += 9.0 * kSpec[l].cin * kSpec[l].cout / std::pow(4.0, kLevel[l]);
  return s + kHeadC;
}

int ctas_nn_conv3x3_dev(const void *x, int32_t x_cs, int32_t x_co, int32_t cin, const void *w,
                        const float *bias, void *y, int32_t y_cs, int32_t y_co, int32_t cout,
                        const void *mask, int32_t m_cs, int32_t m_co, int64_t B, int64_t H,
                        int64_t W, int32_t relu, void *stream) {
  return guarded([&] {
    if (!x || !w || !y) ctas::fail(CTAS_E_ARG, "null argument");
    ctas::ConvArgs c{};
    c.x = (const bf16 *)x;
    c.x_cs = x_cs;
    c.x_co = x_co;
    c.cin = cin;
    c.w = (const bf16 *)w;
    c.bias = bias;
    c.y = (bf16 *)y;
    c.y_cs = y_cs;
    c.y_co = y_co;
    c.cout = cout;
    c.mask = (const bf16 *)mask;
    c.m_cs = m_cs;
    c.m_co = m_co;
    c.B = (int)B;
    c.H = (int)H;
    c.W = (int)W;
    c.relu = relu;
    if (!ctas::conv_shape_ok(c)) ctas::fail(CTAS_E_SHAPE, "convolution shape not supported");
    check_tc_error();
    cuda_check(ctas::launch_conv3x3(c, (cudaStream_t)stream), "convolution");
    return CTAS_OK;
  });
}

int ctas_nn_conv3x3_wgrad_dev(const void *x, int32_t x_cs, int32_t x_co, int32_t cin,
                              const void *dy, int32_t dy_cs, int32_t dy_co, int32_t cout,
                              float *dw, int64_t B, int64_t H, int64_t W, void *stream) {
  return guarded([&] {
    if (!x || !dy || !dw) ctas::fail(CTAS_E_ARG, "null argument");
    ctas::WgradArgs g{};
    g.x = (const bf16 *)x;
    g.x_cs = x_cs;
    g.x_co = x_co;
    g.cin = cin;
    g.dy = (const bf16 *)dy;
    g.dy_cs = dy_cs;
    g.dy_co = dy_co;
    g.cout = cout;
    g.dw = dw;
    g.B = (int)B;
    g.H = (int)H;
    g.W = (int)W;
    cuda_check(ctas::launch_conv3x3_wgrad(g, (cudaStream_t)stream), "weight gradient");
    return CTAS_OK;
  });
}

int ctas_nn_flip_weights_dev(const void *w, int32_t cout, int32_t cin, void *wt, void *stream) {
  return guarded([&] {
    if (!w || !wt) ctas::fail(CTAS_E_ARG, "null argument");
    if (cout < 1 || cin < 1) ctas::fail(CTAS_E_ARG, "bad channel counts");
    cuda_check(ctas::launch_flip_weights((const bf16 *)w, cout, cin, (bf16 *)wt,
                                         (cudaStream_t)stream),
               "flip weights");
    return CTAS_OK;
  });
}

}  // extern "C"
