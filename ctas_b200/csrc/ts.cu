// ts.cu -- tomosynthesis step ts_add (ctas src/common/lct.cpp:731-787) on the
// device: the row filter of the reference's unpadded FFT, and the
// single-angle clamped nearest-sample backprojection.
//
// Filter.  The reference filters each row of length n (= pixels) with
// HC2R(R2HC(z) * f) / n, f = Filter::fill(n): a circular convolution of length
// n with the real, even kernel g = IDFT_n(f).  The device FFT is a power of two
// P >= 2n - 1 (the CT padding rule), so the row is extended periodically (two
// periods from offset n/2; filter kernel "periodic" mode) and multiplied by
// G_P = DFT_P(h), h the kernel g laid out symmetrically about 0 (|d| <= n/2;
// for even n the d = n/2 tap is split between +-n/2).  For outputs n/2 ..
// 3n/2 - 1 every tap reads inside the two periods, so the result is the
// circular convolution up to float rounding.
//
// Backprojection.  One thread per result pixel adds the n images' terms in
// order, with the reference's float expression for the sample index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ctas_fbp.h"
#include "../../include/ctas_ts.h"
#include "fbp_host.hpp"
#include "fbp_kernels.hpp"

namespace {

struct TsBpLaunch {
  const float *q;     // images x rows x Wp, sample c at column kRowOff + c
  int64_t img_stride;
  int rows, W, Wp, n;
  const float2 *cs;   // per image (cos(angle), (plane - center) * sin(angle))
  float rc;           // Rcenter = pixels * 0.5 + center
  float *result;      // rows x W
};

__global__ void ts_bp_kernel(TsBpLaunch a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= a.W) return;
  float *r = a.result + (int64_t)y * a.W + x;
  float acc = *r;
  const float wf = (float)a.W, wl = (float)(a.W - 1);
  const float dx = __fsub_rn((float)x, a.rc);  // (xcur - Rcenter)
  const float *row = a.q + (int64_t)y * a.Wp + ctas::kRowOff;
  for (int i = 0; i < a.n; i++) {
    const float2 c = a.cs[i];
    // di = (xcur - Rcenter)*cur_cos - plane_cos + Rcenter  (lct.cpp:778)
    float di = __fadd_rn(__fsub_rn(__fmul_rn(dx, c.x), c.y), a.rc);
    di = (di < 0.f) ? 0.f : ((di >= wf) ? wl : di);
    acc = __fadd_rn(acc, row[(int64_t)i * a.img_stride + (int)di]);
  }
  *r = acc;
}

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
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = CTAS_E_NODEVICE;
  cudaGetLastError();
  ctas::fail(code, std::string("tomosynthesis: ") + what + ": " + cudaGetErrorString(e));
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

}  // namespace

struct ctas_ts {
  int device = 0;
  int64_t rows = 0, W = 0, P = 0, Wp = 0;
  int32_t contrast = 2;
  std::vector<int> radices;
  cudaStream_t stream = nullptr;  // host calls
  Buf tw, gperm, q, cs, host_in, host_out;
  int64_t chunk = 1;  // images filtered per launch
  ~ctas_ts() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    tw.release();
    gperm.release();
    q.release();
    cs.release();
    host_in.release();
    host_out.release();
    if (stream) cudaStreamDestroy(stream);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

namespace {

// G_P[f] = DFT_P of the symmetric layout of g = IDFT_n(fwin), f = 0 .. P-1.
std::vector<double> ts_window(const std::vector<float> &fwin, int64_t n, int64_t P) {
  std::vector<double> cn((size_t)n), cp((size_t)P);
  for (int64_t m = 0; m < n; m++) cn[(size_t)m] = std::cos(2.0 * M_PI * (double)m / (double)n);
  for (int64_t m = 0; m < P; m++) cp[(size_t)m] = std::cos(2.0 * M_PI * (double)m / (double)P);
  const int64_t half = n / 2;
  std::vector<double> g((size_t)half + 1);
  for (int64_t d = 0; d <= half; d++) {
    double s = 0.0;
    for (int64_t k = 0; k < n; k++) s += (double)fwin[(size_t)k] * cn[(size_t)((k * d) % n)];
    g[(size_t)d] = s / (double)n;
  }
  // tap weights of h on d = 0 .. half: w_0 = g0, w_d = 2 g_d, and for even n
  // the d = n/2 tap once (split between +-n/2)
  std::vector<double> w((size_t)half + 1);
  w[0] = g[0];
  for (int64_t d = 1; d <= half; d++) w[(size_t)d] = (n % 2 == 0 && d == half) ? g[(size_t)d] : 2.0 * g[(size_t)d];
  std::vector<double> G((size_t)P);
  for (int64_t f = 0; f < P; f++) {
    double s = 0.0;
    for (int64_t d = 0; d <= half; d++) s += w[(size_t)d] * cp[(size_t)((f * d) % P)];
    G[(size_t)f] = s;
  }
  return G;
}

void ts_create(ctas_ts *h, int64_t rows, int64_t pixels, int32_t ftype, float fparam,
               int32_t contrast, int32_t device) {
  if (rows < 1 || pixels < 2)
    ctas::fail(CTAS_E_SHAPE, "tomosynthesis: image must have at least 1 row and 2 columns");
  if (contrast < 0 || contrast > 3) ctas::fail(CTAS_E_ARG, "unknown contrast");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    ctas::fail(CTAS_E_NODEVICE, "no CUDA device");
  }
  int dev = device;
  if (dev < 0) cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= ndev) ctas::fail(CTAS_E_ARG, "device ordinal out of range");
  h->device = dev;
  h->rows = rows;
  h->W = pixels;
  h->P = ctas::padded_width(pixels);
  if (h->P > 16384)  // the row-pair FFT lives in shared memory
    ctas::fail(CTAS_E_UNSUPPORTED, "tomosynthesis: rows wider than 8192 pixels are not supported");
  h->Wp = ctas::padded_pitch(pixels);
  // ts_add filters for every contrast; ABS adds -log, REF the running sum
  h->contrast = contrast == CTAS_FLT ? CTAS_PHS : contrast;
  h->radices = ctas::fft_radices(h->P);
  const std::vector<float> fwin = ctas::filter_fill(ftype, fparam, pixels);  // Filter::fill(n)
  const std::vector<double> G = ts_window(fwin, pixels, h->P);
  const auto perm = ctas::fft_output_order(h->P, h->radices);
  std::vector<float> gp((size_t)h->P);
  const float invP = 1.0f / (float)h->P;
  for (int64_t p = 0; p < h->P; p++) gp[(size_t)p] = (float)G[(size_t)perm[(size_t)p]] * invP;
  const auto tw = ctas::fft_twiddles(h->P);
  DevGuard g(dev);
  cuda_check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  h->tw.ensure(sizeof(float) * tw.size());
  h->gperm.ensure(sizeof(float) * gp.size());
  cuda_check(cudaMemcpy(h->tw.p, tw.data(), sizeof(float) * tw.size(), cudaMemcpyHostToDevice),
             "cudaMemcpy");
  cuda_check(cudaMemcpy(h->gperm.p, gp.data(), sizeof(float) * gp.size(), cudaMemcpyHostToDevice),
             "cudaMemcpy");
  const int64_t per = rows * h->Wp * (int64_t)sizeof(float);
  h->chunk = std::max<int64_t>(1, std::min<int64_t>(65535, ((int64_t)2 << 30) / per));
}

// n images of projections (device) added into result (device), in order.
void ts_run(ctas_ts *h, float *proj, const float *angles, int64_t n, float *result, float center,
            int32_t plane, uint32_t flags, cudaStream_t st) {
  const int64_t rows = h->rows, W = h->W;
  const float rc = (float)((double)W * 0.5 + (double)center);  // Rcenter
  std::vector<float2> cs((size_t)n);
  for (int64_t i = 0; i < n; i++) {
    const float cur_sin = std::sin(angles[i]), cur_cos = std::cos(angles[i]);  // sinf / cosf
    const float plane_cos = ((float)plane - center) * cur_sin;
    cs[(size_t)i] = make_float2(cur_cos, plane_cos);
  }
  const int64_t C = std::min(h->chunk, n);
  h->q.ensure(sizeof(float) * (size_t)(C * rows * h->Wp));
  h->cs.ensure(sizeof(float2) * (size_t)n);
  cuda_check(cudaMemcpyAsync(h->cs.p, cs.data(), sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice,
                             st),
             "cudaMemcpyAsync");
  for (int64_t i0 = 0; i0 < n; i0 += C) {
    const int64_t m = std::min(C, n - i0);
    float *x = proj + i0 * rows * W;
    ctas::FilterLaunch a{};
    a.x = x;
    a.x_slice_stride = rows * W;
    a.q = h->q.p;
    a.q_slice_stride = rows * h->Wp;
    a.tw = h->tw.as<float2>();
    a.gperm = h->gperm.as<float>();
    a.minmax = nullptr;  // ABS: plain -log (lct.cpp:735-736)
    a.N = (int)rows;
    a.W = (int)W;
    a.Wp = (int)h->Wp;
    a.P = (int)h->P;
    a.zs = (int)(W / 2);
    a.contrast = h->contrast;
    a.store = 0;
    a.nradix = (int)h->radices.size();
    for (size_t k = 0; k < h->radices.size(); k++) a.radix[k] = h->radices[k];
    a.S = (int)m;
    a.guard = 0;
    a.periodic = 1;
    cuda_check(ctas::launch_filter(a, st), "filter kernel");
    TsBpLaunch b{};
    b.q = h->q.as<float>();
    b.img_stride = rows * h->Wp;
    b.rows = (int)rows;
    b.W = (int)W;
    b.Wp = (int)h->Wp;
    b.n = (int)m;
    b.cs = h->cs.as<float2>() + i0;
    b.rc = rc;
    b.result = result;
    ts_bp_kernel<<<dim3((unsigned)((W + 255) / 256), (unsigned)rows), 256, 0, st>>>(b);
    cuda_check(cudaGetLastError(), "tomosynthesis kernel");
    if (!(flags & CTAS_FLAG_NO_WRITEBACK))
      cuda_check(ctas::launch_unpad(h->q.p, rows * h->Wp, nullptr, 0, (int)rows, (int)W,
                                    (int)h->Wp, (int)m, x, rows * W, st),
                 "unpad kernel");
  }
}

}  // namespace

extern "C" {

int ctas_ts_create(ctas_ts **out, int64_t rows, int64_t pixels, int32_t ftype, float fparam,
                   int32_t contrast, int32_t device) {
  return guarded([&] {
    if (!out) ctas::fail(CTAS_E_ARG, "null output");
    *out = nullptr;
    ctas_ts *h = new ctas_ts();
    try {
      ts_create(h, rows, pixels, ftype, fparam, contrast, device);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return CTAS_OK;
  });
}

int ctas_ts_destroy(ctas_ts *h) {
  delete h;
  return CTAS_OK;
}

int ctas_ts_add_dev(ctas_ts *h, float *projection_dev, float *result_dev, float center,
                    float angle, int32_t plane, uint32_t flags, void *stream) {
  return guarded([&] {
    if (!h || !projection_dev || !result_dev) ctas::fail(CTAS_E_ARG, "null argument");
    DevGuard g(h->device);
    const cudaStream_t st = (cudaStream_t)stream;
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");  // parameter buffer reuse
    ts_run(h, projection_dev, &angle, 1, result_dev, center, plane, flags, st);
    return CTAS_OK;
  });
}

int ctas_ts_add_batch_dev(ctas_ts *h, float *projections_dev, const float *angles, int64_t n,
                          float *result_dev, float center, int32_t plane, uint32_t flags,
                          void *stream) {
  return guarded([&] {
    if (!h || !projections_dev || !result_dev || !angles) ctas::fail(CTAS_E_ARG, "null argument");
    if (n < 1) ctas::fail(CTAS_E_ARG, "no projections");
    DevGuard g(h->device);
    const cudaStream_t st = (cudaStream_t)stream;
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    ts_run(h, projections_dev, angles, n, result_dev, center, plane, flags, st);
    return CTAS_OK;
  });
}

int ctas_ts_add(ctas_ts *h, float *projection, float *result, float center, float angle,
                int32_t plane, uint32_t flags) {
  return guarded([&] {
    if (!h || !projection || !result) ctas::fail(CTAS_E_ARG, "null argument");
    DevGuard g(h->device);
    const size_t bytes = sizeof(float) * (size_t)(h->rows * h->W);
    h->host_in.ensure(bytes);
    h->host_out.ensure(bytes);
    cuda_check(cudaMemcpyAsync(h->host_in.p, projection, bytes, cudaMemcpyHostToDevice, h->stream),
               "cudaMemcpyAsync");
    cuda_check(cudaMemcpyAsync(h->host_out.p, result, bytes, cudaMemcpyHostToDevice, h->stream),
               "cudaMemcpyAsync");
    ts_run(h, h->host_in.as<float>(), &angle, 1, h->host_out.as<float>(), center, plane, flags,
           h->stream);
    cuda_check(cudaMemcpyAsync(result, h->host_out.p, bytes, cudaMemcpyDeviceToHost, h->stream),
               "cudaMemcpyAsync");
    if (!(flags & CTAS_FLAG_NO_WRITEBACK))
      cuda_check(cudaMemcpyAsync(projection, h->host_in.p, bytes, cudaMemcpyDeviceToHost,
                                 h->stream),
                 "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
    return CTAS_OK;
  });
}

}  // extern "C"
