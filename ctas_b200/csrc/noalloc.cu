// noalloc.cu -- filtered backprojection that allocates nothing.
//
// Some callers cannot allocate device memory while they reconstruct: code that
// runs inside a framework owning every device allocation (a memory pool or a
// graph-replay runtime that forbids cudaMalloc), real-time acquisition loops
// with a fixed memory budget, or plug-ins loaded into a host process whose
// allocator they must not touch.  For them, ctas_fbp_reconstruct_dev_noalloc
// runs the same filter and backprojection kernels as a handle does, with all
// of its scratch -- the padded filtered sinogram, the FFT twiddles, the
// window and the angle table -- in one fixed array of this file
// (g_noalloc_scratch, kNoAllocScratchBytes), and its host-side tables in
// fixed host arrays.  It calls no cudaMalloc, cudaFree or allocating library
// routine; the caller passes the input sinogram and the output slice.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <mutex>
#include <string>

#include "../../include/ctas_fbp.h"
#include "bp_fast.hpp"
#include "fbp_host.hpp"
#include "fbp_kernels.hpp"

namespace {

// 32 MiB: a 1800 x 2560 sinogram at FFT length 8192 needs 18.5 MiB.  Every
// GPU that loads this library holds the array until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int64_t kMaxPad = 16384;        // FFT length (shared-memory FFT limit)
constexpr int64_t kMaxAngles = 16384;     // host table capacity
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mutex;                       // serialises calls (shared scratch)
void *g_scratch_addr[kMaxDevices] = {};   // device address, per device

// host staging, reused by every call under g_mutex
std::complex<double> h_fft[kMaxPad];
float h_window[kMaxPad];
float h_gperm[kMaxPad];
float h_tw[2 * kMaxPad];
float h_tab[2 * kMaxAngles];
int h_err = 0;

int fail_with(int code, const std::string &m) {
  ctas::set_last_error(m);  // read back by ctas_fbp_last_error()
  return code;
}

size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" int ctas_fbp_reconstruct_dev_noalloc(const float *sino_dev, float *slice_dev,
                                                int64_t n_angles, int64_t width,
                                                int32_t contrast, int32_t ftype, float fparam,
                                                float arc_deg, int64_t pad, float center,
                                                float pixel_size_m, float lambda_m,
                                                void *stream) {
  try {
    if (!sino_dev || !slice_dev) return fail_with(CTAS_E_ARG, "null buffer");
    if (width < 2)
      return fail_with(CTAS_E_SHAPE, "Number of pixels in the CT reconstruction less than 2.");
    if (n_angles <= 0) return fail_with(CTAS_E_SHAPE, "Zero projections in sinogram.");
    if (contrast == CTAS_ABS)
      return fail_with(CTAS_E_UNSUPPORTED,
                       "absorption contrast needs a device reduction; use a handle");
    if (contrast < 0 || contrast > 3) return fail_with(CTAS_E_ARG, "unknown contrast");
    ctas::filter_check(ftype, fparam);
    const int64_t P = pad ? pad : ctas::padded_width(width);
    if (pad && ((pad & (pad - 1)) != 0 || pad < width))
      return fail_with(CTAS_E_ARG, "pad must be a power of two >= width");
    if (P < 4 || P > kMaxPad)
      return fail_with(CTAS_E_SHAPE, "padded width " + std::to_string(P) +
                                         " outside the supported range [4, 16384]");
    if (n_angles > kMaxAngles)
      return fail_with(CTAS_E_SHAPE, "at most 16384 projections per call");
    if (!(std::fabs(center) < (float)(width / 2)))
      return fail_with(CTAS_E_CENTER, "Rotation center " + std::to_string(center) +
                                          " is outside the sinogram width " +
                                          std::to_string(width) + ".");
    // scratch layout: padded filtered rows | twiddles | window | angle table | error word
    const int64_t Wp = ctas::padded_pitch(width);
    const size_t b_filt = round256(sizeof(float) * (size_t)(n_angles * Wp));
    const size_t b_tw = round256(sizeof(float) * 2 * (size_t)P);
    const size_t b_g = round256(sizeof(float) * (size_t)P);
    const size_t b_tab = round256(sizeof(float) * 2 * (size_t)n_angles);
    const size_t need = b_filt + b_tw + b_g + b_tab + 256;
    if (need > kNoAllocScratchBytes)
      return fail_with(CTAS_E_SHAPE,
                       "a " + std::to_string(n_angles) + " x " + std::to_string(width) +
                           " sinogram needs " + std::to_string(need) +
                           " bytes of scratch; this entry point holds at most " +
                           std::to_string(kNoAllocScratchBytes) + " bytes (32 MiB)");

    cudaStream_t st = (cudaStream_t)stream;
    // The call copies a result word back and waits for its stream, neither of
    // which a capturing stream allows.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
      cudaGetLastError();
      return fail_with(CTAS_E_ARG, "invalid stream");
    }
    if (cap != cudaStreamCaptureStatusNone)
      return fail_with(CTAS_E_ARG, "ctas_fbp_reconstruct_dev_noalloc cannot run on a capturing "
                                   "stream (it waits for its own work before returning)");

    std::lock_guard<std::mutex> lock(g_mutex);
    // Declared after the lock, so destroyed before it: whatever way the call
    // leaves once work is queued, the stream is drained while the lock is
    // still held, and the next call cannot overwrite scratch that queued
    // kernels still read.  The kernels' device waits are bounded, so the
    // drain ends.
    struct Drain {
      cudaStream_t st;
      bool armed = false;
      ~Drain() {
        if (armed) {
          cudaStreamSynchronize(st);
          cudaGetLastError();
        }
      }
    } drain{st};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
      return fail_with(CTAS_E_NODEVICE, "no current CUDA device");
    // set-up, once per device with that device current: the array's name is a
    // host-side stand-in, the kernels need its device address
    if (!g_scratch_addr[dev]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail_with(CTAS_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_addr[dev] = p;
    }
    unsigned char *base = static_cast<unsigned char *>(g_scratch_addr[dev]);
    float *d_filt = reinterpret_cast<float *>(base);
    float *d_tw = reinterpret_cast<float *>(base + b_filt);
    float *d_g = reinterpret_cast<float *>(base + b_filt + b_tw);
    float *d_tab = reinterpret_cast<float *>(base + b_filt + b_tw + b_g);
    int *d_err = reinterpret_cast<int *>(base + b_filt + b_tw + b_g + b_tab);

    // host tables (the handle computes the same ones at create time)
    ctas::filter_fill_into(ftype, fparam, P, h_window, h_fft);
    const float scale = (float)P / (float)width;               // lct.cpp:506
    for (int64_t k = 0; k < P; k++) h_window[k] = h_window[k] * scale;
    if (contrast == CTAS_REF) h_window[0] = 0.0f;              // lct.cpp:507-508
    const float invP = 1.0f / (float)P;
    for (int64_t p = 0; p < P; p++) h_gperm[p] = h_window[ctas::fft_output_frequency(P, p)] * invP;
    ctas::fft_twiddles_into(P, h_tw);
    ctas::angle_table_into(arc_deg, n_angles, h_tab);
    bool sines_nonneg = true;
    for (int64_t i = 0; i < n_angles; i++)
      if (h_tab[2 * i] < 0.0f) sines_nonneg = false;

    auto ck = [](cudaError_t e, const char *what) {
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw ctas::Error{CTAS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
      }
    };
    // the array keeps the previous call's contents: clear what must start at 0
    drain.armed = true;
    ck(cudaMemsetAsync(d_filt, 0, b_filt, st), "cudaMemsetAsync");
    ck(cudaMemsetAsync(d_err, 0, sizeof(int), st), "cudaMemsetAsync");
    ck(cudaMemcpyAsync(d_tw, h_tw, sizeof(float) * 2 * (size_t)P, cudaMemcpyHostToDevice, st),
       "cudaMemcpyAsync");
    ck(cudaMemcpyAsync(d_g, h_gperm, sizeof(float) * (size_t)P, cudaMemcpyHostToDevice, st),
       "cudaMemcpyAsync");
    ck(cudaMemcpyAsync(d_tab, h_tab, sizeof(float) * 2 * (size_t)n_angles,
                       cudaMemcpyHostToDevice, st),
       "cudaMemcpyAsync");

    ctas::FilterLaunch fl{};
    fl.x = sino_dev;
    fl.x_slice_stride = n_angles * width;
    fl.q = d_filt;
    fl.q_slice_stride = n_angles * Wp;
    fl.tw = reinterpret_cast<const float2 *>(d_tw);
    fl.gperm = d_g;
    fl.N = (int)n_angles;
    fl.W = (int)width;
    fl.Wp = (int)Wp;
    fl.P = (int)P;
    fl.zs = (int)((P - width) / 2);
    fl.contrast = contrast;
    fl.store = 0;
    int lg = 0;
    while ((int64_t(1) << lg) < P) lg++;
    for (int s = 0; s < lg / 3; s++) fl.radix[fl.nradix++] = 8;
    if (lg % 3 == 1) fl.radix[fl.nradix++] = 2;
    if (lg % 3 == 2) fl.radix[fl.nradix++] = 4;
    fl.S = 1;
    fl.guard = 1;
    ck(ctas::launch_filter(fl, st), "filter kernel");

    ctas::BpLaunch bl{};
    bl.q = d_filt;
    bl.q_slice_stride = n_angles * Wp;
    bl.store = 0;
    bl.N = (int)n_angles;
    bl.W = (int)width;
    bl.Wp = (int)Wp;
    bl.tab = reinterpret_cast<const float2 *>(d_tab);
    bl.center = center;
    bl.rec_cof = ctas::rec_cof(pixel_size_m, lambda_m);
    bl.out = slice_dev;
    bl.out_slice_stride = width * width;
    bl.S = 1;
    bl.err = d_err;
    bl.out_rows = (int)width;
    bl.out_cols = (int)width;
    bl.geo_oj = 0.f;
    bl.geo_oi = 0.f;
    bl.geo_p = 1.f;
    bl.interp = 0;
    bl.lin = nullptr;
    // a fixed tile: the autotuner would synchronise and create events
    if (sines_nonneg && ctas::bp_fast_supported(bl)) {
      const cudaError_t e = ctas::launch_bp_fast(bl, st, 1);
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw ctas::Error{CTAS_E_CUDA, std::string("backprojection kernel: ") +
                                           cudaGetErrorString(e) + " " +
                                           ctas::bp_fast_error_detail()};
      }
    } else {
      ck(ctas::launch_bp_generic(bl, st), "backprojection kernel");
    }

    // wait for this call's work: the next call reuses the scratch and tables
    ck(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st),
       "cudaMemcpyAsync");
    ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    drain.armed = false;
    if (h_err & 4)
      return fail_with(CTAS_E_TIMEOUT, "a device wait timed out in the backprojection kernel");
    if (h_err) return fail_with(CTAS_E_CUDA, "device error word " + std::to_string(h_err));
    return CTAS_OK;
  } catch (const ctas::Error &e) {
    return fail_with(e.code, e.msg);
  }
}
