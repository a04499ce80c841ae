// volume.cu -- output sample conversion of the streamed volume writer.
//
// The reference converts each reconstructed slice on the host before it is
// written: limit<T> (src/common/external.world.cpp:69-90), called by SaveImage
// (1625-1680) and HDFwrapper::write (737-760) for the ct tool's -i/-m/-M
// (src/executables/ct.cpp:110-116).  Here the conversion runs on the device
// before the device->host copy, so an 8- or 16-bit volume also moves 4x or
// 2x fewer bytes over PCIe.  Each element follows the reference's float
// operations in order, each rounded once (no contraction):
//   interim = (v - mincon) / (maxcon - mincon)
//   interim < 0 -> min, interim > 1 -> max, else T(float(min) + interim * (float(max) - float(min)))
// with C++'s truncation toward zero for the final conversion.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <limits>
#include <string>

#include "../../include/ctas_volume.h"
#include "fbp_host.hpp"
#include "fbp_kernels.hpp"

namespace ctas {
namespace {

// float -> T truncating toward zero.  The PTX conversions saturate, which is
// where C++ is undefined (a float that reaches 2^31, 2^32, 2^63 or 2^64).
template <class T> __device__ __forceinline__ T trunc_to(float v);
template <> __device__ __forceinline__ int8_t trunc_to<int8_t>(float v) {
  return (int8_t)__float2int_rz(v);
}
template <> __device__ __forceinline__ uint8_t trunc_to<uint8_t>(float v) {
  return (uint8_t)__float2uint_rz(v);
}
template <> __device__ __forceinline__ int16_t trunc_to<int16_t>(float v) {
  return (int16_t)__float2int_rz(v);
}
template <> __device__ __forceinline__ uint16_t trunc_to<uint16_t>(float v) {
  return (uint16_t)__float2uint_rz(v);
}
template <> __device__ __forceinline__ int32_t trunc_to<int32_t>(float v) {
  return __float2int_rz(v);
}
template <> __device__ __forceinline__ uint32_t trunc_to<uint32_t>(float v) {
  return __float2uint_rz(v);
}
template <> __device__ __forceinline__ int64_t trunc_to<int64_t>(float v) {
  return (int64_t)__float2ll_rz(v);
}
template <> __device__ __forceinline__ uint64_t trunc_to<uint64_t>(float v) {
  return (uint64_t)__float2ull_rz(v);
}

template <class T>
__device__ __forceinline__ T limit_one(float v, float mn, float lw) {
  constexpr float lo = (float)std::numeric_limits<T>::min();
  constexpr float tw = (float)std::numeric_limits<T>::max() - (float)std::numeric_limits<T>::min();
  const float interim = __fdiv_rn(__fsub_rn(v, mn), lw);
  if (interim < 0.f) return std::numeric_limits<T>::min();
  if (interim > 1.f) return std::numeric_limits<T>::max();
  return trunc_to<T>(__fadd_rn(lo, __fmul_rn(interim, tw)));
}

template <class T> struct alignas(4 * sizeof(T) < 16 ? 4 * sizeof(T) : 16) Pack4 {
  T v[4];
};

// blockIdx.y = image; grid-stride over its pixels, four per step when vec.
template <class T>
__global__ void __launch_bounds__(256)
    quantize_kernel(const float *__restrict__ src, int64_t pixels, float mincon, float maxcon,
                    const float2 *__restrict__ range, T *__restrict__ dst, int vec) {
  const int64_t img = blockIdx.y;
  float mn = mincon, mx = maxcon;
  if (mn == mx) {  // limit<T>: the image's own range (external.world.cpp:71-74)
    const float2 r = range[img];
    mn = r.x;
    mx = r.y;
  }
  const float *p = src + img * pixels;
  T *q = dst + img * pixels;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (mn == mx) {  // all values equal: zeros (external.world.cpp:75-78)
    for (int64_t i = t0; i < pixels; i += stride) q[i] = T(0);
    return;
  }
  const float lw = __fsub_rn(mx, mn);
  if (vec) {
    const int64_t n4 = pixels >> 2;
    const float4 *p4 = reinterpret_cast<const float4 *>(p);
    Pack4<T> *q4 = reinterpret_cast<Pack4<T> *>(q);
    for (int64_t i = t0; i < n4; i += stride) {
      const float4 v = __ldcs(p4 + i);
      Pack4<T> o;
      o.v[0] = limit_one<T>(v.x, mn, lw);
      o.v[1] = limit_one<T>(v.y, mn, lw);
      o.v[2] = limit_one<T>(v.z, mn, lw);
      o.v[3] = limit_one<T>(v.w, mn, lw);
      q4[i] = o;
    }
  } else {
    for (int64_t i = t0; i < pixels; i += stride) q[i] = limit_one<T>(p[i], mn, lw);
  }
}

template <class T>
cudaError_t launch_t(const float *src, int64_t pixels, int S, float mincon, float maxcon,
                     const float2 *range, void *dst, cudaStream_t st) {
  const bool vec = pixels % 4 == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(dst) & (alignof(Pack4<T>) - 1)) == 0;
  const int64_t work = vec ? pixels / 4 : pixels;
  const int64_t want = (work + 255) / 256;
  const int64_t cap = std::max<int64_t>(1, 2368 / std::max(1, S));  // about 16 blocks per SM
  const unsigned nb = (unsigned)std::max<int64_t>(1, std::min(want, cap));
  quantize_kernel<T><<<dim3(nb, (unsigned)S), 256, 0, st>>>(src, pixels, mincon, maxcon, range,
                                                            static_cast<T *>(dst), vec ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace

int quantize_sample_bytes(int bpp) {
  switch (bpp) {
    case 0: return 4;
    case 8: case -8: return 1;
    case 16: case -16: return 2;
    case 32: case -32: return 4;
    case 64: case -64: return 8;
    default: return 0;
  }
}

cudaError_t launch_quantize(const float *src, int64_t pixels, int S, int bpp, float mincon,
                            float maxcon, const float2 *range, void *dst, cudaStream_t st) {
  if (S <= 0 || pixels <= 0) return cudaSuccess;
  switch (bpp) {
    case 8: return launch_t<uint8_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case -8: return launch_t<int8_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case 16: return launch_t<uint16_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case -16: return launch_t<int16_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case 32: return launch_t<uint32_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case -32: return launch_t<int32_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case 64: return launch_t<uint64_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    case -64: return launch_t<int64_t>(src, pixels, S, mincon, maxcon, range, dst, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ctas

namespace {

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

void cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  ctas::fail(e == cudaErrorMemoryAllocation ? CTAS_E_NOMEM : CTAS_E_CUDA,
             std::string("sample conversion: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int32_t ctas_vol_sample_bytes(int32_t bpp) { return ctas::quantize_sample_bytes(bpp); }

int ctas_vol_quantize_dev(const float *src, int64_t n_images, int64_t pixels, int32_t bpp,
                          float mincon, float maxcon, void *dst, void *stream) {
  return guarded([&] {
    if (bpp == 0 || ctas::quantize_sample_bytes(bpp) == 0)
      ctas::fail(CTAS_E_ARG, "bits per sample must be one of +-8, +-16, +-32, +-64");
    if (n_images < 0 || pixels < 0) ctas::fail(CTAS_E_ARG, "negative size");
    if (n_images == 0 || pixels == 0) return CTAS_OK;
    if (!src || !dst) ctas::fail(CTAS_E_ARG, "null buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t sb = ctas::quantize_sample_bytes(bpp);
    const bool own_range = mincon == maxcon;
    for (int64_t i0 = 0; i0 < n_images; i0 += 65535) {
      const int S = (int)std::min<int64_t>(65535, n_images - i0);
      const float *s = src + i0 * pixels;
      void *d = static_cast<char *>(dst) + i0 * pixels * sb;
      float2 *scratch = nullptr;
      if (own_range) {
        cuda_ok(cudaMallocAsync((void **)&scratch,
                                sizeof(float2) * (size_t)S * (ctas::kMinMaxBlocks + 1), st),
                "cudaMallocAsync");
        cuda_ok(ctas::launch_minmax(s, pixels, pixels, S, scratch + S, scratch, nullptr, st),
                "range kernel");
      }
      const cudaError_t e =
          ctas::launch_quantize(s, pixels, S, bpp, mincon, maxcon, scratch, d, st);
      if (scratch) cudaFreeAsync(scratch, st);
      cuda_ok(e, "conversion kernel");
    }
    return CTAS_OK;
  });
}

}  // extern "C"
