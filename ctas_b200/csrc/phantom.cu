// phantom.cu -- the synthetic-input generator for tests and benchmarks:
// exact projections of ellipse phantoms on the device (FP64), and ray-marched
// projections of images (the band-limited texture added to the phantoms).
#include <cuda_runtime.h>

#include <string>

#include "../../include/ctas_fbp.h"
#include "../../include/ctas_phantom.h"

namespace {

__global__ void ellipse_sino_kernel(const double *__restrict__ el, int ne, int N, int W,
                                    const double *__restrict__ th, double center, float *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y, s = blockIdx.z;
  if (k >= W) return;
  double sn, cs;
  sincos(th[n], &sn, &cs);
  const double u = (double)k + 0.5 - ((double)(W / 2) + center);
  const double *e = el + (size_t)s * ne * 6;
  double acc = 0.0;
  for (int m = 0; m < ne; m++, e += 6) {
    const double a = e[2], b = e[3];
    if (a <= 0.0 || b <= 0.0) continue;
    double sp, cp;
    sincos(e[4], &sp, &cp);
    const double na = cs * cp + sn * sp, nb = -cs * sp + sn * cp;
    const double r2 = a * a * na * na + b * b * nb * nb;
    const double d = u - (cs * e[0] + sn * e[1]);
    const double q = r2 - d * d;
    if (q > 0.0) acc += 2.0 * e[5] * a * b * sqrt(q) / r2;
  }
  out[((size_t)s * N + n) * W + k] = (float)acc;
}

// Line integrals of S images (W x W; the value of pixel (j, i) sits at object
// point (i - W/2, j - W/2 - center)), added to out: the ray of detector sample
// k of projection n, x cos th + y sin th = u with u = k + 0.5 - W/2 - center,
// is sampled every `step` pixels along the chord of the disc of radius `R`
// around the axis, bilinearly (zero outside the image).
__global__ void image_sino_kernel(const float *__restrict__ img, int W, int N,
                                  const double *__restrict__ th, double center, float R,
                                  float step, float *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y, s = blockIdx.z;
  if (k >= W) return;
  double sn, cs;
  sincos(th[n], &sn, &cs);
  const float hp = (float)(W / 2);
  const float u = (float)((double)k + 0.5 - ((double)(W / 2) + center));
  float *o = out + ((size_t)s * N + n) * W + k;
  if (fabsf(u) >= R) return;
  const float half = sqrtf(R * R - u * u);
  const float c = (float)cs, sv = (float)sn;
  const float fi0 = u * c + hp, fj0 = u * sv + hp + (float)center;
  const float *im = img + (size_t)s * W * W;
  const int steps = (int)(2.f * half / step) + 1;
  float acc = 0.f;
  for (int m = 0; m < steps; m++) {
    const float t = -half + ((float)m + 0.5f) * step;
    const float fi = fi0 - t * sv, fj = fj0 + t * c;
    const float i0f = floorf(fi), j0f = floorf(fj);
    const int i0 = (int)i0f, j0 = (int)j0f;
    const float wx = fi - i0f, wy = fj - j0f;
    float v = 0.f;
    if (j0 >= 0 && j0 < W) {
      if (i0 >= 0 && i0 < W) v += (1.f - wx) * (1.f - wy) * im[(size_t)j0 * W + i0];
      if (i0 + 1 >= 0 && i0 + 1 < W) v += wx * (1.f - wy) * im[(size_t)j0 * W + i0 + 1];
    }
    if (j0 + 1 >= 0 && j0 + 1 < W) {
      if (i0 >= 0 && i0 < W) v += (1.f - wx) * wy * im[(size_t)(j0 + 1) * W + i0];
      if (i0 + 1 >= 0 && i0 + 1 < W) v += wx * wy * im[(size_t)(j0 + 1) * W + i0 + 1];
    }
    acc += v;
  }
  *o += acc * step;
}

}  // namespace

extern "C" int ctas_phantom_project_image_dev(const float *img, int64_t S, int64_t N, int64_t W,
                                              const double *th, double center, double radius,
                                              double step, float *out, void *stream) {
  if (!img || !th || !out || S <= 0 || N <= 0 || W <= 0 || N > 65535 || S > 65535 ||
      !(radius > 0.0) || !(step > 0.0))
    return CTAS_E_ARG;
  const dim3 grid((unsigned)((W + 127) / 128), (unsigned)N, (unsigned)S);
  image_sino_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(img, (int)W, (int)N, th, center,
                                                            (float)radius, (float)step, out);
  return cudaGetLastError() == cudaSuccess ? CTAS_OK : CTAS_E_CUDA;
}

extern "C" int ctas_phantom_sinogram_dev(const double *el, int64_t ne, int64_t S, int64_t N,
                                         int64_t W, const double *th, double center, float *out,
                                         void *stream) {
  if (!el || !th || !out || ne < 0 || S <= 0 || N <= 0 || W <= 0 || N > 65535 || S > 65535)
    return CTAS_E_ARG;
  const dim3 grid((unsigned)((W + 127) / 128), (unsigned)N, (unsigned)S);
  ellipse_sino_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(el, (int)ne, (int)N, (int)W, th,
                                                               center, out);
  return cudaGetLastError() == cudaSuccess ? CTAS_OK : CTAS_E_CUDA;
}
