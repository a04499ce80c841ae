// phantom.cu -- exact projections of ellipse phantoms on the device (FP64),
// the synthetic-input generator for tests and benchmarks.
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

}  // namespace

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
