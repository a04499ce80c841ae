// probe.cu -- shared-memory gather throughput probe and bounded-wait check
// (see include/ctas_probe.h).
#include <cuda_runtime.h>

#include "../../include/ctas_fbp.h"
#include "../../include/ctas_probe.h"

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeIters = 4096;
constexpr int kUnroll = 16;

__global__ void __launch_bounds__(kProbeThreads) smem_gather_kernel(float *out, int salt) {
  __shared__ float buf[2048];
  for (int k = threadIdx.x; k < 2048; k += blockDim.x) buf[k] = (float)(k ^ salt);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  // each warp reads 32 distinct consecutive-ish words per load: one bank each
  uint32_t base = (uint32_t)__cvta_generic_to_shared(buf) + 4u * (uint32_t)((threadIdx.x >> 5) * 64);
  float acc[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; u++) acc[u] = 0.f;
  for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
    for (int u = 0; u < kUnroll; u++) {
      const uint32_t a = base + 4u * (uint32_t)((lane + u * 5 + it) & 63);
      float v;
      asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
      acc[u] = __fadd_rn(acc[u], v);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int u = 0; u < kUnroll; u++) s += acc[u];
  if (s == 123.456f) out[blockIdx.x] = s;  // keeps the loads alive
}

// An mbarrier that nothing arrives at, waited on with the same bounded
// try-wait loop the pipelined kernels use: the wait must give up after
// `limit` tries, set bit 2 of the error word (the kernels' timeout bit) and
// return, leaving the context usable.
__global__ void bounded_wait_kernel(uint32_t limit, int *err, unsigned long long *tries) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t it = 0, ok = 0;
  for (; it < limit && !ok; ++it)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(b), "r"(0u)
        : "memory");
  if (!ok) atomicOr(err, 4);
  if (threadIdx.x == 0) atomicAdd(tries, (unsigned long long)it);
}

}  // namespace

extern "C" int ctas_probe_bounded_wait(int device, uint32_t limit, int32_t *timed_out,
                                       double *seconds) {
  if (!timed_out || !seconds || limit == 0) return CTAS_E_ARG;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return CTAS_E_NODEVICE;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return CTAS_E_ARG;
  int *err = nullptr;
  unsigned long long *tries = nullptr;
  int rc = CTAS_OK;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&tries, sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(err);
    cudaSetDevice(prev);
    return CTAS_E_NOMEM;
  }
  cudaMemset(err, 0, sizeof(int));
  cudaMemset(tries, 0, sizeof(unsigned long long));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  bounded_wait_kernel<<<1, 32>>>(limit, err, tries);
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess) rc = CTAS_E_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  int herr = 0;
  if (rc == CTAS_OK && cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = CTAS_E_CUDA;
  *timed_out = (herr & 4) ? 1 : 0;
  *seconds = ms * 1e-3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(err);
  cudaFree(tries);
  cudaSetDevice(prev);
  return rc;
}

extern "C" int ctas_probe_smem_gather(int device, double *bytes_per_s, double *seconds) {
  if (!bytes_per_s || !seconds) return CTAS_E_ARG;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return CTAS_E_NODEVICE;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return CTAS_E_ARG;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  cudaEvent_t e0, e1;
  int rc = CTAS_OK;
  if (cudaMalloc(&out, sizeof(float) * 65536) != cudaSuccess) {
    cudaSetDevice(prev);
    return CTAS_E_NOMEM;
  }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8;
  smem_gather_kernel<<<blocks, kProbeThreads>>>(out, 1);  // warm-up
  cudaEventRecord(e0);
  const int reps = 4;
  for (int r = 0; r < reps; r++) smem_gather_kernel<<<blocks, kProbeThreads>>>(out, r);
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess) rc = CTAS_E_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const double loads = (double)reps * blocks * kProbeThreads * kProbeIters * kUnroll;
  *seconds = ms * 1e-3;
  *bytes_per_s = ms > 0 ? loads * 4.0 / (ms * 1e-3) : 0.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  cudaSetDevice(prev);
  return rc;
}
