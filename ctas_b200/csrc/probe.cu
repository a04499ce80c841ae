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
  // each warp reads 32 distinct words per load, one bank each; the addresses
  // are formed once, so the loop issues one load and one add per gather and
  // the shared-memory pipe, not the issue rate, sets the pace (address
  // arithmetic inside the loop held an earlier form to ~80 % of the pipe).
  // The loads are volatile: nothing stores to `buf` inside the loop, and a
  // plain load at a loop-invariant address may be kept in a register.
  const uint32_t base =
      (uint32_t)__cvta_generic_to_shared(buf) + 4u * (uint32_t)((threadIdx.x >> 5) * 64);
  uint32_t addr[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; u++) addr[u] = base + 4u * (uint32_t)((lane + u * 5) & 63);
  float acc[kUnroll];
#pragma unroll
  for (int u = 0; u < kUnroll; u++) acc[u] = 0.f;
  for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
    for (int u = 0; u < kUnroll; u++) {
      float v;
      asm volatile("ld.volatile.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr[u]));
      acc[u] = __fadd_rn(acc[u], v);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int u = 0; u < kUnroll; u++) s += acc[u];
  if (s == 123.456f) out[blockIdx.x] = s;  // keeps the loads alive
}

// L2 read probe: every CTA reads `chunk` 16-byte words per pass from a buffer
// that L2 holds (loads that bypass L1), starting at its own offset and moving
// on by `chunk` each pass; four independent loads per thread are in flight.
__global__ void __launch_bounds__(256) l2_read_kernel(const float4 *__restrict__ buf, uint32_t n4,
                                                     int passes, float *out) {
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t chunk = n4 / gridDim.x, step = blockDim.x;
  uint32_t s = (uint32_t)(((uint64_t)blockIdx.x * 7919u * 256u) % n4);
  for (int p = 0; p < passes; p++) {
    for (uint32_t i = threadIdx.x; i < chunk; i += 4 * step) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i + u * step < chunk) {
          uint32_t k = s + i + u * step;
          if (k >= n4) k -= n4;
          asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];"
                       : "=f"(v[u].x), "=f"(v[u].y), "=f"(v[u].z), "=f"(v[u].w)
                       : "l"(buf + k));
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        acc.x += v[u].x;
        acc.y += v[u].y;
        acc.z += v[u].z;
        acc.w += v[u].w;
      }
    }
    s += chunk;
    if (s >= n4) s -= n4;
  }
  if (acc.x + acc.y + acc.z + acc.w == 123.456f) out[blockIdx.x] = acc.x;  // keeps the loads
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

extern "C" int ctas_probe_l2_read(int device, double *bytes_per_s, double *seconds) {
  if (!bytes_per_s || !seconds) return CTAS_E_ARG;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return CTAS_E_NODEVICE;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return CTAS_E_ARG;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // 32 MiB: resident in L2 (126 MB) once touched
  const int64_t bytes = (int64_t)32 << 20;
  const uint32_t n4 = (uint32_t)(bytes / 16);
  float4 *buf = nullptr;
  float *out = nullptr;
  if (cudaMalloc(&buf, (size_t)bytes) != cudaSuccess || cudaMalloc(&out, sizeof(float) * 8192) != cudaSuccess) {
    cudaFree(buf);
    cudaSetDevice(prev);
    return CTAS_E_NOMEM;
  }
  cudaMemset(buf, 0, (size_t)bytes);
  const int blocks = sms * 8, passes = 16;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = CTAS_OK;
  l2_read_kernel<<<blocks, 256>>>(buf, n4, 2, out);  // warm-up: brings the buffer into L2
  cudaEventRecord(e0);
  const int reps = 4;
  for (int r = 0; r < reps; r++) l2_read_kernel<<<blocks, 256>>>(buf, n4, passes, out);
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess) rc = CTAS_E_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const double read = (double)reps * passes * (double)(n4 / (uint32_t)blocks) * blocks * 16.0;
  *seconds = ms * 1e-3;
  *bytes_per_s = ms > 0 ? read / (ms * 1e-3) : 0.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  cudaFree(out);
  cudaSetDevice(prev);
  return rc;
}
