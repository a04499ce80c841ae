// bp_common.cuh -- reference arithmetic shared by the backprojection kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace ctas {

// Pixel mask of lct.cpp:693-707 (== ct.cl:21-32), every operation rounded as
// the reference rounds it.  true = pixel is reconstructed.
__device__ __forceinline__ bool ref_mask(int j, int i, int W, float c) {
  const int hp = W / 2;
  const float ac = fabsf(c);
  const float fi = (float)i;
  if (fi <= ac || fi >= __fsub_rn(__fsub_rn((float)W, ac), 1.0f)) return false;
  int ip2 = i - hp;
  ip2 *= ip2;
  float d = __fsub_rn((float)(j - hp), c);
  d = __fmul_rn(d, d);
  d = __fadd_rn(d, (float)ip2);
  const float hpc = __fadd_rn((float)hp, c), hmc = __fsub_rn((float)hp, c);
  const float fj = (float)j;
  if ((fj <= hpc && d >= __fmul_rn(hpc, hpc)) || (fj >= hpc && d >= __fmul_rn(hmc, hmc)))
    return false;
  return true;
}

// The same mask at float coordinates (jj, ii) of an output geometry; for
// integer coordinates it is ref_mask exactly (every value below is exact).
__device__ __forceinline__ bool ref_mask_f(float jj, float ii, int W, float c) {
  const int hp = W / 2;
  const float ac = fabsf(c);
  if (ii <= ac || ii >= __fsub_rn(__fsub_rn((float)W, ac), 1.0f)) return false;
  const float di = __fsub_rn(ii, (float)hp);
  const float ip2 = __fmul_rn(di, di);
  float d = __fsub_rn(__fsub_rn(jj, (float)hp), c);
  d = __fmul_rn(d, d);
  d = __fadd_rn(d, ip2);
  const float hpc = __fadd_rn((float)hp, c), hmc = __fsub_rn((float)hp, c);
  if ((jj <= hpc && d >= __fmul_rn(hpc, hpc)) || (jj >= hpc && d >= __fmul_rn(hmc, hmc)))
    return false;
  return true;
}

// Output geometry coordinate o + p * k (float, as the oracle forms it).
__device__ __forceinline__ float geo(float o, float p, int k) {
  return __fadd_rn(o, __fmul_rn(p, (float)k));
}

// First partial sum of the index expression, c + k0 * hp, with k0 rounded in
// one of two orders (lct.cpp:711-712 == ct.cl:36-37 as written):
//   rule 0: k0 = (1 - s) - co -- the OpenCL kernel, and the CPU path built
//           without -ffast-math;
//   rule 1: k0 = 1 - (s + co) -- the CPU path as the reference's build
//           compiles it: with -ffast-math (CMakeLists.txt:10-11) GCC folds
//           (1 - s) - co into 1 - (s + co) even at -O0.
__device__ __forceinline__ float ref_base(float s, float co, int hp, float c, int rule) {
  const float k0 = rule == 1 ? __fsub_rn(1.0f, __fadd_rn(s, co)) : __fsub_rn(__fsub_rn(1.0f, s), co);
  return __fadd_rn(c, __fmul_rn(k0, (float)hp));
}

// (recCof != 0 ? tot * recCof : tot) / N   (lct.cpp:715-718)
__device__ __forceinline__ float ref_finish(float tot, float rec_cof, int N) {
  if (rec_cof != 0.0f) tot = __fmul_rn(tot, rec_cof);
  return __fdiv_rn(tot, (float)N);
}

__device__ __forceinline__ float load_sample(const float *p) { return __ldg(p); }
__device__ __forceinline__ float load_sample(const __half *p) { return __half2float(*p); }
__device__ __forceinline__ float load_sample(const __nv_bfloat16 *p) {
  return __bfloat162float(*p);
}

}  // namespace ctas
