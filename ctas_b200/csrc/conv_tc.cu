// conv_tc.cu -- 3x3 convolution of the learned stage as an implicit GEMM on the
// fifth-generation tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// GEMM view of one output tile: D[128 pixels][NT channels] += A_t[128][K] * B_t[NT][K]^T
// over the nine taps t = (ky, kx) and the input channels in chunks of CK, where
// A_t row m is input pixel (y0 + m/16 + ky - 1, x0 + m%16 + kx - 1) of an 8 x 16
// pixel block and B_t row n is w[n][t][.].  Both operands are K-major (channels
// contiguous, NHWC activations and [cout][9][cin] weights) and reach shared memory
// by TMA with the hardware swizzle the matrix descriptors expect (128 B rows for
// CK = 64, 64 B for 32, 32 B for 16):
//
//   A: one 10 x 16 pixel box x CK channels per (kx, chunk) -- rows y0-1 .. y0+8,
//      zero-filled outside the image by the TMA unit -- serves the three ky taps:
//      tap ky's 128 x CK operand is the same box shifted by 16 ky rows, which
//      keeps every operand start on a swizzle-atom boundary;
//   B: the weights viewed as a 2-D array [cout][9 cin]; three NT x CK boxes per
//      (kx, chunk), one per ky tap, placed one after another.
//
// Persistent warp-specialised CTA (192 threads): warp 0 issues the TMA loads
// into a ring of stages, one thread of warp 1 issues the MMAs (K = 16 each) and
// releases each stage with tcgen05.commit, warps 2-5 drain the accumulator
// (tcgen05.ld, bias, ReLU or ReLU mask, BF16) while the next tile accumulates in
// the other half of the double-buffered tensor-memory accumulator.  Every wait is
// bounded; on expiry the kernel records an error, drains its copies and MMAs,
// frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/ctas_learned.h"
#include "../../include/ctas_fbp.h"
#include "tma_encode.hpp"
#include "unet_kernels.hpp"

namespace ctas {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kThreads = 192;
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kMaxCout = 512;

struct TcArgs {
  bf16 *y;
  int y_cs, y_co;
  const bf16 *mask;
  int m_cs, m_co;
  const float *bias;
  int cout;
  int relu;
  int H, W;
  int tiles_x, tiles_y, tiles_n;
  int64_t total;
  int cin;
  int kchunks;  // cin / CK
  int *err;     // bit 0: a bounded wait ran out
};

template <int CK, int NT, int ST> struct TcCfg {
  static constexpr int kABytes = 160 * CK * 2;     // 10 x 16 pixels x CK channels
  static constexpr int kBBytes = 3 * NT * CK * 2;  // three ky taps x NT x CK
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kRowB = CK * 2;             // bytes per operand row
  static constexpr int kSBO = 8 * kRowB;           // bytes between 8-row groups
  // descriptor layout type: 128 B / 64 B / 32 B swizzle
  static constexpr uint64_t kLayout = CK == 64 ? 2 : CK == 32 ? 4 : 6;
  // accumulator buffers in tensor memory: as many as fit 256 columns (two CTAs
  // per SM), so the MMAs run ahead of the epilogue on small tiles
  static constexpr int kAcc = 256 / NT >= 8 ? 8 : 256 / NT >= 4 ? 4 : 2;
  static constexpr uint32_t kCols = 256;
  static constexpr int kBarOff = ST * kStage;
  static constexpr int kBiasOff = kBarOff + 256;       // bias of all output channels
  static constexpr int kSmem = kBiasOff + 4 * kMaxCout + 1024;  // + alignment slack
  static_assert(kABytes % 1024 == 0 && kBBytes % 1024 == 0, "stage alignment");
  static_assert(NT % 32 == 0 && NT >= 32 && NT <= 128, "UMMA N, epilogue pairs");
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Test aid (ctas_nn_test_timeout): while g_test_stall is set, each kernel's
// producer leaves its first stage of copies out, so the waits on it run out;
// g_wait_limit bounds every wait (short while the test aid is armed).
__device__ int g_test_stall = 0;
__device__ uint32_t g_wait_limit = kWaitLimit;

// bounded wait; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t limit = __ldg(&g_wait_limit);
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// D[tmem] (+)= A[desc] * B[desc]^T, kind::f16 (BF16 operands, FP32 accumulate)
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// shared-memory matrix descriptor of a K-major swizzled operand
template <class C> __device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) |
         ((uint64_t)((C::kSBO >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46) |
         (C::kLayout << 61);
}

struct Tile {
  int b, ty, tx, nt;
};

__device__ __forceinline__ Tile decode(const TcArgs &a, int64_t t) {
  Tile r;
  r.nt = (int)(t % a.tiles_n);
  t /= a.tiles_n;
  r.tx = (int)(t % a.tiles_x);
  t /= a.tiles_x;
  r.ty = (int)(t % a.tiles_y);
  r.b = (int)(t / a.tiles_y);
  return r;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

template <int CK, int NT, int ST>
__global__ void __launch_bounds__(kThreads, 1)
    conv_tc_kernel(const __grid_constant__ CUtensorMap amap,
                   const __grid_constant__ CUtensorMap bmap, TcArgs a) {
  using C = TcCfg<CK, NT, ST>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t *base = smem_raw + pad;
  uint64_t *full = reinterpret_cast<uint64_t *>(base + C::kBarOff);
  uint64_t *empty = full + ST;
  uint64_t *acc_full = empty + ST;  // [kAcc]
  uint64_t *acc_empty = acc_full + C::kAcc;
  uint64_t *drain = acc_empty + C::kAcc;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_tmem + 1);
  float *s_bias = reinterpret_cast<float *>(base + C::kBiasOff);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int i = 0; i < C::kAcc; i++) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
    }
    mbar_init(drain, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(s_tmem)),
                 "r"(C::kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  for (int c = threadIdx.x; c < a.cout; c += kThreads) s_bias[c] = a.bias ? a.bias[c] : 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const int ksteps = 3 * a.kchunks;

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------ TMA producer
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&amap))
                   : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&bmap))
                   : "memory");
      int stage = 0;
      uint32_t ph = 0;
      uint32_t issued = 0, last_par = 0;  // per-stage bits: used / parity of last issue
      for (int64_t t = blockIdx.x; t < a.total && !*s_abort; t += gridDim.x) {
        const Tile tl = decode(a, t);
        for (int ks = 0; ks < ksteps; ks++) {
          const int kc = ks / 3, kx = ks % 3;
          if (!mbar_wait(&empty[stage], ph ^ 1)) {
            atomicOr(a.err, 1);
            *s_abort = 1;
            break;
          }
          uint8_t *sa = base + stage * C::kStage;
          mbar_expect_tx(&full[stage], (uint32_t)C::kStage);
          if (!(__ldg(&g_test_stall) && t == blockIdx.x && ks == 0)) {
            tma_load_4d(sa, &amap, kc * CK, tl.tx * 16 + kx - 1, tl.ty * 8 - 1, tl.b, &full[stage]);
#pragma unroll
            for (int ky = 0; ky < 3; ky++)
              tma_load_2d(sa + C::kABytes + ky * NT * C::kRowB, &bmap,
                          (ky * 3 + kx) * a.cin + kc * CK, tl.nt * NT, &full[stage]);
          }
          issued |= 1u << stage;
          last_par = (last_par & ~(1u << stage)) | (ph << stage);
          if (++stage == ST) {
            stage = 0;
            ph ^= 1;
          }
        }
      }
      // every issued copy has landed before the CTA may exit
      for (int s = 0; s < ST; s++)
        if ((issued >> s) & 1u)
          if (!mbar_wait(&full[s], (last_par >> s) & 1u)) atomicOr(a.err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------ MMA issuer
      constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                                 ((uint32_t)(128 >> 4) << 24);
      int stage = 0;
      uint32_t ph = 0;
      int acc = 0;
      uint32_t acc_ph = 0;
      for (int64_t t = blockIdx.x; t < a.total && !*s_abort; t += gridDim.x) {
        if (!mbar_wait(&acc_empty[acc], acc_ph ^ 1)) {
          atomicOr(a.err, 1);
          *s_abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * NT);
        bool ok = true;
        for (int ks = 0; ks < ksteps; ks++) {
          if (!mbar_wait(&full[stage], ph)) {
            atomicOr(a.err, 1);
            *s_abort = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(base + stage * C::kStage);
          const uint64_t da = sdesc<C>(sa), db = sdesc<C>(sa + C::kABytes);
#pragma unroll
          for (int ky = 0; ky < 3; ky++)
#pragma unroll
            for (int kk = 0; kk < CK / 16; kk++)
              tc_mma(d, da + (uint64_t)((ky * 16 * C::kRowB + kk * 32) >> 4),
                     db + (uint64_t)((ky * NT * C::kRowB + kk * 32) >> 4), idesc,
                     (ks | ky | kk) != 0 ? 1u : 0u);
          tc_commit(&empty[stage]);  // the stage is free once these MMAs have read it
          if (++stage == ST) {
            stage = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        tc_commit(&acc_full[acc]);
        if (++acc == C::kAcc) {
          acc = 0;
          acc_ph ^= 1;
        }
      }
      // all MMAs of this thread complete before tensor memory is released
      tc_commit(drain);
      if (!mbar_wait(drain, 0)) atomicOr(a.err, 1);
    }
  } else {
    // ---------------------------------------------------- epilogue (warps 2-5)
    const int q = warp & 3;  // tensor-memory lane quarter this warp may access
    const int m = q * 32 + lane;
    int acc = 0;
    uint32_t acc_ph = 0;
    for (int64_t t = blockIdx.x; t < a.total; t += gridDim.x) {
      // warp-uniform decisions: the tensor-memory loads below are warp-collective
      if (__shfl_sync(0xffffffffu, *s_abort, 0)) break;
      if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[acc], acc_ph))) {
        if (lane == 0) {
          atomicOr(a.err, 1);
          *s_abort = 1;
        }
        break;
      }
      tc_fence_after();
      const Tile tl = decode(a, t);
      const int yy = tl.ty * 8 + (m >> 4), xx = tl.tx * 16 + (m & 15);
      const int64_t pix = ((int64_t)tl.b * a.H + yy) * a.W + xx;
      bf16 *yp = a.y + pix * a.y_cs + a.y_co + tl.nt * NT;
      const bf16 *mp = a.mask ? a.mask + pix * a.m_cs + a.m_co + tl.nt * NT : nullptr;
      const float *bp = s_bias + tl.nt * NT;
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * NT);
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += 32) {
        // two 16-column loads in flight per wait
        uint32_t r[2][16];
        tmem_ld16(taddr + (uint32_t)c0, r[0]);
        tmem_ld16(taddr + (uint32_t)c0 + 16u, r[1]);
        tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int cc = c0 + 16 * h;
          float v[16];
#pragma unroll
          for (int j = 0; j < 16; j++) {
            v[j] = __uint_as_float(r[h][j]) + bp[cc + j];
            if (a.relu) v[j] = fmaxf(v[j], 0.f);
          }
          if (mp) {
            const uint4 m0 = *reinterpret_cast<const uint4 *>(mp + cc);
            const uint4 m1 = *reinterpret_cast<const uint4 *>(mp + cc + 8);
            const bf16 *mm0 = reinterpret_cast<const bf16 *>(&m0);
            const bf16 *mm1 = reinterpret_cast<const bf16 *>(&m1);
#pragma unroll
            for (int j = 0; j < 8; j++) {
              if (!(__bfloat162float(mm0[j]) > 0.f)) v[j] = 0.f;
              if (!(__bfloat162float(mm1[j]) > 0.f)) v[8 + j] = 0.f;
            }
          }
          uint4 o0, o1;
          o0.x = pack_bf16(v[0], v[1]);
          o0.y = pack_bf16(v[2], v[3]);
          o0.z = pack_bf16(v[4], v[5]);
          o0.w = pack_bf16(v[6], v[7]);
          o1.x = pack_bf16(v[8], v[9]);
          o1.y = pack_bf16(v[10], v[11]);
          o1.z = pack_bf16(v[12], v[13]);
          o1.w = pack_bf16(v[14], v[15]);
          *reinterpret_cast<uint4 *>(yp + cc) = o0;
          *reinterpret_cast<uint4 *>(yp + cc + 8) = o1;
        }
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[acc]);
      if (++acc == C::kAcc) {
        acc = 0;
        acc_ph ^= 1;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(C::kCols)
                 : "memory");
}

// ------------------------------------------------------------ host side
using EncodeTiledFn = ctas::EncodeTiledFn;
EncodeTiledFn encode_fn() { return ctas::tensor_map_encoder(); }

CUtensorMapSwizzle swizzle_for(int ck) {
  return ck == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                  : ck == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

// activations: (cin, W, H, B) of the channel slice; box {CK, 16, 10, 1}
bool make_act_map(const ConvArgs &a, int ck, CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  std::memset(map, 0, sizeof(*map));
  const cuuint64_t dims[4] = {(cuuint64_t)a.cin, (cuuint64_t)a.W, (cuuint64_t)a.H,
                              (cuuint64_t)a.B};
  const cuuint64_t cs = (cuuint64_t)a.x_cs * 2;
  const cuuint64_t strides[3] = {cs, cs * (cuuint64_t)a.W, cs * (cuuint64_t)a.W * a.H};
  const cuuint32_t box[4] = {(cuuint32_t)ck, 16u, 10u, 1u};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(a.x + a.x_co), dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(ck),
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// weights [cout][9][cin] as a 2-D array (9 cin, cout); box {CK, NT}
bool make_wt_map(const ConvArgs &a, int ck, int nt, CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  std::memset(map, 0, sizeof(*map));
  const cuuint64_t dims[2] = {9 * (cuuint64_t)a.cin, (cuuint64_t)a.cout};
  const cuuint64_t strides[1] = {9 * (cuuint64_t)a.cin * 2};
  const cuuint32_t box[2] = {(cuuint32_t)ck, (cuuint32_t)nt};
  const cuuint32_t estr[2] = {1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(a.w), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(ck),
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// device error word of the tensor-core convolutions (mapped host memory, so
// the host reads it without a device synchronisation)
int *g_err_host = nullptr;
int *g_err_dev = nullptr;
std::mutex g_err_mutex;

cudaError_t err_word(int **dev) {
  std::lock_guard<std::mutex> l(g_err_mutex);
  if (!g_err_host) {
    void *p = nullptr;
    cudaError_t e = cudaHostAlloc(&p, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) return e;
    *static_cast<int *>(p) = 0;
    void *d = nullptr;
    e = cudaHostGetDevicePointer(&d, p, 0);
    if (e != cudaSuccess) {
      cudaFreeHost(p);
      return e;
    }
    g_err_host = static_cast<int *>(p);
    g_err_dev = static_cast<int *>(d);
  }
  *dev = g_err_dev;
  return cudaSuccess;
}

// resident CTAs per SM for `smem` bytes of dynamic shared memory, the
// kernel's registers and `per_sm` (tensor-memory) limit
template <class K> int occupancy(K kernel, int smem, int per_sm) {
  cudaFuncAttributes fa{};
  int regs = 128;
  if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess && fa.numRegs > 0) regs = fa.numRegs;
  const int by_regs = 65536 / (((regs + 7) / 8) * 8 * kThreads);
  const int by_smem = 233472 / (smem + 1024);
  return std::max(1, std::min(per_sm, std::min(by_regs, by_smem)));
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int CK, int NT, int ST>
cudaError_t launch_cfg(const ConvArgs &a, cudaStream_t st) {
  using C = TcCfg<CK, NT, ST>;
  CUtensorMap amap, bmap;
  if (!make_act_map(a, CK, &amap) || !make_wt_map(a, CK, NT, &bmap)) return cudaErrorInvalidValue;
  TcArgs t{};
  t.y = a.y;
  t.y_cs = a.y_cs;
  t.y_co = a.y_co;
  t.mask = a.mask;
  t.m_cs = a.m_cs;
  t.m_co = a.m_co;
  t.bias = a.bias;
  t.cout = a.cout;
  t.relu = a.relu;
  t.H = a.H;
  t.W = a.W;
  t.tiles_x = a.W / 16;
  t.tiles_y = a.H / 8;
  t.tiles_n = a.cout / NT;
  t.total = (int64_t)a.B * t.tiles_y * t.tiles_x * t.tiles_n;
  t.cin = a.cin;
  t.kchunks = a.cin / CK;
  cudaError_t e = err_word(&t.err);
  if (e != cudaSuccess) return e;
  // no more CTAs per SM than tensor memory holds (512 columns): pad the
  // shared-memory request so that one more would not fit
  const int per_sm = 512 / (int)C::kCols;
  const int smem = std::max(C::kSmem, 232448 / (per_sm + 1) + 1024);
  e = cudaFuncSetAttribute(conv_tc_kernel<CK, NT, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(conv_tc_kernel<CK, NT, ST>,
                           cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  const int occ = occupancy(conv_tc_kernel<CK, NT, ST>, smem, per_sm);
  const int64_t grid = std::min<int64_t>(t.total, (int64_t)sm_count() * occ);
  conv_tc_kernel<CK, NT, ST><<<(unsigned)grid, kThreads, smem, st>>>(amap, bmap, t);
  return cudaGetLastError();
}

template <int CK, int NT> cudaError_t launch_ck_nt(const ConvArgs &a, cudaStream_t st) {
  constexpr int kStage = 160 * CK * 2 + 3 * NT * CK * 2;
  constexpr int kSt = (96 * 1024) / kStage < 2 ? 2 : (96 * 1024) / kStage > 6 ? 6 : (96 * 1024) / kStage;
  return launch_cfg<CK, NT, kSt>(a, st);
}

template <int CK> cudaError_t launch_ck(const ConvArgs &a, int nt, cudaStream_t st) {
  switch (nt) {
    case 32: return launch_ck_nt<CK, 32>(a, st);
    case 64: return launch_ck_nt<CK, 64>(a, st);
    case 96: return launch_ck_nt<CK, 96>(a, st);
    case 128: return launch_ck_nt<CK, 128>(a, st);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------ row-streaming form
// For layers whose weights fit in shared memory and whose rows are multiples of
// 128 pixels (the full-resolution layers with few output channels, where the
// tiled form above reads every input pixel 3.75 times from L2 for only NT
// outputs): a CTA walks down a strip 128 pixels wide, each input row is loaded
// once into a ring of row buffers and serves the three output rows and nine
// taps that need it, and the weights stay resident.  An input row is stored as
// 64-channel chunks of 130 pixels x 128 bytes in the 128-byte-swizzled K-major
// layout (one TMA box per chunk; channels beyond cin are zero-filled by the
// TMA unit and never multiplied); the operand of tap (ky, kx) is the buffer of
// row y + ky - 1 started kx pixel rows in.  The weights are stored per (tap,
// channel chunk) as swizzled K-major blocks of cout rows (128-, 64- or 32-byte
// rows for 64-, 32- or 16-channel chunks), written by the threads with the same
// address swizzle the TMA unit applies.
constexpr int kRowPx = 130;                    // 128 output pixels + 2 halo
constexpr int kRowChunkBytes = 17 * 1024;      // 130 x 128 B, padded to the 1 KB atom
constexpr int kRowMaxSlots = 8;
constexpr int kMaxAcc = 8;

struct RowArgs {
  bf16 *y;
  int y_cs, y_co;
  const bf16 *mask;
  int m_cs, m_co;
  const float *bias;
  const bf16 *w;  // [cout][9][cin]
  int cin, cout, relu;
  int H, W;
  int strips_x, strips_y, strip_h;
  int64_t total;  // B * strips_y * strips_x
  int nslots, slot_bytes, wbytes;
  int nacc;       // accumulator buffers in tensor memory
  uint32_t cols;
  int *err;
};

// swizzled K-major descriptor for rows of RB bytes (128, 64 or 32; 8-row groups
// 8 RB apart)
template <int RB> __device__ __forceinline__ uint64_t sdesc_swz(uint32_t addr) {
  constexpr uint64_t layout = RB == 128 ? 2 : RB == 64 ? 4 : 6;
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)((8 * RB) >> 4) << 32) |
         ((uint64_t)1 << 46) | (layout << 61);
}

// byte offset of a swizzled operand (rows of RB bytes, region 1024-byte aligned):
// the 16-byte unit index XOR the row phase, as the hardware swizzle does
template <int RB> __host__ __device__ __forceinline__ uint32_t swz(uint32_t off) {
  constexpr uint32_t mask = RB == 128 ? 7u : RB == 64 ? 3u : 1u;
  return off ^ (((off >> 7) & mask) << 4);
}

// 128-byte-swizzled K-major descriptor (rows of 128 B, 8-row groups 1024 B apart).
// The swizzle is applied to the absolute shared-memory address (bits 4-6 XOR
// bits 7-9), as the TMA unit applies it when writing, so an operand may start
// any whole number of rows past a 1024-byte atom with the base offset left 0.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

template <int CIN>
__global__ void __launch_bounds__(kThreads, 1)
    conv_row_kernel(const __grid_constant__ CUtensorMap amap, RowArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t *base = smem_raw + pad;
  uint8_t *slots = base;                                   // input-row ring (1 KB atoms)
  uint8_t *wsm = base + a.nslots * a.slot_bytes;           // weights
  float *s_bias = reinterpret_cast<float *>(wsm + a.wbytes);
  uint64_t *row_full = reinterpret_cast<uint64_t *>(s_bias + kMaxCout);
  uint64_t *row_empty = row_full + kRowMaxSlots;
  uint64_t *acc_full = row_empty + kRowMaxSlots;  // [kMaxAcc]
  uint64_t *acc_empty = acc_full + kMaxAcc;
  uint64_t *drain = acc_empty + kMaxAcc;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_tmem + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ns = a.nslots, cout = a.cout;
  constexpr int cin = CIN;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ns; s++) {
      mbar_init(&row_full[s], 1);
      mbar_init(&row_empty[s], 1);
    }
    for (int i = 0; i < a.nacc; i++) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
    }
    mbar_init(drain, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(s_tmem)),
                 "r"(a.cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // weights -> swizzled K-major blocks [kx][chunk][3 cout rows][kCKB channels]:
  // in a block, rows p * cout + n hold tap (ky = 2 - p, kx), output channel n,
  // so one MMA with N = 3 cout multiplies an input row by the taps of the three
  // output rows it feeds (rows y + 1, y, y - 1 take ky = 0, 1, 2)
  constexpr int kCKB = CIN % 64 == 0 ? 64 : CIN % 32 == 0 ? 32 : 16;
  constexpr int kRB = kCKB * 2, kUnits = kCKB / 8, kChunks = CIN / kCKB;
  for (int i = threadIdx.x; i < 9 * kChunks * cout * kUnits; i += kThreads) {
    const int u = i % kUnits, rest = i / kUnits;
    const int n = rest % cout, blk = rest / cout;  // blk = tap * kChunks + chunk
    const int tap = blk / kChunks, ch = blk - tap * kChunks;
    const int ky = tap / 3, kx = tap - 3 * ky;
    const uint32_t off = (uint32_t)(((kx * kChunks + ch) * 3 * cout + (2 - ky) * cout + n) * kRB +
                                    u * 16);
    *reinterpret_cast<uint4 *>(wsm + swz<kRB>(off)) = *reinterpret_cast<const uint4 *>(
        a.w + (size_t)n * 9 * cin + tap * cin + ch * kCKB + u * 8);
  }
  for (int c = threadIdx.x; c < cout; c += kThreads) s_bias[c] = a.bias ? a.bias[c] : 0.f;
  // generic-proxy stores must be visible to the tensor cores' reads
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------ TMA producer: input rows
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&amap))
                   : "memory");
      uint32_t j = 0, issued = 0, last_par = 0;
      const int chunks = (cin + 63) / 64;
      const uint32_t row_bytes = (uint32_t)chunks * (uint32_t)(kRowPx * 128);
      for (int64_t t = blockIdx.x; t < a.total && !*s_abort; t += gridDim.x) {
        const int sx = (int)(t % a.strips_x);
        const int64_t r = t / a.strips_x;
        const int sy = (int)(r % a.strips_y), b = (int)(r / a.strips_y);
        const int r0 = sy * a.strip_h, r1 = min(r0 + a.strip_h, a.H);
        bool ok = true;
        for (int yi = r0 - 1; yi <= r1; yi++, j++) {
          const int slot = (int)(j % (uint32_t)ns);
          const uint32_t par = (j / (uint32_t)ns) & 1u;
          if (!mbar_wait(&row_empty[slot], par ^ 1u)) {
            atomicOr(a.err, 1);
            *s_abort = 1;
            ok = false;
            break;
          }
          uint8_t *dst = slots + slot * a.slot_bytes;
          mbar_expect_tx(&row_full[slot], row_bytes);
          if (!(__ldg(&g_test_stall) && j == 0))
            for (int c = 0; c < chunks; c++)
              tma_load_4d(dst + c * kRowChunkBytes, &amap, c * 64, sx * 128 - 1, yi, b,
                          &row_full[slot]);
          issued |= 1u << slot;
          last_par = (last_par & ~(1u << slot)) | (par << slot);
        }
        if (!ok) break;
      }
      for (int s = 0; s < ns; s++)
        if ((issued >> s) & 1u)
          if (!mbar_wait(&row_full[s], (last_par >> s) & 1u)) atomicOr(a.err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------ MMA issuer
      // Input-row stationary: input row yi feeds output rows yi - 1, yi, yi + 1
      // (taps ky = 2, 1, 0), whose accumulators are consecutive blocks of cout
      // columns in a ring of nacc blocks; per (kx, 16-channel step) one MMA with
      // N = 3 cout covers all three (split in two where the ring wraps; fewer
      // rows at a strip's edges).  Each output row still receives its taps in
      // the order ky, kx, channel step.  The first MMA into a block (the row
      // yi + 1 block, at kx = 0 and step 0) overwrites it.
      const uint32_t idesc0 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 >> 4) << 24);
      const uint32_t slots_u = smem_u32(slots);
      constexpr int kCKB = CIN % 64 == 0 ? 64 : CIN % 32 == 0 ? 32 : 16;
      constexpr int kRB = kCKB * 2, kSteps = kCKB / 16, kChunks = CIN / kCKB;
      const uint64_t dw0 = sdesc_swz<kRB>(smem_u32(wsm));
      const uint32_t row16 = (uint32_t)kRB / 16;  // one weight row, 16-byte units
      const uint32_t R = (uint32_t)a.nacc;
      const uint32_t wrow = (uint32_t)cout * row16;  // one block of cout weight rows
      const uint32_t kxblk = 3u * wrow;               // one (kx, chunk) weight block
      // Ring segments of the output-row counters o .. o + nb - 1 (weight rows
      // from block position p), split where the ring wraps: TMEM column,
      // instruction descriptor (N) and weight offset of each, computed once per
      // input row so that the MMA loop below only adds constant offsets
      struct Seg {
        uint32_t d, idesc;
        uint64_t boff;
      };
      auto segments = [&](uint32_t o, uint32_t nb, uint32_t p, Seg *sg) -> int {
        const uint32_t g = o % R, n1 = min(nb, R - g);
        sg[0] = Seg{tmem + g * (uint32_t)cout, idesc0 | (((n1 * (uint32_t)cout) >> 3) << 17),
                    (uint64_t)(p * wrow)};
        if (n1 == nb) return 1;
        sg[1] = Seg{tmem, idesc0 | ((((nb - n1) * (uint32_t)cout) >> 3) << 17),
                    (uint64_t)((p + n1) * wrow)};
        return 2;
      };
      uint32_t j0 = 0, o0 = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < a.total && ok && !*s_abort; t += gridDim.x) {
        const int64_t r = t / a.strips_x;
        const int sy = (int)(r % a.strips_y);
        const int r0 = sy * a.strip_h, r1 = min(r0 + a.strip_h, a.H);
        for (int yi = r0 - 1; yi <= r1 && ok; yi++) {
          const uint32_t jl = j0 + (uint32_t)(yi - r0 + 1);  // load index of input row yi
          ok = mbar_wait(&row_full[jl % (uint32_t)ns], (jl / (uint32_t)ns) & 1u);
          const int lo = max(yi - 1, r0), hi = min(yi + 1, r1 - 1);
          const bool fresh = (yi + 1 <= r1 - 1);  // row yi + 1 starts here
          const uint32_t olo = o0 + (uint32_t)(lo - r0), ohi = o0 + (uint32_t)(hi - r0);
          if (ok && fresh)
            ok = mbar_wait(&acc_empty[ohi % R], ((ohi / R) & 1u) ^ 1u);
          if (!ok) {
            atomicOr(a.err, 1);
            *s_abort = 1;
            break;
          }
          tc_fence_after();
          const uint64_t da = sdesc_sw128(slots_u + (jl % (uint32_t)ns) * (uint32_t)a.slot_bytes);
          const uint32_t nb = (uint32_t)(hi - lo + 1), p0 = (uint32_t)(lo - yi + 1);
          // all rows lo..hi (accumulating), and for the first MMA of a fresh
          // row yi + 1: rows lo..hi - 1 accumulating, row hi overwritten
          Seg all[2], head[3];
          const int nall = segments(olo, nb, p0, all);
          int nhead = 0, nacc_head = 0;
          if (fresh) {
            if (nb > 1) nhead = segments(olo, nb - 1, p0, head);
            nacc_head = nhead;
            nhead += segments(ohi, 1, p0 + nb - 1, head + nhead);
          }
#pragma unroll
          for (int kx = 0; kx < 3; kx++)
#pragma unroll
            for (int st = 0; st < cin / 16; st++) {
              // 16-channel step st: row chunk st / 4, 32-byte column st % 4;
              // weights: block (kx, st / kSteps), 32-byte column st % kSteps
              const uint64_t a_op =
                  da + (uint64_t)(((st >> 2) * kRowChunkBytes + kx * 128 + (st & 3) * 32) >> 4);
              const uint64_t b_op =
                  dw0 + (uint64_t)((uint32_t)(kx * kChunks + st / kSteps) * kxblk +
                                   (uint32_t)((st % kSteps) * 2));
              if (kx == 0 && st == 0 && fresh) {
                for (int q = 0; q < nhead; q++)
                  tc_mma(head[q].d, a_op, b_op + head[q].boff, head[q].idesc, q < nacc_head ? 1u : 0u);
              } else {
                tc_mma(all[0].d, a_op, b_op + all[0].boff, all[0].idesc, 1u);
                if (nall > 1) tc_mma(all[1].d, a_op, b_op + all[1].boff, all[1].idesc, 1u);
              }
            }
          tc_commit(&row_empty[jl % (uint32_t)ns]);       // input row yi is done
          if (yi - 1 >= r0) tc_commit(&acc_full[olo % R]);  // output row yi - 1 is complete
        }
        if (!ok) break;
        j0 += (uint32_t)(r1 - r0) + 2u;
        o0 += (uint32_t)(r1 - r0);
      }
      tc_commit(drain);
      if (!mbar_wait(drain, 0)) atomicOr(a.err, 1);
    }
  } else {
    // ---------------------------------------------------- epilogue (warps 2-5)
    const int q = warp & 3;
    const int m = q * 32 + lane;
    int acc = 0;
    uint32_t acc_ph = 0;
    bool stop = false;
    for (int64_t t = blockIdx.x; t < a.total && !stop; t += gridDim.x) {
      const int sx = (int)(t % a.strips_x);
      const int64_t r = t / a.strips_x;
      const int sy = (int)(r % a.strips_y), b = (int)(r / a.strips_y);
      const int r0 = sy * a.strip_h, r1 = min(r0 + a.strip_h, a.H);
      for (int y = r0; y < r1; y++) {
        if (__shfl_sync(0xffffffffu, *s_abort, 0) ||
            !__all_sync(0xffffffffu, mbar_wait(&acc_full[acc], acc_ph))) {
          if (lane == 0) {
            atomicOr(a.err, 1);
            *s_abort = 1;
          }
          stop = true;
          break;
        }
        tc_fence_after();
        const int64_t pix = ((int64_t)b * a.H + y) * a.W + sx * 128 + m;
        bf16 *yp = a.y + pix * a.y_cs + a.y_co;
        const bf16 *mp = a.mask ? a.mask + pix * a.m_cs + a.m_co : nullptr;
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * cout);
#pragma unroll 1
        for (int c0 = 0; c0 < cout; c0 += 32) {
          uint32_t rr[2][16];
          tmem_ld16(taddr + (uint32_t)c0, rr[0]);
          tmem_ld16(taddr + (uint32_t)c0 + 16u, rr[1]);
          tmem_wait_ld();
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int cc = c0 + 16 * h;
            float v[16];
#pragma unroll
            for (int jx = 0; jx < 16; jx++) {
              v[jx] = __uint_as_float(rr[h][jx]) + s_bias[cc + jx];
              if (a.relu) v[jx] = fmaxf(v[jx], 0.f);
            }
            if (mp) {
              const uint4 m0 = *reinterpret_cast<const uint4 *>(mp + cc);
              const uint4 m1 = *reinterpret_cast<const uint4 *>(mp + cc + 8);
              const bf16 *mm0 = reinterpret_cast<const bf16 *>(&m0);
              const bf16 *mm1 = reinterpret_cast<const bf16 *>(&m1);
#pragma unroll
              for (int jx = 0; jx < 8; jx++) {
                if (!(__bfloat162float(mm0[jx]) > 0.f)) v[jx] = 0.f;
                if (!(__bfloat162float(mm1[jx]) > 0.f)) v[8 + jx] = 0.f;
              }
            }
            uint4 o0, o1;
            o0.x = pack_bf16(v[0], v[1]);
            o0.y = pack_bf16(v[2], v[3]);
            o0.z = pack_bf16(v[4], v[5]);
            o0.w = pack_bf16(v[6], v[7]);
            o1.x = pack_bf16(v[8], v[9]);
            o1.y = pack_bf16(v[10], v[11]);
            o1.z = pack_bf16(v[12], v[13]);
            o1.w = pack_bf16(v[14], v[15]);
            *reinterpret_cast<uint4 *>(yp + cc) = o0;
            *reinterpret_cast<uint4 *>(yp + cc + 8) = o1;
          }
        }
        tc_fence_before();
        mbar_arrive(&acc_empty[acc]);
        if (++acc == a.nacc) {
          acc = 0;
          acc_ph ^= 1;
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.cols)
                 : "memory");
}

constexpr int kRowSmemFixed = 4 * kMaxCout + (2 * kRowMaxSlots + 2 * kMaxAcc + 1) * 8 + 16 + 1024;  // bias, barriers, slack
constexpr int kRowSmemMax = 232448;

// resident weights of the row form: 9 taps x cout rows x cin channels
int row_wbytes(const ConvArgs &a) { return 9 * a.cin * a.cout * 2; }

// shared memory of the row form for `slots` input-row buffers
int row_smem(const ConvArgs &a, int slots) {
  return row_wbytes(a) + slots * ((a.cin + 63) / 64) * kRowChunkBytes + kRowSmemFixed;
}

bool make_row_map(const ConvArgs &a, CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  std::memset(map, 0, sizeof(*map));
  const cuuint64_t dims[4] = {(cuuint64_t)a.cin, (cuuint64_t)a.W, (cuuint64_t)a.H,
                              (cuuint64_t)a.B};
  const cuuint64_t cs = (cuuint64_t)a.x_cs * 2;
  const cuuint64_t strides[3] = {cs, cs * (cuuint64_t)a.W, cs * (cuuint64_t)a.W * a.H};
  const cuuint32_t box[4] = {64u, (cuuint32_t)kRowPx, 1u, 1u};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(a.x + a.x_co), dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// ------------------------------------------------------------ weight gradient
// dw[co][t][ci] += sum_p dy[p][co] x[p + d_t][ci]: per tap t a GEMM D[co][ci] whose
// K is the pixels, split over CTAs; each CTA accumulates in tensor memory and adds
// its partial sums to dw with 16-byte atomics.  Both operands come straight from
// the NHWC tensors in the MN-major (channel-contiguous) 128-byte-swizzled layout:
// per 8 x 16 pixel block one TMA box of 64 channels x 128 pixels per operand half
// (x shifted by the tap, zero-filled outside the image), K = 128 pixels per stage
// as 8 MMAs of K = 16.  M = 128 output channels per tile (zero rows past cout),
// N = 64 or 128 input channels (zero columns past cin).
struct WgTcArgs {
  float *dw;
  int cin, cout;
  int H, W;
  int bx, by;
  int64_t nblk;  // B * by * bx pixel blocks
  int co_tiles, ci_tiles, ksplit;
  int *err;
};

// MN-major 128-byte-swizzled descriptor: 8-row K groups 1024 B apart, MN atoms
// of 64 channels `lbo` bytes apart
__device__ __forceinline__ uint64_t sdesc_mn128(uint32_t addr, uint32_t lbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

template <int NT>
__global__ void __launch_bounds__(kThreads, 1)
    wgrad_tc_kernel(const __grid_constant__ CUtensorMap dymap,
                    const __grid_constant__ CUtensorMap xmap, WgTcArgs a) {
  constexpr int kHalf = 16384;                 // 128 pixels x 64 channels x 2 B
  constexpr int kABytes = 2 * kHalf;           // 128 output channels
  constexpr int kBBytes = (NT / 64) * kHalf;   // NT input channels
  constexpr int kStage = kABytes + kBBytes;
  constexpr int ST = NT == 128 ? 3 : 4;
  constexpr uint32_t kCols = NT;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
  uint8_t *base = smem_raw + pad;
  uint64_t *full = reinterpret_cast<uint64_t *>(base + ST * kStage);
  uint64_t *empty = full + ST;
  uint64_t *done = empty + ST;
  uint64_t *drain = done + 1;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_tmem + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // work item: (tap, co tile, ci tile, K split)
  int64_t w = blockIdx.x;
  const int ks = (int)(w % a.ksplit);
  w /= a.ksplit;
  const int cit = (int)(w % a.ci_tiles);
  w /= a.ci_tiles;
  const int cot = (int)(w % a.co_tiles);
  const int tap = (int)(w / a.co_tiles), ky = tap / 3, kx = tap % 3;
  const int64_t b0 = a.nblk * ks / a.ksplit, b1 = a.nblk * (ks + 1) / a.ksplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    mbar_init(drain, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(s_tmem)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------ TMA producer
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&dymap))
                   : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&xmap))
                   : "memory");
      int stage = 0;
      uint32_t ph = 0, issued = 0, last_par = 0;
      for (int64_t blk = b0; blk < b1; blk++) {
        const int tx = (int)(blk % a.bx);
        const int64_t r = blk / a.bx;
        const int ty = (int)(r % a.by), b = (int)(r / a.by);
        if (!mbar_wait(&empty[stage], ph ^ 1)) {
          atomicOr(a.err, 1);
          *s_abort = 1;
          break;
        }
        uint8_t *sa = base + stage * kStage;
        mbar_expect_tx(&full[stage], (uint32_t)kStage);
        if (!(__ldg(&g_test_stall) && blk == b0)) {
          for (int h = 0; h < 2; h++)
            tma_load_4d(sa + h * kHalf, &dymap, cot * 128 + h * 64, tx * 16, ty * 8, b,
                        &full[stage]);
          for (int h = 0; h < NT / 64; h++)
            tma_load_4d(sa + kABytes + h * kHalf, &xmap, cit * NT + h * 64, tx * 16 + kx - 1,
                        ty * 8 + ky - 1, b, &full[stage]);
        }
        issued |= 1u << stage;
        last_par = (last_par & ~(1u << stage)) | (ph << stage);
        if (++stage == ST) {
          stage = 0;
          ph ^= 1;
        }
      }
      for (int s = 0; s < ST; s++)
        if ((issued >> s) & 1u)
          if (!mbar_wait(&full[s], (last_par >> s) & 1u)) atomicOr(a.err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------ MMA issuer
      constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                 ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
      int stage = 0;
      uint32_t ph = 0;
      bool first = true;
      for (int64_t blk = b0; blk < b1 && !*s_abort; blk++) {
        if (!mbar_wait(&full[stage], ph)) {
          atomicOr(a.err, 1);
          *s_abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(base + stage * kStage);
        const uint64_t da = sdesc_mn128(sa, kHalf), db = sdesc_mn128(sa + kABytes, kHalf);
#pragma unroll
        for (int k = 0; k < 8; k++)
          tc_mma(tmem, da + (uint64_t)(k * 128), db + (uint64_t)(k * 128), idesc,
                 (first && k == 0) ? 0u : 1u);
        first = false;
        tc_commit(&empty[stage]);
        if (++stage == ST) {
          stage = 0;
          ph ^= 1;
        }
      }
      tc_commit(done);
      tc_commit(drain);
      if (!mbar_wait(drain, 0)) atomicOr(a.err, 1);
    }
  } else {
    // ---------------------------------------------------- epilogue (warps 2-5)
    const int q = warp & 3;
    const int co_l = q * 32 + lane;
    const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0));
    if (!ok && lane == 0) {
      atomicOr(a.err, 1);
      *s_abort = 1;
    }
    float *stg = reinterpret_cast<float *>(base);
    constexpr int kPitch = NT + 4;
    if (ok && b1 > b0 && !__shfl_sync(0xffffffffu, *s_abort, 0)) {
      tc_fence_after();
      // tensor memory -> shared staging [128][NT + 4] floats (the pipeline
      // stages are idle: every MMA has completed)
      const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += 32) {
        uint32_t rr[2][16];
        tmem_ld16(taddr + (uint32_t)c0, rr[0]);
        tmem_ld16(taddr + (uint32_t)c0 + 16u, rr[1]);
        tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int j = 0; j < 16; j++)
            stg[co_l * kPitch + c0 + 16 * h + j] = __uint_as_float(rr[h][j]);
      }
    }
    // every epilogue warp passes this barrier exactly once
    asm volatile("bar.sync 1, 128;" ::: "memory");
    if (b1 > b0 && !__shfl_sync(0xffffffffu, *s_abort, 0)) {
      // coalesced 16-byte atomics along ci
      const int t = threadIdx.x - 64;
      constexpr int kV = NT / 4;
      for (int i = t; i < 128 * kV; i += 128) {
        const int row = i / kV, c4 = (i % kV) * 4;
        const int co = cot * 128 + row, ci = cit * NT + c4;
        if (co < a.cout && ci < a.cin) {
          const float *v = stg + row * kPitch + c4;
          atomicAdd(reinterpret_cast<float4 *>(a.dw + ((int64_t)co * 9 + tap) * a.cin + ci),
                    make_float4(v[0], v[1], v[2], v[3]));
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols)
                 : "memory");
}

bool make_nhwc_map(const __nv_bfloat16 *p, int cs, int co, int C, int W, int H, int B,
                   CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  std::memset(map, 0, sizeof(*map));
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t s0 = (cuuint64_t)cs * 2;
  const cuuint64_t strides[3] = {s0, s0 * (cuuint64_t)W, s0 * (cuuint64_t)W * H};
  const cuuint32_t box[4] = {64u, 16u, 8u, 1u};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(p + co), dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int NT> cudaError_t launch_wgrad_nt(const WgradArgs &a, cudaStream_t st) {
  constexpr int ST = NT == 128 ? 3 : 4;
  constexpr int kStage = 2 * 16384 + (NT / 64) * 16384;
  const int smem = ST * kStage + 256 + 1024;  // stages, barriers, alignment slack
  CUtensorMap dymap, xmap;
  if (!make_nhwc_map(a.dy, a.dy_cs, a.dy_co, a.cout, a.W, a.H, a.B, &dymap) ||
      !make_nhwc_map(a.x, a.x_cs, a.x_co, a.cin, a.W, a.H, a.B, &xmap))
    return cudaErrorInvalidValue;
  WgTcArgs w{};
  w.dw = a.dw;
  w.cin = a.cin;
  w.cout = a.cout;
  w.H = a.H;
  w.W = a.W;
  w.bx = a.W / 16;
  w.by = a.H / 8;
  w.nblk = (int64_t)a.B * w.by * w.bx;
  w.co_tiles = (a.cout + 127) / 128;
  w.ci_tiles = (a.cin + NT - 1) / NT;
  const int64_t cols = 9LL * w.co_tiles * w.ci_tiles;
  w.ksplit = (int)std::max<int64_t>(1, std::min<int64_t>(w.nblk, (2LL * sm_count() + cols - 1) / cols));
  cudaError_t e = err_word(&w.err);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(wgrad_tc_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = cols * w.ksplit;
  wgrad_tc_kernel<NT><<<(unsigned)grid, kThreads, smem, st>>>(dymap, xmap, w);
  return cudaGetLastError();
}

}  // namespace

int conv_tc_chunk(int cin) {
  return cin % 64 == 0 ? 64 : cin % 32 == 0 ? 32 : cin == 16 ? 16 : 0;
}

int conv_tc_ntile(int cout) {
  if (cout <= 128) return (cout % 32 == 0) ? cout : 0;
  if (cout % 128 == 0) return 128;
  if (cout % 96 == 0) return 96;
  if (cout % 64 == 0) return 64;
  return cout % 32 == 0 ? 32 : 0;
}

bool conv_row_ok(const ConvArgs &a) {
  return conv_tc_ok(a) && a.W % 128 == 0 &&
         (a.cin == 16 || a.cin == 32 || a.cin == 64 || a.cin == 96 || a.cin == 128) &&
         a.cout % 32 == 0 &&
         a.cout <= 64 && row_wbytes(a) <= 112 * 1024 && row_smem(a, 4) <= kRowSmemMax;
}

cudaError_t launch_conv3x3_row(const ConvArgs &a, cudaStream_t st) {
  if (!conv_row_ok(a)) return cudaErrorInvalidValue;
  CUtensorMap amap;
  if (!make_row_map(a, &amap)) return cudaErrorInvalidValue;
  RowArgs r{};
  r.y = a.y;
  r.y_cs = a.y_cs;
  r.y_co = a.y_co;
  r.mask = a.mask;
  r.m_cs = a.m_cs;
  r.m_co = a.m_co;
  r.bias = a.bias;
  r.w = a.w;
  r.cin = a.cin;
  r.cout = a.cout;
  r.relu = a.relu;
  r.H = a.H;
  r.W = a.W;
  r.nacc = 256 / a.cout >= 8 ? 8 : 256 / a.cout >= 4 ? 4 : 2;
  r.cols = 256u;
  r.wbytes = row_wbytes(a);
  r.slot_bytes = ((a.cin + 63) / 64) * kRowChunkBytes;
  int slots = kRowMaxSlots;
  while (slots > 4 && row_smem(a, slots) > 110 * 1024) slots--;  // two CTAs per SM if possible
  r.nslots = slots;
  cudaError_t e = err_word(&r.err);
  if (e != cudaSuccess) return e;
  const int per_sm = 512 / (int)r.cols;
  const int smem = std::max(row_smem(a, slots), 232448 / (per_sm + 1) + 1024);
  auto kern = a.cin == 16   ? conv_row_kernel<16>
              : a.cin == 32 ? conv_row_kernel<32>
              : a.cin == 64 ? conv_row_kernel<64>
              : a.cin == 96 ? conv_row_kernel<96>
                            : conv_row_kernel<128>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  const int occ = occupancy(kern, smem, per_sm);
  const int64_t ctas = (int64_t)sm_count() * occ;
  r.strips_x = a.W / 128;
  // strips of up to 32 rows; shorter where that leaves too few strips per CTA
  int sh = std::min(32, a.H);
  while (sh > 8 && (int64_t)a.B * r.strips_x * ((a.H + sh - 1) / sh) < 4 * ctas) sh /= 2;
  r.strip_h = sh;
  r.strips_y = (a.H + sh - 1) / sh;
  r.total = (int64_t)a.B * r.strips_y * r.strips_x;
  const int64_t grid = std::min<int64_t>(r.total, ctas);
  kern<<<(unsigned)grid, kThreads, smem, st>>>(amap, r);
  return cudaGetLastError();
}

bool conv_tc_ok(const ConvArgs &a) {
  return conv_shape_ok(a) && conv_tc_chunk(a.cin) != 0 && conv_tc_ntile(a.cout) != 0 &&
         a.y_cs % 8 == 0 && a.y_co % 8 == 0 && (!a.mask || (a.m_cs % 8 == 0 && a.m_co % 8 == 0)) &&
         a.cin <= 65535 && a.cout <= kMaxCout;
}

cudaError_t launch_conv3x3_tc(const ConvArgs &a, cudaStream_t st) {
  if (!conv_tc_ok(a)) return cudaErrorInvalidValue;
  if (conv_row_ok(a)) return launch_conv3x3_row(a, st);
  const int ck = conv_tc_chunk(a.cin), nt = conv_tc_ntile(a.cout);
  if (ck == 64) return launch_ck<64>(a, nt, st);
  if (ck == 32) return launch_ck<32>(a, nt, st);
  return launch_ck<16>(a, nt, st);
}

bool wgrad_tc_ok(const WgradArgs &a) {
  return a.B >= 1 && a.H >= 8 && a.W >= 16 && a.H % 8 == 0 && a.W % 16 == 0 && a.cin % 16 == 0 &&
         a.cout % 16 == 0 && a.x_cs % 8 == 0 && a.x_co % 8 == 0 && a.dy_cs % 8 == 0 &&
         a.dy_co % 8 == 0 && a.x_co + a.cin <= a.x_cs && a.dy_co + a.cout <= a.dy_cs &&
         (reinterpret_cast<uintptr_t>(a.dw) & 15) == 0;
}

cudaError_t launch_conv3x3_wgrad_tc(const WgradArgs &a, cudaStream_t st) {
  if (!wgrad_tc_ok(a)) return cudaErrorInvalidValue;
  return a.cin > 64 ? launch_wgrad_nt<128>(a, st) : launch_wgrad_nt<64>(a, st);
}

int conv_tc_error() {
  std::lock_guard<std::mutex> l(g_err_mutex);
  return g_err_host ? *(volatile int *)g_err_host : 0;
}

void conv_tc_clear_error() {
  std::lock_guard<std::mutex> l(g_err_mutex);
  if (g_err_host) *(volatile int *)g_err_host = 0;
}

}  // namespace ctas

// Test aid of the C ABI (ctas_learned.h): arm or disarm the stall of the
// tcgen05 convolution kernels on the current device.
extern "C" int ctas_nn_test_timeout(int32_t enable) {
  const int stall = enable ? 1 : 0;
  const uint32_t limit = enable ? (1u << 12) : ctas::kWaitLimit;
  if (cudaMemcpyToSymbol(ctas::g_test_stall, &stall, sizeof(stall)) != cudaSuccess ||
      cudaMemcpyToSymbol(ctas::g_wait_limit, &limit, sizeof(limit)) != cudaSuccess) {
    cudaGetLastError();
    return CTAS_E_CUDA;
  }
  return CTAS_OK;
}
