// bp_fast.cu -- staged backprojection for sm_100a (all sines >= 0).
//
// Computes exactly what bp_generic.cu computes -- the reference's per-pixel
// arithmetic of CTrec::reconstructOnCPU (ctas src/common/lct.cpp:688-729) /
// ct.cl:14-43, bit for bit -- for the geometry of every scan whose angles lie
// in [0, pi] (sin >= 0 for all projections, e.g. the reference's default
// 180-degree arc).  For such scans every reconstructed pixel has
// t in (-1, W + 1) (the pixel masks bound it), so:
//   * the truncation (int)t equals floor(t) except on (-1, 0), where floor
//     gives -1; column -1 of the padded filtered row repeats sample 0
//     (fbp_kernels.hpp), so floor is exact.  floor(t) is taken with one
//     rounded-down add of 1.5*2^23, whose float bits then hold the index;
//   * a pixel tile only touches a short detector window per projection.
//
// Design:
//   * CTA tile of kTileY x kTileX output pixels, 8 consumer warps with a
//     register tile of kRY x kRX pixels per thread, plus one producer warp.
//   * Per projection, the producer computes the detector window the tile
//     covers and fetches it from the L2-resident filtered sinogram into shared
//     memory with a TMA tile load (cp.async.bulk.tensor, no multicast);
//     kChunk projections per stage, kStages stages, mbarrier completion.
//   * Consumers gather from shared memory with a 4x8 lane patch per warp
//     (the gathered samples of a warp span < 32 consecutive words: no bank
//     conflicts) and accumulate in projection order with packed f32x2 adds.
//   * Every wait is bounded; on timeout the kernel sets bit 2 of the error
//     word, drains its outstanding copies (bounded) and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "bp_common.cuh"
#include "bp_fast.hpp"

namespace ctas {
namespace {

constexpr int kConsumerWarps = 8;
constexpr int kThreads = (kConsumerWarps + 1) * 32;
constexpr int kTileY = 64, kTileX = 64;
constexpr int kRY = 4, kRX = 4;          // register tile per thread
constexpr int kChunk = 16;               // projections per pipeline stage
constexpr int kStages = 4;
constexpr int kBox = 128;                // window samples fetched per projection
constexpr float kMagic = 12582912.0f;    // 1.5 * 2^23
constexpr uint32_t kMagicBits = 0x4B400000u;
constexpr uint32_t kWaitLimit = 1u << 22;

static_assert(kTileY == 4 * (kConsumerWarps / 2) * kRY, "tile rows");
static_assert(kTileX == 8 * 2 * kRX, "tile cols");

struct __align__(16) AngleParam {
  float sx, cy, base;  // sin, cos, c + ((1 - sin) - cos) * hp
  uint32_t addr;       // smem byte address bias: window - 4*(magic bits + x0)
};

struct SmemLayout {
  float win[kStages][kChunk][kBox];
  AngleParam par[kStages][kChunk];
  unsigned long long full[kStages];
  int abort_flag;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: false when the limit ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_row(void *dst, const CUtensorMap *map, int x, int y,
                                             unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// packed f32x2 arithmetic (sm_100a), explicit rounding
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
  float2 r;
  asm("{\n .reg .b64 ra, rb, rr;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " add.rn.f32x2 rr, ra, rb;\n mov.b64 {%0, %1}, rr;\n}\n"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 add2_rm(float2 a, float2 b) {
  float2 r;
  asm("{\n .reg .b64 ra, rb, rr;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " add.rm.f32x2 rr, ra, rb;\n mov.b64 {%0, %1}, rr;\n}\n"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float lds_f32(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}

// Projection parameters and detector window of one tile (producer side).
// The window start x0 is the lowest index any pixel of the tile can reach,
// minus a margin, rounded down to a multiple of 4 (16-byte TMA alignment).
__device__ __forceinline__ int window_start(float sx, float cy, float base, int j0, int i0,
                                            float c) {
  const float jc0 = __fsub_rn((float)j0, c), jc1 = __fsub_rn((float)(j0 + kTileY - 1), c);
  const float d0 = __fmul_rn(cy, (float)i0), d1 = __fmul_rn(cy, (float)(i0 + kTileX - 1));
  const float b0 = __fadd_rn(base, __fmul_rn(sx, jc0)), b1 = __fadd_rn(base, __fmul_rn(sx, jc1));
  const float tmin = fminf(fminf(__fadd_rn(b0, d0), __fadd_rn(b0, d1)),
                           fminf(__fadd_rn(b1, d0), __fadd_rn(b1, d1)));
  const int lo = (int)floorf(tmin) - 2;
  return lo & ~3;  // floor to a multiple of 4 (two's complement)
}

template <bool kCheck, bool kPacked>
__global__ void __launch_bounds__(kThreads, 2)
    bp_fast_kernel(const __grid_constant__ CUtensorMap qmap, BpLaunch a, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations: 128-byte aligned
  SmemLayout &sm = *reinterpret_cast<SmemLayout *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  const int W = a.W, N = a.N, hp = W / 2;
  const float c = a.center;
  const int i0 = blockIdx.x * kTileX, j0 = blockIdx.y * kTileY, sl = blockIdx.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool producer = (warp == kConsumerWarps);
  float *out = a.out + sl * a.out_slice_stride;

  // thread's pixels: rows j0 + wy*16 + ly + 4*r, columns i0 + wx*32 + lx + 8*b
  const int wy = warp >> 1, wx = warp & 1, ly = lane >> 3, lx = lane & 7;
  const int jb = j0 + wy * 16 + ly, ib = i0 + wx * 32 + lx;

  bool any = false;
  if (!producer) {
#pragma unroll
    for (int r = 0; r < kRY; r++)
#pragma unroll
      for (int b = 0; b < kRX; b++) {
        const int j = jb + 4 * r, i = ib + 8 * b;
        any |= (j < W && i < W) && ref_mask(j, i, W, c);
      }
  }
  if (!__syncthreads_or(any)) {
    if (!producer) {
#pragma unroll
      for (int r = 0; r < kRY; r++)
#pragma unroll
        for (int b = 0; b < kRX; b++) {
          const int j = jb + 4 * r, i = ib + 8 * b;
          if (j < W && i < W) out[(int64_t)j * W + i] = 0.f;
        }
    }
    return;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&sm.full[s], 1);
    sm.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const int nchunks = (N + kChunk - 1) / kChunk;
  const int row0 = sl * N;  // first row of this slice in the tensor map

  // producer: fill stage st with chunk ch
  auto issue = [&](int ch) {
    const int st = ch % kStages;
    const int n0 = ch * kChunk;
    const int cnt = min(kChunk, N - n0);
    if (lane == 0) mbar_arrive_expect_tx(&sm.full[st], (uint32_t)(cnt * kBox * sizeof(float)));
    __syncwarp();
    if (lane < cnt) {
      const int n = n0 + lane;
      const float2 sc = a.tab[n];
      const float base = ref_base(sc.x, sc.y, hp, c);
      const int x0 = window_start(sc.x, sc.y, base, j0, i0, c);
      AngleParam p;
      p.sx = sc.x;
      p.cy = sc.y;
      p.base = base;
      p.addr = smem_u32(&sm.win[st][lane][0]) - 4u * (kMagicBits + (uint32_t)x0);
      sm.par[st][lane] = p;
      tma_load_row(&sm.win[st][lane][0], &qmap, x0 + kRowOff, row0 + n, &sm.full[st]);
    }
  };

  int issued = 0;
  if (producer) {
    for (; issued < min(kStages - 1, nchunks); issued++) issue(issued);
  }

  // per-thread constants
  float2 jcp[kRY / 2];  // (j - c) for row pairs
#pragma unroll
  for (int p = 0; p < kRY / 2; p++)
    jcp[p] = make_float2(__fsub_rn((float)(jb + 8 * p), c), __fsub_rn((float)(jb + 8 * p + 4), c));
  float fib[kRX];
#pragma unroll
  for (int b = 0; b < kRX; b++) fib[b] = (float)(ib + 8 * b);
  float2 acc[kRY / 2][kRX];
#pragma unroll
  for (int p = 0; p < kRY / 2; p++)
#pragma unroll
    for (int b = 0; b < kRX; b++) acc[p][b] = make_float2(0.f, 0.f);
  const float2 magic2 = make_float2(kMagic, kMagic);

  int consumed = 0;
  for (int ch = 0; ch < nchunks; ch++) {
    __syncthreads();  // every consumer is done with chunk ch-1: its stage is free
    if (sm.abort_flag) break;
    if (producer) {
      if (issued < nchunks) issue(issued++);
      continue;
    }
    const int st = ch % kStages;
    if (!mbar_wait(&sm.full[st], (uint32_t)((ch / kStages) & 1))) {
      sm.abort_flag = 1;
      if (lane == 0) atomicOr(err, 4);
      continue;
    }
    consumed = ch + 1;
    const int cnt = min(kChunk, N - ch * kChunk);
#pragma unroll 1
    for (int k = 0; k < cnt; k++) {
      const AngleParam p = sm.par[st][k];
      float2 brow[kRY / 2];
      // Products are formed with scalar __fmul_rn and consumed by scalar
      // __fadd_rn: a packed multiply feeding a packed add may be contracted
      // into a fused multiply-add, which would change the reference's
      // rounding.  Only adds whose inputs are adds or loads are packed.
#pragma unroll
      for (int q = 0; q < kRY / 2; q++) {
        brow[q].x = __fadd_rn(p.base, __fmul_rn(p.sx, jcp[q].x));
        brow[q].y = __fadd_rn(p.base, __fmul_rn(p.sx, jcp[q].y));
      }
#pragma unroll
      for (int b = 0; b < kRX; b++) {
        // + 0.0f (an exact add) keeps the product out of any fused form
        const float db = kPacked ? __fadd_rn(__fmul_rn(p.cy, fib[b]), 0.0f)
                                 : __fmul_rn(p.cy, fib[b]);
        const float2 d = make_float2(db, db);
#pragma unroll
        for (int q = 0; q < kRY / 2; q++) {
          float2 t, u;
          if (kPacked) {
            t = add2_rn(brow[q], d);
            u = add2_rm(t, magic2);
          } else {
            t = make_float2(__fadd_rn(brow[q].x, d.x), __fadd_rn(brow[q].y, d.y));
            u = make_float2(__fadd_rd(t.x, kMagic), __fadd_rd(t.y, kMagic));
          }
          const uint32_t a0 = (__float_as_uint(u.x) << 2) + p.addr;
          const uint32_t a1 = (__float_as_uint(u.y) << 2) + p.addr;
          if (kCheck) {
            const uint32_t lo = smem_u32(&sm.win[st][k][0]);
            const bool ok0 = a0 >= lo && a0 < lo + 4 * kBox, ok1 = a1 >= lo && a1 < lo + 4 * kBox;
            if (!(ok0 && ok1)) atomicOr(err, 8);
            const float v0 = ok0 ? lds_f32(a0) : 0.f, v1 = ok1 ? lds_f32(a1) : 0.f;
            acc[q][b] = kPacked ? add2_rn(acc[q][b], make_float2(v0, v1))
                                : make_float2(__fadd_rn(acc[q][b].x, v0), __fadd_rn(acc[q][b].y, v1));
          } else {
            const float v0 = lds_f32(a0), v1 = lds_f32(a1);
            acc[q][b] = kPacked ? add2_rn(acc[q][b], make_float2(v0, v1))
                                : make_float2(__fadd_rn(acc[q][b].x, v0), __fadd_rn(acc[q][b].y, v1));
          }
        }
      }
    }
  }
  __syncthreads();
  if (sm.abort_flag) {
    // drain copies still in flight before the CTA exits (bounded)
    if (producer && lane == 0)
      for (int ch = consumed; ch < issued; ch++)
        mbar_wait(&sm.full[ch % kStages], (uint32_t)((ch / kStages) & 1));
    __syncthreads();
    return;
  }
  if (producer) return;
#pragma unroll
  for (int q = 0; q < kRY / 2; q++)
#pragma unroll
    for (int b = 0; b < kRX; b++) {
      const int i = ib + 8 * b;
      const int jA = jb + 8 * q, jB = jA + 4;
      if (i < W) {
        if (jA < W)
          out[(int64_t)jA * W + i] = ref_mask(jA, i, W, c) ? ref_finish(acc[q][b].x, a.rec_cof, N) : 0.f;
        if (jB < W)
          out[(int64_t)jB * W + i] = ref_mask(jB, i, W, c) ? ref_finish(acc[q][b].y, a.rec_cof, N) : 0.f;
      }
    }
}

// ------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

}  // namespace

bool bp_fast_supported(const BpLaunch &a) {
  return a.store == 0 && encode_fn() != nullptr && a.Wp >= kBox && (a.Wp % 4) == 0 &&
         (int64_t)a.N * a.S < (1ll << 31);
}

static cudaError_t launch_impl(const BpLaunch &a, cudaStream_t st, bool check) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const cuuint64_t dims[2] = {(cuuint64_t)a.Wp, (cuuint64_t)a.N * (cuuint64_t)a.S};
  const cuuint64_t strides[1] = {(cuuint64_t)a.Wp * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)kBox, 1u};
  const cuuint32_t estr[2] = {1u, 1u};
  // the slices of a launch are contiguous in the padded buffer
  if (a.q_slice_stride != (int64_t)a.N * a.Wp) return cudaErrorInvalidValue;
  CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(a.q), dims,
                   strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  const size_t smem = sizeof(SmemLayout) + 128;
  // CTAS_FBP_SCALAR=1 selects scalar-rounded arithmetic instead of packed f32x2
  static const bool scalar = [] {
    const char *e = std::getenv("CTAS_FBP_SCALAR");
    return e && e[0] == '1';
  }();
  auto kern = check ? (scalar ? bp_fast_kernel<true, false> : bp_fast_kernel<true, true>)
                    : (scalar ? bp_fast_kernel<false, false> : bp_fast_kernel<false, true>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((a.W + kTileX - 1) / kTileX, (a.W + kTileY - 1) / kTileY, a.S);
  kern<<<grid, kThreads, smem, st>>>(map, a, a.err);
  return cudaGetLastError();
}

cudaError_t launch_bp_fast(const BpLaunch &a, cudaStream_t st) {
  return launch_impl(a, st, false);
}

cudaError_t launch_bp_fast_checked(const BpLaunch &a, cudaStream_t st) {
  return launch_impl(a, st, true);
}

}  // namespace ctas
