// bp_fast.cu -- staged backprojection for sm_100a.
//
// Reference truncation mode computes exactly what bp_generic.cu computes -- the
// per-pixel arithmetic of CTrec::reconstructOnCPU (ctas
// src/common/lct.cpp:688-729) / ct.cl:14-43, bit for bit -- for every scan whose
// angles lie in [0, pi] (sin >= 0 for all projections, e.g. the reference's
// default 180-degree arc).  For such scans every reconstructed pixel has
// t in (-1, W + 1) (the pixel masks bound it), so:
//   * the truncation (int)t equals floor(t) except on (-1, 0), where floor
//     gives -1; column -1 of the padded filtered row repeats sample 0
//     (fbp_kernels.hpp), so floor is exact.  floor(t) is one rounded-down add
//     of 1.5*2^23, whose float bits then hold the index;
//   * a pixel tile only touches a short detector window per projection.
// Linear interpolation mode (an extension) uses the same staging with
// FP64-derived projection bases and FP32 increments.
//
// Design:
//   * CTA tile of TY x TX output pixels: WY x WX consumer warps, each thread
//     holding RY x RX pixels in registers (lanes form a 4 x 8 patch, so the
//     samples a warp gathers span < 32 consecutive words: no bank conflicts),
//     plus one producer warp.
//   * Per projection the producer computes the detector window the tile
//     covers and fetches it from the L2-resident filtered sinogram into shared
//     memory with a TMA tile load (cp.async.bulk.tensor.2d, no multicast);
//     kChunk projections per stage, kStages stages.  Stages are handed over
//     with full/empty mbarriers, so consumer warps never wait for each other.
//     Reduced-precision stores and linear interpolation load a raw window that
//     the producer converts (scale, sample pairs) before releasing the stage.
//   * Warps whose pixels all lie outside the reconstruction disc write zeros
//     and leave; the stage barriers count only the warps that stay.
//   * Every wait is bounded: on timeout the kernel sets bit 2 of the error
//     word, the producer drains its outstanding copies (bounded), and the CTA
//     returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "bp_common.cuh"
#include "bp_fast.hpp"
#include "tma_encode.hpp"

namespace ctas {
namespace {

// projections per pipeline stage, and stages: 32 x 3 ran 1.3 % (float32) and
// 1.9 % (16-bit stores) faster than 16 x 4 -- half the barrier round trips and
// prefetch restarts per projection -- while keeping two 16-bit 64 x 128 CTAs per
// SM (32 x 4 does not fit them: 16-bit stores then ran 24 % slower)
constexpr int kChunk = 32;
constexpr int kStages = 3;
constexpr float kMagic = 12582912.0f;    // 1.5 * 2^23
constexpr uint32_t kMagicBits = 0x4B400000u;
constexpr uint32_t kWaitLimit = 1u << 22;

thread_local char t_detail[160];  // last launch failure on this host thread

template <int RY_, int RX_, int WY_, int WX_, int BOX_, int MINB_>
struct Tile {
  static constexpr int RY = RY_, RX = RX_, WY = WY_, WX = WX_, BOX = BOX_;
  static constexpr int MINB = MINB_;  // resident CTAs per SM the registers must allow
  static constexpr int TY = WY * 4 * RY, TX = WX * 8 * RX;
  static constexpr int WARPS = WY * WX;
  static constexpr int THREADS = (WARPS + 1) * 32;
  static_assert(RY % 2 == 0 && RX % 2 == 0, "row and column pairs");
  // window span (TY-1)|sin| + (TX-1)|cos| plus margins (window start 2 below
  // the lowest index, 7 of alignment, 1 of rounding, 1 for the linear pair)
  static_assert((BOX - 12) * (BOX - 12) >= (TY - 1) * (TY - 1) + (TX - 1) * (TX - 1),
                "window too short for the tile");
  static_assert((BOX * 4) % 128 == 0, "128-byte aligned window rows");
};

// tile configurations the autotuner chooses from (index = tile id)
using T0 = Tile<4, 4, 4, 2, 128, 2>;  //  64 x  64, 8 warps, 16 px / thread
using T1 = Tile<4, 8, 4, 2, 160, 2>;  //  64 x 128, 8 warps, 32 px / thread
using T2 = Tile<8, 4, 4, 2, 160, 2>;  // 128 x  64, 8 warps, 32 px / thread
using T3 = Tile<8, 8, 4, 2, 192, 1>;  // 128 x 128, 8 warps, 64 px / thread
using T4 = Tile<4, 8, 2, 2, 160, 4>;  //  32 x 128, 4 warps, 32 px / thread
using T5 = Tile<4, 8, 4, 2, 160, 3>;  // T1 held to 3 CTAs / SM
using T6 = Tile<8, 4, 4, 2, 160, 3>;  // T2 held to 3 CTAs / SM
constexpr int kShapes = 7;

// Calls f with a value of the tile type of `shape`.
template <class F> auto with_shape(int shape, F &&f) {
  switch (shape) {
  case 0: return f(T0{});
  case 1: return f(T1{});
  case 2: return f(T2{});
  case 3: return f(T3{});
  case 4: return f(T4{});
  case 5: return f(T5{});
  default: return f(T6{});
  }
}
// Arithmetic variants of the truncation path (tile id / kShapes):
//   0: t by two scalar adds; floor and accumulation by packed f32x2 adds;
//      address = (index bits << 2) + window bias
//   1: folded address (below) with the shift on the integer ALU (funnel
//      shift); per-projection row and column terms by packed products
//      (mul2z_rn) and adds
//   2: as 1 with t by one packed add per pixel pair (two columns of one row:
//      the column products come paired from the packed product, and the row
//      term is the broadcast operand -- 0.5 % faster than pairing two rows)
// Folded address: the projection's coefficients are scaled by 2^-22 (exact:
// no intermediate is subnormal) and floor(t) is taken by a rounded-down add
// of M = 2 + off * 2^-22, off = window word address - window start index.
// The sum lies in [2, 4), where the float grid step is 2^-22, so it is
// 2 + (off + floor(t)) * 2^-22 exactly and its bits are
// 0x40000000 + off + floor(t); shifted left by 2 (mod 2^32) they are the
// byte address of the sample -- one shift, no add, per update.  M itself
// may lie in [1, 2) (negative off); only the sum must be >= 2, which holds
// because floor(t) >= window start.
constexpr int kVariants = 3;
constexpr int kTiles = kVariants * kShapes;
constexpr float kTwoM22 = 2.384185791015625e-07f;  // 2^-22

struct __align__(16) AngleParam {
  float sx, cy, base;  // truncation: sin, cos, c + ((1 - sin) - cos) * hp
                       // (all times 2^-22 with the folded address)
                       // linear: sin, cos, t0
  uint32_t addr;       // smem byte address bias of the window; folded
                       // address: the bits of M
};

template <class TL, class RawT, int MODE> struct Layout {
  static constexpr bool kTransform = (MODE == 1) || !std::is_same<RawT, float>::value;
  static constexpr int kWin = MODE == 1 ? 2 * TL::BOX : TL::BOX;  // floats per window
  // TMA destinations start on 128-byte boundaries: raw rows are padded to a
  // multiple of 128 bytes (BOX samples are loaded into each)
  static constexpr int kRawStride =
      kTransform ? ((TL::BOX * (int)sizeof(RawT) + 127) / 128) * 128 / (int)sizeof(RawT) : 8;
  static_assert((kWin * 4) % 128 == 0, "window rows on 128-byte boundaries");
  static_assert(!kTransform || (kRawStride * (int)sizeof(RawT)) % 128 == 0,
                "raw rows on 128-byte boundaries");
  float win[kStages][kChunk][kWin];
  RawT raw[kStages][kChunk][kRawStride];
  AngleParam par[kStages][kChunk];
  AngleParam parq[kStages][kChunk];  // converting paths: parameters of raw copies in flight
  float scale[kStages][kChunk];
  uint32_t negmask[kStages];  // wide layout: projections whose indices may be < 0
  unsigned long long full[kStages], empty[kStages], rawfull[kStages];
  int active[32];
  int nactive;
  int barriers_live;  // the stage barriers are initialised
  int abort_flag;     // a wait ran out: stop taking work
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_inval(unsigned long long *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity,
                                          uint32_t limit = kWaitLimit) {
  for (uint32_t it = 0; it < limit; ++it)
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

// packed f32x2 adds (sm_100a), explicit rounding; inputs never come straight
// from a multiply (a packed multiply-add chain may be fused)
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

__device__ __forceinline__ float2 add2_rp(float2 a, float2 b) {
  float2 r;
  asm("{\n .reg .b64 ra, rb, rr;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " add.rp.f32x2 rr, ra, rb;\n mov.b64 {%0, %1}, rr;\n}\n"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

// Packed product a * b formed as fma(a, b, +0): one rounding, like a
// multiply, but the compiler cannot contract it into a following add (a
// packed multiply with explicit rounding does get contracted).  It differs
// from the product only in the sign of a zero result, which changes no
// floor index downstream.
__device__ __forceinline__ float2 mul2z_rn(float2 a, float2 b) {
  float2 r;
  asm("{\n .reg .b64 ra, rb, rz, rr;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " mov.b64 rz, 0;\n fma.rn.f32x2 rr, ra, rb, rz;\n mov.b64 {%0, %1}, rr;\n}\n"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

// x << 2 as a funnel shift of (x : lo) with lo < 2^30, so that it runs on the
// integer ALU rather than as a multiply-add
__device__ __forceinline__ uint32_t shl2_alu(uint32_t x, uint32_t lo) {
  uint32_t r;
  asm("shf.l.wrap.b32 %0, %1, %2, 2;" : "=r"(r) : "r"(lo), "r"(x));
  return r;
}

// Shared loads of a released stage.  Not volatile: the address depends on
// parameters read after the stage's barrier wait, which orders the load.
__device__ __forceinline__ float lds_f32(uint32_t addr) {
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}

__device__ __forceinline__ float2 lds_f32x2(uint32_t addr) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}

template <class T> __device__ __forceinline__ float raw_to_f32(T v) { return (float)v; }
template <> __device__ __forceinline__ float raw_to_f32<float>(float v) { return v; }

// Eight 16-bit samples (one 16-byte word) to floats.
__device__ __forceinline__ float2 pair_to_f32(uint32_t w, __half) {
  return __half22float2(*reinterpret_cast<const __half2 *>(&w));
}
__device__ __forceinline__ float2 pair_to_f32(uint32_t w, __nv_bfloat16) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&w));
}

// Lowest detector index any pixel of the tile can reach, minus a margin,
// rounded down to a multiple of `align` elements (16-byte TMA alignment).
// (ja, jb), (ia, ib): reference coordinates of the tile's first and last
// rows and columns; the index is affine in them, so its minimum is at a
// corner (rounding moves it by far less than the margin).
__device__ __forceinline__ int window_start_trunc(float sx, float cy, float base, float ja,
                                                  float jb, float ia, float ib, float c,
                                                  int align, float *tmin_out = nullptr) {
  const float jc0 = __fsub_rn(ja, c), jc1 = __fsub_rn(jb, c);
  const float d0 = __fmul_rn(cy, ia), d1 = __fmul_rn(cy, ib);
  const float b0 = __fadd_rn(base, __fmul_rn(sx, jc0)), b1 = __fadd_rn(base, __fmul_rn(sx, jc1));
  const float tmin = fminf(fminf(__fadd_rn(b0, d0), __fadd_rn(b0, d1)),
                           fminf(__fadd_rn(b1, d0), __fadd_rn(b1, d1)));
  if (tmin_out) *tmin_out = tmin;
  const int lo = (int)floorf(tmin) - 2;
  return lo & ~(align - 1);
}

__device__ __forceinline__ int window_start_linear(float sx, float cy, float t0, float ja,
                                                   float jb, float ia, float ib, int align) {
  const float a = fmaf(sx, ja, t0), b = fmaf(sx, jb, t0);
  const float tmin = fminf(fminf(fmaf(cy, ia, a), fmaf(cy, ib, a)),
                           fminf(fmaf(cy, ia, b), fmaf(cy, ib, b)));
  const int lo = (int)floorf(tmin) - 2;
  return lo & ~(align - 1);
}

// One slice as the tile routine sees it.
struct SliceJob {
  int W, N, row0;            // row0: first row of the slice in the tensor map
  int R, C;                  // output rows, columns
  float oj, oi, p;           // output geometry (see BpLaunch)
  float c, rec_cof;
  const float2 *tab;         // truncation: float sin/cos table
  const double2 *lin;        // linear interpolation: FP64 sin/cos table
  const float *row_scale;    // reduced-precision store: scales indexed by tensor-map row
  float *out;                // the slice's W x W output
  int rule;                  // rounding order of the index expression (ref_base)
  int off;                   // column of sample 0 in the tensor map's rows
  int wide;                  // wide layout: indices may be negative (truncate toward 0)
  uint32_t wait_limit;       // iterations of each bounded mbarrier wait
  int test_stall;            // test aid: the first chunk's copies are not issued
};

// Reconstructs the TY x TX tile at (j0, i0) of one slice.  Called by every
// thread of the CTA; threads return from it without waiting for each other,
// so a caller that runs several tiles joins them with __syncthreads().
// MODE 0: reference truncation (bit-exact); MODE 1: linear interpolation.
template <class TL, class RawT, int MODE, bool kCheck, int kVar, bool kWide>
__device__ __forceinline__ void stage_tile(Layout<TL, RawT, MODE> &sm, const CUtensorMap *qmap,
                                           const SliceJob &job, int i0, int j0, int *err) {
  using L = Layout<TL, RawT, MODE>;
  constexpr bool kFold = kVar != 0 && !kCheck && MODE == 0;
  // the wide layout (negative sines) is served for float32 windows, by
  // separate instantiations so that the other kernels carry none of it
  constexpr bool kWideCapable = kWide;
  static_assert(!kWide || (MODE == 0 && std::is_same<RawT, float>::value), "wide: float32 trunc");
  constexpr bool kPackRC = kVar != 0;
  constexpr bool kPackT = kVar == 2;
  constexpr int kProjUnroll = MODE == 0 ? 2 : 1;
  const int W = job.W, N = job.N, hp = W / 2, R = job.R, Cc = job.C;
  const float c = job.c, oj = job.oj, oi = job.oi, pg = job.p;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool producer = (warp == TL::WARPS);
  float *out = job.out;

  // pixels of this thread: rows jb + 4r (r < RY), columns ib + 8b (b < RX)
  const int wy = warp / TL::WX, wx = warp % TL::WX, ly = lane >> 3, lx = lane & 7;
  const int jb = j0 + wy * 4 * TL::RY + ly, ib = i0 + wx * 8 * TL::RX + lx;

  bool mine = false;
  if (!producer) {
#pragma unroll
    for (int r = 0; r < TL::RY; r++)
#pragma unroll
      for (int b = 0; b < TL::RX; b++) {
        const int j = jb + 4 * r, i = ib + 8 * b;
        mine |= (j < R && i < Cc) && ref_mask_f(geo(oj, pg, j), geo(oi, pg, i), W, c);
      }
    const bool wact = __any_sync(0xffffffffu, mine);
    if (lane == 0) sm.active[warp] = wact ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int n = 0;
    for (int w = 0; w < TL::WARPS; w++) n += sm.active[w];
    sm.nactive = n;
    if (n) {
      for (int s = 0; s < kStages; s++) {
        mbar_init(&sm.full[s], 1);
        mbar_init(&sm.empty[s], (uint32_t)n);
        mbar_init(&sm.rawfull[s], 1);
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      sm.barriers_live = 1;
    }
  }
  __syncthreads();
  const bool cta_active = sm.nactive > 0;
  if (!producer && (!cta_active || !sm.active[warp])) {
#pragma unroll
    for (int r = 0; r < TL::RY; r++)
#pragma unroll
      for (int b = 0; b < TL::RX; b++) {
        const int j = jb + 4 * r, i = ib + 8 * b;
        if (j < R && i < Cc) out[(int64_t)j * Cc + i] = 0.f;
      }
    return;
  }
  if (!cta_active) return;

  const int nchunks = (N + kChunk - 1) / kChunk;
  const int row0 = job.row0;
  constexpr int kAlign = 16 / (int)sizeof(RawT);

  if (producer) {
    // ------------------------------------------------------------ producer
    // Parameters and window start of projection n0 + lane of chunk ch, whose
    // window goes to stage st.
    auto make_param = [&](int ch, int st, AngleParam &p, float &tmin) -> int {
      const int n = ch * kChunk + lane;
      int x0 = 0;
      tmin = 0.f;
      if (MODE == 0) {
        const float2 sc = job.tab[n];
        p.sx = sc.x;
        p.cy = sc.y;
        p.base = ref_base(sc.x, sc.y, hp, c, job.rule);
        x0 = window_start_trunc(p.sx, p.cy, p.base, geo(oj, pg, j0), geo(oj, pg, j0 + TL::TY - 1),
                                geo(oi, pg, i0), geo(oi, pg, i0 + TL::TX - 1), c, kAlign, &tmin);
        if (kFold) {
          // off = window word address - x0, |off| < 2^22; M = 2 + off 2^-22 is
          // exact (a multiple of 2^-22 in [1, 4))
          const int off = (int)(smem_u32(&sm.win[st][lane][0]) >> 2) - x0;
          p.sx = __fmul_rn(p.sx, kTwoM22);
          p.cy = __fmul_rn(p.cy, kTwoM22);
          p.base = __fmul_rn(p.base, kTwoM22);
          p.addr = __float_as_uint(__fadd_rn(2.0f, __fmul_rn((float)off, kTwoM22)));
        } else {
          p.addr = smem_u32(&sm.win[st][lane][0]) - 4u * (kMagicBits + (uint32_t)x0);
        }
      } else {
        // u = t - 0.5 = t0 + sin j + cos i with
        // t0 = (hp + c)(1 - sin) - cos hp - 0.5, formed in FP64
        const double2 g = job.lin[n];
        const double hc = (double)hp + (double)c;
        p.sx = (float)g.x;
        p.cy = (float)g.y;
        p.base = (float)(hc * (1.0 - g.x) - g.y * (double)hp - 0.5);
        x0 = window_start_linear(p.sx, p.cy, p.base, geo(oj, pg, j0), geo(oj, pg, j0 + TL::TY - 1),
                                 geo(oi, pg, i0), geo(oi, pg, i0 + TL::TX - 1), kAlign);
        // pairs (q[k], q[k+1] - q[k]) of 8 bytes at window position k - x0
        p.addr = smem_u32(&sm.win[st][lane][0]) - 8u * (kMagicBits + (uint32_t)x0);
      }
      return x0;
    };
    // TMA copy of one projection's window; the alignment rules (128-byte
    // destination, 16-byte start column) are checked first: a violation is
    // reported and the copy skipped, so the stage times out instead of faulting
    auto load_window = [&](void *dst, int x0, int n, unsigned long long *bar) {
      // test aid: leave the first chunk's windows out, so every wait on them
      // runs out (bounded) and the kernel reports a timeout
      if (job.test_stall && n < kChunk) return;
      // (a start left of column 0 is allowed: those samples read as 0)
      if ((smem_u32(dst) & 127u) == 0 && (((x0 + job.off) * (int)sizeof(RawT)) & 15) == 0)
        tma_load_row(dst, qmap, x0 + job.off, row0 + n, bar);
      else
        atomicOr(err, 16);
    };
    int issued = 0;
    bool ok = true;
    if constexpr (!L::kTransform) {
      // float32 windows land where the consumers read them
      for (int ch = 0; ch < nchunks && ok; ch++) {
        const int st = ch % kStages;
        if (ch >= kStages && !mbar_wait(&sm.empty[st], (uint32_t)(((ch / kStages) - 1) & 1), job.wait_limit)) {
          if (lane == 0) atomicOr(err, 4);
          sm.abort_flag = 1;
          ok = false;
          break;
        }
        const int n0 = ch * kChunk, cnt = min(kChunk, N - n0);
        AngleParam p;
        int x0 = 0;
        float tmin = 0.f;
        if (lane < cnt) {
          x0 = make_param(ch, st, p, tmin);
          sm.par[st][lane] = p;
        }
        if constexpr (kWide) {
          // wide layout: projections for which some pixel of the tile may have
          // t < 0 (the corner minimum misses the per-pixel rounding by far
          // less than 1) take the truncating path
          const uint32_t neg = __ballot_sync(0xffffffffu, lane < cnt && tmin < 1.0f);
          if (lane == 0) sm.negmask[st] = neg;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&sm.full[st], (uint32_t)(cnt * TL::BOX * sizeof(RawT)));
        __syncwarp();
        if (lane < cnt) load_window(&sm.win[st][lane][0], x0, n0 + lane, &sm.full[st]);
        issued = ch + 1;
      }
      if (!ok && lane == 0) {
        // drain this CTA's copies still in flight (bounded): only the latest
        // use of each stage can be outstanding
        for (int ch = (issued > kStages ? issued - kStages : 0); ch < issued; ch++)
          mbar_wait(&sm.full[ch % kStages], (uint32_t)((ch / kStages) & 1), job.wait_limit);
      }
      return;
    } else {
      // Raw windows (16-bit store, or the linear pairs) are converted into
      // the float windows by this warp.  Their copies run up to kStages chunks
      // ahead of the conversion: chunk ch + kStages is issued into raw stage
      // st as soon as chunk ch has been converted out of it.  Its parameters
      // wait in parq until the consumers have released win[st].
      auto issue = [&](int ch) {
        const int st = ch % kStages;
        const int n0 = ch * kChunk, cnt = min(kChunk, N - n0);
        AngleParam p;
        int x0 = 0;
        float tmin = 0.f;
        if (lane < cnt) {
          x0 = make_param(ch, st, p, tmin);
          sm.parq[st][lane] = p;
          sm.scale[st][lane] = job.row_scale ? job.row_scale[(int64_t)row0 + n0 + lane] : 1.f;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&sm.rawfull[st], (uint32_t)(cnt * TL::BOX * sizeof(RawT)));
        __syncwarp();
        if (lane < cnt) load_window(&sm.raw[st][lane][0], x0, n0 + lane, &sm.rawfull[st]);
      };
      for (; issued < nchunks && issued < kStages; issued++) issue(issued);
      int converted = 0;  // chunks whose raw copy has been waited for
      for (int ch = 0; ch < nchunks; ch++) {
        const int st = ch % kStages;
        if (!mbar_wait(&sm.rawfull[st], (uint32_t)((ch / kStages) & 1), job.wait_limit)) {
          ok = false;
          break;
        }
        converted = ch + 1;
        if (ch >= kStages && !mbar_wait(&sm.empty[st], (uint32_t)(((ch / kStages) - 1) & 1), job.wait_limit)) {
          ok = false;
          break;
        }
        const int cnt = min(kChunk, N - ch * kChunk);
        // convert the raw windows: scale (reduced-precision store) and, for
        // linear interpolation, (sample, next - sample) pairs
        if constexpr (MODE == 0 && sizeof(RawT) == 2) {
          // 16-byte words: eight samples per lane and step, independent steps
          // unrolled so one warp keeps up with the consumers.  This warp shares
          // issue slots with the consumers, so the fewest instructions win:
          // four samples per lane (conflict-free 16-byte stores) ran 4 % slower
          constexpr int G = TL::BOX / 8;
          static_assert(TL::BOX % 8 == 0, "16-byte groups");
#pragma unroll 4
          for (int e = lane; e < cnt * G; e += 32) {
            const int k = e / G, g = e - k * G;
            const float sc = sm.scale[st][k];
            const uint4 w = *reinterpret_cast<const uint4 *>(&sm.raw[st][k][8 * g]);
            const float2 a = pair_to_f32(w.x, RawT{}), b = pair_to_f32(w.y, RawT{});
            const float2 c2 = pair_to_f32(w.z, RawT{}), d = pair_to_f32(w.w, RawT{});
            float4 *dst = reinterpret_cast<float4 *>(&sm.win[st][k][8 * g]);
            dst[0] = make_float4(a.x * sc, a.y * sc, b.x * sc, b.y * sc);
            dst[1] = make_float4(c2.x * sc, c2.y * sc, d.x * sc, d.y * sc);
          }
        } else {
          for (int e = lane; e < cnt * TL::BOX; e += 32) {
            const int k = e / TL::BOX, m = e - k * TL::BOX;
            const float sc = sm.scale[st][k];
            const float v = raw_to_f32(sm.raw[st][k][m]) * sc;
            if (MODE == 0) {
              sm.win[st][k][m] = v;
            } else {
              const float v1 = (m + 1 < TL::BOX) ? raw_to_f32(sm.raw[st][k][m + 1]) * sc : 0.f;
              sm.win[st][k][2 * m] = v;
              sm.win[st][k][2 * m + 1] = v1 - v;
            }
          }
        }
        if (lane < cnt) sm.par[st][lane] = sm.parq[st][lane];
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.full[st]);
        if (issued < nchunks) issue(issued++);
      }
      if (!ok) {
        if (lane == 0) {
          atomicOr(err, 4);
          // drain the raw copies issued but not yet waited for (bounded)
          for (int ch = converted; ch < issued; ch++)
            mbar_wait(&sm.rawfull[ch % kStages], (uint32_t)((ch / kStages) & 1), job.wait_limit);
        }
        sm.abort_flag = 1;
      }
      return;
    }
  }

  // -------------------------------------------------------------- consumers
  constexpr int RP = TL::RY / 2;  // row pairs
  float2 jcp[RP];                 // truncation: (j - c); linear: (j, j + 4)
#pragma unroll
  for (int p = 0; p < RP; p++) {
    const float jA = geo(oj, pg, jb + 8 * p), jB = geo(oj, pg, jb + 8 * p + 4);
    jcp[p] = MODE == 0 ? make_float2(__fsub_rn(jA, c), __fsub_rn(jB, c)) : make_float2(jA, jB);
  }
  float fib[TL::RX];
#pragma unroll
  for (int b = 0; b < TL::RX; b++) fib[b] = geo(oi, pg, ib + 8 * b);
  constexpr int RP2 = MODE == 1 ? RP : 1, RX2 = MODE == 1 ? TL::RX : 1;
  // truncation: accc[r][bp] holds pixels (row jb + 4r, columns ib + 8 (2bp),
  // ib + 8 (2bp + 1)); linear: acc[q][b] holds (rows jb + 8q, jb + 8q + 4, column b)
  constexpr int RA = MODE == 0 ? 1 : RP, XA = MODE == 0 ? 1 : TL::RX;
  constexpr int RC = MODE == 0 ? TL::RY : 1, XC = MODE == 0 ? TL::RX / 2 : 1;
  float2 acc[RA][XA];
  float2 accc[RC][XC];
  float2 acc2[RP2][RX2];
#pragma unroll
  for (int p = 0; p < RA; p++)
#pragma unroll
    for (int b = 0; b < XA; b++) acc[p][b] = make_float2(0.f, 0.f);
#pragma unroll
  for (int r = 0; r < RC; r++)
#pragma unroll
    for (int b = 0; b < XC; b++) accc[r][b] = make_float2(0.f, 0.f);
#pragma unroll
  for (int p = 0; p < RP2; p++)
#pragma unroll
    for (int b = 0; b < RX2; b++) acc2[p][b] = make_float2(0.f, 0.f);
  const float2 magic2 = make_float2(kMagic, kMagic);
  // low word of the funnel shift: any value below 2^30 the compiler cannot
  // fold away
  const uint32_t lo_bits = threadIdx.x;

  for (int ch = 0; ch < nchunks; ch++) {
    const int st = ch % kStages;
    if (!mbar_wait(&sm.full[st], (uint32_t)((ch / kStages) & 1), job.wait_limit)) {
      if (lane == 0) atomicOr(err, 4);
      sm.abort_flag = 1;
      return;  // the producer sees the missing arrivals and drains
    }
    const int cnt = min(kChunk, N - ch * kChunk);
    const uint32_t nmask = kWideCapable ? sm.negmask[st] : 0u;
    // the next projection's parameters are loaded one iteration ahead so the
    // shared-memory latency overlaps the current gathers; with truncation two
    // projections per iteration let one projection's last gathers and adds
    // overlap the next one's address arithmetic (3 % faster at 64 x 128 tiles
    // than one); linear interpolation keeps one (its registers are full)
    AngleParam pnext = sm.par[st][0];
#pragma unroll(kProjUnroll)
    for (int k = 0; k < cnt; k++) {
      const AngleParam p = pnext;
      pnext = sm.par[st][k + 1 < cnt ? k + 1 : k];
      if constexpr (MODE == 0) {
        // products by scalar __fmul_rn, consumed by scalar __fadd_rn: never
        // contracted, so every rounding is the reference's
        float2 brow[RP];
#pragma unroll
        for (int q = 0; q < RP; q++) {
          if (kPackRC) {
            brow[q] = add2_rn(make_float2(p.base, p.base),
                              mul2z_rn(make_float2(p.sx, p.sx), jcp[q]));
          } else {
            brow[q].x = __fadd_rn(p.base, __fmul_rn(p.sx, jcp[q].x));
            brow[q].y = __fadd_rn(p.base, __fmul_rn(p.sx, jcp[q].y));
          }
        }
        float2 dbp[TL::RX / 2];  // column products of columns (2bp, 2bp + 1)
#pragma unroll
        for (int b = 0; b < TL::RX; b += 2) {
          if (kPackRC) {
            dbp[b / 2] = mul2z_rn(make_float2(p.cy, p.cy), make_float2(fib[b], fib[b + 1]));
          } else {
            dbp[b / 2] = make_float2(__fmul_rn(p.cy, fib[b]), __fmul_rn(p.cy, fib[b + 1]));
          }
        }
        // gathers of all pixels; NEG: the wide layout's projections whose
        // indices may be negative, where the reference truncates toward zero:
        // floor (rounded-down add) for t >= 0, ceiling (rounded-up add) below
        auto pixels = [&](auto negc) {
          constexpr bool NEG = decltype(negc)::value;
#pragma unroll
        for (int bp = 0; bp < TL::RX / 2; bp++) {
          const float2 d = dbp[bp];
#pragma unroll
          for (int r = 0; r < TL::RY; r++) {
            // row r's term, pixels (r, 2bp) and (r, 2bp + 1); (with packed
            // products, d comes from an fma: nothing to contract)
            const float br = (r & 1) ? brow[r >> 1].y : brow[r >> 1].x;
            const float2 t = kPackT ? add2_rn(make_float2(br, br), d)
                                    : make_float2(__fadd_rn(br, d.x), __fadd_rn(br, d.y));
            const float2 mg = kFold ? make_float2(__uint_as_float(p.addr), __uint_as_float(p.addr))
                                    : magic2;
            float2 u = add2_rm(t, mg);
            if constexpr (NEG) {
              const float2 uc = add2_rp(t, mg);
              u = make_float2(t.x < 0.f ? uc.x : u.x, t.y < 0.f ? uc.y : u.y);
            }
            uint32_t a0, a1;
            if (kFold) {
              a0 = shl2_alu(__float_as_uint(u.x), lo_bits);
              a1 = shl2_alu(__float_as_uint(u.y), lo_bits);
            } else {
              a0 = (__float_as_uint(u.x) << 2) + p.addr;
              a1 = (__float_as_uint(u.y) << 2) + p.addr;
            }
            float v0, v1;
            if (kCheck) {
              const uint32_t lo = smem_u32(&sm.win[st][k][0]);
              const bool ok0 = a0 >= lo && a0 < lo + 4 * TL::BOX;
              const bool ok1 = a1 >= lo && a1 < lo + 4 * TL::BOX;
              if (!(ok0 && ok1)) atomicOr(err, 8);
              v0 = ok0 ? lds_f32(a0) : 0.f;
              v1 = ok1 ? lds_f32(a1) : 0.f;
            } else {
              v0 = lds_f32(a0);
              v1 = lds_f32(a1);
            }
            accc[r][bp] = add2_rn(accc[r][bp], make_float2(v0, v1));
          }
        }
        };
        if constexpr (kWideCapable) {
          if ((nmask >> k) & 1u) pixels(std::true_type{});
          else pixels(std::false_type{});
        } else {
          pixels(std::false_type{});
        }
      } else {
        // linear interpolation: u = t0 + s j + c i, k = floor(u), f = u - k
        float2 brow[RP];
#pragma unroll
        for (int q = 0; q < RP; q++)
          brow[q] = make_float2(fmaf(p.sx, jcp[q].x, p.base), fmaf(p.sx, jcp[q].y, p.base));
#pragma unroll
        for (int b = 0; b < TL::RX; b++) {
#pragma unroll
          for (int q = 0; q < RP; q++) {
            const float u0 = fmaf(p.cy, fib[b], brow[q].x), u1 = fmaf(p.cy, fib[b], brow[q].y);
            const float m0 = __fadd_rd(u0, kMagic), m1 = __fadd_rd(u1, kMagic);
            const float f0 = u0 - (m0 - kMagic), f1 = u1 - (m1 - kMagic);
            const uint32_t a0 = (__float_as_uint(m0) << 3) + p.addr;
            const uint32_t a1 = (__float_as_uint(m1) << 3) + p.addr;
            float2 w0, w1;
            if (kCheck) {
              const uint32_t lo = smem_u32(&sm.win[st][k][0]);
              const bool ok0 = a0 >= lo && a0 < lo + 8 * (TL::BOX - 1);
              const bool ok1 = a1 >= lo && a1 < lo + 8 * (TL::BOX - 1);
              if (!(ok0 && ok1)) atomicOr(err, 8);
              w0 = ok0 ? lds_f32x2(a0) : make_float2(0.f, 0.f);
              w1 = ok1 ? lds_f32x2(a1) : make_float2(0.f, 0.f);
            } else {
              w0 = lds_f32x2(a0);
              w1 = lds_f32x2(a1);
            }
            acc[q][b].x += w0.x;
            acc[q][b].y += w1.x;
            acc2[q][b].x = fmaf(f0, w0.y, acc2[q][b].x);
            acc2[q][b].y = fmaf(f1, w1.y, acc2[q][b].y);
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);
  }

#pragma unroll
  for (int q = 0; q < RP; q++)
#pragma unroll
    for (int b = 0; b < TL::RX; b++) {
      const int i = ib + 8 * b;
      const int jA = jb + 8 * q, jB = jA + 4;
      float vA, vB;
      if constexpr (MODE == 0) {
        const float2 cA = accc[2 * q][b / 2], cB = accc[2 * q + 1][b / 2];
        vA = (b & 1) ? cA.y : cA.x;
        vB = (b & 1) ? cB.y : cB.x;
      } else {
        vA = acc[q][b].x + acc2[q][b].x;
        vB = acc[q][b].y + acc2[q][b].y;
      }
      if (i < Cc) {
        const float fi = geo(oi, pg, i);
        if (jA < R)
          out[(int64_t)jA * Cc + i] =
              ref_mask_f(geo(oj, pg, jA), fi, W, c) ? ref_finish(vA, job.rec_cof, N) : 0.f;
        if (jB < R)
          out[(int64_t)jB * Cc + i] =
              ref_mask_f(geo(oj, pg, jB), fi, W, c) ? ref_finish(vB, job.rec_cof, N) : 0.f;
      }
    }
}


template <class TL, class RawT, int MODE>
__device__ __forceinline__ Layout<TL, RawT, MODE> &stage_smem() {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  return *reinterpret_cast<Layout<TL, RawT, MODE> *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
}

// One CTA per tile; slices along blockIdx.z.
template <class TL, class RawT, int MODE, bool kCheck, int kVar, bool kWide>
__global__ void __launch_bounds__(TL::THREADS, TL::MINB)
    bp_stage_kernel(const __grid_constant__ CUtensorMap qmap, BpLaunch a) {
  auto &sm = stage_smem<TL, RawT, MODE>();
  const int sl = blockIdx.z;
  if (threadIdx.x == 0) sm.abort_flag = 0;
  SliceJob job;
  job.W = a.W;
  job.N = a.N;
  job.row0 = a.q_slice_stride ? sl * a.N : 0;
  job.c = a.centers ? a.centers[sl] : a.center;
  job.rec_cof = a.rec_cof;
  job.tab = a.tab;
  job.lin = a.lin;
  job.rule = a.rule;
  job.off = a.off ? a.off : kRowOff;
  job.wide = a.wide;
  job.wait_limit = a.wait_limit ? a.wait_limit : kWaitLimit;
  job.test_stall = a.test_stall;
  job.row_scale = a.row_scale;
  job.out = a.out + sl * a.out_slice_stride;
  job.R = a.out_rows;
  job.C = a.out_cols;
  job.oj = a.geo_oj;
  job.oi = a.geo_oi;
  job.p = a.geo_p;
  stage_tile<TL, RawT, MODE, kCheck, kVar, kWide>(sm, &qmap, job, blockIdx.x * TL::TX,
                                             blockIdx.y * TL::TY, a.err);
}

// Persistent form for uneven batches: a grid of resident CTAs takes
// (sinogram, tile) work items from an atomic counter until none are left.
template <class TL, class RawT, int MODE, bool kCheck, int kVar>
__global__ void __launch_bounds__(TL::THREADS, TL::MINB)
    bp_stage_batch_kernel(const __grid_constant__ CUtensorMap qmap, BatchLaunch b) {
  auto &sm = stage_smem<TL, RawT, MODE>();
  __shared__ int s_item;
  if (threadIdx.x == 0) {
    sm.abort_flag = 0;
    sm.barriers_live = 0;
    sm.nactive = 0;
  }
  for (;;) {
    __syncthreads();  // the previous tile is finished by every thread
    if (threadIdx.x == 0) {
      if (sm.nactive > 0 && sm.barriers_live) {
        for (int s = 0; s < kStages; s++) {
          mbar_inval(&sm.full[s]);
          mbar_inval(&sm.empty[s]);
          mbar_inval(&sm.rawfull[s]);
        }
      }
      sm.barriers_live = 0;
      s_item = sm.abort_flag ? b.n_items : atomicAdd(b.counter, 1);
    }
    __syncthreads();
    const int item = s_item;
    if (item >= b.n_items) break;
    // the sinogram owning this item: last job with item_begin <= item
    int lo = 0, hi = b.n_jobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (b.jobs[mid].item_begin <= item) lo = mid;
      else hi = mid - 1;
    }
    const BatchJob &J = b.jobs[lo];
    SliceJob job;
    job.W = J.W;
    job.N = J.N;
    job.row0 = J.row0;
    job.c = J.c;
    job.rec_cof = J.rec_cof;
    job.tab = J.tab;
    job.lin = nullptr;
    job.rule = J.rule;
    job.off = kRowOff;
    job.wide = 0;
    job.wait_limit = kWaitLimit;
    job.test_stall = 0;
    job.row_scale = nullptr;
    job.out = J.out;
    job.R = J.W;
    job.C = J.W;
    job.oj = 0.f;
    job.oi = 0.f;
    job.p = 1.f;
    const int t = item - J.item_begin;
    stage_tile<TL, RawT, MODE, kCheck, kVar, false>(sm, &qmap, job, (t % J.tiles_x) * TL::TX,
                                               (t / J.tiles_x) * TL::TY, b.err);
  }
}

// ------------------------------------------------------------ tensor maps
using EncodeTiledFn = ctas::EncodeTiledFn;
EncodeTiledFn encode_fn() { return ctas::tensor_map_encoder(); }

template <class TL, class RawT, int MODE>
constexpr size_t smem_bytes() { return sizeof(Layout<TL, RawT, MODE>) + 128; }

template <class TL, class RawT, int MODE, bool kCheck, int kVar, bool kWide = false>
cudaError_t launch_tile(const CUtensorMap &map, const BpLaunch &a, cudaStream_t st) {
  auto kern = bp_stage_kernel<TL, RawT, MODE, kCheck, kVar, kWide>;
  const size_t smem = smem_bytes<TL, RawT, MODE>();
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)  // all of the unified L1/shared array as shared memory
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) {
    std::snprintf(t_detail, sizeof(t_detail), "shared memory attribute (%zu B): %s", smem,
                  cudaGetErrorString(e));
    return e;
  }
  const dim3 grid((a.out_cols + TL::TX - 1) / TL::TX, (a.out_rows + TL::TY - 1) / TL::TY, a.S);
  kern<<<grid, TL::THREADS, smem, st>>>(map, a);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    std::snprintf(t_detail, sizeof(t_detail), "launch of tile %dx%d (%d threads, %zu B): %s",
                  TL::TY, TL::TX, TL::THREADS, smem, cudaGetErrorString(e));
  return e;
}

// Arithmetic variants (kVariants) exist for the truncation kernels (16-bit
// stores gather from the converted float windows too); linear interpolation
// runs variant 0.  The checked form is variant 0 with bounds checks.
template <class TL, class RawT, int MODE>
cudaError_t launch_variant(const CUtensorMap &map, const BpLaunch &a, cudaStream_t st, bool check,
                           int var) {
  if constexpr (MODE == 0 && std::is_same<RawT, float>::value) {
    if (a.wide) {  // wide layout: its own instantiations
      if (check) return launch_tile<TL, RawT, MODE, true, 0, true>(map, a, st);
      switch (var) {
      case 1: return launch_tile<TL, RawT, MODE, false, 1, true>(map, a, st);
      case 2: return launch_tile<TL, RawT, MODE, false, 2, true>(map, a, st);
      default: return launch_tile<TL, RawT, MODE, false, 0, true>(map, a, st);
      }
    }
  }
  if (a.wide) return cudaErrorInvalidValue;  // float32 truncation only
  if (check) return launch_tile<TL, RawT, MODE, true, 0>(map, a, st);
  if (MODE == 0) {  // 16-bit stores: their windows are converted to float first
    switch (var) {
    case 1: return launch_tile<TL, RawT, MODE, false, 1>(map, a, st);
    case 2: return launch_tile<TL, RawT, MODE, false, 2>(map, a, st);
    default: break;
    }
  }
  return launch_tile<TL, RawT, MODE, false, 0>(map, a, st);
}

template <class TL>
cudaError_t launch_for_tile(const CUtensorMap &map, const BpLaunch &a, cudaStream_t st, bool check,
                            int var) {
  if (a.interp == 1) {
    if (a.store == 1) return launch_variant<TL, __half, 1>(map, a, st, check, var);
    if (a.store == 2) return launch_variant<TL, __nv_bfloat16, 1>(map, a, st, check, var);
    return launch_variant<TL, float, 1>(map, a, st, check, var);
  }
  if (a.store == 1) return launch_variant<TL, __half, 0>(map, a, st, check, var);
  if (a.store == 2) return launch_variant<TL, __nv_bfloat16, 0>(map, a, st, check, var);
  return launch_variant<TL, float, 0>(map, a, st, check, var);
}

// tile id = shape (id % kShapes) + kShapes * arithmetic variant
cudaError_t launch_tile_id(int tile, const CUtensorMap &map, const BpLaunch &a, cudaStream_t st,
                           bool check) {
  if (tile < 0 || tile >= kTiles) return cudaErrorInvalidValue;
  const int var = tile / kShapes;
  return with_shape(tile % kShapes, [&](auto tl) {
    return launch_for_tile<decltype(tl)>(map, a, st, check, var);
  });
}

int tile_box(int tile) {
  return with_shape(tile % kShapes, [](auto tl) { return decltype(tl)::BOX; });
}

bool make_map(const BpLaunch &a, int box, CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    std::snprintf(t_detail, sizeof(t_detail), "cuTensorMapEncodeTiled unavailable");
    return false;
  }
  std::memset(map, 0, sizeof(*map));
  const size_t es = a.store == 0 ? 4 : 2;
  const CUtensorMapDataType dt = a.store == 0   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : a.store == 1 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const cuuint64_t rows = (cuuint64_t)a.N * (a.q_slice_stride ? (cuuint64_t)a.S : 1u);
  const cuuint64_t dims[2] = {(cuuint64_t)a.Wp, rows};
  const cuuint64_t strides[1] = {(cuuint64_t)a.Wp * es};
  const cuuint32_t boxd[2] = {(cuuint32_t)box, 1u};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = enc(map, dt, 2, const_cast<void *>(a.q), dims, strides, boxd, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    std::snprintf(t_detail, sizeof(t_detail),
                  "tensor map encode failed (CUresult %d; dims %llu x %llu, stride %llu B, box %d)",
                  (int)r, (unsigned long long)dims[0], (unsigned long long)dims[1],
                  (unsigned long long)strides[0], box);
  return r == CUDA_SUCCESS;
}

// ------------------------------------------------------------ autotuner
// Per (device, W, N, store, interp): the tile that ran fastest on this
// machine.  Candidates are timed on one slice of the caller's own launch, and
// the winner is cached for the process.
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int, int, int, int>, int> g_tuned;

int env_tile() {
  static const int t = [] {
    const char *e = std::getenv("CTAS_FBP_TILE");
    return e ? std::atoi(e) : -1;
  }();
  return t;
}

template <class TL>
cudaError_t launch_batch_shape(const CUtensorMap &map, const BatchLaunch &b, cudaStream_t st,
                               int var, int *grid_out) {
  auto kern = var == 1   ? bp_stage_batch_kernel<TL, float, 0, false, 1>
              : var == 2 ? bp_stage_batch_kernel<TL, float, 0, false, 2>
                         : bp_stage_batch_kernel<TL, float, 0, false, 0>;
  const size_t smem = smem_bytes<TL, float, 0>();
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TL::THREADS, smem);
  if (e != cudaSuccess) return e;
  const int grid = std::max(1, std::min(b.n_items, sms * std::max(1, per_sm)));
  if (grid_out) *grid_out = grid;
  kern<<<grid, TL::THREADS, smem, st>>>(map, b);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    std::snprintf(t_detail, sizeof(t_detail), "batch launch of tile %dx%d: %s", TL::TY, TL::TX,
                  cudaGetErrorString(e));
  return e;
}

}  // namespace

int bp_fast_tile_window(int tile) { return tile_box(tile); }

void bp_fast_tile_shape(int tile, int *ty, int *tx) {
  with_shape(tile % kShapes, [&](auto tl) {
    *ty = decltype(tl)::TY;
    *tx = decltype(tl)::TX;
    return 0;
  });
}

cudaError_t launch_bp_batch(const BatchLaunch &b, int tile, cudaStream_t st) {
  BpLaunch shape{};
  shape.q = b.q;
  shape.store = 0;
  shape.Wp = b.Wp;
  shape.N = b.rows;
  shape.S = 1;
  CUtensorMap map;
  t_detail[0] = 0;
  if (!make_map(shape, tile_box(tile), &map)) return cudaErrorInvalidValue;
  const int var = tile / kShapes;
  return with_shape(tile % kShapes, [&](auto tl) {
    return launch_batch_shape<decltype(tl)>(map, b, st, var, nullptr);
  });
}

bool bp_fast_supported(const BpLaunch &a) {
  return encode_fn() != nullptr && a.Wp >= 192 && (a.Wp % 8) == 0 && a.geo_p > 0.f &&
         a.geo_p <= 1.f &&
         (int64_t)a.N * a.S < (1ll << 31) &&
         (a.q_slice_stride == (int64_t)a.N * a.Wp || a.q_slice_stride == 0);
}

int bp_fast_tile_count() { return kTiles; }

const char *bp_fast_error_detail() { return t_detail; }

static cudaError_t run_tile(int tile, const BpLaunch &a, cudaStream_t st, bool check) {
  CUtensorMap map;
  t_detail[0] = 0;
  if (!make_map(a, tile_box(tile), &map)) return cudaErrorInvalidValue;
  return launch_tile_id(tile, map, a, st, check);
}

int bp_fast_search(const std::function<float(int)> &time_ms, bool all_variants) {
  // each candidate runs three times; the faster of the two warm runs (kernel
  // loaded, attributes set) is the one compared
  auto measure = [&](int t) {
    time_ms(t);
    const float a = time_ms(t), b = time_ms(t);
    return (a < 0.f || b < 0.f) ? -1.f : std::min(a, b);
  };
  constexpr int kLead = kVariants - 1;  // variant tried with every shape
  const int lead = all_variants ? kLead : 0;
  // bring the clocks up before the first comparison
  for (int k = 0; k < 3; k++) time_ms(kShapes * lead + 1);
  int best = -1;
  float best_ms = 1e30f;
  for (int sh = 0; sh < kShapes; sh++) {
    const float ms = measure(sh + kShapes * lead);
    if (ms >= 0.f && ms < best_ms) {
      best_ms = ms;
      best = sh + kShapes * lead;
    }
  }
  if (best < 0) return -1;
  if (all_variants) {
    const int sh = best % kShapes;
    for (int v = 0; v < kVariants; v++) {
      if (v == lead) continue;
      const float ms = measure(sh + kShapes * v);
      if (ms >= 0.f && ms < best_ms) {
        best_ms = ms;
        best = sh + kShapes * v;
      }
    }
  }
  return best;
}

int bp_fast_choose_tile(const BpLaunch &a, cudaStream_t st, int requested) {
  if (requested >= 0 && requested < kTiles) return requested;
  if (env_tile() >= 0 && env_tile() < kTiles) return env_tile();
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, a.W, a.N, a.store, a.interp, a.out_rows, a.out_cols);
  {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) return it->second;
  }
  // time the candidates on a few slices of this launch (their output is
  // overwritten by the real launch that follows): enough for about eight
  // waves of 64 x 128 tiles at three per SM, so that the last partial wave
  // weighs on every candidate as it will on the real launch
  BpLaunch one = a;
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tiles = (int64_t)((a.out_rows + 63) / 64) * ((a.out_cols + 127) / 128);
    const int64_t want = (8ll * 3 * sms + tiles - 1) / std::max<int64_t>(tiles, 1);
    one.S = (int)std::max<int64_t>(1, std::min<int64_t>(a.S, want));
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return 1;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return 1;
  }
  const int best = bp_fast_search(
      [&](int t) {
        cudaEventRecord(e0, st);
        if (run_tile(t, one, st, false) != cudaSuccess) {
          cudaGetLastError();
          return -1.f;
        }
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
      },
      a.interp == 0);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int chosen = best >= 0 ? best : 1;
  std::lock_guard<std::mutex> g(g_tune_mutex);
  g_tuned[key] = chosen;
  return chosen;
}

cudaError_t launch_bp_fast(const BpLaunch &a, cudaStream_t st, int tile) {
  return run_tile(tile, a, st, false);
}

cudaError_t launch_bp_fast_checked(const BpLaunch &a, cudaStream_t st, int tile) {
  return run_tile(tile, a, st, true);
}

}  // namespace ctas
