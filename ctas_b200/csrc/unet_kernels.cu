// unet_kernels.cu -- kernels of the learned sparse-angle stage: a 4-level 2-D
// U-Net (3x3 convolutions, ReLU, 2x2 max pooling, nearest 2x upsampling with
// channel concatenation) in BF16 with FP32 accumulation, forward and
// backward, on the BF16 tensor cores (mma.sync m16n8k16).
//
// Activations are NHWC BF16; a tensor may be a channel slice of a wider
// buffer (channel stride cs, offset co), which makes the skip concatenation
// free: the encoder writes its output straight into the decoder's input.
//
// conv3x3_kernel: implicit GEMM.  A CTA computes an 8 x 16 pixel block for
// 32 * WN output channels; for every chunk of CK input channels it stages the
// 10 x 18 halo block and the chunk's 3x3 weights in shared memory (cp.async,
// double-buffered, zero fill outside the image) and runs the nine taps as
// shifted GEMMs (ldmatrix rows point at the shifted pixels).  Epilogue: bias,
// ReLU, or multiplication by (mask > 0) -- the latter turns the kernel into
// the data-gradient of a ReLU convolution when given the flipped, transposed
// weights.  conv3x3_wgrad_kernel: weight gradient, dW[co][tap][ci] =
// sum_p dY[p][co] X[p + tap][ci], one tap and a 64 x 32 (co, ci) tile per CTA,
// pixel blocks split over the grid, per-warp partial sums reduced in shared
// memory and added to the FP32 gradient with atomics.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "unet_kernels.hpp"

namespace ctas {
namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// 16-byte async copy; src_bytes = 0 fills the destination with zeros
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                        uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                          uint32_t &r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

// D += A (16x16 bf16, row) * B (16x8 bf16, col), FP32 accumulate
__device__ __forceinline__ void mma_bf16(float *d, const uint32_t *a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kBH = 8, kBW = 16;                 // output pixel block
constexpr int kHH = kBH + 2, kHW = kBW + 2;      // halo block
constexpr int kHP = kHH * kHW;                   // halo pixels

template <int CK, int WN> struct ConvSmem {
  static constexpr int RS = CK + 8;              // padded row (bf16): conflict-free ldmatrix
  static constexpr int TN = 32 * WN;
  bf16 halo[2][kHP][RS];
  bf16 wt[2][TN][9][RS];
};

template <int CK, int WN>
__global__ void __launch_bounds__(128 * WN) conv3x3_kernel(ConvArgs a) {
  using S = ConvSmem<CK, WN>;
  constexpr int TN = S::TN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S &sm = *reinterpret_cast<S *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;       // 32 pixels x 32 channels per warp
  const int ntile = a.cout / TN;
  const int b = blockIdx.z / ntile, n0 = (blockIdx.z % ntile) * TN;
  const int h0 = blockIdx.y * kBH, w0 = blockIdx.x * kBW;
  const int H = a.H, W = a.W;
  const int nchunk = a.cin / CK;

  auto load = [&](int c, int buf) {
    const int ci0 = c * CK;
    constexpr int HV = CK / 8;                   // 16-byte vectors per pixel
    for (int e = tid; e < kHP * HV; e += blockDim.x) {
      const int p = e / HV, v = e - p * HV;
      const int hh = h0 - 1 + p / kHW, ww = w0 - 1 + p % kHW;
      const bool in = hh >= 0 && hh < H && ww >= 0 && ww < W;
      const bf16 *src = a.x + (in ? (((int64_t)b * H + hh) * W + ww) * a.x_cs + a.x_co + ci0 + v * 8 : 0);
      cp_async16(&sm.halo[buf][p][v * 8], src, in ? 16 : 0);
    }
    for (int e = tid; e < TN * 9 * HV; e += blockDim.x) {
      const int n = e / (9 * HV), r = e - n * 9 * HV, t = r / HV, v = r - t * HV;
      const bf16 *src = a.w + ((int64_t)(n0 + n) * 9 + t) * a.cin + ci0 + v * 8;
      cp_async16(&sm.wt[buf][n][t][v * 8], src, 16);
    }
    cp_async_commit();
  };

  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < 4; k++) acc[i][j][k] = 0.f;

  load(0, 0);
  for (int c = 0; c < nchunk; c++) {
    const int buf = c & 1;
    if (c + 1 < nchunk) {
      load(c + 1, buf ^ 1);
      cp_async_wait_1();
    } else {
      cp_async_wait_0();
    }
    __syncthreads();
#pragma unroll 1
    for (int t = 0; t < 9; t++) {
      const int dy = t / 3 - 1, dx = t % 3 - 1;
#pragma unroll
      for (int kk = 0; kk < CK / 16; kk++) {
        uint32_t af[2][4];
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int pr = wm * 2 + i, pc = lane & 15;
          const int hp = (pr + 1 + dy) * kHW + (pc + 1 + dx);
          ldsm_x4(smem_addr(&sm.halo[buf][hp][kk * 16 + (lane >> 4) * 8]), af[i][0], af[i][1],
                  af[i][2], af[i][3]);
        }
#pragma unroll
        for (int jp = 0; jp < 2; jp++) {
          const int mi = lane >> 3;
          const int n = wn * 32 + jp * 16 + ((mi >> 1) << 3) + (lane & 7);
          uint32_t b0, b1, b2, b3;
          ldsm_x4(smem_addr(&sm.wt[buf][n][t][kk * 16 + (mi & 1) * 8]), b0, b1, b2, b3);
#pragma unroll
          for (int i = 0; i < 2; i++) {
            mma_bf16(acc[i][jp * 2], af[i], b0, b1);
            mma_bf16(acc[i][jp * 2 + 1], af[i], b2, b3);
          }
        }
      }
    }
    __syncthreads();
  }

  // epilogue: row g (and g + 8) of the m16 tile = pixel column, columns
  // 2 tig, 2 tig + 1 of the n8 tile = output channels
  const int g = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const int hh = h0 + wm * 2 + i;
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int ww = w0 + g + half * 8;
      const int64_t pix = ((int64_t)b * H + hh) * W + ww;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int co = n0 + wn * 32 + j * 8 + tig * 2;
        float v0 = acc[i][j][half * 2], v1 = acc[i][j][half * 2 + 1];
        if (a.bias) {
          v0 += a.bias[co];
          v1 += a.bias[co + 1];
        }
        if (a.relu) {
          v0 = fmaxf(v0, 0.f);
          v1 = fmaxf(v1, 0.f);
        }
        if (a.mask) {
          const __nv_bfloat162 m =
              *reinterpret_cast<const __nv_bfloat162 *>(a.mask + pix * a.m_cs + a.m_co + co);
          if (!(__bfloat162float(m.x) > 0.f)) v0 = 0.f;
          if (!(__bfloat162float(m.y) > 0.f)) v1 = 0.f;
        }
        *reinterpret_cast<__nv_bfloat162 *>(a.y + pix * a.y_cs + a.y_co + co) =
            __floats2bfloat162_rn(v0, v1);
      }
    }
  }
}

// ---------------------------------------------------------------- wgrad
// grid: x = pixel-block splits, y = 9 taps x ceil(cin / 32) chunks, z = cout / 64
struct WgSmem {
  bf16 dy[kBH * kBW][64 + 8];   // 128 pixels x 64 output channels
  bf16 halo[kHP][32 + 8];       // 10 x 18 pixels x 32 input channels
};

__global__ void __launch_bounds__(256) conv3x3_wgrad_kernel(WgradArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WgSmem &sm = *reinterpret_cast<WgSmem *>(smem_raw);
  float *red = reinterpret_cast<float *>(smem_raw);  // reused after the loop
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = blockIdx.y % 9, ci0 = (blockIdx.y / 9) * 32, co0 = blockIdx.z * 64;
  const int dy = t / 3 - 1, dx = t % 3 - 1;
  const int H = a.H, W = a.W;
  const int bx = W / kBW, by = H / kBH;
  const int nblk = a.B * bx * by;
  const int mt = a.cout - co0 >= 64 ? 4 : 2;     // m16 tiles in this co tile
  const int ck = a.cin - ci0 >= 32 ? 32 : 16;    // input channels in this chunk
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < 4; k++) acc[i][j][k] = 0.f;

  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const int b = blk / (bx * by), r = blk - b * bx * by;
    const int h0 = (r / bx) * kBH, w0 = (r % bx) * kBW;
    // dY block: 128 pixels x (16 * mt) channels
    for (int e = tid; e < kBH * kBW * 8; e += blockDim.x) {
      const int p = e >> 3, v = e & 7;
      if (v * 8 < mt * 16) {
        const int64_t pix = ((int64_t)b * H + h0 + p / kBW) * W + w0 + p % kBW;
        cp_async16(&sm.dy[p][v * 8], a.dy + pix * a.dy_cs + a.dy_co + co0 + v * 8, 16);
      }
    }
    for (int e = tid; e < kHP * 4; e += blockDim.x) {
      const int p = e >> 2, v = e & 3;
      const int hh = h0 - 1 + p / kHW, ww = w0 - 1 + p % kHW;
      const bool in = hh >= 0 && hh < H && ww >= 0 && ww < W && v * 8 < ck;
      const bf16 *src = a.x + (in ? (((int64_t)b * H + hh) * W + ww) * a.x_cs + a.x_co + ci0 + v * 8 : 0);
      cp_async16(&sm.halo[p][v * 8], src, in ? 16 : 0);
    }
    cp_async_commit();
    cp_async_wait_0();
    __syncthreads();
    // warp w: pixels of block row w (16 pixels = one k16 step)
    const int mi = lane >> 3;
    uint32_t bfr[2][4];
#pragma unroll
    for (int jp = 0; jp < 2; jp++) {
      // B = X_tap (k = pixel, n = ci): rows are pixels; .trans
      const int k = ((mi & 1) << 3) + (lane & 7);
      const int hp = (warp + 1 + dy) * kHW + (k + 1 + dx);
      ldsm_x4_t(smem_addr(&sm.halo[hp][jp * 16 + ((mi >> 1) << 3)]), bfr[jp][0], bfr[jp][1],
                bfr[jp][2], bfr[jp][3]);
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
      if (m >= mt) break;
      // A = dY^T (m = co, k = pixel): rows are pixels; .trans
      const int k = ((mi >> 1) << 3) + (lane & 7);
      uint32_t af[4];
      ldsm_x4_t(smem_addr(&sm.dy[warp * kBW + k][m * 16 + ((mi & 1) << 3)]), af[0], af[1], af[2],
                af[3]);
#pragma unroll
      for (int jp = 0; jp < 2; jp++) {
        mma_bf16(acc[m][jp * 2], af, bfr[jp][0], bfr[jp][1]);
        mma_bf16(acc[m][jp * 2 + 1], af, bfr[jp][2], bfr[jp][3]);
      }
    }
    __syncthreads();
  }
  // reduce the 8 warps' tiles in shared memory, then add to dW
  const int g = lane >> 2, tig = lane & 3;
  for (int w = 0; w < 8; w++) {
    if (warp == w) {
#pragma unroll
      for (int m = 0; m < 4; m++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int row = m * 16 + g + (q >> 1) * 8, col = j * 8 + tig * 2 + (q & 1);
            float *dst = &red[row * 32 + col];
            *dst = (w == 0 ? 0.f : *dst) + acc[m][j][q];
          }
    }
    __syncthreads();
  }
  for (int e = tid; e < mt * 16 * 32; e += blockDim.x) {
    const int row = e / 32, col = e % 32;
    if (col < ck) atomicAdd(&a.dw[((int64_t)(co0 + row) * 9 + t) * a.cin + ci0 + col], red[e]);
  }
}

// ------------------------------------------------------- elementwise kernels
// db[c] += sum over pixels of dY[p][c]
__global__ void bias_grad_kernel(const bf16 *dy, int cs, int co, int C, int64_t npix, float *db) {
  const int c = threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int64_t p = blockIdx.x; p < npix; p += gridDim.x) s += __bfloat162float(dy[p * cs + co + c]);
  atomicAdd(&db[c], s);
}

// y (B, H/2, W/2, C) = 2x2 max of x (B, H, W, C)
__global__ void maxpool_kernel(PoolArgs a) {
  const int64_t n = (int64_t)a.B * (a.H / 2) * (a.W / 2) * a.C;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % a.C);
    const int64_t q = e / a.C;
    const int wo = (int)(q % (a.W / 2)), ho = (int)((q / (a.W / 2)) % (a.H / 2));
    const int b = (int)(q / ((int64_t)(a.W / 2) * (a.H / 2)));
    float m = -INFINITY;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        const int64_t pix = ((int64_t)b * a.H + 2 * ho + i) * a.W + 2 * wo + j;
        m = fmaxf(m, __bfloat162float(a.x[pix * a.x_cs + a.x_co + c]));
      }
    const int64_t po = ((int64_t)b * (a.H / 2) + ho) * (a.W / 2) + wo;
    a.y[po * a.y_cs + a.y_co + c] = __float2bfloat16_rn(m);
  }
}

// dx (the pooled input's gradient slice) += dy routed to the first maximum,
// then dx *= (x > 0): the ReLU of the convolution that produced x
__global__ void maxpool_bwd_kernel(PoolArgs a, const bf16 *dy, int dy_cs, int dy_co, bf16 *dx,
                                   int dx_cs, int dx_co) {
  const int64_t n = (int64_t)a.B * (a.H / 2) * (a.W / 2) * a.C;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % a.C);
    const int64_t q = e / a.C;
    const int wo = (int)(q % (a.W / 2)), ho = (int)((q / (a.W / 2)) % (a.H / 2));
    const int b = (int)(q / ((int64_t)(a.W / 2) * (a.H / 2)));
    float m = -INFINITY;
    int arg = 0;
    for (int k = 0; k < 4; k++) {
      const int64_t pix = ((int64_t)b * a.H + 2 * ho + (k >> 1)) * a.W + 2 * wo + (k & 1);
      const float v = __bfloat162float(a.x[pix * a.x_cs + a.x_co + c]);
      if (v > m) {
        m = v;
        arg = k;
      }
    }
    const int64_t po = ((int64_t)b * (a.H / 2) + ho) * (a.W / 2) + wo;
    const float g = __bfloat162float(dy[po * dy_cs + dy_co + c]);
    for (int k = 0; k < 4; k++) {
      const int64_t pix = ((int64_t)b * a.H + 2 * ho + (k >> 1)) * a.W + 2 * wo + (k & 1);
      bf16 *d = dx + pix * dx_cs + dx_co + c;
      const float xv = __bfloat162float(a.x[pix * a.x_cs + a.x_co + c]);
      const float v = __bfloat162float(*d) + (k == arg ? g : 0.f);
      *d = __float2bfloat16_rn(xv > 0.f ? v : 0.f);
    }
  }
}

// y (B, 2H, 2W) channel slice = nearest upsampling of x (B, H, W, C)
__global__ void upsample_kernel(PoolArgs a) {
  const int64_t n = (int64_t)a.B * (2 * a.H) * (2 * a.W) * a.C;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % a.C);
    const int64_t q = e / a.C;
    const int wo = (int)(q % (2 * a.W)), ho = (int)((q / (2 * a.W)) % (2 * a.H));
    const int b = (int)(q / ((int64_t)(2 * a.W) * (2 * a.H)));
    const int64_t pin = ((int64_t)b * a.H + ho / 2) * a.W + wo / 2;
    a.y[q * a.y_cs + a.y_co + c] = a.x[pin * a.x_cs + a.x_co + c];
  }
}

// dx (B, H, W, C) = sum of the 2x2 gradient block of dy, times (x > 0)
__global__ void upsample_bwd_kernel(PoolArgs a, const bf16 *dy, int dy_cs, int dy_co, bf16 *dx,
                                    int dx_cs, int dx_co) {
  const int64_t n = (int64_t)a.B * a.H * a.W * a.C;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % a.C);
    const int64_t q = e / a.C;
    const int w = (int)(q % a.W), h = (int)((q / a.W) % a.H);
    const int b = (int)(q / ((int64_t)a.W * a.H));
    float s = 0.f;
    for (int k = 0; k < 4; k++) {
      const int64_t po = ((int64_t)b * 2 * a.H + 2 * h + (k >> 1)) * (2 * a.W) + 2 * w + (k & 1);
      s += __bfloat162float(dy[po * dy_cs + dy_co + c]);
    }
    const float xv = __bfloat162float(a.x[q * a.x_cs + a.x_co + c]);
    dx[q * dx_cs + dx_co + c] = __float2bfloat16_rn(xv > 0.f ? s : 0.f);
  }
}

// network input: BF16 NHWC with `cpad` channels, channel 0 = x * scale
__global__ void input_kernel(const float *x, int64_t npix, float scale, bf16 *y, int cpad) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npix;
       p += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < cpad; c++) y[p * cpad + c] = __float2bfloat16_rn(c == 0 ? x[p] * scale : 0.f);
}

// ---------------------------------------------------------------- 8-channel vector forms
// The same operations as the element kernels above, one 16-byte vector of
// eight BF16 channels per access (channel counts, strides and offsets multiples
// of 8, element counts below 2^31); results are identical.
__device__ __forceinline__ void unpack8(const uint4 &u, float (&f)[8]) {
  const bf16 *h = reinterpret_cast<const bf16 *>(&u);
#pragma unroll
  for (int j = 0; j < 8; j++) f[j] = __bfloat162float(h[j]);
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 u;
  bf16 *h = reinterpret_cast<bf16 *>(&u);
#pragma unroll
  for (int j = 0; j < 8; j++) h[j] = __float2bfloat16_rn(f[j]);
  return u;
}

__device__ __forceinline__ uint4 ld8(const bf16 *p) { return *reinterpret_cast<const uint4 *>(p); }
__device__ __forceinline__ void st8(bf16 *p, const uint4 &v) { *reinterpret_cast<uint4 *>(p) = v; }

__global__ void maxpool8_kernel(PoolArgs a, int n) {
  const int cg = a.C >> 3, Wo = a.W >> 1, Ho = a.H >> 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int c = (e % cg) * 8;
    int q = e / cg;
    const int wo = q % Wo;
    q /= Wo;
    const int ho = q % Ho, b = q / Ho;
    const int64_t p00 = ((int64_t)b * a.H + 2 * ho) * a.W + 2 * wo;
    const bf16 *x = a.x + a.x_co + c;
    float m[8], v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = -INFINITY;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      unpack8(ld8(x + (p00 + (k >> 1) * a.W + (k & 1)) * a.x_cs), v);
#pragma unroll
      for (int j = 0; j < 8; j++) m[j] = fmaxf(m[j], v[j]);
    }
    const int64_t po = ((int64_t)b * Ho + ho) * Wo + wo;
    st8(a.y + po * a.y_cs + a.y_co + c, pack8(m));
  }
}

__global__ void maxpool_bwd8_kernel(PoolArgs a, int n, const bf16 *dy, int dy_cs, int dy_co,
                                    bf16 *dx, int dx_cs, int dx_co) {
  const int cg = a.C >> 3, Wo = a.W >> 1, Ho = a.H >> 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int c = (e % cg) * 8;
    int q = e / cg;
    const int wo = q % Wo;
    q /= Wo;
    const int ho = q % Ho, b = q / Ho;
    const int64_t p00 = ((int64_t)b * a.H + 2 * ho) * a.W + 2 * wo;
    float xv[4][8], m[8];
    int arg[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      m[j] = -INFINITY;
      arg[j] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      unpack8(ld8(a.x + (p00 + (k >> 1) * a.W + (k & 1)) * a.x_cs + a.x_co + c), xv[k]);
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (xv[k][j] > m[j]) {
          m[j] = xv[k][j];
          arg[j] = k;
        }
    }
    const int64_t po = ((int64_t)b * Ho + ho) * Wo + wo;
    float g[8], d[8];
    unpack8(ld8(dy + po * dy_cs + dy_co + c), g);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      bf16 *dp = dx + (p00 + (k >> 1) * a.W + (k & 1)) * dx_cs + dx_co + c;
      unpack8(ld8(dp), d);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const float v = d[j] + (k == arg[j] ? g[j] : 0.f);
        d[j] = xv[k][j] > 0.f ? v : 0.f;
      }
      st8(dp, pack8(d));
    }
  }
}

// thread per input vector: four output pixels
__global__ void upsample8_kernel(PoolArgs a, int n) {
  const int cg = a.C >> 3;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int c = (e % cg) * 8;
    int q = e / cg;
    const int w = q % a.W;
    q /= a.W;
    const int h = q % a.H, b = q / a.H;
    const uint4 v = ld8(a.x + (((int64_t)b * a.H + h) * a.W + w) * a.x_cs + a.x_co + c);
    const int64_t o00 = ((int64_t)b * 2 * a.H + 2 * h) * (2 * a.W) + 2 * w;
    bf16 *y = a.y + a.y_co + c;
#pragma unroll
    for (int k = 0; k < 4; k++) st8(y + (o00 + (k >> 1) * 2 * a.W + (k & 1)) * a.y_cs, v);
  }
}

__global__ void upsample_bwd8_kernel(PoolArgs a, int n, const bf16 *dy, int dy_cs, int dy_co,
                                     bf16 *dx, int dx_cs, int dx_co) {
  const int cg = a.C >> 3;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int c = (e % cg) * 8;
    int q = e / cg;
    const int w = q % a.W;
    q /= a.W;
    const int h = q % a.H, b = q / a.H;
    const int64_t o00 = ((int64_t)b * 2 * a.H + 2 * h) * (2 * a.W) + 2 * w;
    float s[8], v[8], xv[8];
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      unpack8(ld8(dy + (o00 + (k >> 1) * 2 * a.W + (k & 1)) * dy_cs + dy_co + c), v);
#pragma unroll
      for (int j = 0; j < 8; j++) s[j] += v[j];
    }
    const int64_t pin = ((int64_t)b * a.H + h) * a.W + w;
    unpack8(ld8(a.x + pin * a.x_cs + a.x_co + c), xv);
#pragma unroll
    for (int j = 0; j < 8; j++) s[j] = xv[j] > 0.f ? s[j] : 0.f;
    st8(dx + pin * dx_cs + dx_co + c, pack8(s));
  }
}

__global__ void input8_kernel(const float *x, int n, float scale, bf16 *y, int cpad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    float f[8] = {x[p] * scale, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    bf16 *o = y + (int64_t)p * cpad;
    st8(o, pack8(f));
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    for (int c = 8; c < cpad; c += 8) st8(o + c, z);
  }
}

__global__ void head8_kernel(HeadArgs a, int n) {
  __shared__ float sw[256];
  for (int c = threadIdx.x; c < a.C; c += blockDim.x) sw[c] = a.w[c];
  __syncthreads();
  const float b0 = a.b[0];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    float s = b0, f[8];
    const bf16 *fp = a.feat + (int64_t)p * a.C;
    for (int c = 0; c < a.C; c += 8) {
      unpack8(ld8(fp + c), f);
#pragma unroll
      for (int j = 0; j < 8; j++) s = fmaf(sw[c + j], f[j], s);
    }
    a.out[p] = fmaf(a.x[p], a.scale, s) * a.out_scale;
  }
}

// out = (x * scale + sum_c w[c] feat[p][c] + b) * out_scale
__global__ void head_kernel(HeadArgs a) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.npix;
       p += (int64_t)gridDim.x * blockDim.x) {
    float s = a.b[0];
    for (int c = 0; c < a.C; c++) s = fmaf(a.w[c], __bfloat162float(a.feat[p * a.C + c]), s);
    a.out[p] = fmaf(a.x[p], a.scale, s) * a.out_scale;
  }
}

// loss partials: sum of (out - target*scale)^2; dout = 2 (out - t) / n;
// dfeat[p][c] = dout w[c] (feat > 0); dw[c] += dout feat[p][c]; db += dout
__global__ void head_bwd_kernel(HeadArgs a, const float *target, double *loss, float *dw,
                                float *db, bf16 *dfeat) {
  __shared__ float sw[64];
  __shared__ double sl[8];
  __shared__ float sdb[8];
  __shared__ float sdw[64];
  if (threadIdx.x < 64) {
    sw[threadIdx.x] = threadIdx.x < a.C ? a.w[threadIdx.x] : 0.f;
    sdw[threadIdx.x] = 0.f;
  }
  __syncthreads();
  double l = 0.0;
  float lb = 0.f;
  float lw[32];
  for (int c = 0; c < 32; c++) lw[c] = 0.f;
  const float inv = 2.0f / (float)a.npix;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.npix;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float d = a.out[p] - target[p] * a.scale;
    l += (double)d * d;
    const float g = d * inv;
    lb += g;
    for (int c = 0; c < a.C; c++) {
      const float f = __bfloat162float(a.feat[p * a.C + c]);
      if (c < 32) lw[c] = fmaf(g, f, lw[c]);
      dfeat[p * a.C + c] = __float2bfloat16_rn(f > 0.f ? g * sw[c] : 0.f);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    l += __shfl_down_sync(0xffffffffu, l, o);
    lb += __shfl_down_sync(0xffffffffu, lb, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sl[warp] = l;
    sdb[warp] = lb;
  }
  for (int c = 0; c < a.C && c < 32; c++) {
    float v = lw[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(&sdw[c], v);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    float sb = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      s += sl[w];
      sb += sdb[w];
    }
    atomicAdd(loss, s);
    atomicAdd(db, sb);
  }
  if (threadIdx.x < a.C && threadIdx.x < 32) atomicAdd(&dw[threadIdx.x], sdw[threadIdx.x]);
}

// Adam (bias-corrected), FP32 master weights; optional BF16 copy of w
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, int64_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2, bf16 *wb) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

// wt[ci][t'][co] = w[co][t][ci], t' = 8 - t: the weights of the data gradient
__global__ void flip_weights_kernel(const bf16 *w, int cout, int cin, bf16 *wt) {
  const int64_t n = (int64_t)cout * 9 * cin;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int ci = (int)(e % cin);
    const int t = (int)((e / cin) % 9);
    const int co = (int)(e / ((int64_t)cin * 9));
    wt[((int64_t)ci * 9 + (8 - t)) * cout + co] = w[e];
  }
}

__global__ void to_bf16_kernel(const float *x, bf16 *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

bool vec_ok(const PoolArgs &a) {
  return a.C % 8 == 0 && a.x_cs % 8 == 0 && a.x_co % 8 == 0 && a.y_cs % 8 == 0 && a.y_co % 8 == 0;
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g < 1 ? 1 : g);
}

template <int CK, int WN> cudaError_t conv_launch(const ConvArgs &a, cudaStream_t st) {
  const size_t smem = sizeof(ConvSmem<CK, WN>);
  cudaError_t e = cudaFuncSetAttribute(conv3x3_kernel<CK, WN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid(a.W / kBW, a.H / kBH, a.B * (a.cout / (32 * WN)));
  conv3x3_kernel<CK, WN><<<grid, 128 * WN, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

bool conv_shape_ok(const ConvArgs &a) {
  return a.B >= 1 && a.H >= kBH && a.W >= kBW && a.H % kBH == 0 && a.W % kBW == 0 &&
         a.cout % 32 == 0 && a.cout >= 32 && (a.cin % 32 == 0 || a.cin == 16) && a.cin >= 16 &&
         a.x_cs % 8 == 0 && a.x_co % 8 == 0 && a.y_cs % 2 == 0 && a.y_co % 2 == 0 &&
         (!a.mask || (a.m_cs % 2 == 0 && a.m_co % 2 == 0 && a.m_co + a.cout <= a.m_cs)) &&
         a.x_co + a.cin <= a.x_cs &&
         a.y_co + a.cout <= a.y_cs;
}

cudaError_t launch_conv3x3(const ConvArgs &a, cudaStream_t st) {
  if (conv_tc_ok(a)) return launch_conv3x3_tc(a, st);
  return launch_conv3x3_mma(a, st);
}

cudaError_t launch_conv3x3_mma(const ConvArgs &a, cudaStream_t st) {
  if (!conv_shape_ok(a)) return cudaErrorInvalidValue;
  const bool wide = a.cout % 64 == 0;
  if (a.cin == 16) return wide ? conv_launch<16, 2>(a, st) : conv_launch<16, 1>(a, st);
  return wide ? conv_launch<32, 2>(a, st) : conv_launch<32, 1>(a, st);
}

cudaError_t launch_conv3x3_wgrad(const WgradArgs &a, cudaStream_t st) {
  if (wgrad_tc_ok(a)) return launch_conv3x3_wgrad_tc(a, st);
  if (a.B < 1 || a.H < kBH || a.W < kBW || a.H % kBH || a.W % kBW ||
      (a.cin % 32 && a.cin != 16) || a.cout % 32 || a.x_cs % 8 || a.x_co % 8 || a.dy_cs % 8 ||
      a.dy_co % 8 || a.x_co + a.cin > a.x_cs || a.dy_co + a.cout > a.dy_cs)
    return cudaErrorInvalidValue;
  const size_t smem = sizeof(WgSmem) > 64 * 32 * 4 ? sizeof(WgSmem) : 64 * 32 * 4;
  cudaError_t e = cudaFuncSetAttribute(conv3x3_wgrad_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t nblk = (int64_t)a.B * (a.H / kBH) * (a.W / kBW);
  const int ygrid = 9 * ((a.cin + 31) / 32), zgrid = (a.cout + 63) / 64;
  int64_t xs = (148 * 4 + ygrid * zgrid - 1) / (ygrid * zgrid);
  if (xs > nblk) xs = nblk;
  if (xs < 1) xs = 1;
  conv3x3_wgrad_kernel<<<dim3((unsigned)xs, ygrid, zgrid), 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bias_grad(const __nv_bfloat16 *dy, int cs, int co, int C, int64_t npix, float *db,
                             cudaStream_t st) {
  int64_t g = npix < 2048 ? npix : 2048;
  if (g < 1) g = 1;
  bias_grad_kernel<<<(unsigned)g, 64 * ((C + 63) / 64), 0, st>>>(dy, cs, co, C, npix, db);
  return cudaGetLastError();
}

cudaError_t launch_maxpool(const PoolArgs &a, cudaStream_t st) {
  const int64_t n8 = (int64_t)a.B * (a.H / 2) * (a.W / 2) * (a.C / 8);
  if (vec_ok(a) && n8 < INT32_MAX)
    maxpool8_kernel<<<grid_for(n8, 256), 256, 0, st>>>(a, (int)n8);
  else
    maxpool_kernel<<<grid_for((int64_t)a.B * a.H * a.W * a.C / 4, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_maxpool_bwd(const PoolArgs &a, const __nv_bfloat16 *dy, int dy_cs, int dy_co,
                               __nv_bfloat16 *dx, int dx_cs, int dx_co, cudaStream_t st) {
  const int64_t n8 = (int64_t)a.B * (a.H / 2) * (a.W / 2) * (a.C / 8);
  if (vec_ok(a) && dy_cs % 8 == 0 && dy_co % 8 == 0 && dx_cs % 8 == 0 && dx_co % 8 == 0 &&
      n8 < INT32_MAX)
    maxpool_bwd8_kernel<<<grid_for(n8, 256), 256, 0, st>>>(a, (int)n8, dy, dy_cs, dy_co, dx, dx_cs,
                                                           dx_co);
  else
    maxpool_bwd_kernel<<<grid_for((int64_t)a.B * a.H * a.W * a.C / 4, 256), 256, 0, st>>>(
        a, dy, dy_cs, dy_co, dx, dx_cs, dx_co);
  return cudaGetLastError();
}

cudaError_t launch_upsample(const PoolArgs &a, cudaStream_t st) {
  const int64_t n8 = (int64_t)a.B * a.H * a.W * (a.C / 8);
  if (vec_ok(a) && n8 < INT32_MAX)
    upsample8_kernel<<<grid_for(n8, 256), 256, 0, st>>>(a, (int)n8);
  else
    upsample_kernel<<<grid_for((int64_t)a.B * a.H * a.W * a.C * 4, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_upsample_bwd(const PoolArgs &a, const __nv_bfloat16 *dy, int dy_cs, int dy_co,
                                __nv_bfloat16 *dx, int dx_cs, int dx_co, cudaStream_t st) {
  const int64_t n8 = (int64_t)a.B * a.H * a.W * (a.C / 8);
  if (vec_ok(a) && dy_cs % 8 == 0 && dy_co % 8 == 0 && dx_cs % 8 == 0 && dx_co % 8 == 0 &&
      n8 < INT32_MAX)
    upsample_bwd8_kernel<<<grid_for(n8, 256), 256, 0, st>>>(a, (int)n8, dy, dy_cs, dy_co, dx,
                                                            dx_cs, dx_co);
  else
    upsample_bwd_kernel<<<grid_for((int64_t)a.B * a.H * a.W * a.C, 256), 256, 0, st>>>(
        a, dy, dy_cs, dy_co, dx, dx_cs, dx_co);
  return cudaGetLastError();
}

cudaError_t launch_unet_input(const float *x, int64_t npix, float scale, __nv_bfloat16 *y, int cpad,
                              cudaStream_t st) {
  if (cpad % 8 == 0 && npix < INT32_MAX)
    input8_kernel<<<grid_for(npix, 256), 256, 0, st>>>(x, (int)npix, scale, y, cpad);
  else
    input_kernel<<<grid_for(npix, 256), 256, 0, st>>>(x, npix, scale, y, cpad);
  return cudaGetLastError();
}

cudaError_t launch_head(const HeadArgs &a, cudaStream_t st) {
  if (a.C % 8 == 0 && a.C <= 256 && a.npix < INT32_MAX)
    head8_kernel<<<grid_for(a.npix, 256), 256, 0, st>>>(a, (int)a.npix);
  else
    head_kernel<<<grid_for(a.npix, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_head_bwd(const HeadArgs &a, const float *target, double *loss, float *dw,
                            float *db, __nv_bfloat16 *dfeat, cudaStream_t st) {
  if (a.C > 32) return cudaErrorInvalidValue;
  const int g = grid_for(a.npix, 256);
  head_bwd_kernel<<<g > 1184 ? 1184 : g, 256, 0, st>>>(a, target, loss, dw, db, dfeat);
  return cudaGetLastError();
}

cudaError_t launch_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float b1,
                        float b2, float eps, int step, __nv_bfloat16 *wb, cudaStream_t st) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<grid_for(n, 256), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, wb);
  return cudaGetLastError();
}

cudaError_t launch_flip_weights(const __nv_bfloat16 *w, int cout, int cin, __nv_bfloat16 *wt,
                                cudaStream_t st) {
  flip_weights_kernel<<<grid_for((int64_t)cout * 9 * cin, 256), 256, 0, st>>>(w, cout, cin, wt);
  return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float *x, __nv_bfloat16 *y, int64_t n, cudaStream_t st) {
  to_bf16_kernel<<<grid_for(n, 256), 256, 0, st>>>(x, y, n);
  return cudaGetLastError();
}

}  // namespace ctas
