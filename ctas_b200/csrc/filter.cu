// filter.cu -- batched shared-memory FFT row filter for sm_100a.
//
// Replaces the host FFTW loop of CTrec::prepare_sino / filter_line
// (ctas src/common/lct.cpp:569-597, 280-291):
//   y = HC2R( R2HC(z) * G ) / P,   z = row zero-padded to P,
// where z[zs + c] = x[r][c] (c < W), z[zs + W] = x[r+1][0] (the reference's
// inclusive blitz Range copies one sample of the next row, lct.cpp:580,584)
// and the write-back keeps y[zs .. zs+W-1] (lct.cpp:586).
//
// Design: two rows share one complex FFT of length P (row a in the real part,
// row b in the imaginary part).  G is real and even, so the product with the
// spectrum keeps the two rows separate and the inverse transform returns
// (a (*) g) + i (b (*) g).  The forward transform is decimation in frequency
// (its output is in digit-reversed order), the window is applied in that
// order (the host permutes it), and the inverse runs the stages backwards, so
// no bit-reversal pass exists.  Radix-8 stages, one CTA per row pair, the
// whole padded row pair in shared memory; one HBM read of the input rows and
// one HBM write of the filtered rows.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fbp_kernels.hpp"

namespace ctas {
namespace {

constexpr int kFftThreads = 256;

__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// multiply by DIR*i
template <int DIR> __device__ __forceinline__ float2 mul_i(float2 a) {
  return DIR > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// Twiddles w^q, q = 1 .. R-1, of butterfly m of a stage from its table entry
// (w, w^4) (fbp_host.cpp, fft_twiddles_into: one 16-byte entry per butterfly
// index, consecutive for consecutive m); w^2, w^3 and w^5..w^7 are at most two
// complex products deep, a few ulps.
template <int R>
__device__ __forceinline__ void twiddles(const float4 *__restrict__ tws, int m, float2 *w) {
  const float4 e = __ldg(&tws[m]);
  w[1] = make_float2(e.x, e.y);
  if (R >= 4) {
    w[2] = cmul(w[1], w[1]);
    w[3] = cmul(w[2], w[1]);
  }
  if (R == 8) {
    w[4] = make_float2(e.z, e.w);
    w[5] = cmul(w[4], w[1]);
    w[6] = cmul(w[4], w[2]);
    w[7] = cmul(w[4], w[3]);
  }
}

// Shared-memory index with one pad slot per 16 entries.  Per half-warp of
// 8-byte accesses (strides P / 8, 64 and 8, and eight consecutive elements per
// thread in the middle stage) this costs 1.2-1.25 wavefronts per ideal one over
// all stages, against 1.5-2.0 with one slot per 32; the filter ran 2 % faster
// at P = 4096 and 12 % faster at P = 8192.  XOR-ing the low four bits with bits
// 3-6 (no padding, 1.0-1.2 wavefronts) needed one more register and ran slower
// at P = 4096.
__device__ __forceinline__ int sidx(int p) { return p + (p >> 4); }

template <int DIR> __device__ __forceinline__ void dft2(float2 *x) {
  const float2 a = x[0];
  x[0] = a + x[1];
  x[1] = a - x[1];
}
template <int DIR> __device__ __forceinline__ void dft4(float2 *x) {
  const float2 a0 = x[0] + x[2], a1 = x[0] - x[2];
  const float2 b0 = x[1] + x[3], b1 = mul_i<DIR>(x[1] - x[3]);
  x[0] = a0 + b0;
  x[2] = a0 - b0;
  x[1] = a1 + b1;
  x[3] = a1 - b1;
}
template <int DIR> __device__ __forceinline__ void dft8(float2 *x) {
  float2 e[4] = {x[0], x[2], x[4], x[6]};
  float2 o[4] = {x[1], x[3], x[5], x[7]};
  dft4<DIR>(e);
  dft4<DIR>(o);
  const float r = 0.70710678118654752440f;
  // o1 * (1 + DIR i)/sqrt2, o2 * DIR i, o3 * (-1 + DIR i)/sqrt2
  const float2 w1 = make_float2((o[1].x - DIR * o[1].y) * r, (o[1].y + DIR * o[1].x) * r);
  const float2 w2 = mul_i<DIR>(o[2]);
  const float2 w3 = make_float2((-o[3].x - DIR * o[3].y) * r, (-o[3].y + DIR * o[3].x) * r);
  x[0] = e[0] + o[0];
  x[4] = e[0] - o[0];
  x[1] = e[1] + w1;
  x[5] = e[1] - w1;
  x[2] = e[2] + w2;
  x[6] = e[2] - w2;
  x[3] = e[3] + w3;
  x[7] = e[3] - w3;
}
template <int R, int DIR> __device__ __forceinline__ void dft(float2 *x) {
  if (R == 2) dft2<DIR>(x);
  if (R == 4) dft4<DIR>(x);
  if (R == 8) dft8<DIR>(x);
}

// Forward (decimation in frequency) stage of radix R, stride h, block R*h.
template <int R>
__device__ void dif_stage(float2 *s, int P, int h, const float4 *__restrict__ tws) {
  // h is a power of two: block index b / h by a shift
  const int L = R * h, nb = P / R, lgh = __ffs(h) - 1;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int m = b & (h - 1), base = (b >> lgh) * L + m;
    float2 x[R];
#pragma unroll
    for (int t = 0; t < R; t++) x[t] = s[sidx(base + t * h)];
    dft<R, -1>(x);
    if (h > 1) {
      float2 w[R];
      twiddles<R>(tws, m, w);
#pragma unroll
      for (int q = 1; q < R; q++) x[q] = cmul(x[q], w[q]);
    }
#pragma unroll
    for (int q = 0; q < R; q++) s[sidx(base + q * h)] = x[q];
  }
}

// Exact inverse of dif_stage (times R).
template <int R>
__device__ void dit_stage(float2 *s, int P, int h, const float4 *__restrict__ tws) {
  // h is a power of two: block index b / h by a shift
  const int L = R * h, nb = P / R, lgh = __ffs(h) - 1;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int m = b & (h - 1), base = (b >> lgh) * L + m;
    float2 x[R];
#pragma unroll
    for (int q = 0; q < R; q++) x[q] = s[sidx(base + q * h)];
    if (h > 1) {
      float2 w[R];
      twiddles<R>(tws, m, w);
#pragma unroll
      for (int q = 1; q < R; q++) x[q] = cmulc(x[q], w[q]);
    }
    dft<R, +1>(x);
#pragma unroll
    for (int t = 0; t < R; t++) s[sidx(base + t * h)] = x[t];
  }
}

// Last forward stage (h == 1), window, first inverse stage, in registers.
template <int R>
__device__ void middle_stage(float2 *s, int P, const float *__restrict__ gperm) {
  const int nb = P / R;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int base = b * R;
    float2 x[R];
#pragma unroll
    for (int t = 0; t < R; t++) x[t] = s[sidx(base + t)];
    dft<R, -1>(x);
    float g[R];
    if (R >= 4) {
#pragma unroll
      for (int v = 0; v < R / 4; v++) {
        const float4 g4 = __ldg(reinterpret_cast<const float4 *>(gperm + base) + v);
        g[4 * v] = g4.x;
        g[4 * v + 1] = g4.y;
        g[4 * v + 2] = g4.z;
        g[4 * v + 3] = g4.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < R; q++) g[q] = __ldg(&gperm[base + q]);
    }
#pragma unroll
    for (int q = 0; q < R; q++) {
      x[q].x *= g[q];
      x[q].y *= g[q];
    }
    dft<R, +1>(x);
#pragma unroll
    for (int t = 0; t < R; t++) s[sidx(base + t)] = x[t];
  }
}

// First forward stage (one block of length P, stride h = P / R) with its
// inputs produced by `ld(position)` -- read straight from global memory, so
// each thread has R independent loads in flight.
template <int R, class Loader>
__device__ __forceinline__ void dif_first_stage(float2 *s, int h, const float4 *__restrict__ tws,
                                                Loader ld) {
  for (int b = threadIdx.x; b < h; b += blockDim.x) {
    float2 x[R];
#pragma unroll
    for (int t = 0; t < R; t++) x[t] = ld(b + t * h);
    dft<R, -1>(x);
    float2 w[R];
    twiddles<R>(tws, b, w);
#pragma unroll
    for (int q = 1; q < R; q++) x[q] = cmul(x[q], w[q]);
#pragma unroll
    for (int q = 0; q < R; q++) s[sidx(b + q * h)] = x[q];
  }
}

// Last inverse stage with its outputs handed to `wr(position, value)`.
template <int R, class Writer>
__device__ __forceinline__ void dit_last_stage(const float2 *s, int h, const float4 *__restrict__ tws,
                                               Writer wr) {
  for (int b = threadIdx.x; b < h; b += blockDim.x) {
    float2 x[R];
#pragma unroll
    for (int q = 0; q < R; q++) x[q] = s[sidx(b + q * h)];
    float2 w[R];
    twiddles<R>(tws, b, w);
#pragma unroll
    for (int q = 1; q < R; q++) x[q] = cmulc(x[q], w[q]);
    dft<R, +1>(x);
#pragma unroll
    for (int t = 0; t < R; t++) wr(b + t * h, x[t]);
  }
}

template <bool FWD>
__device__ __forceinline__ void run_stage(float2 *s, int P, int R, int h, const float4 *tw) {
  if (FWD) {
    if (R == 8) dif_stage<8>(s, P, h, tw);
    else if (R == 4) dif_stage<4>(s, P, h, tw);
    else dif_stage<2>(s, P, h, tw);
  } else {
    if (R == 8) dit_stage<8>(s, P, h, tw);
    else if (R == 4) dit_stage<4>(s, P, h, tw);
    else dit_stage<2>(s, P, h, tw);
  }
}

// deAbs of one sample (physical.world.cpp:88-100): clamp when the sinogram
// minimum is <= 0, then -log.
__device__ __forceinline__ float deabs(float v, float2 mm) {
  if (mm.x <= 0.0f) {
    const float mina = (float)((double)mm.y / 1000000.0);
    if (v <= mina) v = mina;
  }
  return -logf(v);
}

template <typename T> __device__ __forceinline__ T to_store(float v);
template <> __device__ __forceinline__ float to_store<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_store<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Power-of-two scale s with max|v|/s <= 1 (1 for an all-zero row).
__device__ __forceinline__ float pow2_scale(float mx) {
  if (!(mx > 0.0f) || !isfinite(mx)) return 1.0f;
  int e;
  frexpf(mx, &e);          // mx = f * 2^e, f in [0.5, 1)
  return ldexpf(1.0f, e);  // mx / 2^e < 1
}

// Filters rows 2*pair and 2*pair+1 of slice sl.  Called by every thread of
// the CTA with the CTA's dynamic shared memory (P + P/32 float2).
template <typename T>
__device__ __forceinline__ void filter_pair(const FilterLaunch &a, int pair, int sl) {
  extern __shared__ float2 sm[];
  __shared__ float red[2][kFftThreads / 32];
  const int N = a.N, W = a.W, P = a.P, zs = a.zs;
  const int r0 = 2 * pair, r1 = r0 + 1;
  const bool has1 = r1 < N;
  const float *x0 = a.x + sl * a.x_slice_stride + (int64_t)r0 * W;
  const float *x1 = x0 + W;
  const bool abs_mode = (a.contrast == 0);
  // no min/max: plain -log (no deAbs clamp)
  const float2 mm = (abs_mode && a.minmax) ? a.minmax[sl] : make_float2(1.f, 1.f);
  const float *ring = a.ring ? a.ring + (int64_t)sl * W : nullptr;
  // quirk samples: first sample of the row after r0 and after r1
  float qa = 0.f, qb = 0.f;
  if (has1) qa = ring ? __fadd_rn(x1[0], ring[0]) : x1[0];
  if (r1 + 1 < N) qb = ring ? __fadd_rn(x1[W], ring[0]) : x1[W];
  if (abs_mode) {
    if (has1) qa = deabs(qa, mm);
    if (r1 + 1 < N) qb = deabs(qb, mm);
  }

  // element p of the zero-padded row pair
  auto load = [&](int p) -> float2 {
    int c = p - zs;
    if (a.periodic) c = p < 2 * W ? (c + W) % W : -1;
    float2 v = make_float2(0.f, 0.f);
    if (c >= 0 && c < W) {
      v.x = x0[c];
      v.y = has1 ? x1[c] : 0.f;
      if (ring) {
        v.x = __fadd_rn(v.x, ring[c]);
        if (has1) v.y = __fadd_rn(v.y, ring[c]);
      }
      if (abs_mode) {
        v.x = deabs(v.x, mm);
        if (has1) v.y = deabs(v.y, mm);
      }
    } else if (c == W && !a.periodic) {
      v = make_float2(qa, qb);
    }
    return v;
  };

  const int ns = a.nradix;
  int hs[8];
  // twiddle table of stage st: tws + to[st] (h entries; fbp_host.cpp)
  int to[8];
  const float4 *tws = reinterpret_cast<const float4 *>(a.tw);
  {
    int h = P, o = 0;
    for (int st = 0; st < ns; st++) {
      h /= a.radix[st];
      hs[st] = h;
      to[st] = o;
      o += h;
    }
  }
  // rows go straight from the last inverse stage to global memory unless a
  // row-wide epilogue (REF running sum, reduced-precision scale) needs them
  const bool direct = ns >= 2 && a.contrast != 1 && a.store == 0;
  T *q0 = reinterpret_cast<T *>(a.q) + sl * a.q_slice_stride + (int64_t)r0 * a.Wp +
          (a.off ? a.off : kRowOff);
  T *q1 = q0 + a.Wp;

  if (ns >= 2) {
    const int R = a.radix[0];
    if (R == 8) dif_first_stage<8>(sm, hs[0], tws, load);
    else if (R == 4) dif_first_stage<4>(sm, hs[0], tws, load);
    else dif_first_stage<2>(sm, hs[0], tws, load);
  } else {
    for (int p = threadIdx.x; p < P; p += blockDim.x) sm[sidx(p)] = load(p);
  }
  __syncthreads();
  for (int st = (ns >= 2 ? 1 : 0); st < ns - 1; st++) {
    run_stage<true>(sm, P, a.radix[st], hs[st], tws + to[st]);
    __syncthreads();
  }
  {
    const int R = a.radix[ns - 1];
    if (R == 8) middle_stage<8>(sm, P, a.gperm);
    else if (R == 4) middle_stage<4>(sm, P, a.gperm);
    else middle_stage<2>(sm, P, a.gperm);
  }
  __syncthreads();
  for (int st = ns - 2; st >= (direct ? 1 : 0); st--) {
    run_stage<false>(sm, P, a.radix[st], hs[st], tws + to[st]);
    __syncthreads();
  }
  if (direct) {
    auto store = [&](int p, float2 z) {
      const int c = p - zs;
      if (c < 0 || c >= W) return;
      q0[c] = to_store<T>(z.x);
      if (has1) q1[c] = to_store<T>(z.y);
      if (c == 0 && a.guard) {
        // column -1 repeats sample 0; column W of the previous row is sample 0
        // of this row (flat-buffer read one past the row end)
        q0[-1] = to_store<T>(z.x);
        if (r0 > 0) q0[W - a.Wp] = to_store<T>(z.x);
        if (has1) {
          q1[-1] = to_store<T>(z.y);
          q0[W] = to_store<T>(z.y);
          if (r1 == N - 1) q1[W] = to_store<T>(0.f);
        } else {
          q0[W] = to_store<T>(0.f);
        }
      }
    };
    const int R = a.radix[0];
    if (R == 8) dit_last_stage<8>(sm, hs[0], tws, store);
    else if (R == 4) dit_last_stage<4>(sm, hs[0], tws, store);
    else dit_last_stage<2>(sm, hs[0], tws, store);
    return;
  }

  // REF contrast: per-row running sum (lct.cpp:590-595), warp 0 row r0, warp 1 row r1
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (a.contrast == 1) {
    if (warp < 2 && (warp == 0 || has1)) {
      float carry = 0.f;
      for (int c0 = 0; c0 < W; c0 += 32) {
        const int c = c0 + lane;
        float v = 0.f;
        if (c < W) {
          const float2 z = sm[sidx(zs + c)];
          v = warp == 0 ? z.x : z.y;
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const float u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        v += carry;
        if (c < W) {
          float2 &z = sm[sidx(zs + c)];
          if (warp == 0) z.x = v;
          else z.y = v;
        }
        carry = __shfl_sync(0xffffffffu, v, 31);
      }
    }
    __syncthreads();
  }

  // per-row scale for reduced-precision stores
  float s0 = 1.f, s1 = 1.f;
  if (a.store != 0) {
    float m0 = 0.f, m1 = 0.f;
    for (int c = threadIdx.x; c < W; c += blockDim.x) {
      const float2 z = sm[sidx(zs + c)];
      m0 = fmaxf(m0, fabsf(z.x));
      m1 = fmaxf(m1, fabsf(z.y));
    }
    m0 = warp_max(m0);
    m1 = warp_max(m1);
    if (lane == 0) {
      red[0][warp] = m0;
      red[1][warp] = m1;
    }
    __syncthreads();
    m0 = 0.f;
    m1 = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      m0 = fmaxf(m0, red[0][w]);
      m1 = fmaxf(m1, red[1][w]);
    }
    s0 = pow2_scale(m0);
    s1 = pow2_scale(m1);
    if (threadIdx.x == 0) {
      a.row_scale[(int64_t)sl * N + r0] = s0;
      if (has1) a.row_scale[(int64_t)sl * N + r1] = s1;
    }
  }
  const float i0 = 1.f / s0, i1 = 1.f / s1;  // exact: powers of two

  for (int c = threadIdx.x; c < W; c += blockDim.x) {
    const float2 z = sm[sidx(zs + c)];
    q0[c] = to_store<T>(z.x * i0);
    if (has1) q1[c] = to_store<T>(z.y * i1);
  }
  if (threadIdx.x == 0 && a.guard) {
    const float2 z = sm[sidx(zs)];
    // column -1 repeats sample 0; column W of the previous row is sample 0 of
    // this row (flat-buffer read one past the row end)
    q0[-1] = to_store<T>(z.x * i0);
    if (a.store == 0) {
      if (r0 > 0) q0[W - a.Wp] = to_store<T>(z.x);
      if (has1) {
        q1[-1] = to_store<T>(z.y * i1);
        q0[W] = to_store<T>(z.y);
        if (r1 == N - 1) q1[W] = to_store<T>(0.f);
      } else {
        q0[W] = to_store<T>(0.f);
      }
    } else {
      // reduced precision: each row is scaled separately, so the one-past-
      // the-end column (only read when t rounds onto W) is left at 0
      q0[W] = to_store<T>(0.f);
      if (has1) {
        q1[-1] = to_store<T>(z.y * i1);
        q1[W] = to_store<T>(0.f);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kFftThreads) filter_rows_kernel(FilterLaunch a) {
  filter_pair<T>(a, blockIdx.x, blockIdx.y);
}

// Uneven batch: one launch over the row pairs of every sinogram; jobs[k]
// describes sinogram k (its rows start at pair_begin[k]).
template <typename T>
__global__ void __launch_bounds__(kFftThreads)
    filter_batch_kernel(const FilterLaunch *__restrict__ jobs, const int *__restrict__ pair_begin,
                        int n_jobs) {
  const int g = blockIdx.x;
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pair_begin[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  const FilterLaunch a = jobs[lo];
  filter_pair<T>(a, g - pair_begin[lo], 0);
}

// FLT contrast: no filtering, copy into the padded layout.
template <typename T>
__global__ void copy_rows_kernel(FilterLaunch a) {
  const int r = blockIdx.x, sl = blockIdx.y;
  const int N = a.N, W = a.W;
  const float *x = a.x + sl * a.x_slice_stride + (int64_t)r * W;
  T *q = reinterpret_cast<T *>(a.q) + sl * a.q_slice_stride + (int64_t)r * a.Wp +
         (a.off ? a.off : kRowOff);
  const float *ring = a.ring ? a.ring + (int64_t)sl * W : nullptr;
  auto xv = [&](int c) { return ring ? __fadd_rn(x[c], ring[c]) : x[c]; };
  __shared__ float red[32];
  float s = 1.f;
  if (a.store != 0) {
    float m = 0.f;
    for (int c = threadIdx.x; c < W; c += blockDim.x) m = fmaxf(m, fabsf(xv(c)));
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, red[w]);
    s = pow2_scale(m);
    if (threadIdx.x == 0) a.row_scale[(int64_t)sl * N + r] = s;
  }
  const float inv = 1.f / s;
  for (int c = threadIdx.x; c < W; c += blockDim.x) q[c] = to_store<T>(xv(c) * inv);
  if (threadIdx.x == 0 && a.guard) {
    q[-1] = to_store<T>(xv(0) * inv);
    // the next row's first sample: read only where that row exists (on the
    // last row of the last slice x[W] lies past the end of the input)
    float nx = 0.f;
    if (a.store == 0 && r + 1 < N) nx = ring ? __fadd_rn(x[W], ring[0]) : x[W];
    q[W] = to_store<T>(nx);
  }
}

__global__ void minmax_partial_kernel(const float *x, int64_t stride, int64_t count,
                                      float2 *partials, const float *ring, int W) {
  const int sl = blockIdx.y;
  const float *p = x + sl * stride;
  const float *rg = ring ? ring + (int64_t)sl * W : nullptr;
  float mn = INFINITY, mx = -INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float v = rg ? __fadd_rn(p[i], rg[i % W]) : p[i];
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  __shared__ float2 red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_float2(mn, mx);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      mn = fminf(mn, red[w].x);
      mx = fmaxf(mx, red[w].y);
    }
    mn = fminf(mn, red[0].x);
    mx = fmaxf(mx, red[0].y);
    partials[sl * gridDim.x + blockIdx.x] = make_float2(mn, mx);
  }
}

__global__ void minmax_final_kernel(const float2 *partials, int nparts, int S,
                                    float2 *minmax, int *err) {
  const int sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= S) return;
  float mn = INFINITY, mx = -INFINITY;
  for (int k = 0; k < nparts; k++) {
    mn = fminf(mn, partials[sl * nparts + k].x);
    mx = fmaxf(mx, partials[sl * nparts + k].y);
  }
  minmax[sl] = make_float2(mn, mx);
  if (err && mn <= 0.0f && (float)((double)mx / 1000000.0) <= 0.0f) atomicOr(err, 1);
}

// Column means over the projections, summed in projection order (lct.cpp:308-311).
__global__ void ring_avg_kernel(const float *x, int64_t stride, int N, int W, float *avg) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x, sl = blockIdx.y;
  if (c >= W) return;
  const float *p = x + sl * stride + c;
  float s = 0.f;
  for (int r = 0; r < N; r++) s = __fadd_rn(s, p[(int64_t)r * W]);
  avg[(int64_t)sl * W + c] = __fdiv_rn(s, (float)N);
}

// Box mean of half width `box` minus the mean (lct.cpp:313-321), each
// column's operations in the reference's order.
__global__ void ring_tmp_kernel(const float *avg, int W, int box, float *ring) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x, sl = blockIdx.y;
  if (c >= W) return;
  const float *a = avg + (int64_t)sl * W;
  float t = 0.f;
  for (int ii = -box; ii <= box; ii++) {
    const int k = c - ii;
    if (k >= 0 && k < W) t = __fadd_rn(t, a[k]);
  }
  if (c >= box && c <= W - 1 - box) t = __fdiv_rn(t, (float)(2 * box + 1));
  for (int ii = 0; ii < box; ii++) {
    if (c == ii) t = __fdiv_rn(t, (float)(box + ii + 1));
    if (c == W - 1 - ii) t = __fdiv_rn(t, (float)(box + ii + 1));
  }
  ring[(int64_t)sl * W + c] = __fsub_rn(t, a[c]);
}

template <typename T>
__global__ void unpad_kernel(const T *q, int64_t q_slice_stride, const float *row_scale,
                             int N, int W, int Wp, float *out, int64_t out_slice_stride, int off) {
  const int r = blockIdx.x, sl = blockIdx.y;
  const T *src = q + sl * q_slice_stride + (int64_t)r * Wp + off;
  float *dst = out + sl * out_slice_stride + (int64_t)r * W;
  const float s = row_scale ? row_scale[(int64_t)sl * N + r] : 1.f;
  for (int c = threadIdx.x; c < W; c += blockDim.x) dst[c] = (float)src[c] * s;
}

// Wide layout (fbp_kernels.hpp, wide_offset): column off + k of row r holds
// the flat sample r*W + k of the slice -- sample k - dr*W of row r + dr,
// dr = floor(k / W) -- and 0 outside the slice's rows.  Reads only the data
// columns, writes only the halo columns, so rows can be filled in any order.
__global__ void halo_kernel(float *q, int64_t q_slice_stride, int N, int W, int Wp, int off) {
  const int r = blockIdx.x, sl = blockIdx.y;
  float *base = q + sl * q_slice_stride;
  float *row = base + (int64_t)r * Wp;
  for (int c = threadIdx.x; c < Wp; c += blockDim.x) {
    if (c >= off && c < off + W) continue;
    const int k = c - off;
    const int dr = k >= 0 ? k / W : -((-k + W - 1) / W);
    const int rr = r + dr, kk = k - dr * W;
    row[c] = (rr >= 0 && rr < N) ? base[(int64_t)rr * Wp + off + kk] : 0.f;
  }
}

template <typename T> __device__ __forceinline__ float ld_sample(const T *p) { return (float)*p; }
template <> __device__ __forceinline__ float ld_sample<float>(const float *p) { return __ldg(p); }

template <typename T>
cudaError_t launch_filter_t(const FilterLaunch &a, cudaStream_t st) {
  if (a.contrast == 3) {
    copy_rows_kernel<T><<<dim3(a.N, a.S), 256, 0, st>>>(a);
    return cudaGetLastError();
  }
  const size_t smem = sizeof(float2) * (size_t)(a.P + a.P / 16);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(filter_rows_kernel<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  filter_rows_kernel<T><<<dim3((a.N + 1) / 2, a.S), kFftThreads, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_filter_batch(const FilterLaunch *jobs_dev, const int *pair_begin_dev, int n_jobs,
                                int n_pairs, int max_pad, cudaStream_t st) {
  const size_t smem = sizeof(float2) * (size_t)(max_pad + max_pad / 16);
  cudaError_t e = cudaFuncSetAttribute(filter_batch_kernel<float>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  filter_batch_kernel<float><<<n_pairs, kFftThreads, smem, st>>>(jobs_dev, pair_begin_dev, n_jobs);
  return cudaGetLastError();
}

cudaError_t launch_halo(float *q, int64_t q_slice_stride, int N, int W, int Wp, int off, int S,
                        cudaStream_t st) {
  halo_kernel<<<dim3(N, S), 256, 0, st>>>(q, q_slice_stride, N, W, Wp, off);
  return cudaGetLastError();
}

cudaError_t launch_filter(const FilterLaunch &a, cudaStream_t st) {
  if (a.store == 1) return launch_filter_t<__half>(a, st);
  if (a.store == 2) return launch_filter_t<__nv_bfloat16>(a, st);
  return launch_filter_t<float>(a, st);
}

cudaError_t launch_minmax(const float *x, int64_t x_slice_stride, int64_t count, int S,
                          float2 *partials, float2 *minmax, int *err, cudaStream_t st,
                          const float *ring, int W) {
  minmax_partial_kernel<<<dim3(kMinMaxBlocks, S), 256, 0, st>>>(x, x_slice_stride, count,
                                                                partials, ring, W);
  minmax_final_kernel<<<(S + 127) / 128, 128, 0, st>>>(partials, kMinMaxBlocks, S, minmax, err);
  return cudaGetLastError();
}

cudaError_t launch_ring(const float *x, int64_t x_slice_stride, int N, int W, int S, int box,
                        float *avg, float *ring, cudaStream_t st) {
  const dim3 g((W + 127) / 128, S);
  ring_avg_kernel<<<g, 128, 0, st>>>(x, x_slice_stride, N, W, avg);
  ring_tmp_kernel<<<g, 128, 0, st>>>(avg, W, box, ring);
  return cudaGetLastError();
}

cudaError_t launch_unpad(const void *q, int64_t q_slice_stride, const float *row_scale,
                         int store, int N, int W, int Wp, int S, float *out,
                         int64_t out_slice_stride, cudaStream_t st, int off) {
  const dim3 g(N, S);
  if (store == 1)
    unpad_kernel<__half><<<g, 256, 0, st>>>((const __half *)q, q_slice_stride, row_scale, N, W,
                                            Wp, out, out_slice_stride, off);
  else if (store == 2)
    unpad_kernel<__nv_bfloat16><<<g, 256, 0, st>>>((const __nv_bfloat16 *)q, q_slice_stride,
                                                   row_scale, N, W, Wp, out, out_slice_stride, off);
  else
    unpad_kernel<float><<<g, 256, 0, st>>>((const float *)q, q_slice_stride, nullptr, N, W, Wp,
                                           out, out_slice_stride, off);
  return cudaGetLastError();
}

}  // namespace ctas
