// axis.cpp -- rotation-axis search (ctas src/common/lct.cpp:792-1325) on the
// device FBP path: class AverageGradient and the raxis() family.
//
// The search logic (grid, directional march, bisection) is the reference's,
// statement by statement, with its float/double conversions; every trial
// evaluation runs on the GPU: average-gradient trials as multi-centre
// backprojections (ctas_fbp_repeat_multi_dev) followed by the fused
// smoothing/Sobel/mean kernel, projection-pair trials as one reduction
// launch per batch of shifts.  Trials the reference evaluates one by one in
// order (the directional march) are evaluated in speculative batches and
// consumed in order, which gives the sequential result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "../../include/ctas_axis.h"
#include "../../include/ctas_fbp.h"
#include "axis_kernels.hpp"
#include "fbp_host.hpp"

namespace {

template <class F> int guarded(F &&f) {
  try {
    return f();
  } catch (const ctas::Error &e) {
    ctas::set_last_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    ctas::set_last_error("host allocation failed");
    return CTAS_E_NOMEM;
  } catch (const std::exception &e) {
    ctas::set_last_error(e.what());
    return CTAS_E_ARG;
  }
}

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  int code = CTAS_E_CUDA;
  if (e == cudaErrorMemoryAllocation) code = CTAS_E_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = CTAS_E_NODEVICE;
  cudaGetLastError();
  ctas::fail(code, std::string("axis search: ") + what + ": " + cudaGetErrorString(e));
}

// status of a ctas_fbp call -> exception carrying its message
void fbp_check(int st) {
  if (st != CTAS_OK) ctas::fail(st, ctas_fbp_last_error());
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cuda_check(cudaGetDevice(&prev), "cudaGetDevice");
    if (dev != prev) cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DevGuard() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
  void ensure(size_t n) {
    if (n <= bytes) return;
    release();
    cuda_check(cudaMalloc(&p, n), "cudaMalloc");
    bytes = n;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
  ~Buf() { release(); }
};

int resolve_device(int32_t device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    ctas::fail(CTAS_E_NODEVICE, "no CUDA device");
  }
  int dev = device;
  if (dev < 0) cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev >= n) ctas::fail(CTAS_E_ARG, "device ordinal out of range");
  return dev;
}

// improveMe (lct.cpp:1114-1134): bisection towards the smaller neighbour.
float improve_me(float eps, const std::vector<float> &vaxSi, const std::vector<float> &errSi,
                 int idx, int cdir, const std::function<float(float)> &getvx) {
  float aa = vaxSi[(size_t)(idx - cdir)];
  float bb = vaxSi[(size_t)(idx + cdir)];
  float rf = vaxSi[(size_t)idx];
  float vl = errSi[(size_t)idx];
  while (std::fabs(aa - rf) > eps || std::fabs(rf - bb) > eps) {
    const bool afar = std::fabs(aa - rf) > std::fabs(rf - bb);
    float &lo = afar ? aa : bb;
    float &hi = afar ? bb : aa;
    const float x = (rf + lo) / 2;
    const float vx = getvx(x);
    if (vl <= vx) {
      lo = x;
    } else {
      vl = vx;
      hi = rf;
      rf = x;
    }
  }
  return rf;
}

}  // namespace

// ------------------------------------------------------------ AverageGradient
struct ctas_ag {
  int device = 0;
  int64_t N = 0, W = 0;
  float sigma = 0.f;
  int K = 1;
  ctas_fbp *rec = nullptr;
  cudaStream_t stream = nullptr;
  Buf g, slices, crop, psum, pcnt, osum, ocnt;
  int64_t chunk = 0;  // slices per batch
  int64_t evaluations = 0;
  ~ctas_ag() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    g.release();
    slices.release();
    crop.release();
    psum.release();
    pcnt.release();
    osum.release();
    ocnt.release();
    if (stream) cudaStreamDestroy(stream);
    if (rec) ctas_fbp_destroy(rec);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

namespace {

// Slices reconstructed per batch: about 2 GiB of slices, 1 .. 256.
int64_t ag_chunk(int64_t W) {
  const int64_t per = W * W * (int64_t)sizeof(float);
  int64_t c = ((int64_t)2 << 30) / per;
  if (c < 1) c = 1;
  if (c > 256) c = 256;
  return c;
}

void ag_create(ctas_ag *ag, const float *sino, int64_t N, int64_t W, float anarc, int32_t device,
               uint32_t flags) {
  if (!sino) ctas::fail(CTAS_E_ARG, "null sinogram");
  if (N < 1 || W < 1) ctas::fail(CTAS_E_SHAPE, "Average gradient: Empty input sinogram.");
  ag->device = resolve_device(device);
  ag->N = N;
  ag->W = W;
  DevGuard dg(ag->device);
  // ct(ish, Contrast::ABS, anarc) with the default Filter (RAMP); sino() on a copy
  ctas_fbp_opts o;
  std::memset(&o, 0, sizeof(o));
  o.struct_size = sizeof(o);
  o.device = ag->device;
  o.flags = CTAS_FLAG_NO_WRITEBACK | (flags & CTAS_FLAG_SHIPPED_INDEX);
  o.tile = -1;
  fbp_check(ctas_fbp_create(&ag->rec, N, W, CTAS_ABS, CTAS_FILTER_RAMP, 0.f, anarc, &o));
  fbp_check(ctas_fbp_sino(ag->rec, const_cast<float *>(sino)));
  // sigma = angO(anarc, N) * W / pi  (float * ssize_t -> float, / M_PI in double)
  const float ang = ctas::step_rad(anarc, N);
  const float sigma = (float)((double)(ang * (float)W) / M_PI);
  ag->sigma = sigma;
  std::vector<double> taps;
  if (sigma > 1) {
    // g(a, b) = exp(-(a*a + b*b) / sig22) (lct.cpp:839-841); separable taps
    // exp(-a*a / sig22), kept while >= 1e-12 (the rest cannot move a float)
    const float sig22 = 2 * sigma * sigma;
    for (int a = 0;; a++) {
      const float v = std::exp((float)(-(a * a)) / sig22);
      if (v < 1e-12f) break;
      taps.push_back((double)v);
      if ((int)taps.size() > ctas::kAgMaxTaps)
        ctas::fail(CTAS_E_UNSUPPORTED,
                   "Average gradient: smoothing width sigma = " + std::to_string(sigma) +
                       " px needs more than " + std::to_string(ctas::kAgMaxTaps) + " taps");
    }
  } else {
    taps.push_back(1.0);  // no smoothing (lct.cpp:837, 866)
  }
  ag->K = (int)taps.size();
  cuda_check(cudaStreamCreateWithFlags(&ag->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  ag->g.ensure(sizeof(double) * taps.size());
  cuda_check(cudaMemcpy(ag->g.p, taps.data(), sizeof(double) * taps.size(), cudaMemcpyHostToDevice),
             "cudaMemcpy");
  ag->chunk = ag_chunk(W);
}

// values[k] = AverageGradient::apply(axis_r[k]) (lct.cpp:863-913)
void ag_apply(ctas_ag *ag, const float *axis_r, int64_t n, float *values) {
  if (n < 0) ctas::fail(CTAS_E_ARG, "negative count");
  if (n == 0) return;
  if (!axis_r || !values) ctas::fail(CTAS_E_ARG, "null axis positions or values");
  DevGuard dg(ag->device);
  const int64_t W = ag->W;
  const int64_t nblk = ctas::ag_blocks_per_slice((int)W);
  const int64_t C = std::min<int64_t>(ag->chunk, n);
  ag->slices.ensure(sizeof(float) * (size_t)(C * W * W));
  ag->crop.ensure(sizeof(int) * (size_t)C);
  ag->psum.ensure(sizeof(double) * (size_t)(C * nblk));
  ag->pcnt.ensure(sizeof(unsigned long long) * (size_t)(C * nblk));
  ag->osum.ensure(sizeof(double) * (size_t)C);
  ag->ocnt.ensure(sizeof(unsigned long long) * (size_t)C);
  std::vector<float> centres((size_t)C);
  std::vector<int> crops((size_t)C);
  std::vector<double> sums((size_t)C);
  std::vector<unsigned long long> cnts((size_t)C);
  for (int64_t k0 = 0; k0 < n; k0 += C) {
    const int64_t m = std::min<int64_t>(C, n - k0);
    for (int64_t k = 0; k < m; k++) {
      // const float centre = axisR - 0.5*(ish(1)-1);
      const float centre = (float)((double)axis_r[k0 + k] - 0.5 * (double)(W - 1));
      // recCrop: Segment(k, -k) of the rows with k = ceil(abs(c)) (ct.h:276-279).
      // In ct.h only the C library's int abs() is in scope, so the float centre
      // is truncated first: k = |(int)c| (0 for |c| < 1).
      const float cacent = (float)std::abs((int)centre);
      if (W - 2 * (int64_t)cacent <= 0)
        ctas::fail(CTAS_E_CENTER, "Range size: Negative size for the cropped slice");
      centres[(size_t)k] = centre;
      crops[(size_t)k] = (int)cacent;
    }
    fbp_check(ctas_fbp_repeat_multi_dev(ag->rec, centres.data(), m, ag->slices.as<float>(),
                                        ag->stream));
    cuda_check(cudaMemcpyAsync(ag->crop.p, crops.data(), sizeof(int) * (size_t)m,
                               cudaMemcpyHostToDevice, ag->stream),
               "cudaMemcpyAsync");
    ctas::AgLaunch a{};
    a.slices = ag->slices.as<float>();
    a.S = (int)m;
    a.W = (int)W;
    a.crop = ag->crop.as<int>();
    a.g = ag->g.as<double>();
    a.K = ag->K;
    a.count_all = ag->K > 1 ? 1 : 0;
    a.part_sum = ag->psum.as<double>();
    a.part_cnt = ag->pcnt.as<unsigned long long>();
    a.out_sum = ag->osum.as<double>();
    a.out_cnt = ag->ocnt.as<unsigned long long>();
    cuda_check(ctas::launch_ag_measure(a, ag->stream), "average-gradient kernel");
    cuda_check(cudaMemcpyAsync(sums.data(), ag->osum.p, sizeof(double) * (size_t)m,
                               cudaMemcpyDeviceToHost, ag->stream),
               "cudaMemcpyAsync");
    cuda_check(cudaMemcpyAsync(cnts.data(), ag->ocnt.p, sizeof(unsigned long long) * (size_t)m,
                               cudaMemcpyDeviceToHost, ag->stream),
               "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(ag->stream), "cudaStreamSynchronize");
    fbp_check(ctas_fbp_synchronize(ag->rec));
    for (int64_t k = 0; k < m; k++) {
      // const float sm = sum(cSlice); const int nm = ...; return nm ? sm/nm : 0.0;
      const float sm = (float)sums[(size_t)k];
      const int nm = (int)cnts[(size_t)k];
      values[k0 + k] = nm ? sm / (float)nm : 0.0f;
    }
    ag->evaluations += m;
  }
}

float ag_one(ctas_ag *ag, float axis_r) {
  float v = 0.f;
  ag_apply(ag, &axis_r, 1, &v);
  return v;
}

// ------------------------------------------------------------ projection pair
// Device copies of two opposite projection sets (rows x W each).
struct Pair {
  const float *p0 = nullptr, *p180 = nullptr;  // device
  int64_t stride0 = 0, stride180 = 0;
  int rows = 0, W = 0;
  bool add_one = false;
  std::vector<float> host180_first, host180_last;  // columns 0 and W-1 of proj180 (+1 applied)
  cudaStream_t stream = nullptr;
  Buf shifts, out, profile;
};

// raxis(proj0, proj180, maxDev) (lct.cpp:1217-1297) on device data.
float pair_raxis(Pair &P, float maxDev) {
  if (maxDev < 0 || maxDev > 0.5)
    ctas::fail(CTAS_E_ARG, "Axis shift: Invalid maximum relative shift of the rotation axis " +
                               std::to_string(maxDev) + ". Must be within [0, 0.5] range.");
  if (P.rows < 1 || P.W < 1) ctas::fail(CTAS_E_SHAPE, "Axis shift: Empty input projections.");
  const int W = P.W, rows = P.rows;
  const float cent = (float)(0.5 * (W - 1));
  ctas::PairLaunch L{};
  L.p0 = P.p0;
  L.p180 = P.p180;
  L.stride0 = P.stride0;
  L.stride180 = P.stride180;
  L.rows = rows;
  L.W = W;
  L.add_one = P.add_one ? 1 : 0;
  // approximate position: centre of mass of sum |p - 1|
  P.profile.ensure(sizeof(float) * (size_t)W);
  cuda_check(ctas::launch_pair_profile(L, P.profile.as<float>(), P.stream), "pair profile kernel");
  std::vector<float> proj((size_t)W);
  cuda_check(cudaMemcpyAsync(proj.data(), P.profile.p, sizeof(float) * (size_t)W,
                             cudaMemcpyDeviceToHost, P.stream),
             "cudaMemcpyAsync");
  cuda_check(cudaStreamSynchronize(P.stream), "cudaStreamSynchronize");
  double s = 0.0, si = 0.0;
  for (int i = 0; i < W; i++) {
    s += (double)proj[(size_t)i];
    si += (double)((float)i * proj[(size_t)i]);  // i0*proj(i0): int * float -> float
  }
  const float sum = (float)s;
  if (sum == 0.0f)
    ctas::fail(CTAS_E_DATA, "Axis shift: Impossible input projection averaging to zero.");
  const float fcr = (float)(si / (double)sum);
  const int stpsz = 16;
  const float stf = maxDev == 0.0f ? 1.0f : maxDev * (float)W / (float)stpsz;
  const int steps = (int)(1.0f + 2.0f * stf);
  if (steps < 3)
    ctas::fail(CTAS_E_ARG, "Axis shift: maximum shift below one search step (fewer than 3 trials)");
  // aver = (sum(proj180R(all,0)) + sum(proj180R(all,W-1))) / (2 rows)
  double a0 = 0.0, a1 = 0.0;
  for (int j = 0; j < rows; j++) {
    a0 += (double)P.host180_last[(size_t)j];   // proj180R column 0 = proj180 column W-1
    a1 += (double)P.host180_first[(size_t)j];  // proj180R column W-1 = proj180 column 0
  }
  L.aver = (float)((a0 + a1) / (double)(2 * rows));

  std::vector<int> sh;
  std::vector<double> sq;
  auto calc = [&](const std::vector<float> &xs) {
    const int n = (int)xs.size();
    sh.resize((size_t)n);
    sq.resize((size_t)n);
    for (int k = 0; k < n; k++) {
      const double t = std::trunc((double)xs[(size_t)k]);  // float -> ssize_t
      if (std::fabs(t) >= (double)W)
        ctas::fail(CTAS_E_DATA, "Axis shift: trial shift of a whole projection width");
      sh[(size_t)k] = (int)t;
    }
    P.shifts.ensure(sizeof(int) * (size_t)n);
    P.out.ensure(sizeof(double) * (size_t)n);
    cuda_check(cudaMemcpyAsync(P.shifts.p, sh.data(), sizeof(int) * (size_t)n,
                               cudaMemcpyHostToDevice, P.stream),
               "cudaMemcpyAsync");
    L.shifts = P.shifts.as<int>();
    L.out = P.out.as<double>();
    cuda_check(ctas::launch_pair_err(L, n, P.stream), "pair error kernel");
    cuda_check(cudaMemcpyAsync(sq.data(), P.out.p, sizeof(double) * (size_t)n,
                               cudaMemcpyDeviceToHost, P.stream),
               "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(P.stream), "cudaStreamSynchronize");
    std::vector<float> e((size_t)n);
    for (int k = 0; k < n; k++) e[(size_t)k] = (float)std::sqrt(sq[(size_t)k]);
    return e;
  };
  auto calc1 = [&](float x) { return calc(std::vector<float>{x})[0]; };

  std::vector<float> vaxS((size_t)steps);
  for (int ii = 0; ii < steps; ii++)
    vaxS[(size_t)ii] = 2 * (fcr - cent) + (float)(stpsz * (ii - (steps - 1) / 2));
  const std::vector<float> errS = calc(vaxS);
  int idx = 0;
  float minval = std::numeric_limits<float>::max();
  for (int i = 1; i < steps - 1; i++)
    if (errS[(size_t)i] < errS[(size_t)(i - 1)] && errS[(size_t)i] < errS[(size_t)(i + 1)] &&
        errS[(size_t)i] < minval)
      minval = errS[(size_t)(idx = i)];
  if (minval != std::numeric_limits<float>::max())  // local minimum found
    return (float)(cent + 0.5 * improve_me(1.0f, vaxS, errS, idx, 1, calc1));

  idx = errS[0] < errS[(size_t)(steps - 1)] ? 0 : steps - 1;
  const int cdir = idx == 0 ? -1 : 1;
  minval = errS[(size_t)idx];
  const int maxSteps = (int)(((float)(W / 2) - (float)cdir * vaxS[(size_t)idx]) / (float)stpsz);
  if (maxSteps <= 0) ctas::fail(CTAS_E_DATA, "Axis shift: Failed to calculate rotation centre.");
  std::vector<float> vaxS2((size_t)maxSteps + 2), errS2((size_t)maxSteps + 2);
  vaxS2[0] = vaxS[(size_t)(idx - cdir)];
  vaxS2[1] = vaxS[(size_t)idx];
  errS2[0] = errS[(size_t)(idx - cdir)];
  errS2[1] = errS[(size_t)idx];
  int idx2 = 1;
  bool stop = false;
  for (int i0 = 0; i0 < maxSteps && !stop; i0 += 8) {
    const int m = std::min(8, maxSteps - i0);
    std::vector<float> xs((size_t)m);
    for (int k = 0; k < m; k++) xs[(size_t)k] = vaxS[(size_t)idx] + (float)(cdir * (i0 + k + 1) * stpsz);
    const std::vector<float> es = calc(xs);
    for (int k = 0; k < m; k++) {
      const int i = i0 + k;
      vaxS2[(size_t)(i + 2)] = xs[(size_t)k];
      errS2[(size_t)(i + 2)] = es[(size_t)k];
      if (es[(size_t)k] < minval) {
        minval = es[(size_t)k];
        idx2 = i + 2;
      } else {
        stop = true;
        break;
      }
    }
  }
  if (idx2 == maxSteps + 1) ctas::fail(CTAS_E_DATA, "Axis shift: Failed to calculate rotation centre.");
  return (float)(cent + 0.5 * improve_me(1.0f, vaxS2, errS2, idx2, cdir, calc1));
}

// ------------------------------------------------------------ raxis(sino, ...)
float raxis_sino(const float *sino, int64_t N, int64_t W, float anarc, float maxDev, int algo,
                 int device, int64_t *trials) {
  if (!sino) ctas::fail(CTAS_E_ARG, "null sinogram");
  if (N < 3 || W < 3)
    ctas::fail(CTAS_E_SHAPE, "Axis shift: Shape of input sinogram (" + std::to_string(N) + "," +
                                 std::to_string(W) + ") is less than minimal (3,3).");
  const float arc = ctas::arc_rad(anarc, N);
  if (arc == 0.0f) ctas::fail(CTAS_E_ARG, "Axis shift: Zero sinogram arc.");
  if (std::fabs(arc) < M_PI)
    ctas::fail(CTAS_E_ARG, "Axis shift: Sinogram arc " +
                               std::to_string(std::fabs(arc) * 180 / M_PI) +
                               " is less than 180 degree.");
  const float maxDevLM = 0.25f;
  if (maxDev < 0 || maxDev > maxDevLM)
    ctas::fail(CTAS_E_ARG, "Axis shift: Invalid maximum relative shift of the rotation axis " +
                               std::to_string(maxDev) + ".");
  if (algo < 0 || algo > 3)
    ctas::fail(CTAS_E_ARG, "Axis shift: Unknown algorithm for rotation axis " +
                               std::to_string(algo) + ".");
  const float cent = (float)(0.5 * (W - 1));
  const int dev = resolve_device(device);
  DevGuard dg(dev);
  if (trials) *trials = 0;

  // the sinogram on the device (pair and threshold estimates)
  Buf dsino;
  dsino.ensure(sizeof(float) * (size_t)(N * W));
  cudaStream_t stream = nullptr;
  cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  struct StreamOwner {
    cudaStream_t s;
    ~StreamOwner() {
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    }
  } so{stream};
  cuda_check(cudaMemcpyAsync(dsino.p, sino, sizeof(float) * (size_t)(N * W), cudaMemcpyHostToDevice,
                             stream),
             "cudaMemcpyAsync");

  auto raxisQ = [&]() {
    // idx180 = (N-1) * pi / |arcO| ; rows j and j + idx180, both + 1
    const int idx180 = (int)((double)(N - 1) * M_PI / (double)std::fabs(ctas::arc_rad(anarc, N)));
    const int nofln = (int)N - idx180;
    Pair P;
    P.p0 = dsino.as<float>();
    P.p180 = dsino.as<float>() + (int64_t)idx180 * W;
    P.stride0 = P.stride180 = W;
    P.rows = nofln;
    P.W = (int)W;
    P.add_one = true;
    P.stream = stream;
    P.host180_first.resize((size_t)nofln);
    P.host180_last.resize((size_t)nofln);
    for (int j = 0; j < nofln; j++) {
      P.host180_first[(size_t)j] = sino[(int64_t)(j + idx180) * W] + 1;
      P.host180_last[(size_t)j] = sino[(int64_t)(j + idx180) * W + W - 1] + 1;
    }
    return pair_raxis(P, std::min(maxDev, 0.5f));
  };

  float fcr = 0;
  if (algo == 0) return raxisQ();
  if (algo == 1) {
    fcr = cent;
  } else if (algo == 2) {
    fcr = raxisQ();
  } else {
    // projLine = sum over projections; threshold 0.1 max + 0.9 min; first and
    // last column above it (lct.cpp:1162-1177)
    Buf line;
    line.ensure(sizeof(float) * (size_t)W);
    cuda_check(ctas::launch_column_sum(dsino.as<float>(), (int)N, (int)W, line.as<float>(), stream),
               "column sum kernel");
    std::vector<float> pl((size_t)W);
    cuda_check(cudaMemcpyAsync(pl.data(), line.p, sizeof(float) * (size_t)W, cudaMemcpyDeviceToHost,
                               stream),
               "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    float mx = pl[0], mn = pl[0];
    for (float v : pl) {
      mx = std::max(mx, v);
      mn = std::min(mn, v);
    }
    const float threshold = (float)(0.1 * mx + 0.9 * mn);
    auto thrFnd = [&](bool fromStart) {
      for (int64_t i = fromStart ? 0 : W - 1; i >= 0 && i < W; i += fromStart ? 1 : -1)
        if (pl[(size_t)i] > threshold) return (float)i;
      ctas::fail(CTAS_E_DATA, "Axis shift: constant projection profile, no threshold crossing");
    };
    fcr = (thrFnd(true) + thrFnd(false)) / 2.0f;
  }
  if (std::fabs(fcr - cent) / (float)W > maxDev)
    ctas::fail(CTAS_E_DATA, "Axis shift: Rotation axis relative shift " +
                                std::to_string(std::fabs(fcr - cent) / (float)W) +
                                " is larger than maximum shift " + std::to_string(maxDev) + ".");
  const float rbxsz = (float)(1.0 - 2.0 * (maxDev + std::fabs(fcr - cent) / (float)W));
  if (rbxsz < 0.5f)
    ctas::fail(CTAS_E_DATA, "Axis shift: Relative box size " + std::to_string(rbxsz) +
                                " is less than miminum window of 0.5.");

  const int stpsz = 8;
  const float stf = maxDev == 0.0f ? 1.0f : maxDev * (float)W / (float)stpsz;
  const int steps = (int)(1.0f + 2.0f * stf);
  if (steps < 3)
    ctas::fail(CTAS_E_ARG, "Axis shift: maximum shift below one search step (fewer than 3 trials)");

  ctas_ag ag;
  ag_create(&ag, sino, N, W, anarc, dev, 0u);
  auto AG = [&](float vax) { return ag_one(&ag, cent + vax); };

  // exec1: the grid coffee + stpsz * (idx - hfsteps), all trials in batches
  const float coffee = fcr - cent;
  const int hfsteps = (steps - 1) / 2;
  std::vector<float> vaxS((size_t)steps), errS((size_t)steps), axr((size_t)steps);
  for (int i = 0; i < steps; i++) {
    vaxS[(size_t)i] = coffee + (float)(stpsz * (i - hfsteps));
    axr[(size_t)i] = cent + vaxS[(size_t)i];
  }
  ag_apply(&ag, axr.data(), steps, errS.data());
  int idxM = 0;
  float minval = std::numeric_limits<float>::max();
  for (int i = 1; i < steps - 1; i++) {
    const float cval = errS[(size_t)i];
    if (cval < errS[(size_t)(i - 1)] && cval < errS[(size_t)(i + 1)] && cval < minval) {
      idxM = i;
      minval = cval;
    }
  }
  int cdir = 1;
  if (!idxM) {  // no local minimum within the range: march outwards (exec2)
    const int idx = errS[0] < errS[(size_t)(steps - 1)] ? 0 : steps - 1;
    cdir = idx == 0 ? -1 : 1;
    const int coffee2 = (int)vaxS[(size_t)(idx - cdir * 2)];
    const int maxSteps = (int)((float)W * maxDevLM - (float)(cdir * coffee2 / stpsz));
    if (maxSteps <= 0) ctas::fail(CTAS_E_DATA, "Axis shift: Impossible number of steps.");
    std::vector<float> v2((size_t)maxSteps), e2((size_t)maxSteps);
    bool found = false;
    for (int i0 = 0; i0 < maxSteps && !found; i0 += 8) {
      const int m = std::min(8, maxSteps - i0);
      std::vector<float> ax((size_t)m), ev((size_t)m);
      for (int k = 0; k < m; k++) {
        v2[(size_t)(i0 + k)] = (float)coffee2 + (float)(stpsz * (i0 + k) * cdir);
        ax[(size_t)k] = cent + v2[(size_t)(i0 + k)];
      }
      ag_apply(&ag, ax.data(), m, ev.data());
      for (int k = 0; k < m && !found; k++) {
        e2[(size_t)(i0 + k)] = ev[(size_t)k];
        if (ev[(size_t)k] < minval) {
          minval = ev[(size_t)k];
          idxM = i0 + k;
        } else {
          found = true;
        }
      }
    }
    if (idxM == maxSteps - 1 || idxM == 0) {
      if (trials) *trials = ag.evaluations;
      return fcr;
    }
    vaxS.swap(v2);
    errS.swap(e2);
  }
  const float rf = improve_me(0.25f, vaxS, errS, idxM, cdir, AG);
  if (trials) *trials = ag.evaluations;
  return cent + rf;
}

}  // namespace

// ------------------------------------------------------------ C ABI
extern "C" {

int ctas_ag_create(ctas_ag **out, const float *sino, int64_t n_angles, int64_t width, float anarc,
                   int32_t device) {
  return ctas_ag_create_flags(out, sino, n_angles, width, anarc, device, 0u);
}

int ctas_ag_create_flags(ctas_ag **out, const float *sino, int64_t n_angles, int64_t width,
                         float anarc, int32_t device, uint32_t flags) {
  return guarded([&] {
    if (!out) ctas::fail(CTAS_E_ARG, "null output");
    if (flags & ~(uint32_t)CTAS_FLAG_SHIPPED_INDEX) ctas::fail(CTAS_E_ARG, "unknown flag");
    *out = nullptr;
    ctas_ag *ag = new ctas_ag();
    try {
      ag_create(ag, sino, n_angles, width, anarc, device, flags);
    } catch (...) {
      delete ag;
      throw;
    }
    *out = ag;
    return CTAS_OK;
  });
}

int ctas_ag_apply(ctas_ag *ag, const float *axis_r, int64_t n, float *values) {
  return guarded([&] {
    if (!ag) ctas::fail(CTAS_E_ARG, "null handle");
    ag_apply(ag, axis_r, n, values);
    return CTAS_OK;
  });
}

int ctas_ag_sigma(const ctas_ag *ag, float *sigma, int32_t *taps) {
  return guarded([&] {
    if (!ag) ctas::fail(CTAS_E_ARG, "null handle");
    if (sigma) *sigma = ag->sigma;
    if (taps) *taps = ag->K;
    return CTAS_OK;
  });
}

int ctas_ag_destroy(ctas_ag *ag) {
  delete ag;
  return CTAS_OK;
}

int ctas_raxis(const float *sino, int64_t n_angles, int64_t width, float anarc, float max_dev,
               int32_t algo, int32_t device, float *axis, int64_t *trials) {
  return guarded([&] {
    if (!axis) ctas::fail(CTAS_E_ARG, "null output");
    *axis = raxis_sino(sino, n_angles, width, anarc, max_dev, algo, device, trials);
    return CTAS_OK;
  });
}

int ctas_raxis_pair(const float *proj0, const float *proj180, int64_t rows, int64_t width,
                    float max_dev, int32_t device, float *axis) {
  return guarded([&] {
    if (!axis || !proj0 || !proj180) ctas::fail(CTAS_E_ARG, "null argument");
    if (rows < 1 || width < 1) ctas::fail(CTAS_E_SHAPE, "Axis shift: Empty input projections.");
    const int dev = resolve_device(device);
    DevGuard dg(dev);
    Buf d0, d1;
    d0.ensure(sizeof(float) * (size_t)(rows * width));
    d1.ensure(sizeof(float) * (size_t)(rows * width));
    cuda_check(cudaMemcpy(d0.p, proj0, sizeof(float) * (size_t)(rows * width),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    cuda_check(cudaMemcpy(d1.p, proj180, sizeof(float) * (size_t)(rows * width),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    Pair P;
    P.p0 = d0.as<float>();
    P.p180 = d1.as<float>();
    P.stride0 = P.stride180 = width;
    P.rows = (int)rows;
    P.W = (int)width;
    P.add_one = false;
    cuda_check(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    P.host180_first.resize((size_t)rows);
    P.host180_last.resize((size_t)rows);
    for (int64_t j = 0; j < rows; j++) {
      P.host180_first[(size_t)j] = proj180[j * width];
      P.host180_last[(size_t)j] = proj180[j * width + width - 1];
    }
    float r = 0.f;
    try {
      r = pair_raxis(P, max_dev);
    } catch (...) {
      cudaStreamSynchronize(P.stream);
      cudaStreamDestroy(P.stream);
      throw;
    }
    cudaStreamDestroy(P.stream);
    *axis = r;
    return CTAS_OK;
  });
}

}  // extern "C"
