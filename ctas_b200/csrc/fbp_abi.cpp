// fbp_abi.cpp -- the C ABI (include/ctas_fbp.h): reconstruction handles, their
// device state, and the host/device call forms.
//
// A handle is the counterpart of one ctas CTrec object (src/common/ct.h:
// 235-298).  What the reference does per object on the host -- window, FFTW
// plans, angle table, OpenCL program and buffers (lct.cpp:487-526, 334-392) --
// is done once at create time here: the window, twiddles and angle table are
// uploaded once and shared by clones; each handle owns its own work buffers
// and CUDA stream, so clones on different host threads run concurrently
// instead of serialising on a per-device trylock (lct.cpp:399).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

#include "../../include/ctas_fbp.h"
#include "../../include/ctas_volume.h"
#include "bp_fast.hpp"
#include "fbp_host.hpp"
#include "fbp_kernels.hpp"

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string &m) {
  g_last_error = m;
  return code;
}

template <class F> int guarded(F &&f) {
  try {
    return f();
  } catch (const ctas::Error &e) {
    return set_error(e.code, e.msg);
  } catch (const std::bad_alloc &) {
    return set_error(CTAS_E_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return set_error(CTAS_E_ARG, e.what());
  }
}

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  int code = CTAS_E_CUDA;
  if (e == cudaErrorMemoryAllocation) code = CTAS_E_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = CTAS_E_NODEVICE;
  cudaGetLastError();  // clear a sticky-free error so later calls can proceed
  ctas::fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Makes the handle's device current for the duration of a call and restores
// the caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  // `nothrow` is for destructors: a failure to select the device is ignored.
  explicit DeviceGuard(int dev, bool nothrow = false) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
    if (prev != dev) {
      const cudaError_t e = cudaSetDevice(dev);
      if (nothrow) cudaGetLastError();
      else cuda_check(e, "cudaSetDevice");
    }
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  // grows the buffer; returns true when it was (re)allocated
  bool ensure(size_t n) {
    if (n <= bytes) return false;
    release();
    cuda_check(cudaMalloc(&p, n), "cudaMalloc");
    bytes = n;
    return true;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
  ~DevBuf() { release(); }
};

// Device constants of one reconstruction set-up, shared by clones.
struct Consts {
  int device = 0;
  DevBuf tw, gperm, tab, lin;
  ~Consts() {
    DeviceGuard g(device, true);
    tw.release();
    gperm.release();
    tab.release();
    lin.release();
  }
};

// One set of work buffers (the host stack call double-buffers two sets).
struct WorkSet {
  DevBuf raw, filt, scale, slice, part, minmax, ring_avg, ring;
  DevBuf samples;  // converted output samples of the volume call
  int64_t slices = 0;
  cudaEvent_t ev_in = nullptr, ev_done = nullptr, ev_out = nullptr;
};

}  // namespace

namespace ctas {
// Lets other translation units of the library report through
// ctas_fbp_last_error().
void set_last_error(const std::string &m) { g_last_error = m; }
}  // namespace ctas

struct ctas_fbp {
  int64_t N = 0, W = 0, P = 0, Wp = 0, out_rows = 0, out_cols = 0;
  float geo_oj = 0.f, geo_oi = 0.f, geo_p = 1.f;  // output geometry
  int32_t contrast = 2, ftype = 1, interp = 0, store = 0;
  float fparam = 0.f, arc_deg = 180.f, rec_cof = 1.f;
  uint32_t flags = 0;
  int32_t chunk = 0;
  int32_t tile = -1;      // staged kernel tile, -1 = autotune
  int32_t ring_box = 0;   // ring-artefact filter half width, 0 = off
  int last_tile = -1;
  std::vector<float> tab;
  std::vector<int> radices;
  bool sines_nonneg = true;
  // wide layout (negative sines, truncation, float32 store): filtered rows
  // carry their neighbours' samples as halos, so the staged kernel serves
  // them too; off = column of sample 0
  bool wide = false;
  int64_t off = ctas::kRowOff;
  int device = 0;
  std::shared_ptr<Consts> dc;
  cudaStream_t stream = nullptr, s_in = nullptr, s_out = nullptr;
  WorkSet ws[2];
  DevBuf err;
  DevBuf centers;           // per-slice centres of repeat_multi
  int *err_host = nullptr;  // pinned
  bool have_sino = false;
  int last_kernel = 0;
  int64_t launches = 0;
  // kernel timing: (kind, start, stop) events, recycled through a pool
  bool profiling = false;
  struct Rec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  // pinned host rings of the volume call (grown on demand) and the event of
  // the last copy that used each buffer
  struct HostBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaEvent_t ev = nullptr;
  };
  HostBuf vin[3], vout[3];

  ~ctas_fbp() {
    DeviceGuard g(device, true);
    if (stream) cudaStreamSynchronize(stream);
    for (auto &w : ws) {
      if (w.ev_in) cudaEventDestroy(w.ev_in);
      if (w.ev_done) cudaEventDestroy(w.ev_done);
      if (w.ev_out) cudaEventDestroy(w.ev_out);
      w.raw.release();
      w.filt.release();
      w.scale.release();
      w.slice.release();
      w.part.release();
      w.minmax.release();
      w.ring_avg.release();
      w.ring.release();
      w.samples.release();
    }
    for (auto *r : {vin, vout})
      for (int i = 0; i < 3; i++) {
        if (r[i].p) cudaFreeHost(r[i].p);
        if (r[i].ev) cudaEventDestroy(r[i].ev);
      }
    err.release();
    centers.release();
    for (auto &r : recs) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
    if (err_host) cudaFreeHost(err_host);
    if (stream) cudaStreamDestroy(stream);
    if (s_in) cudaStreamDestroy(s_in);
    if (s_out) cudaStreamDestroy(s_out);
  }
};

namespace {

size_t elem_bytes(int store) { return store == 0 ? 4 : 2; }

void init_streams(ctas_fbp *h) {
  cuda_check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking), "cudaStreamCreate");
  for (auto &w : h->ws) {
    cuda_check(cudaEventCreateWithFlags(&w.ev_in, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&w.ev_done, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&w.ev_out, cudaEventDisableTiming), "cudaEventCreate");
  }
  h->err.ensure(sizeof(int));
  cuda_check(cudaMemset(h->err.p, 0, sizeof(int)), "cudaMemset");
  cuda_check(cudaMallocHost((void **)&h->err_host, sizeof(int)), "cudaMallocHost");
  *h->err_host = 0;
}

// Sizes one work set for S slices.  The padded filtered buffer is zeroed on
// allocation: its pad columns are never written afterwards.
void ensure_set(ctas_fbp *h, WorkSet &w, int64_t S, bool need_raw) {
  const int64_t N = h->N, W = h->W;
  if (need_raw) w.raw.ensure(sizeof(float) * (size_t)(S * N * W));
  if (w.filt.ensure(elem_bytes(h->store) * (size_t)(S * N * h->Wp)))
    cuda_check(cudaMemset(w.filt.p, 0, w.filt.bytes), "cudaMemset");
  if (h->store != 0) w.scale.ensure(sizeof(float) * (size_t)(S * N));
  w.slice.ensure(sizeof(float) * (size_t)(S * h->out_rows * h->out_cols));
  if (h->contrast == CTAS_ABS) {
    w.part.ensure(sizeof(float2) * (size_t)(S * ctas::kMinMaxBlocks));
    w.minmax.ensure(sizeof(float2) * (size_t)S);
  }
  if (h->ring_box > 0) {
    w.ring_avg.ensure(sizeof(float) * (size_t)(S * W));
    w.ring.ensure(sizeof(float) * (size_t)(S * W));
  }
  w.slices = std::max(w.slices, S);
}

void check_center(const ctas_fbp *h, float center) {
  // abs(center) >= ish(1)/2 (lct.cpp:614, 651): integer half width
  if (!(std::fabs(center) < (float)(h->W / 2)))
    ctas::fail(CTAS_E_CENTER, "Rotation center " + std::to_string(center) +
                                  " is outside the sinogram width " + std::to_string(h->W) + ".");
}

cudaEvent_t take_event(ctas_fbp *h) {
  if (!h->pool.empty()) {
    cudaEvent_t e = h->pool.back();
    h->pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cuda_check(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

// Brackets one launch with events when profiling is on.
struct KernelTimer {
  ctas_fbp *h;
  int kind;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  KernelTimer(ctas_fbp *h_, int kind_, cudaStream_t st_) : h(h_), kind(kind_), st(st_) {
    if (h->profiling) {
      a = take_event(h);
      cuda_check(cudaEventRecord(a, st), "cudaEventRecord");
    }
  }
  void done() {
    if (!a) return;
    cudaEvent_t b = take_event(h);
    cuda_check(cudaEventRecord(b, st), "cudaEventRecord");
    h->recs.push_back({kind, a, b});
    a = nullptr;
  }
};

// The ring-artefact correction of S slices of x (RingFilter::apply).
const float *run_ring(ctas_fbp *h, const float *x, int64_t S, WorkSet &w, cudaStream_t st) {
  if (h->ring_box <= 0) return nullptr;
  cuda_check(ctas::launch_ring(x, h->N * h->W, (int)h->N, (int)h->W, (int)S, h->ring_box,
                               w.ring_avg.as<float>(), w.ring.as<float>(), st),
             "ring filter kernel");
  h->launches += 2;
  return w.ring.as<float>();
}

// Filter S slices of x (device, dense S x N x W) into w.filt.
void run_filter(ctas_fbp *h, const float *x, int64_t S, WorkSet &w, cudaStream_t st) {
  const float *ring = run_ring(h, x, S, w, st);
  if (h->contrast == CTAS_ABS) {
    cuda_check(ctas::launch_minmax(x, h->N * h->W, h->N * h->W, (int)S, w.part.as<float2>(),
                                   w.minmax.as<float2>(), h->err.as<int>(), st, ring, (int)h->W),
               "minmax kernel");
    h->launches += 2;
  }
  ctas::FilterLaunch a{};
  a.x = x;
  a.x_slice_stride = h->N * h->W;
  a.q = w.filt.p;
  a.q_slice_stride = h->N * h->Wp;
  a.row_scale = h->store ? w.scale.as<float>() : nullptr;
  a.tw = h->dc->tw.as<float2>();
  a.gperm = h->dc->gperm.as<float>();
  a.minmax = h->contrast == CTAS_ABS ? w.minmax.as<float2>() : nullptr;
  a.N = (int)h->N;
  a.W = (int)h->W;
  a.Wp = (int)h->Wp;
  a.P = (int)h->P;
  a.zs = (int)((h->P - h->W) / 2);
  a.contrast = h->contrast;
  a.store = h->store;
  a.nradix = (int)h->radices.size();
  for (size_t k = 0; k < h->radices.size(); k++) a.radix[k] = h->radices[k];
  a.S = (int)S;
  a.guard = h->interp == CTAS_INTERP_TRUNC ? 1 : 0;
  a.ring = ring;
  a.off = (int)h->off;
  KernelTimer tm(h, CTAS_KERNEL_FILTER, st);
  cuda_check(ctas::launch_filter(a, st), "filter kernel");
  if (h->wide) {
    cuda_check(ctas::launch_halo(w.filt.as<float>(), h->N * h->Wp, (int)h->N, (int)h->W,
                                 (int)h->Wp, (int)h->off, (int)S, st),
               "halo kernel");
    h->launches += 1;
  }
  tm.done();
  h->launches += 1;
}

// centers_dev: per-slice centres (device) of S slices that all backproject
// the first filtered sinogram of w; null: S sinograms, one centre.
void run_bp(ctas_fbp *h, const WorkSet &w, int64_t S, float center, float *out, cudaStream_t st,
            const float *centers_dev = nullptr) {
  ctas::BpLaunch b{};
  b.q = w.filt.p;
  b.q_slice_stride = centers_dev ? 0 : h->N * h->Wp;
  b.centers = centers_dev;
  b.row_scale = h->store ? w.scale.as<float>() : nullptr;
  b.store = h->store;
  b.N = (int)h->N;
  b.W = (int)h->W;
  b.Wp = (int)h->Wp;
  b.tab = h->dc->tab.as<float2>();
  b.center = center;
  b.rec_cof = h->rec_cof;
  b.out = out;
  b.out_slice_stride = h->out_rows * h->out_cols;
  b.S = (int)S;
  b.out_rows = (int)h->out_rows;
  b.out_cols = (int)h->out_cols;
  b.geo_oj = h->geo_oj;
  b.geo_oi = h->geo_oi;
  b.geo_p = h->geo_p;
  b.rule = (h->flags & CTAS_FLAG_SHIPPED_INDEX) ? 1 : 0;
  b.off = (int)h->off;
  b.wide = h->wide ? 1 : 0;
  if (h->flags & CTAS_FLAG_TEST_TIMEOUT) {
    b.test_stall = 1;
    b.wait_limit = 1u << 12;
  }
  b.err = h->err.as<int>();
  b.interp = h->interp;
  b.lin = h->interp == CTAS_INTERP_LINEAR ? h->dc->lin.as<double2>() : nullptr;
  const bool fast = ctas::bp_fast_supported(b) &&
                    (h->interp == CTAS_INTERP_LINEAR || h->sines_nonneg || h->wide);
  int tile = -1;
  if (fast)  // may time the tiles once (not for the stalling test aid)
    tile = ctas::bp_fast_choose_tile(b, st, (h->flags & CTAS_FLAG_TEST_TIMEOUT) && h->tile < 0
                                                ? 1 : h->tile);
  KernelTimer tm(h, CTAS_KERNEL_BACKPROJECT, st);
  if (fast) {
    const cudaError_t e = (h->flags & CTAS_FLAG_CHECKED) ? ctas::launch_bp_fast_checked(b, st, tile)
                                                          : ctas::launch_bp_fast(b, st, tile);
    if (e != cudaSuccess)
      cuda_check(e, (std::string("backprojection kernel: ") + ctas::bp_fast_error_detail()).c_str());
    h->last_kernel = 2;
    h->last_tile = tile;
  } else {
    cuda_check(ctas::launch_bp_generic(b, st), "backprojection kernel");
    h->last_kernel = 1;
    h->last_tile = -1;
  }
  tm.done();
  h->launches += 1;
}

// Copies the filtered rows of w's first S slices to the host rows `dst`
// (dense S x N x W) on `st`.  Float32 stores: one pitched copy from w.filt,
// W samples from column off of each Wp-sample row.  16-bit stores: the
// stored samples times their row scales, formed by the unpad kernel in w.raw.
void writeback_rows(ctas_fbp *h, WorkSet &w, int64_t S, float *dst, cudaStream_t st) {
  if (h->store == 0) {
    cuda_check(cudaMemcpy2DAsync(dst, sizeof(float) * (size_t)h->W, w.filt.as<float>() + h->off,
                                 sizeof(float) * (size_t)h->Wp, sizeof(float) * (size_t)h->W,
                                 (size_t)(S * h->N), cudaMemcpyDeviceToHost, st),
               "cudaMemcpy2DAsync");
    return;
  }
  cuda_check(ctas::launch_unpad(w.filt.p, h->N * h->Wp, w.scale.as<float>(), h->store, (int)h->N,
                                (int)h->W, (int)h->Wp, (int)S, w.raw.as<float>(), h->N * h->W, st,
                                (int)h->off),
             "unpad kernel");
  h->launches += 1;
  cuda_check(cudaMemcpyAsync(dst, w.raw.p, sizeof(float) * (size_t)(S * h->N * h->W),
                             cudaMemcpyDeviceToHost, st),
             "cudaMemcpyAsync");
}

void reset_err(ctas_fbp *h, cudaStream_t st) {
  cuda_check(cudaMemsetAsync(h->err.p, 0, sizeof(int), st), "cudaMemsetAsync");
}

// Reads the device error word (synchronises `st`).
int read_err(ctas_fbp *h, cudaStream_t st) {
  cuda_check(cudaMemcpyAsync(h->err_host, h->err.p, sizeof(int), cudaMemcpyDeviceToHost, st),
             "cudaMemcpyAsync");
  cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  return *h->err_host;
}

[[noreturn]] void fail_bad_data() {
  ctas::fail(CTAS_E_DATA, "Bad absorption data (maximum is sub-zero).");
}

// Maps a non-zero device error word to a status (and clears it).
void raise_err_word(ctas_fbp *h, int w) {
  if (!w) return;
  cuda_check(cudaMemset(h->err.p, 0, sizeof(int)), "cudaMemset");
  if (w & 1) fail_bad_data();
  if (w & 4) ctas::fail(CTAS_E_TIMEOUT, "a device wait timed out in the backprojection kernel");
  if (w & 8) ctas::fail(CTAS_E_CUDA, "backprojection window check failed");
  if (w & 16) ctas::fail(CTAS_E_CUDA, "backprojection copy alignment check failed");
  ctas::fail(CTAS_E_CUDA, "device error word " + std::to_string(w));
}

// After a synchronous call: report what the kernels flagged.
void check_err_word(ctas_fbp *h, cudaStream_t st) { raise_err_word(h, read_err(h, st)); }

// For ABS contrast the reference rejects the data before touching it
// (physical.world.cpp:89-94): validate first so the caller's buffer is left
// unmodified on error.
void validate_abs(ctas_fbp *h, const float *x, int64_t S, WorkSet &w, cudaStream_t st) {
  if (h->contrast != CTAS_ABS) return;
  reset_err(h, st);
  const float *ring = run_ring(h, x, S, w, st);
  cuda_check(ctas::launch_minmax(x, h->N * h->W, h->N * h->W, (int)S, w.part.as<float2>(),
                                 w.minmax.as<float2>(), h->err.as<int>(), st, ring, (int)h->W),
             "minmax kernel");
  h->launches += 2;
  if (read_err(h, st)) fail_bad_data();
}

ctas_fbp *checked(ctas_fbp *h) {
  if (!h) ctas::fail(CTAS_E_ARG, "null handle");
  return h;
}

int64_t device_chunk(const ctas_fbp *h, int64_t S) {
  if (h->chunk > 0) return std::min<int64_t>(h->chunk, S);
  const double per = (double)h->N * h->Wp * elem_bytes(h->store) + 8.0 * h->N;
  int64_t cmax = std::max<int64_t>(1, (int64_t)(4.0e9 / per));
  const int64_t nch = (S + cmax - 1) / cmax;
  return (S + nch - 1) / nch;
}

int64_t host_chunk(const ctas_fbp *h, int64_t S) {
  if (h->chunk > 0) return std::min<int64_t>(h->chunk, S);
  const double per = (double)h->N * h->W * 4 + (double)h->N * h->Wp * elem_bytes(h->store) +
                     4.0 * h->out_rows * h->out_cols;
  int64_t cmax = std::max<int64_t>(1, (int64_t)(1.0e9 / per));
  // keep at least a few chunks so copies overlap compute
  cmax = std::min<int64_t>(cmax, std::max<int64_t>(1, (S + 3) / 4));
  const int64_t nch = (S + cmax - 1) / cmax;
  return (S + nch - 1) / nch;
}

// Chunk sizes of the host stack call: chunks of C slices, entered and left
// through chunks of 2, 4, 8, ... slices, so that the first upload and the last
// download (the copies no compute overlaps) are short.
std::vector<int64_t> chunk_plan(int64_t n, int64_t C) {
  std::vector<int64_t> up;
  int64_t ramp = 0;
  for (int64_t c = 2; c < C && ramp + 2 * c <= n / 2; c *= 2) {
    up.push_back(c);
    ramp += 2 * c;
  }
  std::vector<int64_t> plan(up.begin(), up.end());
  const int64_t mid = n - ramp, nmid = (mid + C - 1) / C;
  for (int64_t i = 0; i < nmid; i++) plan.push_back(mid * (i + 1) / nmid - mid * i / nmid);
  plan.insert(plan.end(), up.rbegin(), up.rend());
  return plan;
}

// A closable blocking queue between the volume call's threads.
template <class T> class Chan {
  std::mutex m_;
  std::condition_variable cv_;
  std::deque<T> q_;
  bool closed_ = false;

 public:
  void push(const T &v) {
    {
      std::lock_guard<std::mutex> l(m_);
      q_.push_back(v);
    }
    cv_.notify_all();
  }
  // false once closed and drained
  bool pop(T &v) {
    std::unique_lock<std::mutex> l(m_);
    cv_.wait(l, [&] { return !q_.empty() || closed_; });
    if (q_.empty()) return false;
    v = q_.front();
    q_.pop_front();
    return true;
  }
  void close() {
    {
      std::lock_guard<std::mutex> l(m_);
      closed_ = true;
    }
    cv_.notify_all();
  }
};

void ensure_host(ctas_fbp::HostBuf &b, size_t bytes) {
  if (!b.ev) cuda_check(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming), "cudaEventCreate");
  if (bytes <= b.bytes) return;
  if (b.p) cuda_check(cudaFreeHost(b.p), "cudaFreeHost");
  b.p = nullptr;
  b.bytes = 0;
  cuda_check(cudaHostAlloc(&b.p, bytes, cudaHostAllocDefault), "cudaHostAlloc");
  b.bytes = bytes;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

const char *ctas_fbp_last_error(void) { return g_last_error.c_str(); }
const char *ctas_fbp_version(void) { return "ctas_b200 fbp 0.1"; }

int ctas_filter_from_name(const char *name, int32_t *ftype) {
  return guarded([&] {
    if (!ftype) ctas::fail(CTAS_E_ARG, "null output");
    *ftype = ctas::filter_from_name(name ? name : "");
    return CTAS_OK;
  });
}

const char *ctas_filter_name(int32_t ftype) { return ctas::filter_name(ftype); }

int ctas_filter_check(int32_t ftype, float param) {
  return guarded([&] {
    ctas::filter_check(ftype, param);
    return CTAS_OK;
  });
}

int ctas_filter_parse(const char *spec, int32_t *ftype, float *param) {
  return guarded([&] {
    if (!ftype || !param) ctas::fail(CTAS_E_ARG, "null output");
    ctas::filter_parse(spec ? spec : "", ftype, param);
    return CTAS_OK;
  });
}

int ctas_filter_fill(int32_t ftype, float param, int64_t pixels, float *out) {
  return guarded([&] {
    if (!out) ctas::fail(CTAS_E_ARG, "null output");
    const auto f = ctas::filter_fill(ftype, param, pixels);
    std::memcpy(out, f.data(), sizeof(float) * f.size());
    return CTAS_OK;
  });
}

int ctas_contrast_from_name(const char *name, int32_t *contrast) {
  return guarded([&] {
    if (!contrast) ctas::fail(CTAS_E_ARG, "null output");
    *contrast = ctas::contrast_from_name(name ? name : "");
    return CTAS_OK;
  });
}

const char *ctas_contrast_name(int32_t contrast) { return ctas::contrast_name(contrast); }

int64_t ctas_fbp_padded_width(int64_t width) {
  return width >= 1 ? ctas::padded_width(width) : 0;
}

float ctas_fbp_arc(float anarc, int64_t points) { return ctas::arc_rad(anarc, points); }
float ctas_fbp_angle(float anarc, int64_t points) { return ctas::step_rad(anarc, points); }

int ctas_fbp_angle_table(float arc_deg, int64_t n, float *tab) {
  return guarded([&] {
    if (!tab || n <= 0) ctas::fail(CTAS_E_ARG, "bad arguments");
    const auto t = ctas::angle_table(arc_deg, n);
    std::memcpy(tab, t.data(), sizeof(float) * t.size());
    return CTAS_OK;
  });
}

int ctas_fbp_window(int64_t width, int32_t contrast, int32_t ftype, float fparam, int64_t pad,
                    float *G) {
  return guarded([&] {
    if (!G || width < 2) ctas::fail(CTAS_E_ARG, "bad arguments");
    const int64_t P = pad ? pad : ctas::padded_width(width);
    const auto g = ctas::ctrec_window(ftype, fparam, P, width, contrast);
    std::memcpy(G, g.data(), sizeof(float) * g.size());
    return CTAS_OK;
  });
}

float ctas_fbp_rec_cof(float pixel_size_m, float lambda_m) {
  return ctas::rec_cof(pixel_size_m, lambda_m);
}

int ctas_fbp_create(ctas_fbp **out, int64_t n_angles, int64_t width, int32_t contrast,
                    int32_t ftype, float fparam, float arc_deg, const ctas_fbp_opts *opts) {
  return guarded([&] {
    if (!out) ctas::fail(CTAS_E_ARG, "null output handle");
    *out = nullptr;
    // lct.cpp:500-503
    if (width < 2)
      ctas::fail(CTAS_E_SHAPE, "Number of pixels in the CT reconstruction less than 2.");
    if (n_angles <= 0) ctas::fail(CTAS_E_SHAPE, "Zero projections in sinogram.");
    if (contrast < 0 || contrast > 3) ctas::fail(CTAS_E_ARG, "unknown contrast");
    ctas::filter_check(ftype, fparam);
    ctas_fbp_opts o{};
    o.device = -1;
    o.tile = -1;
    o.ring_box = 0;
    if (opts && opts->struct_size) {
      std::memcpy(&o, opts, std::min<size_t>(opts->struct_size, sizeof(o)));
      if (opts->struct_size < offsetof(ctas_fbp_opts, device) + sizeof(int32_t)) o.device = -1;
      if (opts->struct_size < offsetof(ctas_fbp_opts, tile) + sizeof(int32_t)) o.tile = -1;
    }
    if (o.interp != CTAS_INTERP_TRUNC && o.interp != CTAS_INTERP_LINEAR)
      ctas::fail(CTAS_E_ARG, "unknown interpolation mode");
    if (o.store < 0 || o.store > 2) ctas::fail(CTAS_E_ARG, "unknown store precision");

    std::unique_ptr<ctas_fbp> h(new ctas_fbp());
    h->N = n_angles;
    h->W = width;
    h->P = o.pad ? o.pad : ctas::padded_width(width);
    if (o.pad && ((o.pad & (o.pad - 1)) != 0 || o.pad < width))
      ctas::fail(CTAS_E_ARG, "pad must be a power of two >= width");
    if (h->P > 16384 || h->P < 4)
      ctas::fail(CTAS_E_SHAPE, "padded width " + std::to_string(h->P) +
                                   " outside the supported range [4, 16384]");
    if (n_angles * width > (int64_t)1 << 31 || n_angles > (1 << 24))
      ctas::fail(CTAS_E_SHAPE, "sinogram too large");
    h->Wp = ctas::padded_pitch(width);
    // output geometry (extension): rows x cols pixels of pitch p (detector
    // pixels), centred like the reference's W x W grid, shifted by whole or
    // fractional output pixels; the defaults give the reference grid exactly
    h->out_rows = o.out_rows > 0 ? o.out_rows : width;
    h->out_cols = o.out_cols > 0 ? o.out_cols : width;
    if (o.out_rows < 0 || o.out_cols < 0 || o.out_pixel < 0.0 || !std::isfinite(o.out_pixel) ||
        !std::isfinite(o.out_shift_row) || !std::isfinite(o.out_shift_col))
      ctas::fail(CTAS_E_ARG, "bad output geometry");
    if (h->out_rows > 65536 || h->out_cols > 65536) ctas::fail(CTAS_E_SHAPE, "output too large");
    {
      const double pp = o.out_pixel > 0.0 ? o.out_pixel : 1.0;
      h->geo_p = (float)pp;
      h->geo_oj = (float)((width - 1) / 2.0 - (double)h->geo_p * ((h->out_rows - 1) / 2.0 - o.out_shift_row));
      h->geo_oi = (float)((width - 1) / 2.0 - (double)h->geo_p * ((h->out_cols - 1) / 2.0 - o.out_shift_col));
    }
    h->contrast = contrast;
    h->ftype = ftype;
    h->fparam = fparam;
    h->arc_deg = arc_deg;
    h->interp = o.interp;
    h->store = o.store;
    h->flags = o.flags;
    // test aid: CTAS_FBP_CHECKED=1 forces the bounds-checked staged kernel
    if (const char *e = std::getenv("CTAS_FBP_CHECKED"))
      if (e[0] == '1') h->flags |= CTAS_FLAG_CHECKED;
    h->chunk = o.chunk_slices;
    h->tile = o.tile;
    if (opts && opts->struct_size >= offsetof(ctas_fbp_opts, ring_box) + sizeof(int32_t))
      h->ring_box = o.ring_box;
    if (h->ring_box < 0 || h->ring_box > width) ctas::fail(CTAS_E_ARG, "bad ring filter width");
    h->radices = ctas::fft_radices(h->P);
    if (o.angles) {
      // explicit angle list (extension): the float table of the same form
      h->tab.resize((size_t)(2 * n_angles));
      for (int64_t i = 0; i < n_angles; i++) {
        const float th = (float)o.angles[i];
        h->tab[(size_t)(2 * i)] = std::sin(th);
        h->tab[(size_t)(2 * i + 1)] = std::cos(th);
      }
    } else {
      h->tab = ctas::angle_table(arc_deg, n_angles);
    }
    h->sines_nonneg = true;
    for (int64_t i = 0; i < n_angles; i++)
      if (h->tab[(size_t)(2 * i)] < 0.0f) h->sines_nonneg = false;
    h->wide = !h->sines_nonneg && h->interp == CTAS_INTERP_TRUNC && h->store == CTAS_STORE_F32;
    if (h->wide) {
      h->off = ctas::wide_offset(width);
      h->Wp = ctas::wide_pitch(width);
    }

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      ctas::fail(CTAS_E_NODEVICE, "no CUDA device available (there is no CPU fallback)");
    }
    if (o.device < 0) cuda_check(cudaGetDevice(&h->device), "cudaGetDevice");
    else h->device = o.device;
    if (h->device >= ndev) ctas::fail(CTAS_E_ARG, "device ordinal out of range");
    DeviceGuard g(h->device);

    // constants: twiddles, window in the FFT's output order (divided by P),
    // angle table
    auto dc = std::make_shared<Consts>();
    dc->device = h->device;
    const auto tw = ctas::fft_twiddles(h->P);
    const auto G = ctas::ctrec_window(ftype, fparam, h->P, width, contrast);
    const auto perm = ctas::fft_output_order(h->P, h->radices);
    std::vector<float> gp((size_t)h->P);
    const float invP = 1.0f / (float)h->P;  // exact: P is a power of two
    for (int64_t p = 0; p < h->P; p++) gp[(size_t)p] = G[(size_t)perm[(size_t)p]] * invP;
    dc->tw.ensure(sizeof(float) * tw.size());
    dc->gperm.ensure(sizeof(float) * gp.size());
    dc->tab.ensure(sizeof(float) * h->tab.size());
    cuda_check(cudaMemcpy(dc->tw.p, tw.data(), sizeof(float) * tw.size(), cudaMemcpyHostToDevice),
               "cudaMemcpy");
    cuda_check(cudaMemcpy(dc->gperm.p, gp.data(), sizeof(float) * gp.size(),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    cuda_check(cudaMemcpy(dc->tab.p, h->tab.data(), sizeof(float) * h->tab.size(),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    if (h->interp == CTAS_INTERP_LINEAR) {
      // FP64 projection directions for linear interpolation (extension)
      std::vector<double> lin((size_t)(2 * n_angles));
      double arc = arc_deg;
      if (arc < 1.0) arc *= (double)(n_angles - 1);
      arc *= 3.14159265358979323846 / 180.0;
      for (int64_t i = 0; i < n_angles; i++) {
        const double th = o.angles ? o.angles[i] : (double)i * arc / (double)n_angles;
        lin[(size_t)(2 * i)] = std::sin(th);
        lin[(size_t)(2 * i + 1)] = std::cos(th);
      }
      dc->lin.ensure(sizeof(double) * lin.size());
      cuda_check(cudaMemcpy(dc->lin.p, lin.data(), sizeof(double) * lin.size(),
                            cudaMemcpyHostToDevice),
                 "cudaMemcpy");
    }
    h->dc = dc;
    init_streams(h.get());
    *out = h.release();
    return CTAS_OK;
  });
}

int ctas_fbp_clone(const ctas_fbp *src, ctas_fbp **out) {
  return guarded([&] {
    if (!src || !out) ctas::fail(CTAS_E_ARG, "null argument");
    *out = nullptr;
    DeviceGuard g(src->device);
    std::unique_ptr<ctas_fbp> h(new ctas_fbp());
    h->N = src->N;
    h->W = src->W;
    h->P = src->P;
    h->Wp = src->Wp;
    h->out_rows = src->out_rows;
    h->out_cols = src->out_cols;
    h->geo_oj = src->geo_oj;
    h->geo_oi = src->geo_oi;
    h->geo_p = src->geo_p;
    h->contrast = src->contrast;
    h->ftype = src->ftype;
    h->interp = src->interp;
    h->store = src->store;
    h->fparam = src->fparam;
    h->arc_deg = src->arc_deg;
    h->rec_cof = src->rec_cof;  // lct.cpp:537
    h->flags = src->flags;
    h->chunk = src->chunk;
    h->tile = src->tile;
    h->ring_box = src->ring_box;
    h->tab = src->tab;
    h->radices = src->radices;
    h->sines_nonneg = src->sines_nonneg;
    h->wide = src->wide;
    h->off = src->off;
    h->device = src->device;
    h->dc = src->dc;
    init_streams(h.get());
    *out = h.release();
    return CTAS_OK;
  });
}

int ctas_fbp_destroy(ctas_fbp *h) {
  return guarded([&] {
    delete h;
    return CTAS_OK;
  });
}

int ctas_fbp_set_physics(ctas_fbp *h, float pixel_size_m, float lambda_m) {
  return guarded([&] {
    checked(h)->rec_cof = ctas::rec_cof(pixel_size_m, lambda_m);
    return CTAS_OK;
  });
}

int ctas_fbp_rec_shape(const ctas_fbp *h, float center, int64_t *rows, int64_t *cols) {
  return guarded([&] {
    if (!h || !rows || !cols) ctas::fail(CTAS_E_ARG, "null argument");
    // ceil(abs(center)) with ct.h's int abs(): the centre is truncated first
    *rows = h->W - 2 * (int64_t)std::abs((int)center);
    *cols = h->W;
    return CTAS_OK;
  });
}

int ctas_fbp_out_shape(const ctas_fbp *h, int64_t *rows, int64_t *cols) {
  return guarded([&] {
    if (!h || !rows || !cols) ctas::fail(CTAS_E_ARG, "null argument");
    *rows = h->out_rows;
    *cols = h->out_cols;
    return CTAS_OK;
  });
}

int ctas_fbp_sino_shape(const ctas_fbp *h, int64_t *n_angles, int64_t *width) {
  return guarded([&] {
    if (!h || !n_angles || !width) ctas::fail(CTAS_E_ARG, "null argument");
    *n_angles = h->N;
    *width = h->W;
    return CTAS_OK;
  });
}

int ctas_fbp_sino(ctas_fbp *h, float *sino) {
  return guarded([&] {
    checked(h);
    if (!sino) ctas::fail(CTAS_E_ARG, "null sinogram");
    DeviceGuard g(h->device);
    WorkSet &w = h->ws[0];
    ensure_set(h, w, 1, true);
    const size_t in_bytes = sizeof(float) * (size_t)(h->N * h->W);
    cuda_check(cudaMemcpyAsync(w.raw.p, sino, in_bytes, cudaMemcpyHostToDevice, h->stream),
               "cudaMemcpyAsync");
    validate_abs(h, w.raw.as<float>(), 1, w, h->stream);
    run_filter(h, w.raw.as<float>(), 1, w, h->stream);
    if (!(h->flags & CTAS_FLAG_NO_WRITEBACK)) {
      writeback_rows(h, w, 1, sino, h->stream);
    }
    check_err_word(h, h->stream);
    h->have_sino = true;
    return CTAS_OK;
  });
}

int ctas_fbp_repeat(ctas_fbp *h, float *slice, float center) {
  return guarded([&] {
    checked(h);
    if (!slice) ctas::fail(CTAS_E_ARG, "null slice");
    check_center(h, center);
    if (!h->have_sino) ctas::fail(CTAS_E_STATE, "repeat() called before sino()");
    DeviceGuard g(h->device);
    WorkSet &w = h->ws[0];
    run_bp(h, w, 1, center, w.slice.as<float>(), h->stream);
    cuda_check(cudaMemcpyAsync(slice, w.slice.p, sizeof(float) * (size_t)(h->out_rows * h->out_cols),
                               cudaMemcpyDeviceToHost, h->stream),
               "cudaMemcpyAsync");
    check_err_word(h, h->stream);
    return CTAS_OK;
  });
}

int ctas_fbp_reconstruct(ctas_fbp *h, float *sino, float *slice, float center) {
  return guarded([&] {
    checked(h);
    if (!sino || !slice) ctas::fail(CTAS_E_ARG, "null buffer");
    check_center(h, center);
    DeviceGuard g(h->device);
    WorkSet &w = h->ws[0];
    ensure_set(h, w, 1, true);
    const size_t in_bytes = sizeof(float) * (size_t)(h->N * h->W);
    cuda_check(cudaMemcpyAsync(w.raw.p, sino, in_bytes, cudaMemcpyHostToDevice, h->stream),
               "cudaMemcpyAsync");
    validate_abs(h, w.raw.as<float>(), 1, w, h->stream);
    run_filter(h, w.raw.as<float>(), 1, w, h->stream);
    run_bp(h, w, 1, center, w.slice.as<float>(), h->stream);
    cuda_check(cudaMemcpyAsync(slice, w.slice.p, sizeof(float) * (size_t)(h->out_rows * h->out_cols),
                               cudaMemcpyDeviceToHost, h->stream),
               "cudaMemcpyAsync");
    if (!(h->flags & CTAS_FLAG_NO_WRITEBACK)) {
      writeback_rows(h, w, 1, sino, h->stream);
    }
    check_err_word(h, h->stream);
    h->have_sino = true;
    return CTAS_OK;
  });
}

int ctas_fbp_sino_dev(ctas_fbp *h, const float *sino_dev, float *filtered_dev, void *stream) {
  return guarded([&] {
    checked(h);
    if (!sino_dev) ctas::fail(CTAS_E_ARG, "null sinogram");
    DeviceGuard g(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    WorkSet &w = h->ws[0];
    ensure_set(h, w, 1, false);
    run_filter(h, sino_dev, 1, w, st);
    if (filtered_dev) {
      cuda_check(ctas::launch_unpad(w.filt.p, h->N * h->Wp, h->store ? w.scale.as<float>() : nullptr,
                                    h->store, (int)h->N, (int)h->W, (int)h->Wp, 1, filtered_dev,
                                    h->N * h->W, st, (int)h->off),
                 "unpad kernel");
      h->launches += 1;
    }
    h->have_sino = true;
    return CTAS_OK;
  });
}

int ctas_fbp_repeat_dev(ctas_fbp *h, float *slice_dev, float center, void *stream) {
  return guarded([&] {
    checked(h);
    if (!slice_dev) ctas::fail(CTAS_E_ARG, "null slice");
    check_center(h, center);
    if (!h->have_sino) ctas::fail(CTAS_E_STATE, "repeat() called before sino()");
    DeviceGuard g(h->device);
    run_bp(h, h->ws[0], 1, center, slice_dev, (cudaStream_t)stream);
    return CTAS_OK;
  });
}

int ctas_fbp_repeat_multi_dev(ctas_fbp *h, const float *centers, int64_t n, float *slices_dev,
                              void *stream) {
  return guarded([&] {
    checked(h);
    if (!centers || !slices_dev) ctas::fail(CTAS_E_ARG, "null centres or slices");
    if (n < 1 || n > 65535) ctas::fail(CTAS_E_ARG, "number of centres must be 1 .. 65535");
    for (int64_t k = 0; k < n; k++) check_center(h, centers[k]);
    if (!h->have_sino) ctas::fail(CTAS_E_STATE, "repeat() called before sino()");
    DeviceGuard g(h->device);
    const cudaStream_t st = (cudaStream_t)stream;
    // the centre buffer may still be read by an earlier call on this stream
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    h->centers.ensure(sizeof(float) * (size_t)n);
    cuda_check(cudaMemcpyAsync(h->centers.p, centers, sizeof(float) * (size_t)n,
                               cudaMemcpyHostToDevice, st),
               "cudaMemcpyAsync");
    run_bp(h, h->ws[0], n, 0.f, slices_dev, st, h->centers.as<float>());
    return CTAS_OK;
  });
}

int ctas_fbp_reconstruct_dev(ctas_fbp *h, const float *sino_dev, float *slice_dev, float center,
                             void *stream) {
  return guarded([&] {
    checked(h);
    if (!sino_dev || !slice_dev) ctas::fail(CTAS_E_ARG, "null buffer");
    check_center(h, center);
    DeviceGuard g(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    WorkSet &w = h->ws[0];
    ensure_set(h, w, 1, false);
    run_filter(h, sino_dev, 1, w, st);
    run_bp(h, w, 1, center, slice_dev, st);
    h->have_sino = true;
    return CTAS_OK;
  });
}

int ctas_fbp_synchronize(ctas_fbp *h) {
  return guarded([&] {
    checked(h);
    DeviceGuard g(h->device);
    cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    cuda_check(cudaMemcpy(h->err_host, h->err.p, sizeof(int), cudaMemcpyDeviceToHost),
               "cudaMemcpy");
    raise_err_word(h, *h->err_host);
    return CTAS_OK;
  });
}

int ctas_fbp_reconstruct_stack_dev(ctas_fbp *h, const float *sinos_dev, float *slices_dev,
                                   int64_t n_slices, float center, void *stream) {
  return guarded([&] {
    checked(h);
    if (n_slices < 0) ctas::fail(CTAS_E_ARG, "negative slice count");
    if (n_slices == 0) return CTAS_OK;
    if (!sinos_dev || !slices_dev) ctas::fail(CTAS_E_ARG, "null buffer");
    check_center(h, center);
    DeviceGuard g(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t C = device_chunk(h, n_slices);
    WorkSet &w = h->ws[0];
    ensure_set(h, w, C, false);
    for (int64_t s0 = 0; s0 < n_slices; s0 += C) {
      const int64_t S = std::min(C, n_slices - s0);
      run_filter(h, sinos_dev + s0 * h->N * h->W, S, w, st);
      run_bp(h, w, S, center, slices_dev + s0 * h->out_rows * h->out_cols, st);
    }
    h->have_sino = (n_slices == 1);
    return CTAS_OK;
  });
}

int ctas_fbp_reconstruct_stack(ctas_fbp *h, float *sinos, float *slices, int64_t n_slices,
                               float center) {
  return guarded([&] {
    checked(h);
    if (n_slices < 0) ctas::fail(CTAS_E_ARG, "negative slice count");
    if (n_slices == 0) return CTAS_OK;
    if (!sinos || !slices) ctas::fail(CTAS_E_ARG, "null buffer");
    check_center(h, center);
    DeviceGuard g(h->device);
    const int64_t C = host_chunk(h, n_slices);
    const bool wb = !(h->flags & CTAS_FLAG_NO_WRITEBACK);
    const int64_t NW = h->N * h->W, OO = h->out_rows * h->out_cols;
    for (auto &w : h->ws) ensure_set(h, w, C, true);
    // If a later chunk fails, copies of earlier chunks into the caller's host
    // buffers may still be queued: drain all three streams before returning,
    // so the caller may free those buffers once the call has returned.
    struct Drain {
      ctas_fbp *h;
      bool armed = true;
      ~Drain() {
        if (!armed) return;
        cudaStreamSynchronize(h->s_in);
        cudaStreamSynchronize(h->stream);
        cudaStreamSynchronize(h->s_out);
        cudaGetLastError();
      }
    } drain{h};
    if (h->contrast == CTAS_ABS) {
      // validate every slice before any output is written
      for (int64_t s0 = 0; s0 < n_slices; s0 += C) {
        const int64_t S = std::min(C, n_slices - s0);
        WorkSet &w = h->ws[0];
        cuda_check(cudaMemcpyAsync(w.raw.p, sinos + s0 * NW, sizeof(float) * (size_t)(S * NW),
                                   cudaMemcpyHostToDevice, h->stream),
                   "cudaMemcpyAsync");
        validate_abs(h, w.raw.as<float>(), S, w, h->stream);
      }
    }
    // three-stream pipeline: host->device (s_in), compute (stream),
    // device->host (s_out); two work sets alternate.
    const std::vector<int64_t> plan = chunk_plan(n_slices, C);
    int64_t k = 0, s0 = 0;
    for (const int64_t S : plan) {
      WorkSet &w = h->ws[k & 1];
      if (k >= 2) cuda_check(cudaStreamWaitEvent(h->s_in, w.ev_out, 0), "cudaStreamWaitEvent");
      cuda_check(cudaMemcpyAsync(w.raw.p, sinos + s0 * NW, sizeof(float) * (size_t)(S * NW),
                                 cudaMemcpyHostToDevice, h->s_in),
                 "cudaMemcpyAsync");
      cuda_check(cudaEventRecord(w.ev_in, h->s_in), "cudaEventRecord");
      cuda_check(cudaStreamWaitEvent(h->stream, w.ev_in, 0), "cudaStreamWaitEvent");
      run_filter(h, w.raw.as<float>(), S, w, h->stream);
      run_bp(h, w, S, center, w.slice.as<float>(), h->stream);
      // 16-bit stores: the written-back rows are the stored samples times
      // their row scales, formed by the unpad kernel in w.raw
      if (wb && h->store != 0) {
        cuda_check(ctas::launch_unpad(w.filt.p, h->N * h->Wp, w.scale.as<float>(), h->store,
                                      (int)h->N, (int)h->W, (int)h->Wp, (int)S,
                                      w.raw.as<float>(), NW, h->stream, (int)h->off),
                   "unpad kernel");
        h->launches += 1;
      }
      cuda_check(cudaEventRecord(w.ev_done, h->stream), "cudaEventRecord");
      cuda_check(cudaStreamWaitEvent(h->s_out, w.ev_done, 0), "cudaStreamWaitEvent");
      cuda_check(cudaMemcpyAsync(slices + s0 * OO, w.slice.p, sizeof(float) * (size_t)(S * OO),
                                 cudaMemcpyDeviceToHost, h->s_out),
                 "cudaMemcpyAsync");
      if (wb && h->store == 0) {
        // float32 store: the filtered rows sit in w.filt, W samples from column
        // off of every Wp-sample row (slices follow at N rows each), and one
        // pitched copy brings them back
        cuda_check(cudaMemcpy2DAsync(sinos + s0 * NW, sizeof(float) * (size_t)h->W,
                                     w.filt.as<float>() + h->off, sizeof(float) * (size_t)h->Wp,
                                     sizeof(float) * (size_t)h->W, (size_t)(S * h->N),
                                     cudaMemcpyDeviceToHost, h->s_out),
                   "cudaMemcpy2DAsync");
      } else if (wb) {
        cuda_check(cudaMemcpyAsync(sinos + s0 * NW, w.raw.p, sizeof(float) * (size_t)(S * NW),
                                   cudaMemcpyDeviceToHost, h->s_out),
                   "cudaMemcpyAsync");
      }
      cuda_check(cudaEventRecord(w.ev_out, h->s_out), "cudaEventRecord");
      s0 += S;
      k++;
    }
    cuda_check(cudaStreamSynchronize(h->s_out), "cudaStreamSynchronize");
    drain.armed = false;
    check_err_word(h, h->stream);
    h->have_sino = false;
    return CTAS_OK;
  });
}

int ctas_fbp_reconstruct_volume(ctas_fbp *h, int64_t n_slices, float center, int32_t bpp,
                                float mincon, float maxcon, ctas_vol_read_fn read,
                                ctas_vol_write_fn write, void *user) {
  return guarded([&] {
    checked(h);
    if (n_slices < 0) ctas::fail(CTAS_E_ARG, "negative slice count");
    if (!read || !write) ctas::fail(CTAS_E_ARG, "null callback");
    const int64_t sb = ctas::quantize_sample_bytes(bpp);
    if (sb == 0) ctas::fail(CTAS_E_ARG, "bits per sample must be 0, +-8, +-16, +-32 or +-64");
    if (n_slices == 0) return CTAS_OK;
    check_center(h, center);
    DeviceGuard g(h->device);
    const int64_t C = host_chunk(h, n_slices);
    const int64_t NW = h->N * h->W, OO = h->out_rows * h->out_cols;
    const bool own_range = bpp != 0 && mincon == maxcon;
    for (auto &w : h->ws) {
      ensure_set(h, w, C, true);
      if (bpp != 0) w.samples.ensure((size_t)(sb * C * OO));
      if (own_range) {
        w.part.ensure(sizeof(float2) * (size_t)(C * ctas::kMinMaxBlocks));
        w.minmax.ensure(sizeof(float2) * (size_t)C);
      }
    }
    for (int i = 0; i < 3; i++) {
      ensure_host(h->vin[i], sizeof(float) * (size_t)(C * NW));
      ensure_host(h->vout[i], (size_t)(sb * C * OO));
    }
    const int64_t nch = (n_slices + C - 1) / C;
    struct Out {
      int64_t first, count;
      int buf;
    };
    Chan<int> in_free, in_full, out_free;
    Chan<Out> out_full;
    for (int i = 0; i < 3; i++) {
      in_free.push(i);
      out_free.push(i);
    }
    std::atomic<bool> stop_read{false}, stop_write{false};
    std::mutex em;
    int io_code = 0;
    std::string io_msg;
    auto io_fail = [&](int code, const std::string &m) {
      std::lock_guard<std::mutex> l(em);
      if (!io_code) {
        io_code = code;
        io_msg = m;
      }
    };
    const int dev = h->device;
    // reader: callback -> pinned input ring, in slice order
    std::thread reader([&] {
      cudaSetDevice(dev);
      for (int64_t k = 0; k < nch && !stop_read; k++) {
        int b;
        if (!in_free.pop(b)) break;
        // the buffer's previous host->device copy must be done before refilling
        const cudaError_t e = cudaEventSynchronize(h->vin[b].ev);
        if (e != cudaSuccess) {
          io_fail(CTAS_E_CUDA, std::string("cudaEventSynchronize: ") + cudaGetErrorString(e));
          break;
        }
        const int64_t s0 = k * C, cnt = std::min(C, n_slices - s0);
        const int r = read(user, s0, cnt, static_cast<float *>(h->vin[b].p));
        if (r != 0) {
          io_fail(CTAS_E_IO, "volume read callback returned " + std::to_string(r) +
                                 " for slices " + std::to_string(s0) + ".." +
                                 std::to_string(s0 + cnt - 1));
          break;
        }
        in_full.push(b);
      }
      in_full.close();
    });
    // writer: pinned output ring -> callback, in slice order
    std::thread writer([&] {
      cudaSetDevice(dev);
      Out o;
      while (out_full.pop(o)) {
        const cudaError_t e = cudaEventSynchronize(h->vout[o.buf].ev);
        if (e != cudaSuccess) {
          io_fail(CTAS_E_CUDA, std::string("cudaEventSynchronize: ") + cudaGetErrorString(e));
          stop_write = true;
          stop_read = true;
        } else if (!stop_write) {
          const int r = write(user, o.first, o.count, h->vout[o.buf].p);
          if (r != 0) {
            io_fail(CTAS_E_IO, "volume write callback returned " + std::to_string(r) +
                                   " for slices " + std::to_string(o.first) + ".." +
                                   std::to_string(o.first + o.count - 1));
            stop_write = true;
            stop_read = true;
          }
        }
        out_free.push(o.buf);
      }
    });
    // Ends both threads on every exit path; on an exception the chunks
    // already queued for writing are still written.
    struct Join {
      std::thread &r, &w;
      Chan<int> &in_free, &in_full, &out_free;
      Chan<Out> &out_full;
      std::atomic<bool> &stop_read;
      void finish() {
        stop_read = true;
        in_free.close();
        out_full.close();
        if (w.joinable()) w.join();
        out_free.close();
        if (r.joinable()) r.join();
      }
      ~Join() { finish(); }
    } join{reader, writer, in_free, in_full, out_free, out_full, stop_read};

    int64_t k = 0;
    int b;
    while (!stop_write && in_full.pop(b)) {
      const int64_t s0 = k * C, S = std::min(C, n_slices - s0);
      WorkSet &w = h->ws[k & 1];
      if (k >= 2) cuda_check(cudaStreamWaitEvent(h->s_in, w.ev_out, 0), "cudaStreamWaitEvent");
      cuda_check(cudaMemcpyAsync(w.raw.p, h->vin[b].p, sizeof(float) * (size_t)(S * NW),
                                 cudaMemcpyHostToDevice, h->s_in),
                 "cudaMemcpyAsync");
      cuda_check(cudaEventRecord(h->vin[b].ev, h->s_in), "cudaEventRecord");
      cuda_check(cudaEventRecord(w.ev_in, h->s_in), "cudaEventRecord");
      in_free.push(b);
      cuda_check(cudaStreamWaitEvent(h->stream, w.ev_in, 0), "cudaStreamWaitEvent");
      validate_abs(h, w.raw.as<float>(), S, w, h->stream);  // absorption only; synchronises
      run_filter(h, w.raw.as<float>(), S, w, h->stream);
      run_bp(h, w, S, center, w.slice.as<float>(), h->stream);
      const void *res = w.slice.p;
      if (bpp != 0) {
        if (own_range) {
          cuda_check(ctas::launch_minmax(w.slice.as<float>(), OO, OO, (int)S, w.part.as<float2>(),
                                         w.minmax.as<float2>(), nullptr, h->stream),
                     "range kernel");
          h->launches += 2;
        }
        cuda_check(ctas::launch_quantize(w.slice.as<float>(), OO, (int)S, bpp, mincon, maxcon,
                                         own_range ? w.minmax.as<float2>() : nullptr,
                                         w.samples.p, h->stream),
                   "sample conversion kernel");
        h->launches += 1;
        res = w.samples.p;
      }
      cuda_check(cudaEventRecord(w.ev_done, h->stream), "cudaEventRecord");
      int o;
      if (!out_free.pop(o)) break;
      cuda_check(cudaStreamWaitEvent(h->s_out, w.ev_done, 0), "cudaStreamWaitEvent");
      cuda_check(cudaMemcpyAsync(h->vout[o].p, res, (size_t)(sb * S * OO), cudaMemcpyDeviceToHost,
                                 h->s_out),
                 "cudaMemcpyAsync");
      cuda_check(cudaEventRecord(h->vout[o].ev, h->s_out), "cudaEventRecord");
      cuda_check(cudaEventRecord(w.ev_out, h->s_out), "cudaEventRecord");
      out_full.push(Out{s0, S, o});
      k++;
    }
    out_full.close();
    cuda_check(cudaStreamSynchronize(h->s_out), "cudaStreamSynchronize");
    check_err_word(h, h->stream);
    h->have_sino = false;
    join.finish();  // the threads' errors are final after this
    if (io_code) ctas::fail(io_code, io_msg);
    return CTAS_OK;
  });
}

int ctas_fbp_last_kernel(const ctas_fbp *h) { return h ? h->last_kernel : 0; }

int ctas_fbp_last_tile(const ctas_fbp *h) { return h ? h->last_tile : -1; }

int ctas_fbp_tile_count(void) { return ctas::bp_fast_tile_count(); }

int ctas_fbp_tile_shape(int32_t tile, int32_t *rows, int32_t *cols, int32_t *window) {
  if (!rows || !cols || !window || tile < 0 || tile >= ctas::bp_fast_tile_count()) {
    ctas::set_last_error("bad tile id or null output");
    return CTAS_E_ARG;
  }
  int ty = 0, tx = 0;
  ctas::bp_fast_tile_shape(tile, &ty, &tx);
  *rows = ty;
  *cols = tx;
  *window = ctas::bp_fast_tile_window(tile);
  return CTAS_OK;
}

int64_t ctas_fbp_kernel_launches(const ctas_fbp *h) { return h ? h->launches : 0; }

int ctas_fbp_set_profiling(ctas_fbp *h, int enable) {
  return guarded([&] {
    checked(h)->profiling = enable != 0;
    return CTAS_OK;
  });
}

int ctas_fbp_profile_read(ctas_fbp *h, int kind, double *total_ms, int64_t *launches) {
  return guarded([&] {
    checked(h);
    if (!total_ms || !launches) ctas::fail(CTAS_E_ARG, "null output");
    DeviceGuard g(h->device);
    double tot = 0.0;
    int64_t n = 0;
    std::vector<ctas_fbp::Rec> keep;
    for (auto &r : h->recs) {
      if (r.kind != kind) {
        keep.push_back(r);
        continue;
      }
      cuda_check(cudaEventSynchronize(r.b), "cudaEventSynchronize");
      float ms = 0.f;
      cuda_check(cudaEventElapsedTime(&ms, r.a, r.b), "cudaEventElapsedTime");
      tot += ms;
      n++;
      h->pool.push_back(r.a);
      h->pool.push_back(r.b);
    }
    h->recs.swap(keep);
    *total_ms = tot;
    *launches = n;
    return CTAS_OK;
  });
}

}  // extern "C"

// ===================================================================== batches
struct ctas_fbp_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<ctas_fbp_job> jobs;
  std::vector<ctas::FilterLaunch> fjobs;   // host copies (pointers into dev buffers)
  std::vector<ctas::BatchJob> bjobs;
  std::vector<int> pair_begin;
  int64_t rows = 0;
  int Wp = 0, max_pad = 0, n_pairs = 0, n_items = 0, tile = -1;
  int32_t contrast = CTAS_PHS;
  float rec_cof = 1.f;
  DevBuf filt, tables, d_fjobs, d_pairs, d_bjobs, counter, err;
  int *err_host = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;

  ~ctas_fbp_batch() {
    DeviceGuard g(device, true);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    filt.release();
    tables.release();
    d_fjobs.release();
    d_pairs.release();
    d_bjobs.release();
    counter.release();
    err.release();
    if (err_host) cudaFreeHost(err_host);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// BatchJob tile grid and work-item numbering for one tile shape.
void batch_items(ctas_fbp_batch *b, int tile) {
  int ty = 0, tx = 0;
  ctas::bp_fast_tile_shape(tile, &ty, &tx);
  int item = 0;
  for (auto &j : b->bjobs) {
    j.tiles_x = (j.W + tx - 1) / tx;
    j.tiles_y = (j.W + ty - 1) / ty;
    j.item_begin = item;
    item += j.tiles_x * j.tiles_y;
  }
  b->n_items = item;
  cuda_check(cudaMemcpy(b->d_bjobs.p, b->bjobs.data(), sizeof(ctas::BatchJob) * b->bjobs.size(),
                        cudaMemcpyHostToDevice),
             "cudaMemcpy");
}

ctas::BatchLaunch batch_launch(ctas_fbp_batch *b) {
  ctas::BatchLaunch L{};
  L.jobs = b->d_bjobs.as<ctas::BatchJob>();
  L.n_jobs = (int)b->bjobs.size();
  L.n_items = b->n_items;
  L.counter = b->counter.as<int>();
  L.err = b->err.as<int>();
  L.q = b->filt.p;
  L.Wp = b->Wp;
  L.rows = (int)b->rows;
  return L;
}

void batch_enqueue(ctas_fbp_batch *b, cudaStream_t st) {
  cuda_check(cudaMemsetAsync(b->counter.p, 0, sizeof(int), st), "cudaMemsetAsync");
  if (b->contrast == CTAS_FLT) {
    for (auto &f : b->fjobs) cuda_check(ctas::launch_filter(f, st), "filter kernel");
  } else {
    cuda_check(ctas::launch_filter_batch(b->d_fjobs.as<ctas::FilterLaunch>(), b->d_pairs.as<int>(),
                                         (int)b->fjobs.size(), b->n_pairs, b->max_pad, st),
               "filter kernel");
  }
  const cudaError_t e = ctas::launch_bp_batch(batch_launch(b), b->tile, st);
  if (e != cudaSuccess)
    cuda_check(e, (std::string("backprojection kernel: ") + ctas::bp_fast_error_detail()).c_str());
}

}  // namespace

extern "C" {

int ctas_fbp_batch_create(ctas_fbp_batch **out, const ctas_fbp_job *jobs, int64_t n_jobs,
                          int32_t contrast, int32_t ftype, float fparam, float arc_deg,
                          float pixel_size_m, float lambda_m, const ctas_fbp_opts *opts) {
  return guarded([&] {
    if (!out || !jobs || n_jobs <= 0) ctas::fail(CTAS_E_ARG, "bad job list");
    *out = nullptr;
    if (contrast != CTAS_PHS && contrast != CTAS_REF && contrast != CTAS_FLT)
      ctas::fail(CTAS_E_UNSUPPORTED, "batches take PHS, REF or FLT contrast");
    ctas::filter_check(ftype, fparam);
    ctas_fbp_opts o{};
    o.tile = -1;
    if (opts && opts->struct_size)
      std::memcpy(&o, opts, std::min<size_t>(opts->struct_size, sizeof(o)));
    if (opts && opts->struct_size && opts->struct_size < offsetof(ctas_fbp_opts, tile) + sizeof(int32_t))
      o.tile = -1;
    if (o.interp != CTAS_INTERP_TRUNC || o.store != CTAS_STORE_F32 || o.angles)
      ctas::fail(CTAS_E_UNSUPPORTED, "batches use the float32 truncation path and uniform angles");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      ctas::fail(CTAS_E_NODEVICE, "no CUDA device available (there is no CPU fallback)");
    }
    std::unique_ptr<ctas_fbp_batch> b(new ctas_fbp_batch());
    cuda_check(cudaGetDevice(&b->device), "cudaGetDevice");
    DeviceGuard g(b->device);
    b->contrast = contrast;
    b->rec_cof = ctas::rec_cof(pixel_size_m, lambda_m);
    const int rule = (o.flags & CTAS_FLAG_SHIPPED_INDEX) ? 1 : 0;
    b->jobs.assign(jobs, jobs + n_jobs);
    // layout: every sinogram's padded rows in one buffer of the widest pitch
    int64_t Wp = 0;
    for (auto &j : b->jobs) {
      if (!j.sino_dev || !j.slice_dev) ctas::fail(CTAS_E_ARG, "null buffer in job list");
      if (j.width < 2 || j.n_angles <= 0) ctas::fail(CTAS_E_SHAPE, "bad sinogram shape in job list");
      if (!(std::fabs(j.center) < (float)(j.width / 2)))
        ctas::fail(CTAS_E_CENTER, "Rotation center " + std::to_string(j.center) +
                                      " is outside the sinogram width " + std::to_string(j.width) + ".");
      Wp = std::max(Wp, ctas::padded_pitch(j.width));
    }
    Wp = std::max<int64_t>(Wp, 192);  // at least the widest staged window
    b->Wp = (int)Wp;
    // tables: twiddles per FFT length, window per (width, length), angle table per count
    std::vector<float> host;
    auto put = [&](const std::vector<float> &v) {
      while (host.size() % 64) host.push_back(0.f);  // 256-byte aligned pieces
      const size_t off = host.size();
      host.insert(host.end(), v.begin(), v.end());
      return off;
    };
    std::map<int64_t, size_t> tw_off, tab_off;
    std::map<std::pair<int64_t, int64_t>, size_t> g_off;
    std::vector<std::array<size_t, 3>> offs;
    int64_t row = 0;
    int pairs = 0;
    for (auto &j : b->jobs) {
      const int64_t P = o.pad ? o.pad : ctas::padded_width(j.width);
      if (o.pad && ((o.pad & (o.pad - 1)) != 0 || o.pad < j.width))
        ctas::fail(CTAS_E_ARG, "pad must be a power of two >= every width");
      if (P > 16384) ctas::fail(CTAS_E_SHAPE, "padded width above 16384");
      if (!tw_off.count(P)) tw_off[P] = put(ctas::fft_twiddles(P));
      const auto key = std::make_pair(j.width, P);
      if (!g_off.count(key)) {
        const auto G = ctas::ctrec_window(ftype, fparam, P, j.width, contrast);
        const auto perm = ctas::fft_output_order(P, ctas::fft_radices(P));
        std::vector<float> gp((size_t)P);
        const float invP = 1.0f / (float)P;
        for (int64_t p = 0; p < P; p++) gp[(size_t)p] = G[(size_t)perm[(size_t)p]] * invP;
        g_off[key] = put(gp);
      }
      if (!tab_off.count(j.n_angles)) {
        const auto tab = ctas::angle_table(arc_deg, j.n_angles);
        for (int64_t i = 0; i < j.n_angles; i++)
          if (tab[(size_t)(2 * i)] < 0.0f)
            ctas::fail(CTAS_E_UNSUPPORTED, "batches need every sine >= 0 (an arc of at most 180)");
        tab_off[j.n_angles] = put(tab);
      }
      offs.push_back({tw_off[P], g_off[key], tab_off[j.n_angles]});
      b->max_pad = std::max<int>(b->max_pad, (int)P);
      ctas::FilterLaunch f{};
      f.x = j.sino_dev;
      f.x_slice_stride = j.n_angles * j.width;
      f.q_slice_stride = j.n_angles * Wp;
      f.N = (int)j.n_angles;
      f.W = (int)j.width;
      f.Wp = (int)Wp;
      f.P = (int)P;
      f.zs = (int)((P - j.width) / 2);
      f.contrast = contrast;
      f.store = 0;
      const auto rad = ctas::fft_radices(P);
      f.nradix = (int)rad.size();
      for (size_t k = 0; k < rad.size(); k++) f.radix[k] = rad[k];
      f.S = 1;
      f.guard = 1;
      f.q = reinterpret_cast<void *>((uintptr_t)row);  // row index until the buffer exists
      b->fjobs.push_back(f);
      b->pair_begin.push_back(pairs);
      pairs += (int)((j.n_angles + 1) / 2);
      ctas::BatchJob bj{};
      bj.W = (int)j.width;
      bj.N = (int)j.n_angles;
      bj.row0 = (int)row;
      bj.c = j.center;
      bj.rec_cof = b->rec_cof;
      bj.out = j.slice_dev;
      bj.rule = rule;
      b->bjobs.push_back(bj);
      row += j.n_angles;
    }
    b->rows = row;
    b->n_pairs = pairs;
    if (row * Wp > ((int64_t)1 << 34)) ctas::fail(CTAS_E_SHAPE, "batch too large");
    b->filt.ensure(sizeof(float) * (size_t)(row * Wp));
    cuda_check(cudaMemset(b->filt.p, 0, b->filt.bytes), "cudaMemset");
    b->tables.ensure(sizeof(float) * host.size());
    cuda_check(cudaMemcpy(b->tables.p, host.data(), sizeof(float) * host.size(),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    float *tb = b->tables.as<float>();
    for (size_t k = 0; k < b->fjobs.size(); k++) {
      auto &f = b->fjobs[k];
      const int64_t r0 = (int64_t)(uintptr_t)f.q;
      f.q = b->filt.as<float>() + r0 * Wp;
      f.tw = reinterpret_cast<const float2 *>(tb + offs[k][0]);
      f.gperm = tb + offs[k][1];
      b->bjobs[k].tab = reinterpret_cast<const float2 *>(tb + offs[k][2]);
    }
    b->d_fjobs.ensure(sizeof(ctas::FilterLaunch) * b->fjobs.size());
    cuda_check(cudaMemcpy(b->d_fjobs.p, b->fjobs.data(), sizeof(ctas::FilterLaunch) * b->fjobs.size(),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    b->d_pairs.ensure(sizeof(int) * b->pair_begin.size());
    cuda_check(cudaMemcpy(b->d_pairs.p, b->pair_begin.data(), sizeof(int) * b->pair_begin.size(),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy");
    b->d_bjobs.ensure(sizeof(ctas::BatchJob) * b->bjobs.size());
    b->counter.ensure(sizeof(int));
    b->err.ensure(sizeof(int));
    cuda_check(cudaMemset(b->err.p, 0, sizeof(int)), "cudaMemset");
    cuda_check(cudaMallocHost((void **)&b->err_host, sizeof(int)), "cudaMallocHost");
    cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");

    // autotune the tile on this batch (timing the whole filter + backprojection)
    const int ntiles = ctas::bp_fast_tile_count();
    if (o.tile >= 0 && o.tile < ntiles) {
      b->tile = o.tile;
    } else {
      cudaEvent_t e0, e1;
      cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
      cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
      int best = -1;
      try {
        best = ctas::bp_fast_search(
            [&](int t) {
              b->tile = t;
              batch_items(b.get(), t);
              cuda_check(cudaEventRecord(e0, b->stream), "cudaEventRecord");
              batch_enqueue(b.get(), b->stream);
              cuda_check(cudaEventRecord(e1, b->stream), "cudaEventRecord");
              cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
              float ms = 0.f;
              cudaEventElapsedTime(&ms, e0, e1);
              return ms;
            },
            true);
      } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      o.tile = best >= 0 ? best : 0;
      b->tile = o.tile;
    }
    batch_items(b.get(), b->tile);
    // capture the run as a graph
    cuda_check(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal),
               "cudaStreamBeginCapture");
    try {
      batch_enqueue(b.get(), b->stream);
    } catch (...) {
      cudaGraph_t tmp = nullptr;
      cudaStreamEndCapture(b->stream, &tmp);
      if (tmp) cudaGraphDestroy(tmp);
      throw;
    }
    cuda_check(cudaStreamEndCapture(b->stream, &b->graph), "cudaStreamEndCapture");
    cuda_check(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
    cuda_check(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
    *out = b.release();
    return CTAS_OK;
  });
}

int ctas_fbp_batch_run(ctas_fbp_batch *b, void *stream) {
  return guarded([&] {
    if (!b) ctas::fail(CTAS_E_ARG, "null batch");
    DeviceGuard g(b->device);
    cuda_check(cudaGraphLaunch(b->exec, (cudaStream_t)stream), "cudaGraphLaunch");
    return CTAS_OK;
  });
}

int ctas_fbp_batch_run_loop(ctas_fbp_batch *b, void *stream) {
  return guarded([&] {
    if (!b) ctas::fail(CTAS_E_ARG, "null batch");
    DeviceGuard g(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    for (size_t k = 0; k < b->fjobs.size(); k++) {
      const auto &f = b->fjobs[k];
      const auto &j = b->bjobs[k];
      cuda_check(ctas::launch_filter(f, st), "filter kernel");
      ctas::BpLaunch bl{};
      bl.q = f.q;
      bl.q_slice_stride = (int64_t)j.N * b->Wp;
      bl.store = 0;
      bl.N = j.N;
      bl.W = j.W;
      bl.Wp = b->Wp;
      bl.tab = j.tab;
      bl.center = j.c;
      bl.rec_cof = j.rec_cof;
      bl.out = j.out;
      bl.out_slice_stride = (int64_t)j.W * j.W;
      bl.S = 1;
      bl.err = b->err.as<int>();
      bl.interp = 0;
      bl.out_rows = j.W;
      bl.out_cols = j.W;
      bl.geo_oj = 0.f;
      bl.geo_oi = 0.f;
      bl.geo_p = 1.f;
      bl.rule = j.rule;
      cudaError_t e;
      if (ctas::bp_fast_supported(bl))
        e = ctas::launch_bp_fast(bl, st, ctas::bp_fast_choose_tile(bl, st, -1));
      else
        e = ctas::launch_bp_generic(bl, st);
      if (e != cudaSuccess) cuda_check(e, "backprojection kernel");
    }
    return CTAS_OK;
  });
}

int ctas_fbp_batch_synchronize(ctas_fbp_batch *b) {
  return guarded([&] {
    if (!b) ctas::fail(CTAS_E_ARG, "null batch");
    DeviceGuard g(b->device);
    cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    cuda_check(cudaMemcpy(b->err_host, b->err.p, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    const int w = *b->err_host;
    if (w) {
      cuda_check(cudaMemset(b->err.p, 0, sizeof(int)), "cudaMemset");
      if (w & 4) ctas::fail(CTAS_E_TIMEOUT, "a device wait timed out in the backprojection kernel");
      ctas::fail(CTAS_E_CUDA, "device error word " + std::to_string(w));
    }
    return CTAS_OK;
  });
}

int ctas_fbp_batch_tile(const ctas_fbp_batch *b) { return b ? b->tile : -1; }

int ctas_fbp_batch_destroy(ctas_fbp_batch *b) {
  return guarded([&] {
    delete b;
    return CTAS_OK;
  });
}

}  // extern "C"
