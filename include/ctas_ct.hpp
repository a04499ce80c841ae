// ctas_ct.hpp -- C++ mirror of the ctas reconstruction interface over the C ABI.
//
// The classes keep the names, constructors and methods of ctas
// src/common/ct.h (Filter :87-162, CTrec :235-298, raxis :327-329, ts_add, and
// the AverageGradient class of lct.cpp:800-915), plus the ct tool's slice loop
// over a whole volume (reconstruct_volume, ct.cpp:156-206) and of Contrast
// (src/common/physical.world.h:18-45), so code written against the reference
// (ct.cpp:156-236, axis.cpp:143-155) compiles against this header with only
// its include changed.  Errors are thrown as CtasErr carrying the C-ABI
// status, where the reference throws CtasErr from throw_error
// (common.world.cpp:165-170).
//
// Arrays: any 2-D float container with contiguous row-major storage works as
// the reference's `Map` -- a blitz::Array<float,2> (data(), extent(i),
// resize(rows, cols)) or the small ctas_b200::Map below.
#pragma once

#include <array>
#include <cstdint>
#include <exception>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "ctas_axis.h"
#include "ctas_fbp.h"
#include "ctas_ts.h"
#include "ctas_volume.h"

namespace ctas_b200 {

class CtasErr : public std::runtime_error {
 public:
  int code;
  CtasErr(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void throw_on(int rc) {
  if (rc != CTAS_OK) throw CtasErr(rc, ctas_fbp_last_error());
}

// A two-element shape type: blitz::TinyVector<T,2> (the reference's Shape<2>,
// matrix.world.h:222; blitz marks its length with `numElements`) or
// std::array<T,2>.  blitz::Range, which is also constructible from two
// integers, has neither, so Array::resize(Shape) stays unambiguous.
namespace detail {
template <class V, class = void> struct is_shape2 : std::false_type {};
template <class V>
struct is_shape2<V, std::enable_if_t<(int)V::numElements == 2>> : std::true_type {};
template <class T> struct is_shape2<std::array<T, 2>, void> : std::true_type {};
}  // namespace detail

// recShape()'s result: the reference returns Shape<2> (ct.h:272-274); this
// converts to it (or to std::array<T,2>) so `map.resize(rec.recShape())`
// compiles for a blitz::Array (axis.cpp:149) and for Map below.
struct RecShape {
  int64_t rows = 0, cols = 0;
  int64_t operator()(int i) const { return i == 0 ? rows : cols; }
  int64_t operator[](int i) const { return i == 0 ? rows : cols; }
  template <class V, std::enable_if_t<detail::is_shape2<V>::value, int> = 0> operator V() const {
    V v;
    v[0] = (std::decay_t<decltype(v[0])>)rows;
    v[1] = (std::decay_t<decltype(v[1])>)cols;
    return v;
  }
};

// Segment (matrix.world.h:275-290, size at matrix.world.cpp:41-50): rows
// [from, orgsz + to) for to <= 0, [from, to) otherwise.
struct Segment {
  int64_t from = 0, to = 0;
  int64_t begin() const { return from; }
  int64_t size(int64_t orgsz = 0) const {
    const int64_t sz = to + (to > 0 ? 0 : orgsz) - from;
    if (sz <= 0) throw std::runtime_error("Range size: Negative size for the range.");
    if (to > 0 && orgsz > 0 && orgsz < to)
      throw std::runtime_error("Range size: Range is larger than original size.");
    return sz;
  }
  int64_t end(int64_t orgsz = 0) const { return from + size(orgsz); }
  explicit operator bool() const { return from || to; }
};

// recCrop()'s result (Crop<2>, matrix.world.h:303-327): a row and a column
// segment; shape() is Crop::shape.  The cropped view of a blitz::Array a of
// R rows is a(Range(c.rows.begin(), c.rows.end(R) - 1), Range::all()).
struct RecCrop {
  Segment rows, cols;
  RecShape shape(int64_t R, int64_t C) const {
    return RecShape{rows.size(R), cols.size(C)};
  }
  explicit operator bool() const { return bool(rows) || bool(cols); }
};

// Contiguous row-major float image, for callers without blitz.
class Map {
  std::vector<float> d_;
  int64_t r_ = 0, c_ = 0;

 public:
  Map() = default;
  Map(int64_t rows, int64_t cols) : d_((size_t)(rows * cols)), r_(rows), c_(cols) {}
  // like blitz::Array::resize: keeps the data when the shape is unchanged
  void resize(int64_t rows, int64_t cols) {
    if (rows == r_ && cols == c_) return;
    d_.assign((size_t)(rows * cols), 0.0f);
    r_ = rows;
    c_ = cols;
  }
  void resize(const RecShape &s) { resize(s.rows, s.cols); }
  float *data() { return d_.data(); }
  const float *data() const { return d_.data(); }
  int64_t extent(int i) const { return i == 0 ? r_ : c_; }
  float &operator()(int64_t j, int64_t i) { return d_[(size_t)(j * c_ + i)]; }
  float operator()(int64_t j, int64_t i) const { return d_[(size_t)(j * c_ + i)]; }
};

namespace detail {
template <class M, class = void> struct has_contig : std::false_type {};
template <class M>
struct has_contig<M, std::void_t<decltype(std::declval<const M &>().isStorageContiguous())>>
    : std::true_type {};

template <class M> float *checked_data(M &m, int64_t rows, int64_t cols, const char *what) {
  if (m.extent(0) != rows || m.extent(1) != cols)
    throw CtasErr(CTAS_E_SHAPE, std::string("Wrong ") + what + " shape.");
  if constexpr (has_contig<M>::value) {
    if (!m.isStorageContiguous())
      throw CtasErr(CTAS_E_ARG, std::string(what) + " must be stored contiguously.");
  }
  return const_cast<float *>(m.data());
}

template <class S, class = void> struct call_index : std::false_type {};
template <class S>
struct call_index<S, std::void_t<decltype(std::declval<const S &>()(0))>> : std::true_type {};
template <class S> int64_t shape_at(const S &s, int i) {
  if constexpr (call_index<S>::value) return (int64_t)s(i);
  else return (int64_t)s[i];
}
}  // namespace detail

class Contrast {
 public:
  typedef enum { ABS = CTAS_ABS, REF = CTAS_REF, PHS = CTAS_PHS, FLT = CTAS_FLT } Cntype;
  Contrast(Cntype cn = FLT) : c_(cn) {}
  Contrast(const std::string &name) {
    int32_t v = 0;
    throw_on(ctas_contrast_from_name(name.c_str(), &v));
    c_ = (Cntype)v;
  }
  Cntype contrast() const { return c_; }
  std::string name() const { return ctas_contrast_name(c_); }
  bool operator==(const Contrast &o) const { return c_ == o.c_; }
  bool operator!=(const Contrast &o) const { return c_ != o.c_; }

 private:
  Cntype c_;
};

class Filter {
 public:
  typedef enum {
    NONE = 0, RAMP, BARLETT, WELCH, PARZEN, HANN, HAMMING, BLACKMAN, LANCKZOS, KAISER, GAUSS,
    SHEPP_LOGAN = CTAS_FILTER_SHEPP_LOGAN, COSINE = CTAS_FILTER_COSINE
  } Ftype;
  Filter(Ftype tp = RAMP, float as = 0) : t_(tp), p_(as) { throw_on(ctas_filter_check(t_, p_)); }
  Filter(const std::string &name, float as = 0) : p_(as) {
    int32_t v = 0;
    throw_on(ctas_filter_from_name(name.c_str(), &v));
    t_ = (Ftype)v;
    throw_on(ctas_filter_check(t_, p_));
  }
  Ftype filter() const { return t_; }
  float param() const { return p_; }
  std::string name() const { return ctas_filter_name(t_); }
  std::vector<float> fill(int pixels) const {
    std::vector<float> f((size_t)pixels);
    throw_on(ctas_filter_fill(t_, p_, pixels, f.data()));
    return f;
  }
  bool operator==(const Filter &o) const { return t_ == o.t_; }
  bool operator!=(const Filter &o) const { return t_ != o.t_; }

 private:
  Ftype t_;
  float p_;
};

// _conversion(Filter*, string) (lct.cpp:236-248)
inline bool _conversion(Filter *val, const std::string &in) {
  int32_t t = 0;
  float p = 0;
  if (ctas_filter_parse(in.c_str(), &t, &p) != CTAS_OK) return false;
  *val = Filter((Filter::Ftype)t, p);
  return true;
}

class CTrec {
 public:
  template <class Shape>
  CTrec(const Shape &sinoshape, Contrast cn, float anarc = 180, const Filter &ft = Filter(),
        const ctas_fbp_opts *opts = nullptr)
      : N_(detail::shape_at(sinoshape, 0)), W_(detail::shape_at(sinoshape, 1)) {
    throw_on(ctas_fbp_create(&h_, N_, W_, cn.contrast(), ft.filter(), ft.param(), anarc, opts));
    throw_on(ctas_fbp_out_shape(h_, &R_, &C_));
  }
  // per-thread clone (lct.cpp:529-545)
  CTrec(CTrec &other) : N_(other.N_), W_(other.W_), R_(other.R_), C_(other.C_) {
    throw_on(ctas_fbp_clone(other.h_, &h_));
  }
  CTrec &operator=(const CTrec &) = delete;
  ~CTrec() { ctas_fbp_destroy(h_); }

  // (W - 2k) x W, k = |(int)center| (ct.h:272-274; see ctas_fbp_rec_shape)
  RecShape recShape(const float center = 0.0) const {
    int64_t r = 0, c = 0;
    throw_on(ctas_fbp_rec_shape(h_, center, &r, &c));
    return RecShape{r, c};
  }
  // rows [k, W - k), all columns (ct.h:276-279), k as in recShape
  RecCrop recCrop(const float center = 0.0) const {
    int64_t r = 0, c = 0;
    throw_on(ctas_fbp_rec_shape(h_, center, &r, &c));
    const int64_t k = (W_ - r) / 2;
    return RecCrop{Segment{k, -k}, Segment{}};
  }
  void setPhysics(float pixelSize = 0.0, float lambda = 0.0) {
    throw_on(ctas_fbp_set_physics(h_, pixelSize, lambda));
  }
  template <class M> void sino(M &sinogram) {
    throw_on(ctas_fbp_sino(h_, detail::checked_data(sinogram, N_, W_, "sinogram")));
  }
  template <class M> void repeat(M &slice, float center) {
    slice.resize(R_, C_);
    throw_on(ctas_fbp_repeat(h_, detail::checked_data(slice, R_, C_, "slice"), center));
  }
  template <class M> void reconstruct(M &sinogram, M &slice, float center) {
    float *s = detail::checked_data(sinogram, N_, W_, "sinogram");
    slice.resize(R_, C_);
    throw_on(ctas_fbp_reconstruct(h_, s, detail::checked_data(slice, R_, C_, "slice"), center));
  }
  // The device path is the only path; these keep the reference's call sites
  // (ct.cpp:174, 221) valid.
  void doOnGPU() {}
  void allowCPU() {}

  template <class M>
  static void reconstruct(M &sinogram, M &slice, Contrast cn, float arc = 180,
                          const Filter &ft = Filter(), float center = 0, float pixelSize = 0.0,
                          float lambda = 0.0) {
    CTrec rec(std::array<int64_t, 2>{sinogram.extent(0), sinogram.extent(1)}, cn, arc, ft);
    rec.setPhysics(pixelSize, lambda);
    rec.reconstruct(sinogram, slice, center);
  }

  ctas_fbp *handle() { return h_; }

 private:
  ctas_fbp *h_ = nullptr;
  int64_t N_, W_, R_ = 0, C_ = 0;
};

// Rotation-axis search (ct.h:327-329, lct.cpp:792-1297), as axis.cpp:117-170
// calls it.  The sinogram is an absorption (transmission) image.
class AverageGradient {
 public:
  template <class M>
  explicit AverageGradient(M &sino, const float anarc = 180) {
    const float *d = detail::checked_data(sino, sino.extent(0), sino.extent(1), "sinogram");
    throw_on(ctas_ag_create(&h_, d, sino.extent(0), sino.extent(1), anarc, -1));
  }
  AverageGradient(const AverageGradient &) = delete;
  AverageGradient &operator=(const AverageGradient &) = delete;
  ~AverageGradient() { ctas_ag_destroy(h_); }
  float apply(const float axisR) {
    float v = 0.f;
    throw_on(ctas_ag_apply(h_, &axisR, 1, &v));
    return v;
  }

 private:
  ctas_ag *h_ = nullptr;
};

template <class M>
float raxis(M &sino, const float anarc, const float maxDev, int algo = 0) {
  const float *d = detail::checked_data(sino, sino.extent(0), sino.extent(1), "sinogram");
  float ax = 0.f;
  throw_on(ctas_raxis(d, sino.extent(0), sino.extent(1), anarc, maxDev, algo, -1, &ax, nullptr));
  return ax;
}

template <class M>
float raxis(M &proj0, M &proj180, const float maxDev) {
  if (proj0.extent(0) != proj180.extent(0) || proj0.extent(1) != proj180.extent(1))
    throw CtasErr(CTAS_E_SHAPE, "Different shapes of input projections.");
  const float *a = detail::checked_data(proj0, proj0.extent(0), proj0.extent(1), "proj0");
  const float *b = detail::checked_data(proj180, proj0.extent(0), proj0.extent(1), "proj180");
  float ax = 0.f;
  throw_on(ctas_raxis_pair(a, b, proj0.extent(0), proj0.extent(1), maxDev, -1, &ax));
  return ax;
}

// ts_add (ct.h, lct.cpp:731-787), as ts.cpp:209-217 calls it: filters
// `projection` in place and adds it into `result`.  Each call sets up the
// window and FFT tables for the image shape, like the reference's per-call
// FFTW plans; for a series, keep a ctas_ts handle (ctas_ts.h).
template <class M>
void ts_add(M &projection, M &result, const Filter &filter, const float center,
            const Contrast contrast, const float angle, const int plane) {
  const int64_t rows = projection.extent(0), cols = projection.extent(1);
  if (result.extent(0) != rows || result.extent(1) != cols)
    throw CtasErr(CTAS_E_SHAPE, "tomosynthesis: The size of the result array does not match "
                                "the requested reconstruction.");
  float *p = detail::checked_data(projection, rows, cols, "projection");
  float *r = detail::checked_data(result, rows, cols, "result");
  ctas_ts *h = nullptr;
  throw_on(ctas_ts_create(&h, rows, cols, filter.filter(), filter.param(), contrast.contrast(), -1));
  const int rc = ctas_ts_add(h, p, r, center, angle, plane, 0);
  ctas_ts_destroy(h);
  throw_on(rc);
}

// The ct tool's slice loop (ct.cpp:156-206: readTo, RingFilter::apply,
// reconstruct, save) over a whole volume as one streamed call
// (ctas_volume.h).  read(first, count, float *sinos) fills `count` sinograms
// [count][N][W]; write(first, count, const void *slices) takes `count` slices
// of bpp samples (0 = float32).  Each is called from one library thread, in
// slice order; an exception thrown by either ends the call and is rethrown.
template <class Read, class Write>
void reconstruct_volume(CTrec &rec, int64_t n_slices, float center, Read &&read, Write &&write,
                        int bpp = 0, float mincon = 0, float maxcon = 0) {
  struct Ctx {
    std::remove_reference_t<Read> &r;
    std::remove_reference_t<Write> &w;
    std::exception_ptr err_r, err_w;  // one per callback thread
  } ctx{read, write, nullptr, nullptr};
  ctas_vol_read_fn rd = [](void *u, int64_t first, int64_t count, float *sinos) -> int {
    auto *c = static_cast<Ctx *>(u);
    try {
      c->r(first, count, sinos);
      return 0;
    } catch (...) {
      c->err_r = std::current_exception();
      return -1;
    }
  };
  ctas_vol_write_fn wr = [](void *u, int64_t first, int64_t count, const void *slices) -> int {
    auto *c = static_cast<Ctx *>(u);
    try {
      c->w(first, count, slices);
      return 0;
    } catch (...) {
      c->err_w = std::current_exception();
      return -1;
    }
  };
  const int rc = ctas_fbp_reconstruct_volume(rec.handle(), n_slices, center, bpp, mincon, maxcon,
                                             rd, wr, &ctx);
  if (ctx.err_r) std::rethrow_exception(ctx.err_r);
  if (ctx.err_w) std::rethrow_exception(ctx.err_w);
  throw_on(rc);
}

}  // namespace ctas_b200
