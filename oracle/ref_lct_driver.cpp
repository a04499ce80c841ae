// ref_lct_driver.cpp -- C entry points over the reference's own reconstruction
// code, for the oracle.  Test infrastructure only: compiled (by
// oracle/Makefile, target `lct`) together with the reference's
// common.world.cpp, parallel.world.cpp, physical.world.cpp and
// matrix.world.cpp where they lie, against the stand-in headers of
// oracle/shim/ (no OpenCL device, so CTrec takes its CPU path,
// lct.cpp:519-524; FFTW computed in double).  The reference's lct.cpp is
// compiled as part of this translation unit (the #include below reads it
// where it lies), which makes its file-local AverageGradient class reachable.
// Nothing here restates the reference: every result comes from its code.
//
// Buffers: row-major float32.  A sinogram buffer passed in must hold
// n_angles * width + 1 floats, the last one 0: the reference's padding reads
// one sample past each row (lct.cpp:579-584), which for the last row is the
// float after the array.
#include <malloc.h>
#include <sys/time.h>

#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include "lct.cpp"

namespace {

thread_local std::string t_msg;

template <class F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (CtasErr &e) {
    t_msg = e.consume();
    return -1;
  } catch (std::exception &e) {
    t_msg = e.what();
    return -2;
  } catch (...) {
    t_msg = "unknown exception";
    return -3;
  }
}

Map wrap(float *p, long rows, long cols) {
  return Map(p, Shape<2>(rows, cols), blitz::neverDeleteData);
}

void copy_out(const Map &m, float *dst) {
  const Map s(safe(m));
  std::memcpy(dst, s.data(), sizeof(float) * (size_t)s.size());
}

double now_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

}  // namespace

extern "C" {

const char *ref_lct_last_error(void) { return t_msg.c_str(); }

// Make the C library serve every allocation of at least `bytes` with fresh
// zeroed pages (mallopt M_MMAP_THRESHOLD), for the AverageGradient calls
// above.  Process-wide: call it in a process of its own.
int ref_lct_mmap_threshold(int bytes) { return mallopt(M_MMAP_THRESHOLD, bytes) == 1 ? 0 : -1; }

// Filter::fill(filt, P) (lct.cpp:122-209): the window before the P/W scaling.
int ref_lct_filter_fill(int P, int ftype, float fparam, float *out) {
  return guarded([&] {
    Filter f((Filter::Ftype)ftype, fparam);
    Line w(P);
    f.fill(w);
    copy_out(Map(w.data(), Shape<2>(1, P), blitz::neverDeleteData), out);
  });
}

// CTrec::reconstruct (lct.cpp:649-685) of one sinogram: the sinogram buffer
// (n*w + 1 floats) is filtered in place as the reference does; slice gets w*w.
int ref_lct_reconstruct(float *sino, float *slice, long n, long w, int contrast, int ftype,
                        float fparam, float arc, float center, float pixel_size, float lambda) {
  return guarded([&] {
    Map s = wrap(sino, n, w);
    Map out;
    CTrec rec(Shape<2>(n, w), Contrast((Contrast::Cntype)contrast), arc,
              Filter((Filter::Ftype)ftype, fparam));
    rec.setPhysics(pixel_size, lambda);
    rec.reconstruct(s, out, center);
    copy_out(out, slice);
  });
}

// CTrec::sino then CTrec::repeat for each centre (lct.cpp:600-647): slices
// gets n_centers * w * w floats.
int ref_lct_sino_repeat(float *sino, float *slices, long n, long w, int contrast, int ftype,
                        float fparam, float arc, const float *centers, int n_centers,
                        float pixel_size, float lambda) {
  return guarded([&] {
    Map s = wrap(sino, n, w);
    CTrec rec(Shape<2>(n, w), Contrast((Contrast::Cntype)contrast), arc,
              Filter((Filter::Ftype)ftype, fparam));
    rec.setPhysics(pixel_size, lambda);
    rec.sino(s);
    for (int k = 0; k < n_centers; k++) {
      Map out;
      rec.repeat(out, centers[k]);
      copy_out(out, slices + (size_t)k * w * w);
    }
  });
}

// RingFilter::apply (lct.cpp:295-327), in place.
int ref_lct_ring(float *sino, long n, long w, long box) {
  return guarded([&] {
    Map s = wrap(sino, n, w);
    RingFilter rf(w, box);
    rf.apply(s);
  });
}

// ts_add (lct.cpp:739-787): the projection (rows x cols) is filtered in place
// and its backprojection added into result (rows x cols).
int ref_lct_ts_add(float *projection, float *result, long rows, long cols, int ftype,
                   float fparam, float center, int contrast, float angle, int plane) {
  return guarded([&] {
    Map p = wrap(projection, rows, cols);
    Map r = wrap(result, rows, cols);
    ts_add(p, r, Filter((Filter::Ftype)ftype, fparam), center,
           Contrast((Contrast::Cntype)contrast), angle, plane);
  });
}

// AverageGradient(sino, arc).apply(axis) (lct.cpp:804-915) for each axis
// position: the metric the rotation-axis search minimises.  Evaluated on the
// object that filtered the sinogram.  Its constructor filters a copy of the
// sinogram that it allocates itself (lct.cpp:830-831), so the padding's read
// one float past the last row (lct.cpp:579-584) sees whatever follows that
// allocation; results are reproducible only where that float is 0, e.g. for
// blocks the C library maps fresh from the system (ref_lct_mmap_threshold).  (raxis's own thread pool evaluates it on
// copies, AGinThread::beforeThread; a CTrec copy does not copy the sinogram it
// references (lct.cpp:529-545), so on a machine without OpenCL every copy's
// CPU backprojection reads an empty array and the process crashes.  The
// search itself therefore cannot run here; its metric can.)
int ref_lct_ag_metric(const float *sino, long n, long w, float arc, const float *axes,
                      int n_axes, float *out) {
  return guarded([&] {
    Map s(Shape<2>(n, w));
    std::memcpy(s.data(), sino, sizeof(float) * (size_t)(n * w));
    AverageGradient ag(s, arc);
    for (int k = 0; k < n_axes; k++) out[k] = ag.apply(axes[k]);
  });
}

// raxis(sino, arc, maxDev, algo) (lct.cpp:1133-1215): the rotation-axis
// search; the sinogram is not modified.  Only algorithm 0 (the 0/180 degree
// projection correlation) runs on a machine without OpenCL; see above.
int ref_lct_raxis(const float *sino, long n, long w, float arc, float max_dev, int algo,
                  float *axis) {
  return guarded([&] {
    Map s(Shape<2>(n, w));
    std::memcpy(s.data(), sino, sizeof(float) * (size_t)(n * w));
    *axis = raxis(s, arc, max_dev, algo);
  });
}

// The ct tool's slice loop (ct.cpp:156-236, RecInThread): n_slices sinograms
// (n*w each, contiguous, read-only here) reconstructed by `threads` threads of
// the reference's InThread pool, one CTrec clone per thread, each thread
// copying its slice's sinogram into its own (n*w + 1)-float buffer before
// reconstructing it, as the tool reads each slice into a per-thread map.
// slices gets n_slices * w * w floats (nullable: results dropped).  Returns
// the wall time of the loop in *seconds.
int ref_lct_reconstruct_stack(const float *sinos, float *slices, long n_slices, long n, long w,
                              int contrast, int ftype, float fparam, float arc, float center,
                              float pixel_size, float lambda, int threads, double *seconds) {
  return guarded([&] {
    class Loop : public InThread {
      const float *sinos;
      float *slices;
      long n_slices, n, w;
      float center, pixel_size, lambda;
      CTrec canon;
      std::mutex m;
      struct Mine {
        CTrec *rec;
        std::vector<float> buf;
        Map out;
      };
      std::unordered_map<pthread_t, Mine *> mine;

      bool inThread(long idx) override {
        if (idx >= n_slices) return false;
        const pthread_t me = pthread_self();
        Mine *my = nullptr;
        {
          std::lock_guard<std::mutex> l(m);
          auto it = mine.find(me);
          if (it != mine.end()) my = it->second;
        }
        if (!my) {
          my = new Mine;
          my->rec = n_slices == 1 ? &canon : new CTrec(canon);
          my->rec->setPhysics(pixel_size, lambda);
          my->buf.assign((size_t)(n * w + 1), 0.0f);
          std::lock_guard<std::mutex> l(m);
          mine.emplace(me, my);
        }
        std::memcpy(my->buf.data(), sinos + (size_t)idx * n * w, sizeof(float) * (size_t)(n * w));
        my->buf[(size_t)(n * w)] = 0.0f;
        Map s = wrap(my->buf.data(), n, w);
        my->rec->reconstruct(s, my->out, center);
        if (slices) copy_out(my->out, slices + (size_t)idx * w * w);
        return true;
      }

     public:
      Loop(const float *s, float *o, long ns, long n_, long w_, int cn, int ft, float fp,
           float arc, float c, float ps, float lam)
          : InThread(false, "", 0), sinos(s), slices(o), n_slices(ns), n(n_), w(w_),
            center(c), pixel_size(ps), lambda(lam),
            canon(Shape<2>(n_, w_), Contrast((Contrast::Cntype)cn), arc,
                  Filter((Filter::Ftype)ft, fp)) {}
      ~Loop() {
        for (auto &e : mine) {
          if (e.second->rec != &canon) delete e.second->rec;
          delete e.second;
        }
      }
    };
    Loop loop(sinos, slices, n_slices, n, w, contrast, ftype, fparam, arc, center, pixel_size,
              lambda);
    const double t0 = now_s();
    loop.execute(threads);
    *seconds = now_s() - t0;
  });
}

}  // extern "C"
