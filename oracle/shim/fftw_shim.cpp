// fftw_shim.cpp -- the transforms declared by shim/fftw3.h, in double
// precision.  Test infrastructure only (it stands in for FFTW3f when the
// reference's lct.cpp is compiled for the oracle).  Every transform is the
// exact DFT of its definition evaluated by FFT in double and rounded to float
// once at the end: a radix-2 FFT for power-of-two lengths, Bluestein's
// chirp-z algorithm (through a power-of-two FFT) for other lengths.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "fftw3.h"

namespace {

using cd = std::complex<double>;

// exp(sign * 2 pi i k / n) with k reduced mod n in integers first
cd unit_root(int64_t k, int64_t n, int sign) {
  k %= n;
  if (k < 0) k += n;
  const double a = 2.0 * M_PI * (double)k / (double)n;
  return cd(std::cos(a), sign * std::sin(a));
}

struct Pow2Fft {
  int n = 0;
  std::vector<cd> w;  // w[k] = exp(-2 pi i k / n), k < n/2
  explicit Pow2Fft(int n_) : n(n_), w(n_ / 2 > 0 ? n_ / 2 : 1) {
    for (int k = 0; k < n / 2; k++) w[k] = unit_root(k, n, -1);
  }
  // in-place, sign -1 (forward) or +1 (backward, unnormalised)
  void run(cd *a, int sign) const {
    for (int i = 1, j = 0; i < n; i++) {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int step = n / len;
      for (int i = 0; i < n; i += len)
        for (int k = 0; k < len / 2; k++) {
          cd t = w[k * step];
          if (sign > 0) t = std::conj(t);
          const cd u = a[i + k], v = a[i + k + len / 2] * t;
          a[i + k] = u + v;
          a[i + k + len / 2] = u - v;
        }
    }
  }
};

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// complex DFT of any length n >= 1
struct Dft {
  int n = 0, m = 0;
  Pow2Fft *direct = nullptr, *conv = nullptr;
  std::vector<cd> chirp;           // exp(-i pi k^2 / n), k < n
  std::vector<cd> kernel_fft[2];   // FFT of the conjugate chirp, per sign
  explicit Dft(int n_) : n(n_) {
    if (is_pow2(n)) {
      direct = new Pow2Fft(n);
      return;
    }
    m = 1;
    while (m < 2 * n - 1) m <<= 1;
    conv = new Pow2Fft(m);
    chirp.resize(n);
    for (int64_t k = 0; k < n; k++) chirp[k] = unit_root(k * k, 2 * (int64_t)n, -1);
    for (int s = 0; s < 2; s++) {
      // sign -1 uses the chirp as is; sign +1 its conjugate
      std::vector<cd> b(m, cd(0, 0));
      for (int k = 0; k < n; k++) {
        const cd c = s == 0 ? std::conj(chirp[k]) : chirp[k];
        b[k] = c;
        if (k) b[m - k] = c;
      }
      conv->run(b.data(), -1);
      kernel_fft[s] = std::move(b);
    }
  }
  ~Dft() {
    delete direct;
    delete conv;
  }
  void run(cd *a, int sign) const {
    if (direct) {
      direct->run(a, sign);
      return;
    }
    const int s = sign < 0 ? 0 : 1;
    std::vector<cd> x(m, cd(0, 0));
    for (int k = 0; k < n; k++) x[k] = a[k] * (s == 0 ? chirp[k] : std::conj(chirp[k]));
    conv->run(x.data(), -1);
    for (int k = 0; k < m; k++) x[k] *= kernel_fft[s][k];
    conv->run(x.data(), +1);
    const double inv = 1.0 / (double)m;
    for (int k = 0; k < n; k++) a[k] = x[k] * inv * (s == 0 ? chirp[k] : std::conj(chirp[k]));
  }
};

enum Kind { R2HC, HC2R, C1D, C2D };

}  // namespace

struct ctas_shim_fftwf_plan_s {
  Kind kind;
  int n0 = 0, n1 = 0, sign = -1;
  void *in = nullptr, *out = nullptr;
  Dft *d0 = nullptr, *d1 = nullptr;
};

namespace {

void r2r(const ctas_shim_fftwf_plan_s *p, const float *in, float *out) {
  const int n = p->n0;
  std::vector<cd> a(n);
  if (p->kind == R2HC) {
    for (int j = 0; j < n; j++) a[j] = cd(in[j], 0.0);
    p->d0->run(a.data(), -1);
    std::vector<float> o(n);
    for (int k = 0; k <= n / 2; k++) o[k] = (float)a[k].real();
    for (int k = 1; k < (n + 1) / 2; k++) o[n - k] = (float)a[k].imag();
    for (int k = 0; k < n; k++) out[k] = o[k];
  } else {
    for (int k = 0; k <= n / 2; k++) {
      const double re = in[k];
      const double im = (k > 0 && k < (n + 1) / 2) ? (double)in[n - k] : 0.0;
      a[k] = cd(re, im);
      if (k > 0 && n - k != k) a[n - k] = cd(re, -im);
    }
    p->d0->run(a.data(), +1);
    for (int j = 0; j < n; j++) out[j] = (float)a[j].real();
  }
}

void dft(const ctas_shim_fftwf_plan_s *p, const fftwf_complex *in, fftwf_complex *out) {
  const int r = p->kind == C2D ? p->n0 : 1, c = p->kind == C2D ? p->n1 : p->n0;
  std::vector<cd> a((size_t)r * c);
  for (size_t k = 0; k < a.size(); k++) a[k] = cd(in[k][0], in[k][1]);
  for (int i = 0; i < r; i++) (p->kind == C2D ? p->d1 : p->d0)->run(&a[(size_t)i * c], p->sign);
  if (p->kind == C2D) {
    std::vector<cd> col(r);
    for (int j = 0; j < c; j++) {
      for (int i = 0; i < r; i++) col[i] = a[(size_t)i * c + j];
      p->d0->run(col.data(), p->sign);
      for (int i = 0; i < r; i++) a[(size_t)i * c + j] = col[i];
    }
  }
  for (size_t k = 0; k < a.size(); k++) {
    out[k][0] = (float)a[k].real();
    out[k][1] = (float)a[k].imag();
  }
}

}  // namespace

extern "C" {

fftwf_plan fftwf_plan_r2r_1d(int n, float *in, float *out, fftw_r2r_kind kind, unsigned) {
  if (n < 1) return nullptr;
  auto *p = new ctas_shim_fftwf_plan_s;
  p->kind = kind == FFTW_R2HC ? R2HC : HC2R;
  p->n0 = n;
  p->in = in;
  p->out = out;
  p->d0 = new Dft(n);
  return p;
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned) {
  if (n < 1) return nullptr;
  auto *p = new ctas_shim_fftwf_plan_s;
  p->kind = C1D;
  p->n0 = n;
  p->sign = sign;
  p->in = in;
  p->out = out;
  p->d0 = new Dft(n);
  return p;
}

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned) {
  if (n0 < 1 || n1 < 1) return nullptr;
  auto *p = new ctas_shim_fftwf_plan_s;
  p->kind = C2D;
  p->n0 = n0;
  p->n1 = n1;
  p->sign = sign;
  p->in = in;
  p->out = out;
  p->d0 = new Dft(n0);
  p->d1 = new Dft(n1);
  return p;
}

void fftwf_execute_r2r(const fftwf_plan p, float *in, float *out) { r2r(p, in, out); }

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out) {
  dft(p, in, out);
}

void fftwf_execute(const fftwf_plan p) {
  if (p->kind == R2HC || p->kind == HC2R)
    r2r(p, static_cast<const float *>(p->in), static_cast<float *>(p->out));
  else
    dft(p, static_cast<const fftwf_complex *>(p->in), static_cast<fftwf_complex *>(p->out));
}

void fftwf_destroy_plan(fftwf_plan p) {
  if (!p) return;
  delete p->d0;
  delete p->d1;
  delete p;
}

}  // extern "C"
