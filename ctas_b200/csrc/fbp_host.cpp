// fbp_host.cpp -- host-side set-up of the FBP path.
//
// This translation unit must be compiled without -ffast-math and with
// -ffp-contract=off: the window and the angle table are float computations
// whose rounding the reference fixes (lct.cpp:150-203, 512-517), and the
// backprojection index rule depends on the angle table bit for bit.
#include "fbp_host.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdlib>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace ctas {

void fail(int code, const std::string &msg) { throw Error{code, msg}; }

static std::string upper(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

int64_t padded_width(int64_t W) {
  // zidth(pow(2, ceil(log2(2*ish(1)-1))))
  return (int64_t)std::pow(2.0, std::ceil(std::log2((double)(2 * W - 1))));
}

bool filter_known(int32_t t) { return (t >= 0 && t <= 10) || t == 100 || t == 101; }

const char *filter_name(int32_t t) {
  switch (t) {
  case 0: return "NONE";
  case 1: return "RAMP";
  case 2: return "BARLETT";
  case 3: return "WELCH";
  case 4: return "PARZEN";
  case 5: return "HANN";
  case 6: return "HAMMING";
  case 7: return "BLACKMAN";
  case 8: return "LANCKZOS";
  case 9: return "KAISER";
  case 10: return "GAUSS";
  case 100: return "SHEPP-LOGAN";
  case 101: return "COSINE";
  default: return nullptr;
  }
}

int32_t filter_from_name(const std::string &_name) {
  const std::string n = upper(_name);
  if (n == "NONE") return 0;
  if (n.empty() || n == "RAMP") return 1;
  if (n == "BARLETT") return 1;  // the reference maps BARLETT to RAMP (lct.cpp:74)
  if (n == "WELCH") return 3;
  if (n == "PARZEN") return 4;
  if (n == "HANN") return 5;
  if (n == "HAMMING") return 6;
  if (n == "BLACKMAN") return 7;
  if (n == "LANCKZOS") return 8;
  if (n == "KAISER") return 9;
  if (n == "GAUSS") return 10;
  if (n == "SHEPP-LOGAN" || n == "SHEPP_LOGAN" || n == "SHEPPLOGAN") return 100;
  if (n == "COSINE" || n == "COS") return 101;
  fail(-4, "The string \"" + _name + "\" does not describe any known filter.");
}

void filter_check(int32_t t, float p) {
  if (!filter_known(t)) fail(-4, "Unknown filter type " + std::to_string(t) + ".");
  if (t == 9 && p < 0.0f)
    fail(-4, "Alpha parameter of Kaiser filter must be non-negative (set " +
                 std::to_string(p) + "). ");
  if (t == 10 && p <= 0.0f)
    fail(-4, "Sigma parameter of Guass filter must be strictly positive (set " +
                 std::to_string(p) + "). ");
}

void filter_parse(const std::string &in, int32_t *ftype, float *param) {
  const auto idx = in.find(':');
  float p = 0.0f;
  std::string name = in;
  if (idx != std::string::npos) {
    const std::string v = in.substr(idx + 1);
    char *end = nullptr;
    p = std::strtof(v.c_str(), &end);
    if (v.empty() || end == v.c_str() || *end != '\0')
      fail(-4, "Can not convert \"" + v + "\" to a float filter parameter.");
    name = in.substr(0, idx);
  }
  const int32_t t = filter_from_name(name);
  filter_check(t, p);
  *ftype = t;
  *param = p;
}

int32_t contrast_from_name(const std::string &_name) {
  const std::string n = upper(_name);
  if (n == "A" || n == "ABS" || n == "ABSORPTION") return 0;
  if (n == "R" || n == "REF" || n == "REFRACTION") return 1;
  if (n == "P" || n == "PHS" || n == "PHASE") return 2;
  if (n == "F" || n == "FLT" || n == "FILTERED") return 3;
  fail(-1, "The string \"" + _name + "\" does not describe any known contrast.");
}

const char *contrast_name(int32_t c) {
  switch (c) {
  case 0: return "ABSORPTION";
  case 1: return "REFRACTION";
  case 2: return "PHASE";
  case 3: return "FILTERED";
  default: return nullptr;
  }
}

// ------------------------------------------------------------------ FFT (host)
// Iterative radix-2 transform in double; sign -1 forward, +1 unnormalised
// inverse.  Used once per object to evaluate FFTW's HC2R of the Ram-Lak taps.
static void fft_double(std::vector<std::complex<double>> &a, int sign) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; i++) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const size_t half = len / 2;
    for (size_t k = 0; k < half; k++) {
      const double ang = sign * 2.0 * M_PI * (double)k / (double)len;
      const std::complex<double> w(std::cos(ang), std::sin(ang));
      for (size_t s = 0; s < n; s += len) {
        const std::complex<double> u = a[s + k], v = a[s + k + half] * w;
        a[s + k] = u + v;
        a[s + k + half] = u - v;
      }
    }
  }
}

// Window factor for one float frequency fp (lct.cpp:155-200).  The reference
// evaluates the trigonometric windows in double and stores them in a float.
// I0(x) = sum_k ((x/2)^2)^k / (k!)^2, summed until a term stops changing the
// sum (the reference calls GSL's gsl_sf_bessel_I0, lct.cpp:192-193).
static double bessel_i0(double x) {
  const double q = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; k++) {
    term *= q / ((double)k * (double)k);
    const double next = sum + term;
    if (next == sum) break;
    sum = next;
  }
  return sum;
}

// Window factors of lct.cpp:155-198 in the order the reference's build
// evaluates them: its -ffast-math flag (CMakeLists.txt:10-11) lets GCC
// reassociate the polynomial windows even at -O0, so PARZEN is computed as
// (3 fp^3 - 6 fp^2) + 1 and BLACKMAN as (0.5 cos + 0.08 cos2) + 0.42 -- the
// window a ctas binary actually uses, on its CPU and on its OpenCL path alike.
static float window_factor(int32_t t, float fp, float alsig) {
  switch (t) {
  case 0:
  case 1: return 1.0f;
  case 2: return 1 - fp;
  case 3: return 1 - fp * fp;
  case 4: return (fp <= 0.5f) ? (fp * (fp * fp) * 3.0f - fp * fp * 6.0f) + 1.0f
                              : (fp * (fp * fp) + 1.0f) * 2.0f;
  case 5: return (float)((std::cos((double)fp * M_PI) + 1.0) * 0.5);
  case 6: return (float)(std::cos((double)fp * M_PI) * 0.46 + 0.54);
  case 7: return (float)((std::cos((double)fp * M_PI) * 0.5 +
                          std::cos((double)fp * (2 * M_PI)) * 0.08) + 0.42);
  case 8: return (float)((fp == 0.0f) ? 0.0 : std::fabs(std::sin(M_PI * fp)) / fp);
  case 9: return (float)(bessel_i0((double)(alsig * std::sqrt(1 - fp * fp))) /
                         bessel_i0((double)alsig));
  case 10: return std::pow(2.0f, (-fp) * fp / (alsig * alsig));
  case 100: {
    const double x = M_PI * (double)fp / 2.0;
    return (float)(fp == 0.0f ? 1.0 : std::sin(x) / x);
  }
  case 101: return (float)std::cos(M_PI * (double)fp / 2.0);
  default: return 1.0f;
  }
}

std::vector<float> filter_fill(int32_t ftype, float param, int64_t pixels) {
  if (pixels <= 0) fail(-1, "Zero-size filter requested.");
  filter_check(ftype, param);
  const int64_t P = pixels;
  // Ram-Lak taps (lct.cpp:132-135), float as the reference stores them.
  std::vector<float> f((size_t)P, 0.0f);
  f[0] = 0.25f;
  // lct.cpp:134 writes -1.0/(pix*pix*M_PI*M_PI); the reference's -ffast-math
  // build folds it to (-1/pi^2) / (pix*pix), with pix*pix an int product
  const double neg_inv_pi2 = -1.0 / (M_PI * M_PI);
  for (int64_t pix = 1; pix < P / 2; pix += 2)
    f[(size_t)pix] = (float)(neg_inv_pi2 / (double)(int)(pix * pix));
  // FFTW_HC2R (lct.cpp:138-140): the taps are the real half-spectrum
  // r_0..r_{P/2}; imaginary parts are zero.  For P a power of two the FFT in
  // double is used; other lengths fall back to the direct sum.
  std::vector<double> H((size_t)P);
  if ((P & (P - 1)) == 0) {
    std::vector<std::complex<double>> a((size_t)P);
    for (int64_t k = 0; k <= P / 2 && k < P; k++) {
      a[(size_t)k] = f[(size_t)k];
      if (k > 0 && k < P - k) a[(size_t)(P - k)] = f[(size_t)k];
    }
    fft_double(a, +1);
    for (int64_t m = 0; m < P; m++) H[(size_t)m] = a[(size_t)m].real();
    // make the even symmetry exact
    for (int64_t m = 1; m < (P + 1) / 2; m++) H[(size_t)(P - m)] = H[(size_t)m];
  } else {
    for (int64_t m = 0; m < P; m++) {
      double s = f[0];
      for (int64_t k = 1; 2 * k < P; k++)
        s += 2.0 * f[(size_t)k] * std::cos(2.0 * M_PI * (double)((k * m) % P) / (double)P);
      if (P % 2 == 0) s += f[(size_t)(P / 2)] * ((m & 1) ? -1.0 : 1.0);
      H[(size_t)m] = s;
    }
  }
  std::vector<float> out((size_t)P);
  for (int64_t pix = 0; pix < P; pix++) {
    float fp = (float)((pix < P / 2) ? pix : P - pix);
    fp = (float)((double)fp * (2.0 / (double)P));
    const float w = window_factor(ftype, fp, param);
    const float h = (float)H[(size_t)pix];
    out[(size_t)pix] = (float)((double)h * ((double)w / 2.0));  // lct.cpp:203
  }
  return out;
}

std::vector<float> ctrec_window(int32_t ftype, float param, int64_t P, int64_t W,
                                int32_t contrast) {
  std::vector<float> G = filter_fill(ftype, param, P);
  const float s = (float)P / (float)W;                     // lct.cpp:506
  for (auto &g : G) g = g * s;
  if (contrast == 1) G[0] = 0.0f;                           // lct.cpp:507-508
  return G;
}

float arc_rad(float anarc, int64_t points) {
  float r = anarc;
  if (r < 1.0f) r *= (float)(points - 1);
  r = (float)((double)r * (M_PI / 180));
  return r;
}

float step_rad(float anarc, int64_t points) {
  float r = anarc;
  if (r > 1.0f && points > 1) r /= (float)(points - 1);
  r = (float)((double)r * (M_PI / 180));
  return r;
}

std::vector<float> angle_table(float arc_deg, int64_t N) {
  std::vector<float> tab((size_t)(2 * N));
  const float arc = arc_rad(arc_deg, N);
  for (int64_t i = 0; i < N; i++) {
    const float th = (float)i * arc / (float)N;
    tab[(size_t)(2 * i)] = std::sin(th);      // float overloads: sinf / cosf
    tab[(size_t)(2 * i + 1)] = std::cos(th);
  }
  return tab;
}

float rec_cof(float pixel_size, float lambda) {
  float r = 1.0f;
  if (lambda > 0.0f) r = (float)((double)r * ((double)lambda / (2 * M_PI)));
  if (pixel_size > 0.0f) r = (float)((double)r * (M_PI / (double)pixel_size));
  return r;
}

std::vector<float> fft_twiddles(int64_t P) {
  std::vector<float> tw((size_t)(2 * P));
  fft_twiddles_into(P, tw.data());
  return tw;
}

std::vector<int> fft_radices(int64_t P) {
  int lg = 0;
  while ((int64_t(1) << lg) < P) lg++;
  std::vector<int> r;
  int rem = lg % 3;
  for (int s = 0; s < lg / 3; s++) r.push_back(8);
  if (rem == 1) r.push_back(2);
  if (rem == 2) r.push_back(4);
  return r;
}

std::vector<int64_t> fft_output_order(int64_t P, const std::vector<int> &radices) {
  // Decimation in frequency: after the stage with radix R_s and stride h_s the
  // digit q_s of the output position p = sum q_s h_s selects the residue of the
  // frequency k = q_0 + R_0 q_1 + R_0 R_1 q_2 + ...
  std::vector<int64_t> h(radices.size());
  int64_t L = P;
  for (size_t s = 0; s < radices.size(); s++) {
    h[s] = L / radices[s];
    L = h[s];
  }
  std::vector<int64_t> perm((size_t)P);
  for (int64_t p = 0; p < P; p++) {
    int64_t k = 0, mult = 1;
    for (size_t s = 0; s < radices.size(); s++) {
      const int64_t q = (p / h[s]) % radices[s];
      k += q * mult;
      mult *= radices[s];
    }
    perm[(size_t)p] = k;
  }
  return perm;
}

}  // namespace ctas

// ---------------------------------------------- forms without allocation
namespace ctas {

void filter_fill_into(int32_t ftype, float param, int64_t P, float *out, void *scratch) {
  if (P <= 0 || (P & (P - 1)) != 0) fail(-1, "window length must be a power of two");
  filter_check(ftype, param);
  auto *a = static_cast<std::complex<double> *>(scratch);
  for (int64_t k = 0; k < P; k++) a[k] = 0.0;
  // Ram-Lak taps (lct.cpp:132-135) as the real half-spectrum of FFTW's HC2R
  a[0] = 0.25f;
  const double neg_inv_pi2 = -1.0 / (M_PI * M_PI);  // as folded by the reference's build
  for (int64_t pix = 1; pix < P / 2; pix += 2) {
    const float f = (float)(neg_inv_pi2 / (double)(int)(pix * pix));
    a[pix] = f;
    a[P - pix] = f;
  }
  // unnormalised inverse transform in place (iterative radix 2)
  for (int64_t i = 1, j = 0; i < P; i++) {
    int64_t bit = P >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int64_t len = 2; len <= P; len <<= 1) {
    const int64_t half = len / 2;
    for (int64_t k = 0; k < half; k++) {
      const double ang = 2.0 * M_PI * (double)k / (double)len;
      const std::complex<double> w(std::cos(ang), std::sin(ang));
      for (int64_t s = 0; s < P; s += len) {
        const std::complex<double> u = a[s + k], v = a[s + k + half] * w;
        a[s + k] = u + v;
        a[s + k + half] = u - v;
      }
    }
  }
  for (int64_t m = 1; m < (P + 1) / 2; m++) a[P - m] = a[m];
  for (int64_t pix = 0; pix < P; pix++) {
    float fp = (float)((pix < P / 2) ? pix : P - pix);
    fp = (float)((double)fp * (2.0 / (double)P));
    const float w = window_factor(ftype, fp, param);
    const float h = (float)a[pix].real();
    out[pix] = (float)((double)h * ((double)w / 2.0));
  }
}

void angle_table_into(float arc_deg, int64_t N, float *tab) {
  const float arc = arc_rad(arc_deg, N);
  for (int64_t i = 0; i < N; i++) {
    const float th = (float)i * arc / (float)N;
    tab[2 * i] = std::sin(th);
    tab[2 * i + 1] = std::cos(th);
  }
}

void fft_twiddles_into(int64_t P, float *tw) {
  // Per stage s of the radix plan (radix R_s, stride h_s = P / (R_0 ... R_s),
  // step t_s = P / (R_s h_s)): h_s entries of four floats, (w^(m t_s),
  // w^(4 m t_s)) for m < h_s, w = exp(-2 pi i / P), one 16-byte load per
  // butterfly with consecutive threads on consecutive entries.  In all fewer
  // than P / 2 entries: the rest of the 2 P floats is zero.
  auto put = [&](int64_t k, float *o) {
    const double a = -2.0 * M_PI * (double)(k % P) / (double)P;
    o[0] = (float)std::cos(a);
    o[1] = (float)std::sin(a);
  };
  std::fill(tw, tw + 2 * P, 0.0f);
  // the radix plan of fft_radices, formed here without allocating
  int lg = 0;
  while ((int64_t(1) << lg) < P) lg++;
  const int n8 = lg / 3, last = lg % 3 == 1 ? 2 : lg % 3 == 2 ? 4 : 0;
  int64_t h = P, off = 0;
  for (int s = 0; s < n8 + (last ? 1 : 0); s++) {
    const int R = s < n8 ? 8 : last;
    h /= R;
    const int64_t t = P / (R * h);
    for (int64_t m = 0; m < h; m++) {
      put(m * t, tw + 4 * (off + m));
      put(4 * m * t, tw + 4 * (off + m) + 2);
    }
    off += h;
  }
}

int64_t fft_output_frequency(int64_t P, int64_t p) {
  int lg = 0;
  while ((int64_t(1) << lg) < P) lg++;
  int radix[8], ns = 0;
  for (int s = 0; s < lg / 3; s++) radix[ns++] = 8;
  if (lg % 3 == 1) radix[ns++] = 2;
  if (lg % 3 == 2) radix[ns++] = 4;
  int64_t h = P, k = 0, mult = 1;
  for (int s = 0; s < ns; s++) {
    h /= radix[s];
    k += ((p / h) % radix[s]) * mult;
    mult *= radix[s];
  }
  return k;
}

}  // namespace ctas
