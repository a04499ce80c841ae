/*
 * fbp_oracle.c -- CPU restatement of the ctas parallel-beam FBP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * ctas_b200/: it is loaded by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py, never by the product library.
 *
 * It restates, function by function, the reference code of ctas v0.7.0
 * (paths relative to the ctas source tree):
 *
 *   orc_padded_width      src/common/lct.cpp:490        (zidth = 2^ceil(log2(2W-1)))
 *   orc_filter_fill       src/common/lct.cpp:122-209    (Filter::fill) and :505-508
 *   orc_arc               src/common/lct.cpp:470-476    (arcO)
 *   orc_angle_table       src/common/lct.cpp:512-517
 *   orc_deabs             src/common/physical.world.cpp:88-100 (deAbs)
 *   orc_prepare_sino      src/common/lct.cpp:569-597    (prepare_sino) + :280-291 (filter_line)
 *   orc_bp_compat         src/common/lct.cpp:688-729    (reconstructOnCPU) == src/common/ct.cl:14-43
 *   orc_rec_cof           src/common/lct.cpp:558-566    (setPhysics)
 *
 * Two precisions are offered:
 *   - "compat" (FP32): every operation the reference performs in float is
 *     performed in float here, in the reference's order; the FFTW float
 *     transform (absent from this container) is stood in for by an FP64 FFT
 *     whose output is rounded to float.
 *   - "fp64": the same algorithm with FP64 samples, FP64 window and FP64
 *     accumulation.  In compat-index mode the detector index of every update
 *     is still chosen with the reference's float expression (index choice is
 *     geometry, not precision).
 * A linear-interpolation backprojector (an extension with no reference
 * counterpart) is provided in FP64 only.
 *
 * Parity pin: the backprojector is checked bit for bit against the
 * reference's own ct.cl compiled for the host (oracle/Makefile -> oracle/_ref);
 * the filter stage depends on FFTW, which is absent, and is pinned only by
 * known-answer tests (impulse response, independent numpy FFT).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Filter::Ftype (src/common/ct.h:92-132), extended with two windows that the
 * reference does not have. */
enum {
  ORC_NONE = 0, ORC_RAMP, ORC_BARLETT, ORC_WELCH, ORC_PARZEN, ORC_HANN,
  ORC_HAMMING, ORC_BLACKMAN, ORC_LANCKZOS, ORC_KAISER, ORC_GAUSS,
  ORC_SHEPP_LOGAN = 100, ORC_COSINE = 101
};
/* Contrast::Cntype (src/common/physical.world.h:22-27) */
enum { ORC_ABS = 0, ORC_REF = 1, ORC_PHS = 2, ORC_FLT = 3 };

/* ------------------------------------------------------------------ FFT */

/* In-place iterative radix-2 complex FFT in double, length n (power of 2).
 * sign = -1: forward (e^{-2 pi i k m / n}); sign = +1: unnormalised inverse. */
static void fft_c2c(double *re, double *im, int64_t n, int sign) {
  int64_t j = 0;
  for (int64_t i = 1; i < n; i++) {
    int64_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double t = re[i]; re[i] = re[j]; re[j] = t;
      t = im[i]; im[i] = im[j]; im[j] = t;
    }
  }
  for (int64_t len = 2; len <= n; len <<= 1) {
    int64_t half = len >> 1;
    for (int64_t k = 0; k < half; k++) {
      double ang = sign * 2.0 * M_PI * (double)k / (double)len;
      double wr = cos(ang), wi = sin(ang);
      for (int64_t s = 0; s < n; s += len) {
        int64_t a = s + k, b = a + half;
        double xr = re[b] * wr - im[b] * wi;
        double xi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - xr; im[b] = im[a] - xi;
        re[a] += xr; im[a] += xi;
      }
    }
  }
}

/* ------------------------------------------------------- CTrec set-up */

int64_t orc_padded_width(int64_t W) {
  /* lct.cpp:490: zidth(pow(2, ceil(log2(2*ish(1)-1)))) */
  return (int64_t)pow(2.0, ceil(log2((double)(2 * W - 1))));
}

/* I0 by its power series, summed until a term stops changing the sum (GSL's
 * gsl_sf_bessel_I0, which the reference calls, is absent here). */
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

/* Window value for one normalised frequency fp in [0,1] (lct.cpp:150-200).
 * The reference evaluates each window on a float fp and stores the result in
 * a float; 'as_float' selects that rounding (compat) or keeps double.  The
 * compat form follows the reference as its build compiles it: -ffast-math
 * (CMakeLists.txt:10-11) lets GCC reassociate PARZEN into (3 fp^3 - 6 fp^2) + 1
 * and BLACKMAN into (0.5 cos + 0.08 cos2) + 0.42 even at -O0. */
static double window_value(int ftype, double fpd, float fpf, float alsig,
                           int as_float) {
  double r;
  float ff = fpf;
  switch (ftype) {
  case ORC_NONE:
  case ORC_RAMP: r = 1.0; break;
  case ORC_BARLETT: r = as_float ? (double)(1 - ff) : 1 - fpd; break;
  case ORC_WELCH: r = as_float ? (double)(1 - ff * ff) : 1 - fpd * fpd; break;
  case ORC_PARZEN:
    if (as_float)
      r = (ff <= 0.5) ? (double)((ff * (ff * ff) * 3.0f - ff * ff * 6.0f) + 1.0f)
                      : (double)((ff * (ff * ff) + 1.0f) * 2.0f);
    else
      r = (fpd <= 0.5) ? 1 - 6 * fpd * fpd + 3 * fpd * fpd * fpd
                       : 2 * (1 + fpd * fpd * fpd);
    break;
  case ORC_HANN: r = 0.5 * (1 + cos(M_PI * fpd)); break;
  case ORC_HAMMING: r = 0.54 + 0.46 * cos(M_PI * fpd); break;
  case ORC_BLACKMAN:
    r = (cos(M_PI * fpd) * 0.5 + cos(2 * M_PI * fpd) * 0.08) + 0.42;
    break;
  case ORC_LANCKZOS: r = (fpd == 0.0) ? 0.0 : fabs(sin(M_PI * fpd)) / fpd; break;
  case ORC_KAISER: {
    double a1 = as_float ? (double)(alsig * sqrtf(1 - ff * ff))
                         : alsig * sqrt(1 - fpd * fpd);
    r = bessel_i0(a1) / bessel_i0((double)alsig);
    break;
  }
  case ORC_GAUSS:
    if (as_float)
      r = (double)powf(2.0f, ((float)-ff) * ff / (alsig * alsig));
    else
      r = pow(2.0, -fpd * fpd / ((double)alsig * alsig));
    break;
  case ORC_SHEPP_LOGAN: {
    /* sinc window sin(pi f/2)/(pi f/2): no reference counterpart */
    double x = M_PI * fpd / 2.0;
    r = (fpd == 0.0) ? 1.0 : sin(x) / x;
    break;
  }
  case ORC_COSINE: r = cos(M_PI * fpd / 2.0); break; /* no reference counterpart */
  default: r = 1.0;
  }
  return as_float ? (double)(float)r : r;
}

/* Filter::fill (lct.cpp:122-209) followed by the CTrec scaling
 * (lct.cpp:505-508).  Writes P values into G (float, compat) or Gd (double).
 * Returns 0 on success, -1 for an unknown filter. */
int orc_filter_fill(int ftype, float alsig, int64_t P, int64_t W, int contrast,
                    float *G, double *Gd) {
  if (P <= 0) return -1;
  double *re = (double *)calloc((size_t)P, sizeof(double));
  double *im = (double *)calloc((size_t)P, sizeof(double));
  float *f = (float *)calloc((size_t)P, sizeof(float));
  /* lct.cpp:132-135 */
  f[0] = 0.25f;
  /* lct.cpp:134 as the reference's -ffast-math build folds it:
   * (-1/pi^2) / (pix*pix), pix*pix an int product */
  const double neg_inv_pi2 = -1.0 / (M_PI * M_PI);
  for (int pix = 1; pix < P / 2; pix += 2)
    f[pix] = (float)(neg_inv_pi2 / (double)(pix * pix));
  /* FFTW_HC2R of f (lct.cpp:138-140): f holds real parts r_0..r_{P/2}
   * (imaginary parts are all zero), H[m] = r0 + 2 sum r_k cos(2 pi k m/P). */
  for (int64_t k = 0; k <= P / 2; k++) {
    re[k] = f[k];
    if (k > 0 && k < P - k) re[P - k] = f[k];
  }
  fft_c2c(re, im, P, +1);
  for (int64_t pix = 0; pix < P; pix++) {
    float fpf = (float)((pix < P / 2) ? pix : P - pix);
    fpf = (float)((double)fpf * (2.0 / (double)P));       /* lct.cpp:152-153 */
    double fpd = (double)((pix < P / 2) ? pix : P - pix) * (2.0 / (double)P);
    if (G) {
      float H = (float)re[pix];
      double w = window_value(ftype, (double)fpf, fpf, alsig, 1);
      float g = (float)((double)H * (w / 2.0));             /* lct.cpp:203 */
      g = g * ((float)P / (float)W);                         /* lct.cpp:506 */
      G[pix] = g;
    }
    if (Gd) {
      double w = window_value(ftype, fpd, fpf, alsig, 0);
      Gd[pix] = re[pix] * (w / 2.0) * ((double)P / (double)W);
    }
  }
  if (contrast == ORC_REF) {                                 /* lct.cpp:507-508 */
    if (G) G[0] = 0.0f;
    if (Gd) Gd[0] = 0.0;
  }
  free(re); free(im); free(f);
  return 0;
}

/* arcO (lct.cpp:470-476) */
float orc_arc(float anarc, int64_t points) {
  float r = anarc;
  if (r < 1.0f) r *= (float)(points - 1);
  r = (float)((double)r * (M_PI / 180));
  return r;
}

/* Angle table (lct.cpp:512-517): tab[2i] = sinf(th_i), tab[2i+1] = cosf(th_i)
 * with th_i = i*arc/N in float. */
void orc_angle_table(float anarc, int64_t N, float *tab) {
  const float arc = orc_arc(anarc, N);
  for (int64_t i = 0; i < N; i++) {
    float th = (float)i * arc / (float)N;
    tab[2 * i] = sinf(th);
    tab[2 * i + 1] = cosf(th);
  }
}

/* Table for an explicit angle list (extension): sinf/cosf of the angles
 * rounded to float, the same form as the uniform table. */
void orc_angle_table_list(const double *th, int64_t N, float *tab) {
  for (int64_t i = 0; i < N; i++) {
    const float t = (float)th[i];
    tab[2 * i] = sinf(t);
    tab[2 * i + 1] = cosf(t);
  }
}

/* FP64 table for the linear-interpolation extension. */
void orc_angle_table_f64(double anarc, int64_t N, double *tab) {
  double arc = anarc;
  if (arc < 1.0) arc *= (double)(N - 1);
  arc *= M_PI / 180.0;
  for (int64_t i = 0; i < N; i++) {
    double th = (double)i * arc / (double)N;
    tab[2 * i] = sin(th);
    tab[2 * i + 1] = cos(th);
  }
}

/* setPhysics (lct.cpp:558-566) */
float orc_rec_cof(float pixelSize, float lambda) {
  float r = 1.0f;
  if (lambda > 0.0f) r = (float)((double)r * ((double)lambda / (2 * M_PI)));
  if (pixelSize > 0.0f) r = (float)((double)r * (M_PI / (double)pixelSize));
  return r;
}

/* deAbs (physical.world.cpp:88-100).  Returns -1 on "bad absorption data". */
int orc_deabs(float *x, int64_t n) {
  if (n <= 0) return 0;
  float mn = x[0], mx = x[0];
  for (int64_t i = 1; i < n; i++) {
    if (x[i] < mn) mn = x[i];
    if (x[i] > mx) mx = x[i];
  }
  if (mn <= 0.0f) {
    const float mina = (float)((double)mx / 1000000.0);
    if (mina <= 0.0f) return -1;
    for (int64_t i = 0; i < n; i++)
      if (x[i] <= mina) x[i] = mina;
  }
  for (int64_t i = 0; i < n; i++) x[i] = -logf(x[i]);
  return 0;
}

/* prepare_sino (lct.cpp:569-597) with filter_line (lct.cpp:280-291).
 *
 * x:    N*W input (row = projection).  For ABS contrast it is deAbs'ed
 *       in place first, as the reference does.
 * q:    N*W float output (may alias x); qd: optional N*W double output.
 * G/Gd: the P-point window (float as the reference holds it; double for the
 *       fp64 form).
 *
 * The padded line is z[zs+c] = x[r][c] for c < W and, because blitz Range is
 * inclusive (lct.cpp:580,584), also z[zs+W] = x[r+1][0]: the first sample of
 * the next, still unfiltered row; 0 after the last row.  The write-back copies
 * z[zs .. zs+W-1] only (lct.cpp:586). */
int orc_prepare_sino(float *x, int64_t N, int64_t W, int64_t P, int contrast,
                     const float *G, const double *Gd, float *q, double *qd) {
  if (contrast == ORC_ABS)
    if (orc_deabs(x, N * W)) return -1;
  const int64_t zs = (P - W) / 2;
  double *re = (double *)malloc(sizeof(double) * (size_t)P);
  double *im = (double *)malloc(sizeof(double) * (size_t)P);
  double *rowd = (double *)malloc(sizeof(double) * (size_t)W);
  float *next0 = (float *)malloc(sizeof(float) * (size_t)(N + 1));
  for (int64_t r = 0; r < N; r++) next0[r] = (r + 1 < N) ? x[(r + 1) * W] : 0.0f;
  for (int64_t r = 0; r < N; r++) {
    if (contrast == ORC_FLT) {
      for (int64_t c = 0; c < W; c++) rowd[c] = x[r * W + c];
    } else {
      memset(re, 0, sizeof(double) * (size_t)P);
      memset(im, 0, sizeof(double) * (size_t)P);
      for (int64_t c = 0; c < W; c++) re[zs + c] = x[r * W + c];
      if (zs + W < P) re[zs + W] = next0[r];
      fft_c2c(re, im, P, -1);
      for (int64_t k = 0; k < P; k++) {
        /* R2HC -> *G -> HC2R multiplies complex bin k by G[k] (and its
         * mirror P-k by G[P-k]; G is even so both agree). */
        double g = Gd ? Gd[k] : (double)G[k];
        re[k] *= g; im[k] *= g;
      }
      fft_c2c(re, im, P, +1);
      for (int64_t c = 0; c < W; c++) rowd[c] = re[zs + c] / (double)P;
    }
    if (contrast == ORC_REF) {
      /* partial_sum in float (compat) / double (fp64), lct.cpp:590-595 */
      float accf = 0.0f; double accd = 0.0;
      for (int64_t c = 0; c < W; c++) {
        float v = (float)rowd[c];
        accf += v; accd += rowd[c];
        if (q) q[r * W + c] = accf;
        if (qd) qd[r * W + c] = accd;
      }
    } else {
      for (int64_t c = 0; c < W; c++) {
        if (q) q[r * W + c] = (float)rowd[c];
        if (qd) qd[r * W + c] = rowd[c];
      }
    }
  }
  free(re); free(im); free(rowd); free(next0);
  return 0;
}

/* Pixel mask of lct.cpp:693-707 / ct.cl:21-32, evaluated in float exactly as
 * the reference does.  Returns 1 when the pixel is reconstructed. */
static int in_mask(int64_t j, int64_t i, int64_t W, float center) {
  const int hp = (int)(W / 2);
  const float acent = fabsf(center);
  int ip2 = (int)(i - hp);
  ip2 *= ip2;
  if ((float)i <= acent || (float)i >= ((float)W - acent) - 1.0f) return 0;
  float ijp2 = (float)(j - hp) - center;
  ijp2 *= ijp2;
  ijp2 += (float)ip2;
  const float hpc = (float)hp + center, hmc = (float)hp - center;
  if (((float)j <= hpc && ijp2 >= hpc * hpc) ||
      ((float)j >= hpc && ijp2 >= hmc * hmc))
    return 0;
  return 1;
}

int orc_in_mask(int64_t j, int64_t i, int64_t W, float center) {
  return in_mask(j, i, W, center);
}

/* Which rounding order the first term of the index expression follows.
 *   0: ct.cl:36-37 as written, c + ((1 - s) - co) * hp -- the OpenCL kernel,
 *      and lct.cpp:711-712 built without -ffast-math;
 *   1: lct.cpp:711-712 as the reference's build compiles it (-ffast-math,
 *      CMakeLists.txt:10-11): GCC folds (1 - s) - co into 1 - (s + co), even
 *      at -O0, so the as-shipped CPU path computes c + (1 - (s + co)) * hp.
 * Everything after the first term is the same in both. */
static int g_index_rule = 0;
void orc_set_index_rule(int rule) { g_index_rule = rule; }
int orc_index_rule(void) { return g_index_rule; }

/* The reference's detector index for projection n and pixel (j,i): the float
 * expression of lct.cpp:711-712 (== ct.cl:36-37), truncated toward zero. */
static int64_t ref_index(float sx, float cy, int hp, float center, int64_t j,
                         int64_t i) {
  const float k0 = g_index_rule == 1 ? 1.0f - (sx + cy) : (1.0f - sx) - cy;
  float t = center + k0 * (float)hp;
  t = t + sx * ((float)j - center);
  t = t + cy * (float)i;
  return (int64_t)t;
}

/* Sample at flat offset n*W + k of an N*W buffer; outside the buffer the
 * reference reads unrelated memory, defined here as 0. */
static double flat_sample_f(const float *q, int64_t N, int64_t W, int64_t n,
                            int64_t k) {
  int64_t o = n * W + k;
  return (o < 0 || o >= N * W) ? 0.0 : (double)q[o];
}
static double flat_sample_d(const double *q, int64_t N, int64_t W, int64_t n,
                            int64_t k) {
  int64_t o = n * W + k;
  return (o < 0 || o >= N * W) ? 0.0 : q[o];
}

/* reconstructOnCPU (lct.cpp:688-729), rows [r0, r1) of the W*W slice.
 * tab: float sin/cos table.  With q (float) the sum is accumulated in float
 * in projection order (bit-compatible with the reference); with qd (double)
 * it is accumulated in double. */
void orc_bp_compat(const float *q, const double *qd, int64_t N, int64_t W,
                   const float *tab, float center, float recCof, int64_t r0,
                   int64_t r1, float *slice, double *sliced) {
  const int hp = (int)(W / 2);
  for (int64_t j = r0; j < r1; j++) {
    for (int64_t i = 0; i < W; i++) {
      float outf = 0.0f;
      double outd = 0.0;
      if (in_mask(j, i, W, center)) {
        float totf = 0.0f;
        double totd = 0.0;
        for (int64_t n = 0; n < N; n++) {
          int64_t k = ref_index(tab[2 * n], tab[2 * n + 1], hp, center, j, i);
          if (q) totf += (float)flat_sample_f(q, N, W, n, k);
          if (qd) totd += flat_sample_d(qd, N, W, n, k);
        }
        if (recCof != 0.0f) {
          totf *= recCof;
          totd *= (double)recCof;
        }
        outf = totf / (float)N;
        outd = totd / (double)N;
      }
      if (slice) slice[(j - r0) * W + i] = outf;
      if (sliced) sliced[(j - r0) * W + i] = outd;
    }
  }
}

/* Linear-interpolation backprojector (extension; no reference counterpart).
 * FP64 throughout.  Sample k is centred at detector coordinate k + 0.5, so the
 * geometry agrees with the reference's nearest-lower rule; samples outside
 * [0, W) are 0.  Same pixel mask as the reference. */
void orc_bp_linear(const double *qd, int64_t N, int64_t W, const double *tab,
                   double center, double recCof, int64_t r0, int64_t r1,
                   double *sliced) {
  const int hp = (int)(W / 2);
  for (int64_t j = r0; j < r1; j++) {
    for (int64_t i = 0; i < W; i++) {
      double out = 0.0;
      if (in_mask(j, i, W, (float)center)) {
        double tot = 0.0;
        const double y = (double)j - hp - center, x = (double)i - hp;
        for (int64_t n = 0; n < N; n++) {
          double u = ((double)hp + center) + tab[2 * n] * y + tab[2 * n + 1] * x - 0.5;
          double kf = floor(u);
          double f = u - kf;
          int64_t k = (int64_t)kf;
          double a = (k >= 0 && k < W) ? qd[n * W + k] : 0.0;
          double b = (k + 1 >= 0 && k + 1 < W) ? qd[n * W + k + 1] : 0.0;
          tot += a + f * (b - a);
        }
        if (recCof != 0.0) tot *= recCof;
        out = tot / (double)N;
      }
      sliced[(j - r0) * W + i] = out;
    }
  }
}

/* Output geometry (extension): output pixel (j, i) of an R x C grid stands
 * for the reference coordinates jj = oj + p*j, ii = oi + p*i (float), and every
 * float expression of the reference mask and index rule is evaluated at them.
 * With R = C = W, p = 1, oj = oi = 0 this is orc_bp_compat. */
static int in_mask_f(float jj, float ii, int64_t W, float center) {
  const int hp = (int)(W / 2);
  const float acent = fabsf(center);
  if (ii <= acent || ii >= ((float)W - acent) - 1.0f) return 0;
  const float di = ii - (float)hp;
  const float ip2 = di * di;
  float ijp2 = (jj - (float)hp) - center;
  ijp2 *= ijp2;
  ijp2 += ip2;
  const float hpc = (float)hp + center, hmc = (float)hp - center;
  if ((jj <= hpc && ijp2 >= hpc * hpc) || (jj >= hpc && ijp2 >= hmc * hmc)) return 0;
  return 1;
}

void orc_bp_compat_geom(const float *q, int64_t N, int64_t W, const float *tab, float center,
                        float recCof, int64_t R, int64_t C, float oj, float oi, float p,
                        float *slice) {
  const int hp = (int)(W / 2);
  for (int64_t j = 0; j < R; j++) {
    const float jj = oj + p * (float)j;
    for (int64_t i = 0; i < C; i++) {
      const float ii = oi + p * (float)i;
      float out = 0.0f;
      if (in_mask_f(jj, ii, W, center)) {
        float tot = 0.0f;
        for (int64_t n = 0; n < N; n++) {
          const float sx = tab[2 * n], cy = tab[2 * n + 1];
          const float k0 = g_index_rule == 1 ? 1.0f - (sx + cy) : (1.0f - sx) - cy;
          float t = center + k0 * (float)hp;
          t = t + sx * (jj - center);
          t = t + cy * ii;
          tot += (float)flat_sample_f(q, N, W, n, (int64_t)t);
        }
        if (recCof != 0.0f) tot *= recCof;
        out = tot / (float)N;
      }
      slice[j * C + i] = out;
    }
  }
}

void orc_bp_linear_geom(const double *qd, int64_t N, int64_t W, const double *tab, double center,
                        double recCof, int64_t R, int64_t C, float oj, float oi, float p,
                        double *sliced) {
  const int hp = (int)(W / 2);
  for (int64_t j = 0; j < R; j++) {
    const float jj = oj + p * (float)j;
    for (int64_t i = 0; i < C; i++) {
      const float ii = oi + p * (float)i;
      double out = 0.0;
      if (in_mask_f(jj, ii, W, (float)center)) {
        double tot = 0.0;
        const double y = (double)jj - hp - center, x = (double)ii - hp;
        for (int64_t n = 0; n < N; n++) {
          double u = ((double)hp + center) + tab[2 * n] * y + tab[2 * n + 1] * x - 0.5;
          double kf = floor(u);
          double f = u - kf;
          int64_t k = (int64_t)kf;
          double a = (k >= 0 && k < W) ? qd[n * W + k] : 0.0;
          double b = (k + 1 >= 0 && k + 1 < W) ? qd[n * W + k + 1] : 0.0;
          tot += a + f * (b - a);
        }
        if (recCof != 0.0) tot *= recCof;
        out = tot / (double)N;
      }
      sliced[j * C + i] = out;
    }
  }
}

/* RingFilter::apply (lct.cpp:295-327) without a mask: column means over the
 * projections (float, projection order), a box mean of half width `box`
 * (dstR/srcR of matrix.world.h:261-267; the box shrinks at the edges), and the
 * difference added back to every projection.  In place on x (N x W). */
void orc_ring(float *x, int64_t N, int64_t W, int64_t box) {
  if (box <= 0 || N <= 0) return;
  float *avg = (float *)calloc((size_t)W, sizeof(float));
  float *tmp = (float *)calloc((size_t)W, sizeof(float));
  for (int64_t r = 0; r < N; r++)
    for (int64_t c = 0; c < W; c++) avg[c] += x[r * W + c];
  for (int64_t c = 0; c < W; c++) avg[c] /= (float)N;
  for (int64_t ii = -box; ii <= box; ii++) {
    const int64_t d0 = ii > 0 ? ii : 0, d1 = W - 1 + (ii < 0 ? ii : 0);
    for (int64_t d = d0; d <= d1; d++) tmp[d] += avg[d - ii];
  }
  for (int64_t d = box; d <= W - 1 - box; d++) tmp[d] /= (float)(2 * box + 1);
  for (int64_t ii = 0; ii < box; ii++) {
    tmp[ii] /= (float)(box + ii + 1);
    tmp[W - 1 - ii] /= (float)(box + ii + 1);
  }
  for (int64_t c = 0; c < W; c++) tmp[c] -= avg[c];
  for (int64_t r = 0; r < N; r++)
    for (int64_t c = 0; c < W; c++) x[r * W + c] += tmp[c];
  free(avg);
  free(tmp);
}

/* ------------------------------------------------------------------------
 * Rotation-axis search (lct.cpp:792-1325).  Test infrastructure.
 * ---------------------------------------------------------------------- */

/* AverageGradient::apply (lct.cpp:863-913) after ct.repeat(): the metric of
 * one reconstructed W x W slice at `centre`.
 *  - Smoothing (sigma > 1): the reference multiplies the slice's FFT by the FFT
 *    of g(a, b) = expf(-(a*a + b*b) / sig22), a, b in [0, W) (lct.cpp:839-841),
 *    and divides the inverse by W^2: a circular convolution with that table,
 *    evaluated here exactly in double and rounded to float.
 *  - Crop k = |(int)c| rows top and bottom (ct.h:276-279 writes ceil(abs(c)),
 *    but only the C library's int abs() is in scope there; no crop when 0).
 *  - derH / derV: six statements each (lct.cpp:879-902), every statement a
 *    pass over its destination range with a float add.
 *  - cSlice = sqrt(derH*derH + derV*derV) assigns full-size arrays to the
 *    cropped view: blitz walks each operand from its own first element, so
 *    cropped row y takes full row y.
 *  - Borders zeroed, sum in double (blitz sums float in double), count > 0.
 *    With smoothing the reference's float FFT leaves rounding noise in every
 *    pixel, so every magnitude of the region is positive there; the exact
 *    convolution here has none, so the count is then taken over the whole
 *    region (rows >= k, inside the zeroed borders).
 * Returns nm ? sm/nm : 0 with sm = (float)sum; *sum_out / *cnt_out (nullable)
 * receive the double sum and the count. */
float orc_ag_metric(const float *slice, int64_t W, float centre, float sigma,
                    double *sum_out, int64_t *cnt_out) {
  const int64_t n = W * W;
  float *B = (float *)malloc(sizeof(float) * (size_t)n);
  if (sigma > 1) {
    const float sig22 = 2 * sigma * sigma;
    /* nonzero part of the table: a*a + b*b below the float underflow */
    int64_t amax = 0;
    while (amax < W && expf((float)(-(int)(amax * amax)) / sig22) > 0.0f) amax++;
    float *g = (float *)malloc(sizeof(float) * (size_t)(amax * amax + 1));
    for (int64_t a = 0; a < amax; a++)
      for (int64_t b = 0; b < amax; b++)
        g[a * amax + b] = expf((float)(-(int)(a * a + b * b)) / sig22);
    for (int64_t y = 0; y < W; y++)
      for (int64_t x = 0; x < W; x++) {
        double acc = 0.0;
        for (int64_t a = 0; a < amax; a++) {
          const int64_t yy = ((y - a) % W + W) % W;
          for (int64_t b = 0; b < amax; b++) {
            const float gv = g[a * amax + b];
            if (gv == 0.0f) continue;
            const int64_t xx = ((x - b) % W + W) % W;
            acc += (double)gv * (double)slice[yy * W + xx];
          }
        }
        B[y * W + x] = (float)acc;
      }
    free(g);
  } else {
    memcpy(B, slice, sizeof(float) * (size_t)n);
  }
  /* ceil(abs(center)) in ct.h:277 calls the C library's int abs(): the
   * centre is truncated first */
  const float cacent = (float)abs((int)centre);
  const int64_t cc = (int64_t)cacent;
  const int64_t R = W - 2 * cc;
  float *dH = (float *)calloc((size_t)n, sizeof(float));
  float *dV = (float *)calloc((size_t)n, sizeof(float));
  /* statement (s0, s1, k): dst(r, x) += k * C(r - s0, x - s1) over the
   * destination ranges dstR(R, s0) x dstR(W, s1) (matrix.world.h:261-272) */
  static const int sh[6][3] = {{-1, -1, -1}, {-1, 0, -2}, {-1, 1, -1},
                               {1, -1, 1},   {1, 0, 2},   {1, 1, 1}};
  static const int sv[6][3] = {{-1, -1, -1}, {0, -1, -2}, {1, -1, -1},
                               {-1, 1, 1},   {0, 1, 2},   {1, 1, 1}};
  for (int pass = 0; pass < 2; pass++) {
    float *D = pass ? dV : dH;
    const int (*S)[3] = pass ? sv : sh;
    for (int t = 0; t < 6; t++) {
      const int s0 = S[t][0], s1 = S[t][1];
      const float k = (float)S[t][2];
      const int64_t r0 = s0 > 0 ? s0 : 0, r1 = R - 1 + (s0 < 0 ? s0 : 0);
      const int64_t c0 = s1 > 0 ? s1 : 0, c1 = W - 1 + (s1 < 0 ? s1 : 0);
      for (int64_t r = r0; r <= r1; r++)
        for (int64_t x = c0; x <= c1; x++) {
          const float cv = B[(cc + r - s0) * W + (x - s1)];
          float *d = &D[(cc + r) * W + x];
          *d = *d + k * cv;
        }
    }
  }
  double sum = 0.0;
  int64_t cnt = 0;
  const int noisy = sigma > 1;
  for (int64_t y = 0; y < R; y++)
    for (int64_t x = 0; x < W; x++) {
      float m = 0.0f;
      const int border = x == 0 || x == W - 1 || y == 0 || y == R - 1;
      if (!border) {
        const float h = dH[y * W + x], v = dV[y * W + x];
        const float hh = h * h, vv = v * v;
        m = sqrtf(hh + vv);
      }
      sum += (double)m;
      if (m > 0.0f || (noisy && !border && y >= cc)) cnt++;
    }
  free(B);
  free(dH);
  free(dV);
  if (sum_out) *sum_out = sum;
  if (cnt_out) *cnt_out = cnt;
  const float sm = (float)sum;
  return cnt ? sm / (float)cnt : 0.0f;
}

/* calcErr of raxis(proj0, proj180, maxDev) (lct.cpp:1246-1252) before the
 * square root: dlt = aver, then columns dstR(W, xs) <- mirrored proj180
 * columns srcR(W, xs), minus proj0; sum of float squares in double, row
 * order.  xs is the trial shift already truncated to an integer. */
double orc_pair_sq(const float *p0, const float *p180, int64_t rows, int64_t W, float aver,
                   int64_t xs) {
  double s = 0.0;
  const int64_t lo = xs > 0 ? xs : 0, hi = W - 1 + (xs < 0 ? xs : 0);
  for (int64_t j = 0; j < rows; j++)
    for (int64_t i = 0; i < W; i++) {
      float d = aver;
      if (i >= lo && i <= hi) d = p180[j * W + (W - 1 - (i - xs))];
      d = d - p0[j * W + i];
      const float dd = d * d;
      s += (double)dd;
    }
  return s;
}

/* ------------------------------------------------------------------------
 * Tomosynthesis ts_add (lct.cpp:731-787).  Test infrastructure.
 * ---------------------------------------------------------------------- */

/* Filter::fill(filt, n) (lct.cpp:122-209) for any length n: the Ram-Lak taps,
 * FFTW_HC2R of them (here a direct double sum), the window factor evaluated
 * as the reference rounds it, / 2.  Float window of n values. */
int orc_filter_fill_plain(int ftype, float alsig, int64_t n, float *out) {
  if (n <= 0) return -1;
  float *f = (float *)calloc((size_t)n, sizeof(float));
  f[0] = 0.25f;
  const double neg_inv_pi2 = -1.0 / (M_PI * M_PI);  /* as the reference's build folds it */
  for (int64_t pix = 1; pix < n / 2; pix += 2)
    f[pix] = (float)(neg_inv_pi2 / (double)(int)(pix * pix));
  for (int64_t m = 0; m < n; m++) {
    /* HC2R: r_0 + 2 sum_{0<k<n/2} r_k cos(2 pi k m / n) + r_{n/2} (-1)^m */
    double s = f[0];
    for (int64_t k = 1; 2 * k < n; k++)
      s += 2.0 * (double)f[k] * cos(2.0 * M_PI * (double)((k * m) % n) / (double)n);
    if (n % 2 == 0) s += (double)f[n / 2] * ((m & 1) ? -1.0 : 1.0);
    const float H = (float)s;
    float fpf = (float)((m < n / 2) ? m : n - m);
    fpf = (float)((double)fpf * (2.0 / (double)n));
    const double w = window_value(ftype, (double)fpf, fpf, alsig, 1);
    out[m] = (float)((double)H * (w / 2.0));
  }
  free(f);
  return 0;
}

/* ts_add (lct.cpp:731-787) with the row filter evaluated exactly in double
 * (circular convolution with g = IDFT_n(fwin), then rounded to float, where
 * the reference uses FFTW's float transforms).  proj (rows x n) is left as
 * the reference leaves it: -log for ABS, filtered, running sum for REF;
 * result is accumulated. */
void orc_ts_add(float *proj, float *result, int64_t rows, int64_t n, const float *fwin,
                float center, int contrast, float angle, int plane) {
  double *g = (double *)malloc(sizeof(double) * (size_t)n);
  for (int64_t m = 0; m < n; m++) {
    double s = 0.0;
    for (int64_t k = 0; k < n; k++)
      s += (double)fwin[k] * cos(2.0 * M_PI * (double)((k * m) % n) / (double)n);
    g[m] = s / (double)n;
  }
  if (contrast == ORC_ABS)
    for (int64_t i = 0; i < rows * n; i++) proj[i] = -logf(proj[i]);
  double *z = (double *)malloc(sizeof(double) * (size_t)n);
  const float cur_sin = sinf(angle), cur_cos = cosf(angle);
  const float plane_cos = ((float)plane - center) * cur_sin;
  const float Rcenter = (float)(n * 0.5 + center);
  for (int64_t y = 0; y < rows; y++) {
    float *ln = proj + y * n;
    for (int64_t x = 0; x < n; x++) z[x] = ln[x];
    for (int64_t x = 0; x < n; x++) {
      double s = 0.0;
      for (int64_t m = 0; m < n; m++) s += g[m] * z[((x - m) % n + n) % n];
      ln[x] = (float)s;
    }
    if (contrast == ORC_REF)
      for (int64_t x = 1; x < n; x++) ln[x] = ln[x - 1] + ln[x];
    for (int64_t x = 0; x < n; x++) {
      float di = ((float)x - Rcenter) * cur_cos - plane_cos + Rcenter;
      di = (di < 0) ? 0 : (di >= (float)n) ? (float)(n - 1) : di;
      result[y * n + x] += ln[(int64_t)di];
    }
  }
  free(z);
  free(g);
}

/* ------------------------------------------------------------------------
 * Output sample conversion of the volume writer: limit<T>
 * (src/common/external.world.cpp:69-90) for one image of n floats.
 * bpp: 8, 16, 32, 64 unsigned; -8, -16, -32, -64 signed.  With
 * mincon == maxcon the image's own minimum and maximum are used; an image of
 * equal values becomes 0.  Each float operation is rounded on its own
 * (the reference is built for x86-64 without FMA); the final conversion
 * truncates toward zero and saturates where C++ leaves it undefined (a float
 * that reaches 2^31, 2^32, 2^63 or 2^64).  Returns -1 for a bad bpp.
 */
#define ORC_LIMIT_T(T, LO, HI, TOPF)                                               \
  {                                                                                \
    T *q = (T *)dst;                                                               \
    if (mn == mx) {                                                                \
      for (int64_t i = 0; i < n; i++) q[i] = 0;                                    \
      return 0;                                                                    \
    }                                                                              \
    const float tw = (float)(HI) - (float)(LO);                                    \
    const float lw = mx - mn;                                                      \
    for (int64_t i = 0; i < n; i++) {                                              \
      const float interim = (src[i] - mn) / lw;                                    \
      if (interim < 0) q[i] = (LO);                                                \
      else if (interim > 1) q[i] = (HI);                                           \
      else {                                                                       \
        const float prod = interim * tw;                                           \
        const float v = (float)(LO) + prod;                                        \
        q[i] = v >= (TOPF) ? (HI) : (T)v;                                          \
      }                                                                            \
    }                                                                              \
    return 0;                                                                      \
  }

int orc_limit(const float *src, int64_t n, int bpp, float mincon, float maxcon, void *dst) {
  float mn = mincon, mx = maxcon;
  if (mn == mx && n > 0) {
    mn = src[0];
    mx = src[0];
    for (int64_t i = 1; i < n; i++) {
      if (src[i] < mn) mn = src[i];
      if (src[i] > mx) mx = src[i];
    }
  }
  switch (bpp) {
    case 8: ORC_LIMIT_T(uint8_t, 0, UINT8_MAX, 256.0f)
    case -8: ORC_LIMIT_T(int8_t, INT8_MIN, INT8_MAX, 128.0f)
    case 16: ORC_LIMIT_T(uint16_t, 0, UINT16_MAX, 65536.0f)
    case -16: ORC_LIMIT_T(int16_t, INT16_MIN, INT16_MAX, 32768.0f)
    case 32: ORC_LIMIT_T(uint32_t, 0, UINT32_MAX, 4294967296.0f)
    case -32: ORC_LIMIT_T(int32_t, INT32_MIN, INT32_MAX, 2147483648.0f)
    case 64: ORC_LIMIT_T(uint64_t, 0, UINT64_MAX, 18446744073709551616.0f)
    case -64: ORC_LIMIT_T(int64_t, INT64_MIN, INT64_MAX, 9223372036854775808.0f)
    default: return -1;
  }
}
