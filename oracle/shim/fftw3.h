/*
 * fftw3.h -- stand-in for the single-precision FFTW3 interface, for compiling
 * the reference's reconstruction code (ctas src/common/lct.cpp) without FFTW.
 * Test infrastructure only.  It declares the handful of FFTW names lct.cpp
 * uses (call sites lct.cpp:50-61, 138-140, 285-287, 509-510, 757-759,
 * 824-827, 1310-1311) with FFTW's documented signatures and transform
 * definitions; fftw_shim.cpp computes every transform in double precision
 * (an exact-order DFT by FFT) and rounds the result to float once.  FFTW's own
 * single-precision rounding is therefore not reproduced: results differ from
 * a real FFTW build by about one float ulp of the transform's magnitude.
 *
 * Transform definitions (FFTW manual, "What FFTW Really Computes"):
 *   R2HC  r[k] = sum_j x[j] cos(2 pi j k / n), k = 0..n/2;
 *         i[k] = -sum_j x[j] sin(2 pi j k / n), k = 1..(n+1)/2-1;
 *         stored as r0, r1, ..., r_{n/2}, i_{(n+1)/2-1}, ..., i1.
 *   HC2R  the unnormalised inverse of R2HC.
 *   DFT   y[k] = sum_j x[j] exp(sign * 2 pi i j k / n), unnormalised,
 *         row-major for two dimensions.
 */
#ifndef CTAS_ORACLE_SHIM_FFTW3_H
#define CTAS_ORACLE_SHIM_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct ctas_shim_fftwf_plan_s *fftwf_plan;

typedef enum { FFTW_R2HC = 0, FFTW_HC2R = 1 } fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_r2r_1d(int n, float *in, float *out, fftw_r2r_kind kind,
                             unsigned flags);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_r2r(const fftwf_plan p, float *in, float *out);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
#endif
