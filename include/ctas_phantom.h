/*
 * ctas_phantom.h -- seeded synthetic inputs on the device (extension; the
 * reference has no phantom generator).
 *
 * Exact parallel-beam projections of sums of ellipses, in the detector
 * geometry of the reference backprojector (ctas src/common/lct.cpp:711-713):
 * sample k of projection n is the line integral at detector coordinate
 * t = k + 0.5, the rotation axis projecting to t = W/2 + center.
 */
#ifndef CTAS_PHANTOM_H
#define CTAS_PHANTOM_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ellipses_dev: n_slices x n_ellipses x 6 doubles (x0, y0, a, b, phi, rho)
 * in pixel units relative to the rotation axis; angles_dev: n_angles
 * projection angles in radians; out_dev: n_slices x n_angles x width float32.
 * Asynchronous on `stream` (a cudaStream_t). */
int ctas_phantom_sinogram_dev(const double *ellipses_dev, int64_t n_ellipses, int64_t n_slices,
                              int64_t n_angles, int64_t width, const double *angles_dev,
                              double center, float *out_dev, void *stream);

/* Line integrals of n_slices images (width x width float32 on the device; the
 * value of pixel (j, i) sits at object point (i - W/2, j - W/2 - center)),
 * ADDED to out_dev (n_slices x n_angles x width): each ray is sampled every
 * `step` pixels (bilinear, zero outside the image) along its chord of the disc
 * of `radius` pixels around the axis, so content outside that disc is not
 * projected.  For texture fields, whose line integrals have no closed form. */
int ctas_phantom_project_image_dev(const float *image_dev, int64_t n_slices, int64_t n_angles,
                                   int64_t width, const double *angles_dev, double center,
                                   double radius, double step, float *out_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif
