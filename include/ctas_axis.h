/*
 * ctas_axis.h -- C ABI of the rotation-axis search (ctas `axis` tool), on the
 * same device path as ctas_fbp.h.
 *
 * Reference: class AverageGradient and the raxis() family,
 * src/common/lct.cpp:792-1325, declared in src/common/ct.h:327-329; the
 * caller is src/executables/axis.cpp:117-170.  Statuses and the last-error
 * message are those of ctas_fbp.h (ctas_fbp_last_error()).  Axis positions are
 * absolute detector coordinates (the image centre is 0.5 * (width - 1)), as
 * raxis() returns them.
 *
 * Deliberate differences from the reference, each where it is undefined:
 *  - the directional search after the grid runs its trials in order (the
 *    reference's worker threads may finish them out of order, which makes its
 *    stopping point scheduling-dependent);
 *  - a grid of fewer than 3 points (maximum shift below one step), a constant
 *    threshold profile (algorithm 3) and a trial shift of a whole width or more
 *    (projection pair) are reported as errors instead of reading out of range.
 */
#ifndef CTAS_AXIS_H
#define CTAS_AXIS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctas_ag ctas_ag;

/* AverageGradient(Map &sino, float anarc) (lct.cpp:814-843): filters a copy of
 * the n_angles x width sinogram (absorption contrast, RAMP window; the
 * caller's buffer is not modified) and prepares the Gaussian smoothing of
 * width sigma = angO(anarc, n_angles) * width / pi.  device: CUDA ordinal,
 * -1 = current.  Fails with CTAS_E_UNSUPPORTED if sigma needs more than 157
 * taps (sigma > 21 pixels). */
int ctas_ag_create(ctas_ag **out, const float *sino, int64_t n_angles, int64_t width,
                   float anarc, int32_t device);
/* The same with flags: CTAS_FLAG_SHIPPED_INDEX (ctas_fbp.h) backprojects with
 * the index rounding of the reference's CPU path as built; the default is
 * that of its OpenCL kernel, the path on which the reference's axis tool
 * runs (its CPU path cannot: AGinThread evaluates on CTrec copies, which do
 * not copy the sinogram, lct.cpp:529-545). */
int ctas_ag_create_flags(ctas_ag **out, const float *sino, int64_t n_angles, int64_t width,
                         float anarc, int32_t device, uint32_t flags);
/* AverageGradient::apply(axisR) (lct.cpp:863-913) for n axis positions:
 * values[k] = mean gradient magnitude of the smoothed, cropped slice
 * reconstructed about axis_r[k].  The n backprojections run as batched
 * multi-centre launches.  Synchronous. */
int ctas_ag_apply(ctas_ag *ag, const float *axis_r, int64_t n, float *values);
/* Smoothing width sigma and the number of Gaussian taps used (1 = none). */
int ctas_ag_sigma(const ctas_ag *ag, float *sigma, int32_t *taps);
int ctas_ag_destroy(ctas_ag *ag);

/* raxis(Map &sino, float anarc, float maxDev, int algo) (lct.cpp:1137-1212):
 * rotation axis of an n_angles x width absorption sinogram.  algo 0: the
 * 0/180-degree projection pair only; 1: average-gradient search from the
 * image centre; 2: from the pair estimate; 3: from a threshold of the summed
 * projections.  max_dev: maximum relative shift, 0 .. 0.25.  *axis receives the
 * absolute axis position; *trials (nullable) the number of average-gradient
 * evaluations (reconstructions) made: the grid in batches, the directional
 * march in speculative batches of 8 (up to 7 trials past the reference's
 * stopping point), the bisection one by one. */
int ctas_raxis(const float *sino, int64_t n_angles, int64_t width, float anarc, float max_dev,
               int32_t algo, int32_t device, float *axis, int64_t *trials);

/* raxis(Map &proj0, Map &proj180, float maxDev) (lct.cpp:1217-1297): rotation
 * axis from two opposite rows x width projections; max_dev 0 .. 0.5. */
int ctas_raxis_pair(const float *proj0, const float *proj180, int64_t rows, int64_t width,
                    float max_dev, int32_t device, float *axis);

#ifdef __cplusplus
}
#endif

#endif /* CTAS_AXIS_H */
