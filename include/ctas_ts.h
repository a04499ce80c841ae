/*
 * ctas_ts.h -- C ABI of the tomosynthesis step of ctas (the `ts` tool), on the
 * same device path as ctas_fbp.h.
 *
 * Reference: ts_add(Map &projection, Map &result, const Filter &filter,
 * float center, Contrast contrast, float angle, int plane),
 * src/common/lct.cpp:731-787, declared in src/common/ct.h; called once per
 * projection by src/executables/ts.cpp:209-217.  For every row of the
 * projection image: -log for absorption contrast, the filter window applied
 * with an FFT of the row's own length (no padding: a circular convolution),
 * a running sum for refraction contrast, then
 *   result(y, x) += projection(y, (ssize_t) clamp(di, 0, pixels-1)),
 *   di = (x - Rc) * cos(angle) - (plane - center) * sin(angle) + Rc,
 *   Rc = pixels / 2 + center,
 * in float, rounded as the reference rounds it.
 *
 * Statuses and the last-error message are those of ctas_fbp.h
 * (ctas_fbp_last_error()).  Images are row-major float32 [rows][pixels].
 */
#ifndef CTAS_TS_H
#define CTAS_TS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ctas_ts ctas_ts;

/* Set-up for projection images of rows x pixels: the window of
 * Filter(ftype, fparam).fill(pixels) (lct.cpp:122-209) and the device FFT
 * tables.  contrast: CTAS_ABS (-log first), CTAS_REF (running sum after the
 * filter); PHS and FLT filter only, as ts_add does.  device: CUDA ordinal,
 * -1 = current. */
int ctas_ts_create(ctas_ts **out, int64_t rows, int64_t pixels, int32_t ftype, float fparam,
                   int32_t contrast, int32_t device);
int ctas_ts_destroy(ctas_ts *h);

/* ts_add on host images (synchronous): `projection` is replaced by its
 * filtered rows as the reference leaves it (unless flags has
 * CTAS_FLAG_NO_WRITEBACK), `result` is accumulated in place. */
int ctas_ts_add(ctas_ts *h, float *projection, float *result, float center, float angle,
                int32_t plane, uint32_t flags);
/* Device form, asynchronous on `stream` (a cudaStream_t). */
int ctas_ts_add_dev(ctas_ts *h, float *projection_dev, float *result_dev, float center,
                    float angle, int32_t plane, uint32_t flags, void *stream);
/* Extension: n projections (n x rows x pixels, device) at angles[n] (host,
 * radians) added into result_dev in one filter launch and one backprojection
 * launch; every result pixel receives its n terms in order, so the result is
 * that of n ts_add calls.  Synchronises `stream` on entry (the angles are
 * staged in a handle-owned buffer). */
int ctas_ts_add_batch_dev(ctas_ts *h, float *projections_dev, const float *angles, int64_t n,
                          float *result_dev, float center, int32_t plane, uint32_t flags,
                          void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTAS_TS_H */
