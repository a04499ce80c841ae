/*
 * ctas_volume.h -- streamed volume reconstruction: the ct tool's slice loop
 * (src/executables/ct.cpp:156-206) as one pipelined call.
 *
 * The reference reads each sinogram (ReadVolumeBySlice::readTo,
 * src/common/external.world.cpp:1320), ring-filters it (RingFilter::apply),
 * reconstructs it (CTrec::reconstruct) and saves the slice
 * (SaveVolumeBySlice::save, external.world.cpp:1457-1494), one slice per host
 * thread.  Here one call streams a whole volume through a ctas_fbp handle:
 *
 *   reader thread   read callback -> pinned input ring (3 chunks)
 *   copy stream     host -> device of chunk k+1
 *   compute stream  ring filter, filter, backprojection, sample conversion of chunk k
 *   copy stream     device -> host of chunk k-1 into a pinned output ring (3 chunks)
 *   writer thread   write callback from the output ring
 *
 * so file reads, both copy directions, the kernels and file writes overlap.
 * The file formats (HDF5, TIFF, image series) stay with the caller, behind
 * the two callbacks; ctas_vol_raw_reconstruct is the built-in pair for raw
 * contiguous float32 volumes at a byte offset -- the layout the reference
 * memory-maps for contiguous HDF5 datasets and files in /dev/shm
 * (HDFwrapper::mmapMeIfYouCan, external.world.cpp:191-280).
 *
 * Output samples (the ct tool's -i/-m/-M, ct.cpp:110-116): bpp 0 writes
 * float32; bpp in {8, 16, 32, 64} writes unsigned and {-8, -16, -32, -64}
 * signed integers of that width, converted on the device as the reference's
 * limit<T> does (external.world.cpp:69-90): with equal mincon and maxcon each
 * slice's own minimum and maximum are used (an all-equal slice becomes 0);
 * v -> (v - mincon) / (maxcon - mincon), below 0 -> the type's minimum, above
 * 1 -> its maximum, else min + interim * (max - min) in float, truncated
 * toward zero.  Where that float reaches 2^32, 2^31, 2^64 or 2^63 (32- and
 * 64-bit types at interim == 1) C++ leaves the conversion undefined; here it
 * saturates to the type's maximum.
 *
 * Statuses and the last-error message as in ctas_fbp.h.
 */
#ifndef CTAS_VOLUME_H
#define CTAS_VOLUME_H

#include <stdint.h>

#include "ctas_fbp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bytes of one output sample for bpp (0 -> 4); 0 for an unsupported bpp. */
int32_t ctas_vol_sample_bytes(int32_t bpp);

/* limit<T> on the device: n_images images of `pixels` float32 values at src
 * (contiguous) -> the same count of bpp samples at dst.  bpp != 0.
 * Asynchronous on `stream` (cudaStream_t); stream-ordered scratch when the
 * range is per image. */
int ctas_vol_quantize_dev(const float *src, int64_t n_images, int64_t pixels, int32_t bpp,
                          float mincon, float maxcon, void *dst, void *stream);

/* Fill `count` sinograms starting at slice `first` into sinos
 * ([count][n_angles][width] float32, pinned host memory).  Non-zero aborts. */
typedef int (*ctas_vol_read_fn)(void *user, int64_t first, int64_t count, float *sinos);
/* Consume `count` slices starting at slice `first` ([count][rows][cols]
 * samples of the call's bpp, pinned host memory, valid during the call).
 * Non-zero aborts. */
typedef int (*ctas_vol_write_fn)(void *user, int64_t first, int64_t count, const void *slices);

/* Reconstruct n_slices sinograms of the handle's shape, all with the same
 * centre, reading them through `read` and handing the slices to `write`.
 * Each callback is called from one library thread, in slice order, with
 * chunks of the same size (the last one shorter); the two run concurrently
 * with each other and with the device.  The handle's options apply
 * (ring_box, store, geometry, tile); the filtered sinograms are not returned.
 * A callback's non-zero return ends the call with CTAS_E_IO after the chunks
 * already on their way are written; absorption data that fail deAbs end it
 * with CTAS_E_DATA, the earlier chunks written.  Synchronous. */
int ctas_fbp_reconstruct_volume(ctas_fbp *h, int64_t n_slices, float center, int32_t bpp,
                                float mincon, float maxcon, ctas_vol_read_fn read,
                                ctas_vol_write_fn write, void *user);

/* Raw contiguous volumes: sinograms as float32 [n_slices][n_angles][width]
 * at byte in_offset of in_path; slices written as bpp samples
 * [n_slices][rows][cols] at byte out_offset of out_path (created if absent,
 * never truncated).  io_threads: threads per chunk read or write (0 = auto).
 * A short input file is CTAS_E_IO. */
int ctas_vol_raw_reconstruct(ctas_fbp *h, const char *in_path, int64_t in_offset,
                             int64_t n_slices, const char *out_path, int64_t out_offset,
                             float center, int32_t bpp, float mincon, float maxcon,
                             int32_t io_threads);

#ifdef __cplusplus
}
#endif

#endif /* CTAS_VOLUME_H */
