/*
 * ctas_probe.h -- measurement entry points (no reference counterpart).
 *
 * The backprojection gathers every sample from shared memory, so its roofline
 * is the shared-memory load throughput of the GPU rather than HBM or the
 * tensor cores.  ctas_probe_smem_gather measures that ceiling on the current
 * device with a kernel that does nothing but conflict-free 32-bit shared
 * loads and adds, the same instruction mix as the backprojection's inner loop
 * without the index arithmetic.
 */
#ifndef CTAS_PROBE_H
#define CTAS_PROBE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Achieved shared-memory load bandwidth in bytes/s (4 bytes per lane per
 * load) and the measured kernel time in seconds.  Synchronous. */
int ctas_probe_smem_gather(int device, double *bytes_per_s, double *seconds);

#ifdef __cplusplus
}
#endif
#endif
