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

/* L2 read bandwidth in bytes/s: every CTA streams 16-byte loads that bypass L1
 * (ld.global.cg) through a 32 MiB buffer held in L2, and the kernel time in
 * seconds.  The staged backprojection fetches its detector windows from L2 by
 * TMA; this is the ceiling of that traffic.  Synchronous. */
int ctas_probe_l2_read(int device, double *bytes_per_s, double *seconds);

/* Failure-detection check: one CTA waits, with the bounded try-wait loop of
 * the pipelined kernels, on an mbarrier that nothing ever arrives at.  After
 * `limit` tries the wait gives up, sets the timeout bit of an error word and
 * the kernel returns; *timed_out receives 1 when that bit was set, *seconds
 * the kernel time.  The device stays usable (no fault, no hang).
 * Synchronous. */
int ctas_probe_bounded_wait(int device, uint32_t limit, int32_t *timed_out, double *seconds);

#ifdef __cplusplus
}
#endif
#endif
