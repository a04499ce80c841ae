/*
 * ref_ctcl_driver.c -- host driver for the reference's OpenCL kernel `fbp`
 * (ctas src/common/ct.cl:5-44) compiled as C by oracle/Makefile.
 *
 * TEST INFRASTRUCTURE ONLY.  It plays the role of the OpenCL runtime in
 * CTrec::ForCLdev::reconstruct (src/common/lct.cpp:394-416): one call of the
 * kernel body per work item (i = column, j = row) of the W x W NDRange, with
 * the arguments that lct.cpp:357-362 and :408 bind.  Rows are spread over
 * POSIX threads, one contiguous band per thread, like the reference's own
 * slice-level thread pool spreads slices.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include "ref_ctcl_prelude.h"

__thread size_t ref_ctcl_gid[2];

/* The reference kernel, compiled from ct.cl. */
void fbp(const float *sino, float *slice, int pixels, int thetas,
         const float2 *cossins, float center, float coeff);

typedef struct {
  const float *sino; float *slice; int W, N; const float2 *tab;
  float center, coeff; int64_t r0, r1;
  const int64_t *rows; int64_t nrows; int stride;
} job_t;

/* rows rows[t], rows[t + stride], ... of a row list */
static void *run_row_list(void *arg) {
  job_t *jb = (job_t *)arg;
  for (int64_t r = jb->r0; r < jb->nrows; r += jb->stride) {
    const int64_t j = jb->rows[r];
    for (int64_t i = 0; i < jb->W; i++) {
      ref_ctcl_gid[0] = (size_t)i;
      ref_ctcl_gid[1] = (size_t)j;
      fbp(jb->sino, jb->slice, jb->W, jb->N, jb->tab, jb->center, jb->coeff);
    }
  }
  return NULL;
}

static void *run_rows(void *arg) {
  job_t *jb = (job_t *)arg;
  for (int64_t j = jb->r0; j < jb->r1; j++)
    for (int64_t i = 0; i < jb->W; i++) {
      ref_ctcl_gid[0] = (size_t)i;
      ref_ctcl_gid[1] = (size_t)j;
      fbp(jb->sino, jb->slice, jb->W, jb->N, jb->tab, jb->center, jb->coeff);
    }
  return NULL;
}

/* Reconstruct rows [r0, r1) of the W x W slice.  `slice` must hold the full
 * W x W image (the kernel indexes it by i + j*W).  tab: N (sin, cos) pairs as
 * CTrec builds them (lct.cpp:512-517).  Returns 0 or -1. */
int ref_ctcl_fbp(const float *sino, float *slice, int W, int N,
                 const float *tab, float center, float coeff, int64_t r0,
                 int64_t r1, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (r1 <= r0) return 0;
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
  char *live = (char *)calloc((size_t)nthreads, 1);
  job_t *jobs = (job_t *)malloc(sizeof(job_t) * (size_t)nthreads);
  int64_t rows = r1 - r0;
  for (int t = 0; t < nthreads; t++) {
    int64_t a = r0 + rows * t / nthreads, b = r0 + rows * (t + 1) / nthreads;
    jobs[t] = (job_t){sino, slice, W, N, (const float2 *)tab, center, coeff, a, b, NULL, 0, 1};
    if (b <= a) continue;
    if (nthreads > 1 && pthread_create(&th[t], NULL, run_rows, &jobs[t]) == 0)
      live[t] = 1;
    else
      run_rows(&jobs[t]);
  }
  for (int t = 0; t < nthreads; t++)
    if (live[t]) pthread_join(th[t], NULL);
  free(live);
  free(th); free(jobs);
  return 0;
}

/* Reconstruct the listed rows (each 0 <= row < W) of the W x W slice, rows
 * dealt round-robin to `nthreads` threads.  Returns 0. */
int ref_ctcl_fbp_rows(const float *sino, float *slice, int W, int N, const float *tab,
                      float center, float coeff, const int64_t *rows, int64_t nrows,
                      int nthreads) {
  if (nthreads < 1) nthreads = 1;
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
  char *live = (char *)calloc((size_t)nthreads, 1);
  job_t *jobs = (job_t *)malloc(sizeof(job_t) * (size_t)nthreads);
  for (int t = 0; t < nthreads; t++) {
    jobs[t] = (job_t){sino, slice, W, N, (const float2 *)tab, center, coeff, t, 0,
                      rows, nrows, nthreads};
    if (nthreads > 1 && pthread_create(&th[t], NULL, run_row_list, &jobs[t]) == 0)
      live[t] = 1;
    else
      run_row_list(&jobs[t]);
  }
  for (int t = 0; t < nthreads; t++)
    if (live[t]) pthread_join(th[t], NULL);
  free(th); free(live); free(jobs);
  return 0;
}
