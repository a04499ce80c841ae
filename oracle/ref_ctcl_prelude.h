/*
 * ref_ctcl_prelude.h -- OpenCL C builtins needed to compile the reference's
 * backprojection kernel (src/common/ct.cl of ctas) as plain C99 with gcc.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle/Makefile).  Nothing here comes from the
 * reference: it defines the OpenCL C spellings that ct.cl uses -- the
 * address-space and kernel qualifiers, the float2 vector type with .x/.y, and
 * get_global_id() -- so that the kernel body runs once per work item on the
 * host.  The work-item id lives in thread-local storage set by the driver
 * (ref_ctcl_driver.c).
 */
#ifndef REF_CTCL_PRELUDE_H
#define REF_CTCL_PRELUDE_H
#include <math.h>
#include <stddef.h>

#define kernel
#define __kernel
#define global
#define __global

typedef struct { float x, y; } float2;

extern __thread size_t ref_ctcl_gid[2];
#define get_global_id(d) (ref_ctcl_gid[(d)])

#endif
