/*
 * CL/cl.h -- stand-in for the OpenCL API header, for compiling the reference's
 * reconstruction code (ctas src/common/lct.cpp, parallel.world.*) on a machine
 * without an OpenCL SDK.  Test infrastructure only: it declares the types,
 * constants and entry points those files name, with the signatures of the
 * OpenCL 2.2 API, and every entry point reports that no platform exists.  The
 * reference then finds no OpenCL device (parallel.world.cpp, _CL_intialize),
 * CL_isReady() is false and CTrec runs its CPU path (lct.cpp:519-524,
 * 688-729), which is the code the oracle wants to run.
 */
#ifndef CTAS_ORACLE_SHIM_CL_H
#define CTAS_ORACLE_SHIM_CL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef float cl_float;
typedef cl_uint cl_bool;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_device_type;
typedef cl_bitfield cl_mem_flags;
typedef cl_bitfield cl_device_exec_capabilities;
typedef cl_bitfield cl_queue_properties;
typedef intptr_t cl_context_properties;
typedef cl_uint cl_device_info;
typedef cl_uint cl_context_info;
typedef cl_uint cl_program_info;
typedef cl_uint cl_program_build_info;
typedef cl_int cl_build_status;
typedef cl_uint cl_kernel_info;
typedef cl_uint cl_kernel_work_group_info;
typedef cl_uint cl_command_queue_info;
typedef cl_uint cl_image_info;
typedef cl_uint cl_mem_object_type;
typedef cl_uint cl_channel_order;
typedef cl_uint cl_channel_type;

typedef struct _cl_platform_id *cl_platform_id;
typedef struct _cl_device_id *cl_device_id;
typedef struct _cl_context *cl_context;
typedef struct _cl_command_queue *cl_command_queue;
typedef struct _cl_mem *cl_mem;
typedef struct _cl_program *cl_program;
typedef struct _cl_kernel *cl_kernel;
typedef struct _cl_event *cl_event;

/* vector types: .s[], .x/.y(/.z/.w) name the same storage */
typedef union {
  cl_float s[2];
  struct { cl_float x, y; };
  struct { cl_float s0, s1; };
} __attribute__((aligned(8))) cl_float2;

typedef union {
  cl_float s[4];
  struct { cl_float x, y, z, w; };
  struct { cl_float s0, s1, s2, s3; };
} __attribute__((aligned(16))) cl_float4;

typedef struct {
  cl_channel_order image_channel_order;
  cl_channel_type image_channel_data_type;
} cl_image_format;

typedef struct {
  cl_mem_object_type image_type;
  size_t image_width;
  size_t image_height;
  size_t image_depth;
  size_t image_array_size;
  size_t image_row_pitch;
  size_t image_slice_pitch;
  cl_uint num_mip_levels;
  cl_uint num_samples;
  union { cl_mem buffer; cl_mem mem_object; };
} cl_image_desc;

#define CL_SUCCESS 0
#define CL_DEVICE_NOT_FOUND (-1)
#define CL_INVALID_VALUE (-30)
#define CL_INVALID_PLATFORM (-32)
#define CL_PLATFORM_NOT_FOUND_KHR (-1001)
#define CL_FALSE 0
#define CL_TRUE 1

#define CL_DEVICE_TYPE_GPU (1 << 2)
#define CL_DEVICE_GLOBAL_MEM_SIZE 0x101F
#define CL_DEVICE_AVAILABLE 0x1027
#define CL_DEVICE_COMPILER_AVAILABLE 0x1028
#define CL_DEVICE_EXECUTION_CAPABILITIES 0x1029
#define CL_EXEC_KERNEL (1 << 0)
#define CL_CONTEXT_DEVICES 0x1081
#define CL_CONTEXT_NUM_DEVICES 0x1083
#define CL_QUEUE_CONTEXT 0x1090
#define CL_QUEUE_DEVICE 0x1091
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_MEM_OBJECT_IMAGE2D 0x10F1
#define CL_MEM_OBJECT_IMAGE3D 0x10F2
#define CL_IMAGE_WIDTH 0x1114
#define CL_IMAGE_HEIGHT 0x1115
#define CL_IMAGE_DEPTH 0x1116
#define CL_PROGRAM_CONTEXT 0x1161
#define CL_PROGRAM_BUILD_STATUS 0x1181
#define CL_PROGRAM_BUILD_OPTIONS 0x1182
#define CL_PROGRAM_BUILD_LOG 0x1183
#define CL_BUILD_SUCCESS 0
#define CL_KERNEL_FUNCTION_NAME 0x1190
#define CL_KERNEL_CONTEXT 0x1193
#define CL_KERNEL_PROGRAM 0x1194
#define CL_KERNEL_PREFERRED_WORK_GROUP_SIZE_MULTIPLE 0x11B3
#define CL_R 0x10B0
#define CL_FLOAT 0x10DE

/* Every entry point fails: there is no OpenCL platform. */
#define CTAS_SHIM_NO_CL(ret) { return ret; }

static inline cl_int clGetPlatformIDs(cl_uint n, cl_platform_id *p, cl_uint *np) {
  (void)n; (void)p;
  if (np) *np = 0;
  return CL_PLATFORM_NOT_FOUND_KHR;
}
static inline cl_int clGetDeviceIDs(cl_platform_id, cl_device_type, cl_uint, cl_device_id *,
                                    cl_uint *nd) {
  if (nd) *nd = 0;
  return CL_DEVICE_NOT_FOUND;
}
static inline cl_int clGetDeviceInfo(cl_device_id, cl_device_info, size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_context clCreateContext(const cl_context_properties *, cl_uint,
                                         const cl_device_id *,
                                         void (*)(const char *, const void *, size_t, void *),
                                         void *, cl_int *e) {
  if (e) *e = CL_DEVICE_NOT_FOUND;
  return 0;
}
static inline cl_command_queue clCreateCommandQueueWithProperties(cl_context, cl_device_id,
                                                                  const cl_queue_properties *,
                                                                  cl_int *e) {
  if (e) *e = CL_DEVICE_NOT_FOUND;
  return 0;
}
static inline cl_int clGetContextInfo(cl_context, cl_context_info, size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clGetCommandQueueInfo(cl_command_queue, cl_command_queue_info, size_t,
                                           void *, size_t *) CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_program clCreateProgramWithSource(cl_context, cl_uint, const char **,
                                                   const size_t *, cl_int *e) {
  if (e) *e = CL_INVALID_VALUE;
  return 0;
}
static inline cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id *, const char *,
                                    void (*)(cl_program, void *), void *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info,
                                           size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clGetProgramInfo(cl_program, cl_program_info, size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clReleaseProgram(cl_program) CTAS_SHIM_NO_CL(CL_SUCCESS)
static inline cl_kernel clCreateKernel(cl_program, const char *, cl_int *e) {
  if (e) *e = CL_INVALID_VALUE;
  return 0;
}
static inline cl_int clReleaseKernel(cl_kernel) CTAS_SHIM_NO_CL(CL_SUCCESS)
static inline cl_int clGetKernelInfo(cl_kernel, cl_kernel_info, size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clGetKernelWorkGroupInfo(cl_kernel, cl_device_id, cl_kernel_work_group_info,
                                              size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t *,
                                            const size_t *, const size_t *, cl_uint,
                                            const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clFinish(cl_command_queue) CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void *, cl_int *e) {
  if (e) *e = CL_INVALID_VALUE;
  return 0;
}
static inline cl_int clReleaseMemObject(cl_mem) CTAS_SHIM_NO_CL(CL_SUCCESS)
static inline cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t,
                                          const void *, cl_uint, const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t,
                                         void *, cl_uint, const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueReadBufferRect(cl_command_queue, cl_mem, cl_bool, const size_t *,
                                             const size_t *, const size_t *, size_t, size_t,
                                             size_t, size_t, void *, cl_uint, const cl_event *,
                                             cl_event *) CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueFillBuffer(cl_command_queue, cl_mem, const void *, size_t, size_t,
                                         size_t, cl_uint, const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_mem clCreateImage(cl_context, cl_mem_flags, const cl_image_format *,
                                   const cl_image_desc *, void *, cl_int *e) {
  if (e) *e = CL_INVALID_VALUE;
  return 0;
}
static inline cl_int clGetImageInfo(cl_mem, cl_image_info, size_t, void *, size_t *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueFillImage(cl_command_queue, cl_mem, const void *, const size_t *,
                                        const size_t *, cl_uint, const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueReadImage(cl_command_queue, cl_mem, cl_bool, const size_t *,
                                        const size_t *, size_t, size_t, void *, cl_uint,
                                        const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)
static inline cl_int clEnqueueWriteImage(cl_command_queue, cl_mem, cl_bool, const size_t *,
                                         const size_t *, size_t, size_t, const void *, cl_uint,
                                         const cl_event *, cl_event *)
    CTAS_SHIM_NO_CL(CL_INVALID_VALUE)

#undef CTAS_SHIM_NO_CL

#ifdef __cplusplus
}
#endif
#endif
