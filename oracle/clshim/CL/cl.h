/* Declaration-only OpenCL 1.1 header used to compile the reference
 * interpreter as a CPU oracle. Written from the public OpenCL 1.1 API
 * (Khronos specification, section 4 and 5 signatures). No OpenCL runtime
 * exists on this machine: every entry point is stubbed in clstub.c to report
 * failure, so the reference finds zero platforms (vendor/OCLinit.cpp:12-24)
 * and DeviceMap builds only the interpreter (runtime/DeviceMap.cpp:17-23).
 *
 * Test infrastructure only; nothing in the product includes this file. */
#ifndef CHAI_ORACLE_CL_SHIM_H
#define CHAI_ORACLE_CL_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t  cl_int;
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef cl_uint  cl_bool;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_device_type;
typedef cl_uint  cl_platform_info;
typedef cl_uint  cl_device_info;
typedef cl_bitfield cl_command_queue_properties;
typedef intptr_t cl_context_properties;
typedef cl_bitfield cl_mem_flags;
typedef cl_uint  cl_program_build_info;
typedef cl_uint  cl_channel_order;
typedef cl_uint  cl_channel_type;

typedef struct _cl_platform_id*   cl_platform_id;
typedef struct _cl_device_id*     cl_device_id;
typedef struct _cl_context*       cl_context;
typedef struct _cl_command_queue* cl_command_queue;
typedef struct _cl_mem*           cl_mem;
typedef struct _cl_program*       cl_program;
typedef struct _cl_kernel*        cl_kernel;
typedef struct _cl_event*         cl_event;

typedef struct _cl_image_format {
    cl_channel_order image_channel_order;
    cl_channel_type  image_channel_data_type;
} cl_image_format;

#define CL_SUCCESS                  0
#define CL_DEVICE_NOT_FOUND        -1
#define CL_INVALID_VALUE          -30
#define CL_INVALID_PLATFORM       -32

#define CL_FALSE 0
#define CL_TRUE  1

#define CL_DEVICE_TYPE_CPU          (1 << 1)
#define CL_DEVICE_TYPE_GPU          (1 << 2)
#define CL_DEVICE_TYPE_ACCELERATOR  (1 << 3)
#define CL_DEVICE_TYPE_ALL          0xFFFFFFFF

#define CL_DEVICE_TYPE                 0x1000
#define CL_DEVICE_MAX_WORK_GROUP_SIZE  0x1004
#define CL_DEVICE_NAME                 0x102B
#define CL_DEVICE_VENDOR               0x102C

#define CL_QUEUE_OUT_OF_ORDER_EXEC_MODE_ENABLE (1 << 0)
#define CL_QUEUE_PROFILING_ENABLE              (1 << 1)

#define CL_CONTEXT_PLATFORM 0x1084

#define CL_MEM_READ_WRITE     (1 << 0)
#define CL_MEM_WRITE_ONLY     (1 << 1)
#define CL_MEM_READ_ONLY      (1 << 2)
#define CL_MEM_USE_HOST_PTR   (1 << 3)
#define CL_MEM_ALLOC_HOST_PTR (1 << 4)

#define CL_RGBA            0x10B5
#define CL_SIGNED_INT32    0x10D9
#define CL_UNSIGNED_INT32  0x10DC
#define CL_FLOAT           0x10DE

#define CL_PROGRAM_BUILD_LOG 0x1183

cl_int clGetPlatformIDs(cl_uint, cl_platform_id*, cl_uint*);
cl_int clGetDeviceIDs(cl_platform_id, cl_device_type, cl_uint, cl_device_id*, cl_uint*);
cl_int clGetDeviceInfo(cl_device_id, cl_device_info, size_t, void*, size_t*);
cl_context clCreateContext(const cl_context_properties*, cl_uint, const cl_device_id*,
                           void (*)(const char*, const void*, size_t, void*), void*, cl_int*);
cl_int clReleaseContext(cl_context);
cl_command_queue clCreateCommandQueue(cl_context, cl_device_id, cl_command_queue_properties, cl_int*);
cl_int clReleaseCommandQueue(cl_command_queue);
cl_mem clCreateBuffer(cl_context, cl_mem_flags, size_t, void*, cl_int*);
cl_mem clCreateImage2D(cl_context, cl_mem_flags, const cl_image_format*, size_t, size_t, size_t,
                       void*, cl_int*);
cl_int clReleaseMemObject(cl_mem);
cl_program clCreateProgramWithSource(cl_context, cl_uint, const char**, const size_t*, cl_int*);
cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id*, const char*,
                      void (*)(cl_program, void*), void*);
cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t, void*, size_t*);
cl_int clReleaseProgram(cl_program);
cl_kernel clCreateKernel(cl_program, const char*, cl_int*);
cl_int clReleaseKernel(cl_kernel);
cl_int clSetKernelArg(cl_kernel, cl_uint, size_t, const void*);
cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel, cl_uint, const size_t*, const size_t*,
                              const size_t*, cl_uint, const cl_event*, cl_event*);
cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, void*, cl_uint,
                           const cl_event*, cl_event*);
cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem, cl_bool, size_t, size_t, const void*, cl_uint,
                            const cl_event*, cl_event*);
cl_int clEnqueueReadImage(cl_command_queue, cl_mem, cl_bool, const size_t*, const size_t*, size_t,
                          size_t, void*, cl_uint, const cl_event*, cl_event*);
cl_int clEnqueueWriteImage(cl_command_queue, cl_mem, cl_bool, const size_t*, const size_t*, size_t,
                           size_t, const void*, cl_uint, const cl_event*, cl_event*);
cl_int clWaitForEvents(cl_uint, const cl_event*);
cl_int clReleaseEvent(cl_event);

#ifdef __cplusplus
}
#endif

#endif
