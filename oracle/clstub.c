/* OpenCL entry points for the oracle build of the reference interpreter.
 * Every call fails, so the reference sees no OpenCL platform
 * (vendor/OCLinit.cpp:12-24) and schedules every trace on its CPU
 * interpreter device (runtime/DeviceMap.cpp:17-23).
 *
 * Test infrastructure only; nothing in the product links this file. */
#include "CL/cl.h"

cl_int clGetPlatformIDs(cl_uint n, cl_platform_id* p, cl_uint* num)
{
    (void)n; (void)p;
    if (num) *num = 0;
    return CL_INVALID_PLATFORM;
}
cl_int clGetDeviceIDs(cl_platform_id a, cl_device_type b, cl_uint c, cl_device_id* d, cl_uint* e)
{
    (void)a; (void)b; (void)c; (void)d;
    if (e) *e = 0;
    return CL_DEVICE_NOT_FOUND;
}
cl_int clGetDeviceInfo(cl_device_id a, cl_device_info b, size_t c, void* d, size_t* e)
{ (void)a; (void)b; (void)c; (void)d; (void)e; return CL_INVALID_VALUE; }
cl_context clCreateContext(const cl_context_properties* a, cl_uint b, const cl_device_id* c,
                           void (*d)(const char*, const void*, size_t, void*), void* e, cl_int* f)
{ (void)a; (void)b; (void)c; (void)d; (void)e; if (f) *f = CL_INVALID_VALUE; return 0; }
cl_int clReleaseContext(cl_context a) { (void)a; return CL_INVALID_VALUE; }
cl_command_queue clCreateCommandQueue(cl_context a, cl_device_id b, cl_command_queue_properties c, cl_int* d)
{ (void)a; (void)b; (void)c; if (d) *d = CL_INVALID_VALUE; return 0; }
cl_int clReleaseCommandQueue(cl_command_queue a) { (void)a; return CL_INVALID_VALUE; }
cl_mem clCreateBuffer(cl_context a, cl_mem_flags b, size_t c, void* d, cl_int* e)
{ (void)a; (void)b; (void)c; (void)d; if (e) *e = CL_INVALID_VALUE; return 0; }
cl_mem clCreateImage2D(cl_context a, cl_mem_flags b, const cl_image_format* c, size_t d, size_t e,
                       size_t f, void* g, cl_int* h)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; if (h) *h = CL_INVALID_VALUE; return 0; }
cl_int clReleaseMemObject(cl_mem a) { (void)a; return CL_INVALID_VALUE; }
cl_program clCreateProgramWithSource(cl_context a, cl_uint b, const char** c, const size_t* d, cl_int* e)
{ (void)a; (void)b; (void)c; (void)d; if (e) *e = CL_INVALID_VALUE; return 0; }
cl_int clBuildProgram(cl_program a, cl_uint b, const cl_device_id* c, const char* d,
                      void (*e)(cl_program, void*), void* f)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; return CL_INVALID_VALUE; }
cl_int clGetProgramBuildInfo(cl_program a, cl_device_id b, cl_program_build_info c, size_t d, void* e, size_t* f)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; return CL_INVALID_VALUE; }
cl_int clReleaseProgram(cl_program a) { (void)a; return CL_INVALID_VALUE; }
cl_kernel clCreateKernel(cl_program a, const char* b, cl_int* c)
{ (void)a; (void)b; if (c) *c = CL_INVALID_VALUE; return 0; }
cl_int clReleaseKernel(cl_kernel a) { (void)a; return CL_INVALID_VALUE; }
cl_int clSetKernelArg(cl_kernel a, cl_uint b, size_t c, const void* d)
{ (void)a; (void)b; (void)c; (void)d; return CL_INVALID_VALUE; }
cl_int clEnqueueNDRangeKernel(cl_command_queue a, cl_kernel b, cl_uint c, const size_t* d, const size_t* e,
                              const size_t* f, cl_uint g, const cl_event* h, cl_event* i)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; return CL_INVALID_VALUE; }
cl_int clEnqueueReadBuffer(cl_command_queue a, cl_mem b, cl_bool c, size_t d, size_t e, void* f, cl_uint g,
                           const cl_event* h, cl_event* i)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; return CL_INVALID_VALUE; }
cl_int clEnqueueWriteBuffer(cl_command_queue a, cl_mem b, cl_bool c, size_t d, size_t e, const void* f,
                            cl_uint g, const cl_event* h, cl_event* i)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; return CL_INVALID_VALUE; }
cl_int clEnqueueReadImage(cl_command_queue a, cl_mem b, cl_bool c, const size_t* d, const size_t* e, size_t f,
                          size_t g, void* h, cl_uint i, const cl_event* j, cl_event* k)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; (void)j; (void)k;
  return CL_INVALID_VALUE; }
cl_int clEnqueueWriteImage(cl_command_queue a, cl_mem b, cl_bool c, const size_t* d, const size_t* e, size_t f,
                           size_t g, const void* h, cl_uint i, const cl_event* j, cl_event* k)
{ (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; (void)j; (void)k;
  return CL_INVALID_VALUE; }
cl_int clWaitForEvents(cl_uint a, const cl_event* b) { (void)a; (void)b; return CL_INVALID_VALUE; }
cl_int clReleaseEvent(cl_event a) { (void)a; return CL_INVALID_VALUE; }
