/* Types-only stand-in for the OpenCL API header, written for this project so
 * that the reference's CPU_RUN build (which includes clinterface.h but makes
 * no OpenCL calls) compiles on a machine without OpenCL headers.  Declares
 * the scalar/vector typedefs and opaque handles the reference's headers
 * name; no function is declared or defined. */
#ifndef QG_REF_STUB_CL_H
#define QG_REF_STUB_CL_H
#include <stddef.h>
#include <stdint.h>
typedef int8_t   cl_char;
typedef uint8_t  cl_uchar;
typedef int16_t  cl_short;
typedef uint16_t cl_ushort;
typedef int32_t  cl_int;
typedef uint32_t cl_uint;
typedef int64_t  cl_long;
typedef uint64_t cl_ulong;
typedef float    cl_float;
typedef double   cl_double;
typedef cl_uint  cl_bool;
typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_device_type;
typedef cl_uint  cl_platform_info;
typedef cl_uint  cl_device_info;
typedef cl_bitfield cl_command_queue_properties;
typedef cl_bitfield cl_mem_flags;
typedef cl_uint  cl_program_build_info;
typedef cl_uint  cl_kernel_work_group_info;
typedef cl_uint  cl_profiling_info;
typedef struct _cl_platform_id *cl_platform_id;
typedef struct _cl_device_id *cl_device_id;
typedef struct _cl_context *cl_context;
typedef struct _cl_command_queue *cl_command_queue;
typedef struct _cl_mem *cl_mem;
typedef struct _cl_program *cl_program;
typedef struct _cl_kernel *cl_kernel;
typedef struct _cl_event *cl_event;
typedef union { cl_float s[2]; struct { cl_float x, y; }; } cl_float2;
typedef union { cl_float s[4]; struct { cl_float x, y, z, w; }; } cl_float4;
typedef union { cl_double s[2]; struct { cl_double x, y; }; } cl_double2;
typedef union { cl_double s[4]; struct { cl_double x, y, z, w; }; } cl_double4;
typedef union { cl_uint s[2]; struct { cl_uint x, y; }; } cl_uint2;
typedef union { cl_uint s[4]; struct { cl_uint x, y, z, w; }; } cl_uint4;
typedef union { cl_int s[4]; struct { cl_int x, y, z, w; }; } cl_int4;
#endif
