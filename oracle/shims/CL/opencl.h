/* Minimal OpenCL type names so the reference's host sources compile as a CPU
 * oracle.  No OpenCL runtime exists here; every OCLwrapper method is a link
 * stub (oracle/ref_stubs.cc) that aborts if called. */
#ifndef GF_ORACLE_OPENCL_SHIM_H
#define GF_ORACLE_OPENCL_SHIM_H
#include <stddef.h>
#include <stdint.h>
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef uint32_t cl_bool;
typedef uint64_t cl_ulong;
typedef uint64_t cl_mem_flags;
typedef struct _cl_mem* cl_mem;
typedef struct _cl_program* cl_program;
typedef struct _cl_kernel* cl_kernel;
typedef struct _cl_command_queue* cl_command_queue;
typedef struct _cl_context* cl_context;
typedef struct _cl_platform_id* cl_platform_id;
typedef struct _cl_device_id* cl_device_id;
typedef struct _cl_event* cl_event;
#define CL_FALSE 0
#define CL_TRUE 1
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#endif
