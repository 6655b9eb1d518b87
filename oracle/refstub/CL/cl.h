/*
 * Stand-in for the OpenCL header, so the reference's host file
 * src/calc_grad.c (the DFT-gradient assembly) compiles as plain C on the
 * host for the oracle pin.  TEST INFRASTRUCTURE ONLY: only the type names
 * that the reference's headers mention are declared; no OpenCL call is made.
 */
#ifndef SEISCL_REFSTUB_CL_H
#define SEISCL_REFSTUB_CL_H
#include <stddef.h>
#include <stdint.h>
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef int8_t cl_char;
typedef uint64_t cl_ulong;
typedef uint64_t cl_device_type;
typedef struct refstub_opaque *cl_mem, *cl_command_queue, *cl_event, *cl_kernel, *cl_program, *cl_context,
    *cl_device_id, *cl_platform_id;
typedef union {
    float s[2];
    struct { float x, y; };
} cl_float2;
#define CL_SUCCESS 0
#endif
