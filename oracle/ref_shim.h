/*
 * ref_shim.h -- lets the reference's OpenCL kernel sources compile as plain C
 * on the host, so the oracle can be pinned against them.
 *
 * TEST INFRASTRUCTURE ONLY.  Used by oracle/ref_tu.c, which includes the
 * reference kernel files in place (they are not copied into this repository).
 * Each work-item index comes from a thread-local array the glue code sets.
 */
#ifndef SEISCL_REF_SHIM_H
#define SEISCL_REF_SHIM_H
#define __OPENCL_VERSION__ 120
#define __kernel
#define __global
#define __local
#define CLK_LOCAL_MEM_FENCE 0
#define barrier(x) ((void)0)
extern __thread int fdo_ref_gid[3];
#define get_global_id(d) (fdo_ref_gid[(d)])
#define get_local_size(d) 1
#define get_local_id(d) 0
typedef struct { float x, y; } float2;
typedef unsigned short half;
typedef struct { half x, y; } half2;
#endif
