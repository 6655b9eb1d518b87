/*
 * ref_gpu_tu.cu -- one of the reference's CUDA kernel files, compiled in place.
 *
 * TEST INFRASTRUCTURE ONLY (the reference's own GPU kernels on the B200, for
 * parity and for timing beside this package's kernels).  oracle/build.py
 * compiles this file once per kernel file with -DREF_KERNEL_FILE=<file.cl>,
 * the entry point renamed by a -D (update_v -> ref_gpu_update_v, ...),
 * -DREF_ENTRY=<renamed entry>, -DREF_LAUNCH=<launcher name> and the -D
 * constants the reference passes to NVRTC (src/clprogram.c:449-571) with
 * LOCAL_OFF=0.  nvcc does not define __OPENCL_VERSION__, so
 * header_CUDACL.cl takes its CUDA branch as under NVRTC: the kernels are
 * extern "C" __global__ functions whose tiles live in dynamic shared memory
 * (LOCDEF), launched as src/clprogram.c:1030-1056 launches them.  The kernel
 * sources are read from the reference tree through the include path; nothing
 * of them is copied into this repository.
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "header_CUDACL.cl"
#include "header_FD.cl"
#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_KERNEL_FILE)

// Launch the file's kernel: grid and block as three unsigned each, the
// dynamic shared memory in bytes, and the kernel's arguments as
// cudaLaunchKernel takes them (one pointer per argument).  Returns the
// cudaError_t of the launch.
extern "C" int REF_LAUNCH(const unsigned *grid, const unsigned *block, unsigned smem, void **args, void *stream)
{
    return (int)cudaLaunchKernel((const void *)REF_ENTRY, dim3(grid[0], grid[1], grid[2]),
                                 dim3(block[0], block[1], block[2]), args, smem, (cudaStream_t)stream);
}
