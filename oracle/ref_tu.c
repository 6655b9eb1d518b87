/*
 * ref_tu.c -- one translation unit per reference kernel file.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build_ref.py compiles this file once per
 * kernel with -DREF_KERNEL_FILE=<file.cl> and the kernel's entry point renamed,
 * plus the grid and physics constants the reference would pass as -D options
 * (src/clprogram.c:449-571).  The kernel sources are read in place from the
 * reference tree through the include path.
 */
#include "ref_shim.h"
#include "header_CUDACL.cl"
#include "header_FD.cl"
#ifdef REF_WITH_INJECT
#include "header_injectbnd.cl"
#endif
#define REF_STR2(x) #x
#define REF_STR(x) REF_STR2(x)
#include REF_STR(REF_KERNEL_FILE)
