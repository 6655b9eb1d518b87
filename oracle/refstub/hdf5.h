/*
 * Stand-in for the HDF5 header (type names only), for compiling the
 * reference's src/calc_grad.c in place.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef SEISCL_REFSTUB_HDF5_H
#define SEISCL_REFSTUB_HDF5_H
#include <stdint.h>
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#endif
