/*
 * Type stubs so that the reference header util.h (which includes <hdf5.h>)
 * compiles without libhdf5.  The HDF5 I/O functions are declared but never
 * defined or called by the oracle build.  TEST INFRASTRUCTURE ONLY.
 */
#pragma once
#include <stdint.h>
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
