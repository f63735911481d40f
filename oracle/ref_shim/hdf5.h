/* Minimal HDF5 type declarations needed by the reference's include/TypeTraits.hpp.
 * Test infrastructure only (oracle build). */
#pragma once
typedef long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#define H5T_NATIVE_DOUBLE 1
#define H5T_NATIVE_INT 2
#define H5T_NATIVE_CHAR 3
static inline hid_t H5Tcopy(hid_t t) { return t; }
