/*
 * Type-only HDF5 shim.  TEST INFRASTRUCTURE ONLY: euler_2d_par.h:75-80 declares
 * hid_t/herr_t globals, so the reference hot-path sources need these typedefs
 * to compile into the CPU oracle.  No HDF5 function is declared here; the
 * oracle never performs file I/O through HDF5.
 */
#ifndef HOS_ORACLE_SHIM_HDF5_H
#define HOS_ORACLE_SHIM_HDF5_H

typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#endif
