/*
 * hdf5.h -- the HDF5 calls of the reference's host driver, over this
 * library's own HDF5 subset (no libhdf5).
 *
 * hdf5_routines_2d_par.c reads the run parameters and the initial condition
 * (get_params :13-101, get_ic_2d :104-188) and writes snapshots
 * (create_file_2d, write_header_2d, write_field_2d, write_coordinates_2d,
 * write_extra_2d, :191-537) through the calls declared below, on one rank
 * with a hyperslab selection that covers the whole [Nx][Ny] field.
 * libhos_hostshim.so implements them with hos_h5_info / hos_h5_read_f64 /
 * hos_h5_write (include/hos_gpu.h): reads convert the stored values as
 * H5Dread with H5T_IEEE_F64LE / F32LE does; a file created with H5Fcreate
 * collects its datasets in memory and is written at H5Fclose.  Datasets are
 * 2-D or lower; selections are H5S_ALL or one hyperslab block without
 * strides.  A call outside that subset returns a negative status and prints
 * the reason.  A host that has HDF5 uses its own header and library instead.
 */
#ifndef HOS_HOSTSHIM_HDF5_H
#define HOS_HOSTSHIM_HDF5_H

#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

typedef enum { H5S_SELECT_SET = 0 } H5S_seloper_t;

#define H5F_ACC_RDONLY 0x0000u
#define H5F_ACC_RDWR 0x0001u
#define H5F_ACC_TRUNC 0x0002u
#define H5F_ACC_EXCL 0x0004u

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5P_FILE_ACCESS ((hid_t)0x1000000001LL)
#define H5P_DATASET_XFER ((hid_t)0x1000000002LL)
#define H5T_IEEE_F64LE ((hid_t)0x2000000001LL)
#define H5T_IEEE_F32LE ((hid_t)0x2000000002LL)
#define H5T_NATIVE_DOUBLE H5T_IEEE_F64LE
#define H5T_NATIVE_FLOAT H5T_IEEE_F32LE

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t file);

hid_t H5Dopen(hid_t file, const char* name, hid_t dapl);
hid_t H5Dcreate(hid_t file, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
herr_t H5Dread(hid_t dset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t xfer, void* buf);
herr_t H5Dwrite(hid_t dset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t xfer, const void* buf);
hid_t H5Dget_space(hid_t dset);
herr_t H5Dclose(hid_t dset);

hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims);
herr_t H5Sselect_hyperslab(hid_t space, H5S_seloper_t op, const hsize_t* start, const hsize_t* stride,
                           const hsize_t* count, const hsize_t* block);
herr_t H5Sclose(hid_t space);

hid_t H5Pcreate(hid_t cls);
herr_t H5Pset_fapl_mpio(hid_t fapl, MPI_Comm comm, MPI_Info info);
herr_t H5Pclose(hid_t plist);

hid_t H5Tcopy(hid_t type);
herr_t H5Tclose(hid_t type);

#ifdef __cplusplus
}
#endif

#endif
