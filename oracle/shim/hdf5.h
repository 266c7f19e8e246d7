/*
 * Minimal stand-in for the HDF5 C API subset used by GAMERA-OP's
 * src/hdf5_io.c, so the reference compiles and runs as the CPU oracle on a
 * machine without libhdf5.  Test infrastructure only.
 *
 * Every "HDF5 file" is written as a flat little-endian record file
 * ("GOPRAW01" format, read back by oracle/ref_io.py): for each dataset its
 * name, element type, shape and raw row-major data.  Names, shapes and dtypes
 * are exactly the ones hdf5_io.c asks for, so the per-step layout
 * (/gas[NS1][18][NI][NJ][NK], /gem[18][NI][NJ][NK], ...) is preserved.
 * Chunking and deflate settings are accepted and ignored.
 *
 * Setting GOP_H5_DISCARD=1 in the environment drops all writes (used when the
 * reference is timed: output is disabled during timing).
 */
#ifndef GOP_SHIM_HDF5_H
#define GOP_SHIM_HDF5_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef int H5S_seloper_t;

#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u
#define H5P_DEFAULT ((hid_t)0)
#define H5P_DATASET_CREATE ((hid_t)-100)
#define H5S_ALL ((hid_t)0)
#define H5S_SELECT_SET 0
#define H5S_MAX_RANK 32
#define H5T_NATIVE_DOUBLE ((hid_t)-1)
#define H5T_NATIVE_INT ((hid_t)-2)

hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl);
hid_t H5Fopen(const char *name, unsigned flags, hid_t fapl);
herr_t H5Fclose(hid_t file);

hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *maxdims);
herr_t H5Sclose(hid_t space);
herr_t H5Sselect_hyperslab(hid_t space, H5S_seloper_t op, const hsize_t *start,
                           const hsize_t *stride, const hsize_t *count,
                           const hsize_t *block);
int H5Sget_simple_extent_ndims(hid_t space);
int H5Sget_simple_extent_dims(hid_t space, hsize_t *dims, hsize_t *maxdims);

hid_t H5Pcreate(hid_t cls);
herr_t H5Pclose(hid_t plist);
herr_t H5Pset_chunk(hid_t plist, int ndims, const hsize_t *dims);
herr_t H5Pset_deflate(hid_t plist, unsigned level);

hid_t H5Dcreate2(hid_t loc, const char *name, hid_t type, hid_t space,
                 hid_t lcpl, hid_t dcpl, hid_t dapl);
hid_t H5Dopen2(hid_t loc, const char *name, hid_t dapl);
#define H5Dopen H5Dopen2
herr_t H5Dclose(hid_t dset);
hid_t H5Dget_space(hid_t dset);
herr_t H5Dwrite(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace,
                hid_t plist, const void *buf);
herr_t H5Dread(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace,
               hid_t plist, void *buf);

#ifdef __cplusplus
}
#endif
#endif
