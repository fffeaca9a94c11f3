/*
 * In-memory stand-in for the part of the HDF5 C interface that the
 * reference's data readers use (src/reconstruct/aps_data/XT_HDFIO.c and
 * std_data/XT_HDFIO.c), so that those readers compile unmodified as CPU
 * oracles on a machine without libhdf5.  Test infrastructure only: nothing in
 * the product links it.
 *
 * A "file" is a name; its datasets are arrays registered beforehand with
 * ref_h5_register (h5_shim.c).  H5Dread copies the file space's selected
 * hyperslab (start and count per dimension, unit stride and block) into the
 * memory buffer, contiguous and in row-major order, which is what the
 * readers' memory spaces (the whole buffer selected) describe.
 */
#ifndef ORACLE_H5_STANDIN_H
#define ORACLE_H5_STANDIN_H

#include <stdint.h>

typedef int64_t hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;

#define H5F_ACC_RDONLY 0u
#define H5P_DEFAULT 0
#define H5S_SELECT_SET 0
#define H5T_NATIVE_UINT16 2
#define H5T_NATIVE_FLOAT 4

typedef int H5S_seloper_t;

hid_t H5Fopen(const char *name, unsigned flags, hid_t plist);
hid_t H5Dopen(hid_t file, const char *name, hid_t plist);
hid_t H5Dget_space(hid_t dset);
int H5Sget_simple_extent_ndims(hid_t space);
int H5Sget_simple_extent_dims(hid_t space, hsize_t *dims, hsize_t *maxdims);
herr_t H5Sselect_hyperslab(hid_t space, H5S_seloper_t op, const hsize_t *start, const hsize_t *stride,
                           const hsize_t *count, const hsize_t *block);
hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *maxdims);
herr_t H5Dread(hid_t dset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t plist, void *buf);
herr_t H5Sclose(hid_t space);
herr_t H5Dclose(hid_t dset);
herr_t H5Fclose(hid_t file);

/* registry (not HDF5): dataset `dset` of file `file`, element size 2 or 4 bytes */
int ref_h5_register(const char *file, const char *dset, const void *data, int elem_bytes, int rank,
                    const hsize_t *dims);
void ref_h5_clear(void);

#endif
