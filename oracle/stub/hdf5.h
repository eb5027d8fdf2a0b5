/* Minimal stand-in for <hdf5.h> so that the reference's hot-path translation
 * units (global, knn, voronoi, hydro) compile without libhdf5.  Only the three
 * integer typedefs that those headers name are provided; no HDF5 function is
 * declared, so any accidental use of the HDF5 API fails at compile time.
 * hsize_t is HDF5's unsigned 64-bit size type. */
#ifndef PGPU_ORACLE_STUB_HDF5_H
#define PGPU_ORACLE_STUB_HDF5_H
typedef unsigned long long hsize_t;
typedef long long hid_t;
typedef int herr_t;
#endif
