/* Stand-in: the reference only needs hsize_t outside its H5_HAVE_PARALLEL blocks. */
#ifndef ORACLE_REFSHIM_HDF5_H
#define ORACLE_REFSHIM_HDF5_H
typedef unsigned long long hsize_t;
#endif
