/*
 * hdf5.h -- type-only HDF5 shim (test infrastructure only).  The reference
 * path needs hvl_t for its Trigger record (search/network/openmp/struct.h:6,
 * 211-215).  The HDF5 writer itself (io.c) is replaced by oracle/ref_io.c, so
 * no HDF5 function is declared here.  hvl_t keeps HDF5's layout:
 * { size_t len; void *p; }.  Like the real header it brings in <stdlib.h>
 * and <stdio.h>, which the reference's sources rely on.
 */
#ifndef TDF_SHIM_HDF5_H
#define TDF_SHIM_HDF5_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

typedef struct {
     size_t len;
     void *p;
} hvl_t;

#endif
