/*
 * H5Epublic.h -- empty stand-in (test infrastructure only): the coincidence
 * program includes it (coincidences/coincidences.c:1) but uses no HDF5
 * error API; its HDF5 I/O is replaced by oracle/coinc_io.c.
 */
#ifndef TDF_SHIM_H5EPUBLIC_H
#define TDF_SHIM_H5EPUBLIC_H
#include "hdf5.h"
#endif
