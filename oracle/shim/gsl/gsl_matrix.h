/* gsl_matrix.h -- forwards to the minimal GSL-API shim (test infrastructure only). */
#include "gsl_shim_all.h"
