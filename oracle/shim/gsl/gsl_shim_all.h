/*
 * gsl_shim_all.h -- minimal GSL-API shim (test infrastructure only) so that
 * the reference's own sources compile where GSL is absent.  The reference
 * path uses GSL only to solve the 4x4 grid system in dimless_to_code()
 * (search/network/openmp/auxi.c:63-90, reached from set_search_range() for
 * the directed_range / allsky_range grid types, init.c:630).  The
 * eigen-solver used by the coincidences tool (init.c:1094-1111) is declared
 * but aborts if called; the search never calls it.
 *
 * Type layouts follow GSL's public headers (size/stride/data fields).
 */
#ifndef TDF_SHIM_GSL_ALL_H
#define TDF_SHIM_GSL_ALL_H

#include <stddef.h>

typedef struct {
     size_t size;
     size_t stride;
     double *data;
     void *block;
     int owner;
} gsl_vector;

typedef struct {
     gsl_vector vector;
} gsl_vector_view;

typedef struct {
     size_t size1;
     size_t size2;
     size_t tda;
     double *data;
     void *block;
     int owner;
} gsl_matrix;

typedef struct {
     gsl_matrix matrix;
} gsl_matrix_view;

typedef struct {
     size_t size;
     size_t *data;
} gsl_permutation;

typedef struct {
     size_t size;
} gsl_eigen_symmv_workspace;

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
int gsl_matrix_transpose(gsl_matrix *m);
gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j);

gsl_permutation *gsl_permutation_alloc(size_t n);
void gsl_permutation_free(gsl_permutation *p);

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b, gsl_vector *x);

gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);

#endif
