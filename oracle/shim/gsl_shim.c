/*
 * gsl_shim.c -- implementation of the minimal GSL-API shim (test
 * infrastructure only); see gsl/gsl_shim_all.h for why it exists.
 * LU factorisation: Doolittle elimination with partial (row) pivoting, the
 * method GSL documents for gsl_linalg_LU_decomp (P A = L U).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_shim_all.h"

gsl_vector *gsl_vector_alloc(size_t n)
{
     gsl_vector *v = (gsl_vector *)calloc(1, sizeof(gsl_vector));
     v->size = n;
     v->stride = 1;
     v->data = (double *)calloc(n ? n : 1, sizeof(double));
     v->owner = 1;
     return v;
}

void gsl_vector_free(gsl_vector *v)
{
     if (!v) return;
     if (v->owner) free(v->data);
     free(v);
}

double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }

gsl_vector_view gsl_vector_view_array(double *base, size_t n)
{
     gsl_vector_view w;
     w.vector.size = n;
     w.vector.stride = 1;
     w.vector.data = base;
     w.vector.block = NULL;
     w.vector.owner = 0;
     return w;
}

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2)
{
     gsl_matrix *m = (gsl_matrix *)calloc(1, sizeof(gsl_matrix));
     m->size1 = n1;
     m->size2 = n2;
     m->tda = n2;
     m->data = (double *)calloc(n1 * n2 ? n1 * n2 : 1, sizeof(double));
     m->owner = 1;
     return m;
}

void gsl_matrix_free(gsl_matrix *m)
{
     if (!m) return;
     if (m->owner) free(m->data);
     free(m);
}

gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2)
{
     gsl_matrix_view w;
     w.matrix.size1 = n1;
     w.matrix.size2 = n2;
     w.matrix.tda = n2;
     w.matrix.data = base;
     w.matrix.block = NULL;
     w.matrix.owner = 0;
     return w;
}

int gsl_matrix_transpose(gsl_matrix *m)
{
     for (size_t i = 0; i < m->size1; i++)
          for (size_t j = i + 1; j < m->size2; j++) {
               double t = m->data[i * m->tda + j];
               m->data[i * m->tda + j] = m->data[j * m->tda + i];
               m->data[j * m->tda + i] = t;
          }
     return 0;
}

gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j)
{
     gsl_vector_view w;
     w.vector.size = m->size1;
     w.vector.stride = m->tda;
     w.vector.data = m->data + j;
     w.vector.block = NULL;
     w.vector.owner = 0;
     return w;
}

gsl_permutation *gsl_permutation_alloc(size_t n)
{
     gsl_permutation *p = (gsl_permutation *)calloc(1, sizeof(gsl_permutation));
     p->size = n;
     p->data = (size_t *)calloc(n ? n : 1, sizeof(size_t));
     for (size_t i = 0; i < n; i++) p->data[i] = i;
     return p;
}

void gsl_permutation_free(gsl_permutation *p)
{
     if (!p) return;
     free(p->data);
     free(p);
}

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum)
{
     size_t n = A->size1, t = A->tda;
     double *a = A->data;
     *signum = 1;
     for (size_t i = 0; i < n; i++) p->data[i] = i;
     for (size_t j = 0; j + 1 < n; j++) {
          size_t ip = j;
          double mx = fabs(a[j * t + j]);
          for (size_t i = j + 1; i < n; i++)
               if (fabs(a[i * t + j]) > mx) { mx = fabs(a[i * t + j]); ip = i; }
          if (ip != j) {
               for (size_t k = 0; k < n; k++) {
                    double tmp = a[j * t + k];
                    a[j * t + k] = a[ip * t + k];
                    a[ip * t + k] = tmp;
               }
               size_t tp = p->data[j];
               p->data[j] = p->data[ip];
               p->data[ip] = tp;
               *signum = -*signum;
          }
          double piv = a[j * t + j];
          if (piv != 0.0) {
               for (size_t i = j + 1; i < n; i++) {
                    double f = a[i * t + j] / piv;
                    a[i * t + j] = f;
                    for (size_t k = j + 1; k < n; k++) a[i * t + k] -= f * a[j * t + k];
               }
          }
     }
     return 0;
}

int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b, gsl_vector *x)
{
     size_t n = LU->size1, t = LU->tda;
     const double *a = LU->data;
     for (size_t i = 0; i < n; i++) x->data[i * x->stride] = b->data[p->data[i] * b->stride];
     for (size_t i = 0; i < n; i++) {
          double s = x->data[i * x->stride];
          for (size_t k = 0; k < i; k++) s -= a[i * t + k] * x->data[k * x->stride];
          x->data[i * x->stride] = s;
     }
     for (size_t ii = n; ii-- > 0;) {
          double s = x->data[ii * x->stride];
          for (size_t k = ii + 1; k < n; k++) s -= a[ii * t + k] * x->data[k * x->stride];
          x->data[ii * x->stride] = s / a[ii * t + ii];
     }
     return 0;
}

gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n)
{
     gsl_eigen_symmv_workspace *w = (gsl_eigen_symmv_workspace *)calloc(1, sizeof(*w));
     w->size = n;
     return w;
}

void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { free(w); }

int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w)
{
     (void)A; (void)eval; (void)evec; (void)w;
     fprintf(stderr, "gsl shim: gsl_eigen_symmv is not provided (coincidences-only path)\n");
     abort();
}
