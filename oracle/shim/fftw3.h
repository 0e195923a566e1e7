/*
 * fftw3.h -- minimal FFTW3-API shim so that the reference's own C sources
 * under search/network/openmp compile in this image, where FFTW 3.3.10
 * (Makefile:14) is absent.  Test infrastructure only: it is linked into the
 * oracle builds under oracle/_ref and never into the product.
 *
 * Only the calls the reference path makes are declared
 * (init.c:717-753 plans, jobcore.c:333-355,477-478 new-array execute,
 * init.c:838-852 cleanup).  Complex types are the C99 complex types, as FFTW
 * defines them when <complex.h> is included first.  Plans compute with the
 * textbook transform in oracle/fft_core.c; the float plans compute in float.
 */
#ifndef TDF_SHIM_FFTW3_H
#define TDF_SHIM_FFTW3_H

#include <complex.h>
#include <stddef.h>

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)

typedef double _Complex fftw_complex;
typedef float _Complex fftwf_complex;
typedef struct shim_fftw_plan_s *fftw_plan;
typedef struct shim_fftw_plan_s *fftwf_plan;

int fftw_init_threads(void);
int fftwf_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftwf_plan_with_nthreads(int nthreads);

void *fftw_malloc(size_t n);
void *fftwf_malloc(size_t n);
void fftw_free(void *p);
void fftwf_free(void *p);

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftwf_execute(const fftwf_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);

void fftw_destroy_plan(fftw_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void fftw_cleanup(void);
void fftwf_cleanup(void);

#endif
