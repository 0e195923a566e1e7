/*
 * fft_core.h -- textbook complex FFT used by the CPU oracle (test
 * infrastructure only; nothing in the product links it).
 *
 * The reference computes its FFTs with FFTW 3.3.10 (third-party, absent from
 * this image; install path pinned in search/network/openmp/Makefile:14).  Its
 * semantics, which this file restates, are the DFT definition:
 *     X[k] = sum_{n<N} x[n] * exp(sign * 2*pi*i * n*k / N)
 * unnormalised, sign = -1 for FFTW_FORWARD and +1 for FFTW_BACKWARD
 * (calls at search/network/openmp/jobcore.c:333-334,354-355,477-478).
 * Power-of-two lengths only (every nfft / Ninterp / nfftf of the path is a
 * power of two: search/network/openmp/settings.c:33,73,75).
 *
 * Algorithm: iterative radix-2 decimation in time (Cooley-Tukey 1965) with a
 * bit-reversal permutation and a per-plan twiddle table computed in double.
 * The float variant keeps float data and float twiddles, as FFTW's float
 * plans do.  Stages are parallelised with OpenMP.
 */
#ifndef TDF_ORACLE_FFT_CORE_H
#define TDF_ORACLE_FFT_CORE_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fftc_plan_s {
     int n;          /* transform length (power of two) */
     int sign;       /* -1 forward, +1 backward */
     int log2n;
     double *twd;    /* 2*(n/2) doubles: cos, sin of sign*2*pi*k/n */
     float *twf;     /* same, rounded to float */
     int *rev;       /* bit-reversal permutation */
} fftc_plan;

/* returns NULL if n is not a power of two >= 1 */
fftc_plan *fftc_plan_create(int n, int sign);
void fftc_plan_destroy(fftc_plan *p);

/* in may equal out (in-place) */
void fftc_execute_d(const fftc_plan *p, const double complex *in, double complex *out);
void fftc_execute_f(const fftc_plan *p, const float complex *in, float complex *out);

#ifdef __cplusplus
}
#endif

#endif
