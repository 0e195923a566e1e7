/*
 * fft_time.c -- times the FFT the reference binaries here are linked with:
 * the FFTW-API shim (shim/fftw_shim.c over fft_core.c), built with the
 * reference's FLOAT-build flags like oracle/_ref/gwsearch-ref-f32.  Runs
 * single-precision in-place transforms of length n through
 * fftwf_plan_dft_1d / fftwf_execute_dft as jobcore.c:477-478 does and prints
 * the seconds per transform.  TEST INFRASTRUCTURE ONLY: bench.py's CPU
 * baseline uses it to report the FFT share of the reference's time.
 * Transforms run untimed for at least half a second first, so that the
 * OpenMP threads exist and the cores have left their idle clocks, as they
 * have inside a search that has been running for seconds.
 *
 *     fft-time-f32 <n> <reps>
 */
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "fftw3.h"

int main(int argc, char **argv)
{
     if (argc < 3) {
          fprintf(stderr, "usage: %s n reps\n", argv[0]);
          return 2;
     }
     const int n = atoi(argv[1]), reps = atoi(argv[2]);
     if (n < 2 || reps < 1) return 2;
     fftwf_complex *x = (fftwf_complex *)fftwf_malloc((size_t)n * sizeof(fftwf_complex));
     for (int i = 0; i < n; i++) x[i] = (float)((i * 7) % 13 - 6) + (float)((i * 5) % 11 - 5) * 1.0fi;
     fftwf_plan p = fftwf_plan_dft_1d(n, x, x, FFTW_FORWARD, FFTW_ESTIMATE);
     struct timespec t0, t1;
     clock_gettime(CLOCK_MONOTONIC, &t0);
     do {   /* warm-up: >= 0.5 s */
          fftwf_execute_dft(p, x, x);
          clock_gettime(CLOCK_MONOTONIC, &t1);
     } while ((double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec) < 0.5);
     clock_gettime(CLOCK_MONOTONIC, &t0);
     for (int r = 0; r < reps; r++) fftwf_execute_dft(p, x, x);
     clock_gettime(CLOCK_MONOTONIC, &t1);
     printf("%.9e\n", ((double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec)) / reps);
     fftwf_destroy_plan(p);
     fftwf_free(x);
     return 0;
}
