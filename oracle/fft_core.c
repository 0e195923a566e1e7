/*
 * fft_core.c -- textbook radix-2 complex FFT for the CPU oracle (test
 * infrastructure only).  See fft_core.h for the semantics it restates.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fft_core.h"

#define FFTC_OMP_MIN 16384   /* parallelise stages only for long transforms */

fftc_plan *fftc_plan_create(int n, int sign)
{
     if (n < 1 || (n & (n - 1)) != 0) return NULL;
     fftc_plan *p = (fftc_plan *)calloc(1, sizeof(fftc_plan));
     p->n = n;
     p->sign = sign < 0 ? -1 : 1;
     int l = 0;
     while ((1 << l) < n) l++;
     p->log2n = l;
     int h = n / 2 > 0 ? n / 2 : 1;
     p->twd = (double *)malloc(2 * (size_t)h * sizeof(double));
     p->twf = (float *)malloc(2 * (size_t)h * sizeof(float));
     for (int k = 0; k < h; k++) {
          /* k/n is exact for a power-of-two n */
          double a = 2.0 * M_PI * ((double)k / (double)n);
          double c = cos(a), s = sin(a) * p->sign;
          p->twd[2 * k] = c;
          p->twd[2 * k + 1] = s;
          p->twf[2 * k] = (float)c;
          p->twf[2 * k + 1] = (float)s;
     }
     p->rev = (int *)malloc((size_t)n * sizeof(int));
     for (int i = 0; i < n; i++) {
          int r = 0, v = i;
          for (int b = 0; b < l; b++) { r = (r << 1) | (v & 1); v >>= 1; }
          p->rev[i] = r;
     }
     return p;
}

void fftc_plan_destroy(fftc_plan *p)
{
     if (!p) return;
     free(p->twd);
     free(p->twf);
     free(p->rev);
     free(p);
}

#define FFTC_BODY(CT, RT, TW, MK)                                                \
     const int n = p->n;                                                       \
     if (in != out) memcpy(out, in, (size_t)n * sizeof(CT));                   \
     if (n == 1) return;                                                       \
     const int *rev = p->rev;                                                  \
     for (int i = 0; i < n; i++) {                                             \
          int j = rev[i];                                                      \
          if (j > i) { CT t = out[i]; out[i] = out[j]; out[j] = t; }           \
     }                                                                         \
     const long nh = n / 2;                                                    \
     for (int hs = 1; hs < n; hs <<= 1) {                                      \
          const int tstride = n / (2 * hs);                                    \
          _Pragma("omp parallel for schedule(static) if(n >= FFTC_OMP_MIN)")   \
          for (long b = 0; b < nh; b++) {                                      \
               long j = b % hs;                                                \
               long a0 = (b / hs) * 2 * hs + j;                                \
               long a1 = a0 + hs;                                              \
               RT wr = TW[2 * j * tstride], wi = TW[2 * j * tstride + 1];      \
               RT xr = creal(out[a1]), xi = cimag(out[a1]);                    \
               RT tr = wr * xr - wi * xi;                                      \
               RT ti = wr * xi + wi * xr;                                      \
               RT ur = creal(out[a0]), ui = cimag(out[a0]);                    \
               out[a0] = MK(ur + tr, ui + ti);                                 \
               out[a1] = MK(ur - tr, ui - ti);                                 \
          }                                                                    \
     }

void fftc_execute_d(const fftc_plan *p, const double complex *in, double complex *out)
{
     FFTC_BODY(double complex, double, p->twd, CMPLX)
}

void fftc_execute_f(const fftc_plan *p, const float complex *in, float complex *out)
{
     FFTC_BODY(float complex, float, p->twf, CMPLXF)
}
