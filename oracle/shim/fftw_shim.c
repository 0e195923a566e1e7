/*
 * fftw_shim.c -- implementation of the FFTW3-API shim declared in fftw3.h
 * (test infrastructure only).  Each plan wraps an oracle/fft_core.c plan and
 * remembers the arrays it was planned on, so that fftw_execute() works as in
 * FFTW; fftw_execute_dft() (the new-array interface the reference uses) runs
 * the same transform on the arrays it is given.
 */
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"
#include "../fft_core.h"

struct shim_fftw_plan_s {
     fftc_plan *core;
     int is_float;
     void *in, *out;
};

int fftw_init_threads(void) { return 1; }
int fftwf_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }

static void *shim_alloc(size_t n)
{
     void *p = NULL;
     if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
     return p;
}

void *fftw_malloc(size_t n) { return shim_alloc(n); }
void *fftwf_malloc(size_t n) { return shim_alloc(n); }
void fftw_free(void *p) { free(p); }
void fftwf_free(void *p) { free(p); }

static struct shim_fftw_plan_s *shim_plan(int n, void *in, void *out, int sign, int is_float)
{
     struct shim_fftw_plan_s *p = (struct shim_fftw_plan_s *)calloc(1, sizeof(*p));
     p->core = fftc_plan_create(n, sign);
     if (!p->core) { free(p); return NULL; }
     p->is_float = is_float;
     p->in = in;
     p->out = out;
     return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
     (void)flags;
     return shim_plan(n, in, out, sign, 0);
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags)
{
     (void)flags;
     return shim_plan(n, in, out, sign, 1);
}

static void shim_exec(const struct shim_fftw_plan_s *p, void *in, void *out)
{
     if (p->is_float)
          fftc_execute_f(p->core, (const float complex *)in, (float complex *)out);
     else
          fftc_execute_d(p->core, (const double complex *)in, (double complex *)out);
}

void fftw_execute(const fftw_plan p) { shim_exec(p, p->in, p->out); }
void fftwf_execute(const fftwf_plan p) { shim_exec(p, p->in, p->out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) { shim_exec(p, in, out); }
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out) { shim_exec(p, in, out); }

void fftw_destroy_plan(fftw_plan p)
{
     if (!p) return;
     fftc_plan_destroy(p->core);
     free(p);
}
void fftwf_destroy_plan(fftwf_plan p) { fftw_destroy_plan(p); }
void fftw_cleanup(void) {}
void fftwf_cleanup(void) {}
