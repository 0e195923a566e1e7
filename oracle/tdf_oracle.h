/*
 * tdf_oracle.h -- CPU restatement of TDFstat's job_core() chain in FP64
 * (the reference's PREC=DOUBLE, SIMD=NONE build).  TEST INFRASTRUCTURE ONLY:
 * the parity checker for libtdfcuda.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may load it; the product never does.
 *
 * Pinned against the reference itself: tests compare it with the reference's
 * own sources compiled here (oracle/_ref/gwsearch-ref-f64, built by
 * oracle/Makefile) on the committed golden cases.
 *
 * Inputs and outputs use the descriptor types of include/tdfcuda.h.
 */
#ifndef TDF_ORACLE_H
#define TDF_ORACLE_H

#include <complex.h>
#include "tdfcuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Whole chain for npts sky points; same contract as tdf_search_points(). */
int orc_search_points(const tdf_segment *seg, const tdf_search_opts *opts, int npts,
                      const int32_t *pm, const float *mm, const float *nn, const float *sst,
                      tdf_record *recs, int64_t max_recs, int64_t *nrec,
                      float *pairs, int64_t max_pairs, int64_t *npairs,
                      int32_t *nrec_per_point);

/* Full F over [fr0, fr1] for one template; same contract as tdf_fstat_spectrum(). */
int orc_fstat_spectrum(const tdf_segment *seg, const tdf_search_opts *opts,
                       int32_t pm, float mm, float nn, float ss, double *F, int64_t nF);

/* Sky stage of one sky point (jobcore.c:243-391).  Outputs, per detector n:
   xa[n*N + i], xb[n*N + i] (xDatma/xDatmb after resampling and /sig2),
   tmp1[n*N + i], shft[n*N + i]; and the sums aa, bb.  Returns 0, or 1 if the
   point lies outside the sky ellipse (nothing written). */
int orc_sky_stage(const tdf_segment *seg, int32_t pm, float mm, float nn,
                  double complex *xa, double complex *xb, double *tmp1, double *shft,
                  double *aa, double *bb);

/* modvir (settings.c:254-294) for one detector. */
void orc_modvir(const tdf_segment *seg, int det, double sinal, double cosal,
                double sindel, double cosdel, double *aa, double *bb);

/* natural cubic spline resampling (auxi.c:93-169): ya[0..interpftpad*N) */
void orc_splintpad(const double complex *ya, const double *shftf, int N,
                   int interpftpad, double complex *out);

/* add_signal (init.c:365-504): adds h0*s_n[i] to seg->det[n].xdat[i] where
   it is nonzero, in place (the xdat arrays must be the caller's writable
   copies).  sig->snr > 0 sets h0 from the network SNR (tdf_signal).
   Returns 1 if the signal lies outside [fpo, fpo + B] (nothing added),
   else 0; *h0 receives the amplitude used. */
int orc_add_signal(const tdf_segment *seg, const tdf_signal *sig, double *h0);
/* the same, and h0*s_n[i] into signal_out[n*N + i] (if not NULL) */
int orc_add_signal_out(const tdf_segment *seg, const tdf_signal *sig, double *h0, double *signal_out);

/* textbook FFT (fft_core.c), exposed for the FFT tests */
int orc_fft(int n, int sign, const double complex *in, double complex *out);

#ifdef __cplusplus
}
#endif

#endif
