/*
 * tdf_oracle.c -- CPU restatement of TDFstat's job_core() chain in FP64.
 * TEST INFRASTRUCTURE ONLY (see tdf_oracle.h).  Every function cites the
 * reference lines it follows (paths relative to the TDFstat tree).  The
 * arithmetic is written out component by component in the order the
 * reference's C expressions evaluate, so that with -ffp-contract=off it
 * tracks the reference's DOUBLE build to rounding level.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fft_core.h"
#include "tdf_oracle.h"

#define SQR(x) ((x) * (x))

/* search/network/openmp/auxi.c:22-29 */
static void orc_lin2ast(double be1, double be2, int pm, double sepsm, double cepsm,
                        double *sinal, double *cosal, double *sindel, double *cosdel)
{
     *sindel = be1 * sepsm - (2 * pm - 3) * sqrt(1. - SQR(be1) - SQR(be2)) * cepsm;
     *cosdel = sqrt(1. - SQR(*sindel));
     *sinal = (be1 - sepsm * (*sindel)) / (cepsm * (*cosdel));
     *cosal = be2 / (*cosdel);
}

/* search/network/openmp/settings.c:254-294 */
void orc_modvir(const tdf_segment *seg, int det, double sinal, double cosal,
                double sindel, double cosdel, double *aa, double *bb)
{
     const tdf_detector *d = &seg->det[det];
     const double c1 = d->amod[0], c2 = d->amod[1], c3 = d->amod[2], c4 = d->amod[3],
                  c5 = d->amod[4], c6 = d->amod[5], c7 = d->amod[6], c8 = d->amod[7],
                  c9 = d->amod[8];
     double cosalfr = cosal * (d->cphir) + sinal * (d->sphir);
     double sinalfr = sinal * (d->cphir) - cosal * (d->sphir);
     double c2d = SQR(cosdel);
     double c2sd = sindel * cosdel;
     for (int t = 0; t < seg->N; t++) {
          if (fabs(d->xdat[t]) > DBL_MIN) {
               double c = cosalfr * seg->cosmodf[t] + sinalfr * seg->sinmodf[t];
               double s = sinalfr * seg->cosmodf[t] - cosalfr * seg->sinmodf[t];
               double c2s = 2. * SQR(c);
               double cs = c * s;
               aa[t] = c1 * (2. - c2d) * c2s + c2 * (2. - c2d) * 2. * cs +
                       c3 * c2sd * c + c4 * c2sd * s - c1 * (2. - c2d) + c5 * c2d;
               bb[t] = c6 * sindel * c2s + c7 * sindel * 2. * cs +
                       c8 * cosdel * c + c9 * cosdel * s - c6 * sindel;
          } else {
               aa[t] = 0.;
               bb[t] = 0.;
          }
     }
}

/* search/network/openmp/init.c:365-504 (add_signal), 'amp' form, with the
   'snr' form as the network SNR (the reference's reads sig2 of ifo[nifo],
   init.c:462-464).  Expressions in the reference's evaluation order. */
int orc_add_signal(const tdf_segment *seg, const tdf_signal *sig, double *h0_out)
{
     return orc_add_signal_out(seg, sig, h0_out, NULL);
}

/* the same, and h0*s_n[i] into signal_out[n*N + i] when it is not NULL: what
   the reference writes with mods=write_signal (init.c:475-497) */
int orc_add_signal_out(const tdf_segment *seg, const tdf_signal *sig, double *h0_out, double *signal_out)
{
     const int N = seg->N, nifo = seg->nifo;
     const int dseg = sig->seg - sig->reffr;
     double freqo0 = 2 * M_PI * sig->freq * seg->dt;
     const double freqo1 = M_PI * sig->fdot * seg->dt * seg->dt;
     freqo0 += 2. * freqo1 * (seg->N) * dseg;                              /* init.c:386 */
     if (freqo0 / (2 * M_PI * seg->dt) < sig->fpo || freqo0 / (2 * M_PI * seg->dt) > sig->fpo + sig->B)
          return 1;                                                         /* init.c:389-395 */
     const double sinalpha = sin(sig->ra), cosalpha = cos(sig->ra);
     const double sindelta = sin(sig->dec), cosdelta = cos(sig->dec);
     const double cosi = cos(sig->iota), psi = sig->psi, phi = sig->phase;
     const double cosip = (1. + cosi * cosi) / 2.;
     double amplit[4];                                                      /* init.c:411-414 */
     amplit[0] = cos(2. * psi) * cosip * cos(phi) - sin(2. * psi) * cosi * sin(phi);
     amplit[1] = sin(2. * psi) * cosip * cos(phi) + cos(2. * psi) * cosi * sin(phi);
     amplit[2] = -cos(2. * psi) * cosip * sin(phi) - sin(2. * psi) * cosi * cos(phi);
     amplit[3] = -sin(2. * psi) * cosip * sin(phi) + cos(2. * psi) * cosi * cos(phi);
     const double phaseshift = freqo0 * seg->N * dseg - freqo1 * pow(seg->N * dseg, 2);   /* init.c:417-418 */
     double *s = (double *)malloc((size_t)nifo * N * sizeof(double));
     double *aa = (double *)malloc((size_t)N * sizeof(double));
     double *bb = (double *)malloc((size_t)N * sizeof(double));
     double net = 0.;
     for (int n = 0; n < nifo; n++) {
          const tdf_detector *d = &seg->det[n];
          orc_modvir(seg, n, sinalpha, cosalpha, sindelta, cosdelta, aa, bb);
          const double nSource[3] = {cosalpha * cosdelta, sinalpha * cosdelta, sindelta};
          double sum = 0.;
          for (int i = 0; i < N; i++) {
               double shiftadd = 0.;
               for (int j = 0; j < 3; j++) shiftadd += nSource[j] * d->detssb[i * 3 + j];
               double phaseadd = freqo0 * (i + shiftadd) +
                                 freqo1 * (2. * shiftadd * i + SQR((double)i) + shiftadd * shiftadd) + phaseshift;
               phaseadd -= 2 * M_PI * seg->dt * sig->fpo * i;                 /* init.c:444-447 */
               const double v = amplit[0] * (aa[i]) * cos(phaseadd) + amplit[1] * (bb[i]) * cos(phaseadd) +
                                amplit[2] * (aa[i]) * sin(phaseadd) + amplit[3] * (bb[i]) * sin(phaseadd);
               s[(size_t)n * N + i] = v;
               sum += v * v;
          }
          net += sum / d->sig2;
     }
     const double h0 = sig->snr > 0. ? sig->snr / sqrt(net) : sig->h0;
     for (int n = 0; n < nifo; n++) {
          float *x = (float *)seg->det[n].xdat;
          for (int i = 0; i < N; i++)
               if (x[i]) x[i] += h0 * s[(size_t)n * N + i];                   /* init.c:468-473 */
     }
     if (signal_out)
          for (size_t k = 0; k < (size_t)nifo * N; k++) signal_out[k] = h0 * s[k];   /* init.c:491 */
     free(s);
     free(aa);
     free(bb);
     if (h0_out) *h0_out = h0;
     return 0;
}

/* search/network/openmp/auxi.c:93-117 (natural cubic spline, unit spacing).
   The forward-sweep factors are real: y2[i] = -0.5*invp, invp = 2/(y2[i-1]+4). */
static void orc_spline(const double complex *y, int n, double complex *y2)
{
     double *g = (double *)malloc((size_t)n * sizeof(double));
     double complex *u = (double complex *)malloc((size_t)(n > 1 ? n - 1 : 1) * sizeof(double complex));
     g[0] = 0.;
     u[0] = 0.;
     for (int i = 1; i < n - 1; ++i) {
          double invp = 2. / (g[i - 1] + 4.);
          g[i] = -.5 * invp;
          double dr = creal(y[i - 1]) - 2. * creal(y[i]) + creal(y[i + 1]);
          double di = cimag(y[i - 1]) - 2. * cimag(y[i]) + cimag(y[i + 1]);
          double ur = (-.5 * creal(u[i - 1]) + 3. * dr) * invp;
          double ui = (-.5 * cimag(u[i - 1]) + 3. * di) * invp;
          u[i] = CMPLX(ur, ui);
     }
     /* qn = un = 0: y2[n-1] = 0 */
     y2[n - 1] = 0.;
     for (int k = n - 2; k >= 0; --k) {
          double yr = g[k] * creal(y2[k + 1]) + creal(u[k]);
          double yi = g[k] * cimag(y2[k + 1]) + cimag(u[k]);
          y2[k] = CMPLX(yr, yi);
     }
     free(u);
     free(g);
}

/* search/network/openmp/auxi.c:120-133 */
static double complex orc_splint(const double complex *ya, const double complex *y2a, int n, double x)
{
     if (x < 0 || x > n - 1) return 0.;
     int klo = (int)floor(x);
     int khi = klo + 1;
     double a = khi - x;
     double b = x - klo;
     /* the reference reads ya[n], y2a[n] when x == n-1 exactly (there b == 0) */
     double complex yh = khi < n ? ya[khi] : 0., y2h = khi < n ? y2a[khi] : 0.;
     double ca = a * a * a - a, cb = b * b * b - b;
     double re = a * creal(ya[klo]) + b * creal(yh) + (ca * creal(y2a[klo]) + cb * creal(y2h)) / 6.0;
     double im = a * cimag(ya[klo]) + b * cimag(yh) + (ca * cimag(y2a[klo]) + cb * cimag(y2h)) / 6.0;
     return CMPLX(re, im);
}

/* search/network/openmp/auxi.c:136-169 */
void orc_splintpad(const double complex *ya, const double *shftf, int N,
                   int interpftpad, double complex *out)
{
     int n = interpftpad * N;
     double complex *y2 = (double complex *)malloc((size_t)n * sizeof(double complex));
     orc_spline(ya, n, y2);
     for (int i = 0; i < N; ++i) {
          double x = interpftpad * (i - shftf[i]);
          out[i] = orc_splint(ya, y2, n, x);
     }
     free(y2);
}

int orc_fft(int n, int sign, const double complex *in, double complex *out)
{
     fftc_plan *p = fftc_plan_create(n, sign);
     if (!p) return 1;
     fftc_execute_d(p, in, out);
     fftc_plan_destroy(p);
     return 0;
}

/* search/network/openmp/jobcore.c:243-391 */
typedef struct {
     double sinalt, cosalt, sindelt, cosdelt, het0;
     double ra, dec;
} orc_sky;

static int orc_sky_geometry(const tdf_segment *seg, int32_t pm, float mm, float nn, orc_sky *sk)
{
     const double *M = seg->M;
     double al1 = nn * M[10] + mm * M[14];
     double al2 = nn * M[11] + mm * M[15];
     double cof = seg->oms;
     if ((SQR(al1) + SQR(al2)) / SQR(cof) > 1.) return 1;   /* jobcore.c:248 */
     orc_lin2ast(al1 / cof, al2 / cof, pm, seg->sepsm, seg->cepsm,
                 &sk->sinalt, &sk->cosalt, &sk->sindelt, &sk->cosdelt);
     sk->dec = asin(sk->sindelt);
     sk->ra = fmod(atan2(sk->sinalt, sk->cosalt) + 2. * M_PI, 2. * M_PI);
     sk->het0 = fmod(nn * M[8] + mm * M[12], M[0]);
     return 0;
}

int orc_sky_stage(const tdf_segment *seg, int32_t pm, float mm, float nn,
                  double complex *xam, double complex *xbm, double *tmp1, double *shft_out,
                  double *aa_out, double *bb_out)
{
     orc_sky sk;
     if (orc_sky_geometry(seg, pm, mm, nn, &sk)) return 1;
     const int N = seg->N, nfft = seg->nfft, Ninterp = seg->Ninterp;
     const int nyqst = nfft / 2 + 1;
     double *aa = (double *)malloc((size_t)N * seg->nifo * sizeof(double));
     double *bb = (double *)malloc((size_t)N * seg->nifo * sizeof(double));
     double *shftf = (double *)malloc((size_t)N * sizeof(double));
     int alen = seg->nfftf > Ninterp ? seg->nfftf : Ninterp;
     double complex *xa = (double complex *)malloc((size_t)alen * sizeof(double complex));
     double complex *xb = (double complex *)malloc((size_t)alen * sizeof(double complex));
     fftc_plan *pl_int = fftc_plan_create(nfft, -1);
     fftc_plan *pl_inv = fftc_plan_create(Ninterp, +1);

     for (int n = 0; n < seg->nifo; ++n) {
          const tdf_detector *d = &seg->det[n];
          double *an = aa + (size_t)n * N, *bn = bb + (size_t)n * N;
          double *sh = shft_out + (size_t)n * N;
          double *t1 = tmp1 + (size_t)n * N;
          double complex *xdma = xam + (size_t)n * N, *xdmb = xbm + (size_t)n * N;

          orc_modvir(seg, n, sk.sinalt, sk.cosalt, sk.sindelt, sk.cosdelt, an, bn);

          double nS0 = sk.cosalt * sk.cosdelt, nS1 = sk.sinalt * sk.cosdelt, nS2 = sk.sindelt;
          double shft1 = nS0 * d->detssb[0] + nS1 * d->detssb[1] + nS2 * d->detssb[2];
          for (int i = 0; i < N; ++i) {
               sh[i] = nS0 * d->detssb[i * 3] + nS1 * d->detssb[i * 3 + 1] + nS2 * d->detssb[i * 3 + 2];
               shftf[i] = sh[i] - shft1;
               t1[i] = SQR((double)i) + (double)(2 * i) * sh[i];  /* aux->t2[i] = i*i, init.c:234 */
          }
          for (int i = 0; i < N; ++i) {
               double phase = sk.het0 * i + seg->oms * sh[i];
               double sp, cp;
               sincos(phase, &sp, &cp);
               /* xDat*aa*exph with exph = cp - i*sp (jobcore.c:305-311) */
               double ra = d->xdat[i] * an[i], rb = d->xdat[i] * bn[i];
               xdma[i] = CMPLX(ra * cp, ra * -sp);
               xdmb[i] = CMPLX(rb * cp, rb * -sp);
          }
          for (int i = 0; i < N; ++i) { xa[i] = xdma[i]; xb[i] = xdmb[i]; }
          for (int i = N; i < nfft; ++i) { xa[i] = 0.; xb[i] = 0.; }

          fftc_execute_d(pl_int, xa, xa);                      /* jobcore.c:333-334 */
          fftc_execute_d(pl_int, xb, xb);
          for (int i = nyqst + Ninterp - nfft, j = nyqst; i < Ninterp; ++i, ++j) xa[i] = xa[j];
          for (int i = nyqst; i < nyqst + Ninterp - nfft; ++i) xa[i] = 0.;
          for (int i = nyqst + Ninterp - nfft, j = nyqst; i < Ninterp; ++i, ++j) xb[i] = xb[j];
          for (int i = nyqst; i < nyqst + Ninterp - nfft; ++i) xb[i] = 0.;
          fftc_execute_d(pl_inv, xa, xa);                      /* jobcore.c:354-355 */
          fftc_execute_d(pl_inv, xb, xb);
          double ft = (double)seg->interpftpad / Ninterp;
          for (int i = 0; i < Ninterp; ++i) {
               xa[i] = CMPLX(creal(xa[i]) * ft, cimag(xa[i]) * ft);
               xb[i] = CMPLX(creal(xb[i]) * ft, cimag(xb[i]) * ft);
          }
          orc_splintpad(xa, shftf, N, seg->interpftpad, xdma);   /* jobcore.c:366-367 */
          orc_splintpad(xb, shftf, N, seg->interpftpad, xdmb);
     }

     /* jobcore.c:373-391 */
     double aas = 0., bbs = 0.;
     for (int n = 0; n < seg->nifo; ++n) {
          const double *an = aa + (size_t)n * N, *bn = bb + (size_t)n * N;
          double aatemp = 0., bbtemp = 0.;
          for (int i = 0; i < N; ++i) {
               aatemp += SQR(an[i]);
               bbtemp += SQR(bn[i]);
          }
          double s2 = seg->det[n].sig2;
          aas += aatemp / s2;
          bbs += bbtemp / s2;
          double complex *xdma = xam + (size_t)n * N, *xdmb = xbm + (size_t)n * N;
          for (int i = 0; i < N; ++i) {
               xdma[i] = CMPLX(creal(xdma[i]) / s2, cimag(xdma[i]) / s2);
               xdmb[i] = CMPLX(creal(xdmb[i]) / s2, cimag(xdmb[i]) / s2);
          }
     }
     *aa_out = aas;
     *bb_out = bbs;

     fftc_plan_destroy(pl_int);
     fftc_plan_destroy(pl_inv);
     free(xa); free(xb); free(shftf); free(aa); free(bb);
     return 0;
}

/* spinmod.c:490-514 (GNUSINCOS, DOUBLE) + jobcore.c:473-515: the F-statistic
   of one spindown over [fr0, fr1] into F (indexed by absolute bin). */
static void orc_fstat_one(const tdf_segment *seg, const tdf_search_opts *opts,
                          const double complex *xam, const double complex *xbm,
                          const double *tmp1, double aa, double bb,
                          double het1, double spnd, double complex *fxa, double complex *fxb,
                          const fftc_plan *plan, double *F)
{
     const int N = seg->N, nfftf = seg->nfftf;
     for (int n = 0; n < seg->nifo; ++n) {
          const double complex *xa = xam + (size_t)n * N, *xb = xbm + (size_t)n * N;
          const double *t1 = tmp1 + (size_t)n * N;
          for (int i = N - 1; i > -1; --i) {
               double phase = het1 * i + spnd * t1[i];
               double sp, cp;
               sincos(phase, &sp, &cp);
               double er = cp, ei = -sp;
               /* complex product, naive formula */
               double pr = creal(xa[i]) * er - cimag(xa[i]) * ei;
               double pi = creal(xa[i]) * ei + cimag(xa[i]) * er;
               double qr = creal(xb[i]) * er - cimag(xb[i]) * ei;
               double qi = creal(xb[i]) * ei + cimag(xb[i]) * er;
               if (n == 0) {
                    fxa[i] = CMPLX(pr, pi);
                    fxb[i] = CMPLX(qr, qi);
               } else {
                    fxa[i] = CMPLX(creal(fxa[i]) + pr, cimag(fxa[i]) + pi);
                    fxb[i] = CMPLX(creal(fxb[i]) + qr, cimag(fxb[i]) + qi);
               }
          }
     }
     for (int i = nfftf - 1; i > N - 1; --i) fxa[i] = fxb[i] = 0.;
     fftc_execute_d(plan, fxa, fxa);
     fftc_execute_d(plan, fxb, fxb);
     for (int i = opts->fr[0]; i <= opts->fr[1]; ++i) {
          double na = creal(fxa[i]) * creal(fxa[i]) + cimag(fxa[i]) * cimag(fxa[i]);
          double nb = creal(fxb[i]) * creal(fxb[i]) + cimag(fxb[i]) * cimag(fxb[i]);
          F[i] = na / aa + nb / bb;
     }
     if (opts->blocks_avg) {
          /* FStat(F + fr0, fr1 - fr0, NAVFSTAT, 0), auxi.c:336-363 */
          double *fr = F + opts->fr[0];
          int nfft = opts->fr[1] - opts->fr[0], nav = TDF_NAVFSTAT;
          for (int j = 0; j < nfft / nav; j++) {
               double mu = 0.;
               for (int i = 0; i < nav; i++) mu += *fr++;
               mu /= 2. * nav;
               fr -= nav;
               for (int i = 0; i < nav; i++) *fr++ /= mu;
          }
     }
}

/* per-template scalars (jobcore.c:427-468), DOUBLE build */
typedef struct {
     int iss_size;
     float smin;
} orc_srange;

static orc_srange orc_spindown_range(const tdf_segment *seg, const tdf_search_opts *opts,
                                     float mm, float nn, float sst)
{
     const double *M = seg->M;
     float smin = sst, smax = opts->spndr[1];
     if (opts->allsky) {
          smin = trunc((seg->Smin - nn * M[9] - mm * M[13]) / M[5]);
          smax = trunc(-(nn * M[9] + mm * M[13] + seg->Smax) / M[5]);
          if (smin > smax) {
               smin = smin + smax;
               smax = smin - smax;
               smin = smin - smax;
          }
     }
     orc_srange r;
     r.iss_size = (smax - smin) / opts->sstep + 1;
     r.smin = smin;
     return r;
}

int orc_search_points(const tdf_segment *seg, const tdf_search_opts *opts, int npts,
                      const int32_t *pm, const float *mm, const float *nn, const float *sst,
                      tdf_record *recs, int64_t max_recs, int64_t *nrec,
                      float *pairs, int64_t max_pairs, int64_t *npairs,
                      int32_t *nrec_per_point)
{
     const int N = seg->N, nifo = seg->nifo, nfftf = seg->nfftf;
     const double *M = seg->M;
     double complex *xam = (double complex *)malloc((size_t)N * nifo * sizeof(double complex));
     double complex *xbm = (double complex *)malloc((size_t)N * nifo * sizeof(double complex));
     double *tmp1 = (double *)malloc((size_t)N * nifo * sizeof(double));
     double *shft = (double *)malloc((size_t)N * nifo * sizeof(double));
     double complex *fxa = (double complex *)malloc((size_t)nfftf * sizeof(double complex));
     double complex *fxb = (double complex *)malloc((size_t)nfftf * sizeof(double complex));
     double *F = (double *)malloc((size_t)(2 * seg->nfft > nfftf ? 2 * seg->nfft : nfftf) * sizeof(double));
     fftc_plan *plan = fftc_plan_create(nfftf, -1);
     int64_t r = 0, p = 0;
     int status = TDF_OK;

     for (int ip = 0; ip < npts; ip++) {
          float s0 = sst ? sst[ip] : opts->spndr[0];
          double aa, bb;
          orc_sky sk;
          int out = orc_sky_geometry(seg, pm[ip], mm[ip], nn[ip], &sk);
          if (nrec_per_point) nrec_per_point[ip] = 0;
          if (out) continue;
          orc_sky_stage(seg, pm[ip], mm[ip], nn[ip], xam, xbm, tmp1, shft, &aa, &bb);
          orc_srange sr = orc_spindown_range(seg, opts, mm[ip], nn[ip], s0);
          if (nrec_per_point) nrec_per_point[ip] = sr.iss_size > 0 ? sr.iss_size : 0;
          for (int iss = 0; iss < sr.iss_size; ++iss) {
               float ss = sr.smin + iss * opts->sstep;
               double spnd = ss * M[5] + nn[ip] * M[9] + mm[ip] * M[13];   /* sgnlt[1] */
               if (r < max_recs) {
                    recs[r].m = mm[ip];
                    recs[r].n = nn[ip];
                    recs[r].s = ss;
                    recs[r].ra = (float)sk.ra;
                    recs[r].dec = (float)sk.dec;
                    recs[r].fdot = (float)(spnd / (M_PI * seg->dt * seg->dt));
                    recs[r].len = 0;
                    recs[r].pad = 0;
                    recs[r].offset = p;
               }
               double het1 = fmod(ss * M[4], M[0]);
               if (het1 < 0) het1 += M[0];
               double sgnl0 = sk.het0 + het1;
               orc_fstat_one(seg, opts, xam, xbm, tmp1, aa, bb, het1, spnd, fxa, fxb, plan, F);
               /* MAX_ALG 3, single thread (jobcore.c:552-603) */
               int itrig = 0;
               for (int i = opts->fr[0] + 1; i < opts->fr[1] - 1; ++i) {
                    if (F[i] < opts->thr || F[i - 1] > F[i] || F[i] < F[i + 1]) continue;
                    int ic = i;
                    double Fc = F[ic];
                    i++;
                    double f_ = (double)(2 * ic) / (double)nfftf * M_PI + sgnl0;
                    int veto = 0;
                    for (int k = 0; k < opts->numlines; k++)
                         if (f_ >= opts->lines[2 * k] && f_ <= opts->lines[2 * k + 1]) { veto = 1; break; }
                    if (veto) continue;
                    if (itrig >= opts->bufsize / 2) { status = TDF_ERR_TRIGGER_OVERFLOW; goto done; }
                    if (p + 2 <= max_pairs) {
                         pairs[p] = (float)f_;
                         pairs[p + 1] = (float)Fc;
                    }
                    p += 2;
                    itrig++;
                    if (r < max_recs) recs[r].len += 2;
               }
               r++;
          }
     }
done:
     *nrec = r;
     *npairs = p;
     if (status == TDF_OK && (r > max_recs || p > max_pairs)) status = TDF_ERR_CAPACITY;
     fftc_plan_destroy(plan);
     free(xam); free(xbm); free(tmp1); free(shft); free(fxa); free(fxb); free(F);
     return status;
}

int orc_fstat_spectrum(const tdf_segment *seg, const tdf_search_opts *opts,
                       int32_t pm, float mm, float nn, float ss, double *Fout, int64_t nF)
{
     const int N = seg->N, nifo = seg->nifo, nfftf = seg->nfftf;
     const double *M = seg->M;
     if (nF < (int64_t)opts->fr[1] - opts->fr[0] + 1) return TDF_ERR_CAPACITY;
     orc_sky sk;
     if (orc_sky_geometry(seg, pm, mm, nn, &sk)) return TDF_ERR_INVALID;
     double complex *xam = (double complex *)malloc((size_t)N * nifo * sizeof(double complex));
     double complex *xbm = (double complex *)malloc((size_t)N * nifo * sizeof(double complex));
     double *tmp1 = (double *)malloc((size_t)N * nifo * sizeof(double));
     double *shft = (double *)malloc((size_t)N * nifo * sizeof(double));
     double complex *fxa = (double complex *)malloc((size_t)nfftf * sizeof(double complex));
     double complex *fxb = (double complex *)malloc((size_t)nfftf * sizeof(double complex));
     double *F = (double *)malloc((size_t)(2 * seg->nfft > nfftf ? 2 * seg->nfft : nfftf) * sizeof(double));
     fftc_plan *plan = fftc_plan_create(nfftf, -1);
     double aa, bb;
     orc_sky_stage(seg, pm, mm, nn, xam, xbm, tmp1, shft, &aa, &bb);
     double spnd = ss * M[5] + nn * M[9] + mm * M[13];
     double het1 = fmod(ss * M[4], M[0]);
     if (het1 < 0) het1 += M[0];
     orc_fstat_one(seg, opts, xam, xbm, tmp1, aa, bb, het1, spnd, fxa, fxb, plan, F);
     for (int i = opts->fr[0]; i <= opts->fr[1]; i++) Fout[i - opts->fr[0]] = F[i];
     fftc_plan_destroy(plan);
     free(xam); free(xbm); free(tmp1); free(shft); free(fxa); free(fxb); free(F);
     return TDF_OK;
}
