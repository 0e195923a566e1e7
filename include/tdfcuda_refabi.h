/*
 * tdfcuda_refabi.h -- drop-in entry point with the reference's own
 * signature: libtdfcuda exports
 *
 *   int job_core(int pm, float mm, float nn, Search_settings *sett,
 *                Command_line_opts *opts, Search_range *s_range,
 *                FFTW_plans *plans, FFTW_arrays *fftw_arr, Aux_arrays *aux,
 *                int *sgnlc, Trigger *sgnlv, int *FNum);
 *
 * replacing search/network/openmp/jobcore.c:193-630 (declared jobcore.h:21-33),
 * plus the same function under the name tdf_job_core_ref().  It reads the
 * host's global detector array `ifo` (main.c:29, struct.h:175) like the
 * reference does.  The host program keeps its own headers; the declarations
 * below only restate the layout of the reference's structs (struct.h:19-215,
 * LP64) so that the library reads the same bytes.  FFTW plan and array
 * pointers are accepted and ignored.
 *
 * Behaviour matches the reference: one record per spindown of the point
 * written to sgnlv[0..nrec), ffstat.p malloc'd with sett->bufsize floats when
 * NULL, *FNum += nrec, *sgnlc += triggers, the same ">>FNum mm nn [smin..smax:step]"
 * line on stdout; returns 0; on trigger-buffer overflow it prints the
 * reference's message and exits with EXIT_FAILURE (jobcore.c:586-590).
 * Environment: TDF_FORM = split (default) | fp64, TDF_DEVICE = CUDA device.
 */
#ifndef TDFCUDA_REFABI_H
#define TDFCUDA_REFABI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDF_REF_MAX_DETECTORS 8    /* struct.h:8  */
#define TDF_REF_DETNAME_LENGTH 2   /* struct.h:9  */
#define TDF_REF_FNAME_LENGTH 2048  /* struct.h:10 */
#define TDF_REF_MAXL 512           /* struct.h:14 */

typedef struct { size_t len; void *p; } tdf_ref_hvl_t;   /* HDF5 hvl_t */

typedef struct {                                          /* Command_line_opts, struct.h:19-32 */
     int checkp_flag, veto_flag, help_flag;
     int seg, band, hemi;
     double thr;
     double fpo_val, narrowdown, overlap;
     const char *indir, *outdir, *grid_file, *dump_range_file,
          *usedet, *addsig, *fstat_norm, *label, *mods,
          *gtype, *gcenter, *gsizes, *gsteps;
     char state_file[TDF_REF_FNAME_LENGTH];
} tdf_ref_Command_line_opts;

typedef struct {                                          /* Signals, struct.h:36-55 */
     float *xDat;
     double *DetSSB;
     double *aa, *bb;
     double *shftf, *shft;
     double epsm, phir, sepsm, cepsm, sphir, cphir, crf0, sig2;
     int Nzeros;
     void *xDatma, *xDatmb;                               /* double complex * */
} tdf_ref_Signals;

typedef struct {                                          /* Search_range, struct.h:69-82 */
     int pmr[2], fr[2];
     float mr[2], nr[2], spndr[2];
     float mstep, nstep, sstep;
     float mst, nst, sst;
     int pst;
} tdf_ref_Search_range;

typedef struct {                                          /* Aux_arrays, struct.h:96-101 */
     double *sinmodf, *cosmodf;
     double *t2;
} tdf_ref_Aux_arrays;

typedef struct {                                          /* Search_settings, struct.h:105-145 */
     double fpo, dt, B, oms, omr, Smin, Smax, sepsm, cepsm;
     int nfft, nod, N, nfftf, nmax, nmin, s, nd, interpftpad, fftpad, Ninterp,
         nifo, numlines_band, nvlines_all_inband, bufsize, dd;
     double M[16];
     double invM[4][4];
     double vedva[4][4];
     double lines[TDF_REF_MAXL][2];
} tdf_ref_Search_settings;

typedef struct { double c1, c2, c3, c4, c5, c6, c7, c8, c9; } tdf_ref_Ampl_mod_coeff;  /* struct.h:149-153 */

typedef struct {                                          /* Detector_settings, struct.h:157-172 */
     char xdatname[TDF_REF_FNAME_LENGTH];
     char name[TDF_REF_DETNAME_LENGTH];
     double ephi, elam, eheight, egam;
     tdf_ref_Ampl_mod_coeff amod;
     tdf_ref_Signals sig;
     double start_time;
} tdf_ref_Detector_settings;

typedef struct {                                          /* Trigger, struct.h:211-215 */
     float m, n, s;
     float ra, dec, fdot;
     tdf_ref_hvl_t ffstat;
} tdf_ref_Trigger;

int job_core(int pm, float mm, float nn, tdf_ref_Search_settings *sett, tdf_ref_Command_line_opts *opts,
             tdf_ref_Search_range *s_range, void *plans, void *fftw_arr, tdf_ref_Aux_arrays *aux,
             int *sgnlc, tdf_ref_Trigger *sgnlv, int *FNum);

int tdf_job_core_ref(int pm, float mm, float nn, tdf_ref_Search_settings *sett, tdf_ref_Command_line_opts *opts,
                     tdf_ref_Search_range *s_range, void *plans, void *fftw_arr, tdf_ref_Aux_arrays *aux,
                     int *sgnlc, tdf_ref_Trigger *sgnlv, int *FNum);

/* Releases the engine the drop-in entry keeps between calls. */
void tdf_job_core_release(void);

/* sizeof of each restated struct, for layout checks by bindings */
size_t tdf_ref_struct_size(int which);

#ifdef __cplusplus
}
#endif

#endif
