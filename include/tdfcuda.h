/*
 * tdfcuda.h -- C ABI of libtdfcuda, the B200 (sm_100a) engine for the
 * coherent F-statistic search hot path of TDFstat: the per-sky-point
 * job_core() chain of search/network/openmp.
 *
 * Plain C types only (pointers, sizes, scalars).  All input pointers are HOST
 * pointers unless a name says otherwise; the library copies what it needs to
 * the device.  Every function returns a tdf_status; tdf_last_error() gives a
 * message for the calling thread's last failure.
 *
 * Reference interfaces replaced (paths relative to the TDFstat tree):
 *   job_core()            search/network/openmp/jobcore.c:193-630,
 *                         declared jobcore.h:21-33   -> tdf_search_points(),
 *                         tdf_job_core_ref() / job_core() in tdfcuda_refabi.h
 *   spindown_modulation() search/network/openmp/spinmod.c:17-538 (inside)
 *   modvir()/rogcvir()    search/network/openmp/settings.c:226-294 (inside)
 *   splintpad()/spline()  search/network/openmp/auxi.c:93-169 (inside)
 *   FStat()               search/network/openmp/auxi.c:336-363 (inside)
 * The driver loop search() (jobcore.c:28-188) stays on the host; it may call
 * tdf_search_points() for a whole sky patch instead of job_core() per point.
 */
#ifndef TDFCUDA_H
#define TDFCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDF_MAX_DETECTORS 8   /* MAX_DETECTORS, struct.h:8 */
#define TDF_MAX_LINES 512     /* MAXL, struct.h:14 */
#define TDF_NAVFSTAT 4096     /* NAVFSTAT, auxi.h:12 */

typedef enum tdf_status {
     TDF_OK = 0,
     TDF_ERR_INVALID = 1,          /* bad argument, size or layout */
     TDF_ERR_CUDA = 2,             /* a CUDA runtime call failed */
     TDF_ERR_TRIGGER_OVERFLOW = 3, /* > bufsize/2 triggers in one spindown (jobcore.c:586-590) */
     TDF_ERR_OUT_OF_MEMORY = 4,
     TDF_ERR_CAPACITY = 5,         /* caller's output arrays are too small */
     TDF_ERR_UNSUPPORTED = 6,      /* size or option outside what this build handles */
     TDF_ERR_NO_DEVICE = 7,
     TDF_ERR_NOT_BUILT = 8         /* this entry point is not available in this build */
} tdf_status;

/* Arithmetic form of the engine. */
typedef enum tdf_form {
     /* FP64 sky stage (shift, phase, FFT interpolation, spline); FP32
        resampled series, demodulation sincos, FFTs and F-statistic, with the
        spindown phase argument formed and reduced mod 2*pi in FP64. */
     TDF_FORM_SPLIT = 0,
     /* every step in FP64: the reference's PREC=DOUBLE build */
     TDF_FORM_FP64 = 1
} tdf_form;

/* One detector's inputs: the fields of ifo[n] (struct.h:36-55,157-172) that
   job_core() reads. */
typedef struct tdf_detector {
     const float *xdat;     /* [N] time series, ifo[n].sig.xDat */
     const double *detssb;  /* [3N] detector position w.r.t. the SSB, ifo[n].sig.DetSSB */
     double sig2;           /* ifo[n].sig.sig2 = crf0 * var(xDat) (common.c:68-78) */
     double sphir, cphir;   /* ifo[n].sig.sphir, cphir (common.c:123-124) */
     double amod[9];        /* ifo[n].amod.c1..c9 from rogcvir (settings.c:226-248) */
} tdf_detector;

/* One data segment: Search_settings (struct.h:105-145) fields the path reads,
   the aux arrays (struct.h:96-101) and the detectors. */
typedef struct tdf_segment {
     int32_t N;             /* samples */
     int32_t nfft;          /* 2^ceil(log2 N) */
     int32_t nfftf;         /* fftpad * nfft: spindown FFT length */
     int32_t Ninterp;       /* interpftpad * nfft: interpolation FFT length */
     int32_t interpftpad;   /* 2 (settings.c:56) */
     int32_t nifo;          /* detectors, 1..TDF_MAX_DETECTORS */
     double dt, oms, sepsm, cepsm, Smin, Smax;
     double M[16];          /* grid generator matrix, column-major (jobcore.c:218-240) */
     const double *cosmodf; /* [N] cos(omr*i) (init.c:232-237) */
     const double *sinmodf; /* [N] sin(omr*i) */
     tdf_detector det[TDF_MAX_DETECTORS];
} tdf_segment;

/* Search options: Command_line_opts / Search_range / Search_settings fields
   the path reads. */
typedef struct tdf_search_opts {
     double thr;            /* opts->thr: trigger threshold on F */
     int32_t fr[2];         /* s_range->fr: F-statistic bins [fr0, fr1] */
     int32_t allsky;        /* opts->gtype == "allsky": spindown range per sky point
                               from Smin/Smax (jobcore.c:399-411) */
     int32_t blocks_avg;    /* opts->fstat_norm == "blocks_avg" (jobcore.c:513-515) */
     float spndr[2];        /* s_range->spndr (non-allsky spindown range) */
     float sstep;           /* s_range->sstep */
     int32_t bufsize;       /* sett->bufsize: floats per record; at most bufsize/2 triggers */
     int32_t numlines;      /* sett->numlines_band */
     const double *lines;   /* [numlines][2] veto intervals in radians (sett->lines) */
} tdf_search_opts;

/* One output record: the Trigger compound (struct.h:211-215) with the hvl_t
   replaced by an offset into the caller's pair array. */
typedef struct tdf_record {
     float m, n, s, ra, dec, fdot;
     uint32_t len;          /* ffstat.len: floats, two per trigger (f, F) */
     uint32_t pad;
     int64_t offset;        /* index (in floats) of the first pair in pairs[] */
} tdf_record;

typedef struct tdf_engine tdf_engine;

/* Bits set in a kernel's error word when a bounded wait gave up (the search
   then returns TDF_ERR_CUDA with a message): a wait on an asynchronous copy,
   and a fused pass's row block waiting for its template's column blocks. */
#define TDF_WAIT_TIMEOUT_BIT 2u
#define TDF_ORDER_TIMEOUT_BIT 8u

/* Health check of the bounded waits: one warp on `device` waits, `probes`
   probes at most (1..2^20), on a barrier whose copy never arrives, then one
   thread on a block count that nothing raises, and returns; *status receives
   the kernel's error word (TDF_WAIT_TIMEOUT_BIT and TDF_ORDER_TIMEOUT_BIT
   set when the waits gave up, as they must).  The device stays usable. */
int tdf_check_bounded_wait(int device, int32_t probes, uint32_t *status);

/* Diagnostic (no device needed): the item that ticket `ticket` names in a
   fused pass launch (TDF_FUSED_PASSES=1) of `nt` templates with `blocks`
   column and `blocks` row blocks per template and a row lag of `lag`
   templates (clamped to [1, nt] as the launcher does): template *tmpl,
   block *block, *row = 1 for a row block.  The same code the kernel runs. */
int tdf_spin_order_item(int32_t nt, int32_t blocks, int32_t lag, uint32_t ticket, int32_t *tmpl, int32_t *block,
                        int32_t *row);

const char *tdf_status_string(int status);
/* message of the calling thread's last failed call ("" if none) */
const char *tdf_last_error(void);
int tdf_device_count(int *count);

/* Create an engine on CUDA device `device`: validates sizes, allocates the
   device buffers for up to `max_sky_batch` sky points in flight (0 = library
   default), uploads the segment's inputs.  Replaces the per-run setup that
   job_core() relies on (init_arrays, plan_fftw: init.c:247-294,710-755). */
int tdf_engine_create(const tdf_segment *seg, const tdf_search_opts *opts,
                      int form, int device, int max_sky_batch, tdf_engine **out);

/* Copy new inputs (same sizes as at creation) into the engine's device
   buffers without allocating; e.g. the next segment of a run. */
int tdf_engine_upload(tdf_engine *e, const tdf_segment *seg);

int tdf_engine_destroy(tdf_engine *e);

/* Run npts sky points (hemisphere pm[i], grid position mm[i], nn[i]); the
   work of npts job_core() calls (jobcore.c:193-630).  Records come out in
   the reference order (point, then spindown), one per spindown of every
   point inside the sky ellipse; points outside it give none (jobcore.c:248).
   sst may be NULL (start of the spindown range = spndr[0]) or hold the
   restart spindown per point (s_range->sst, jobcore.c:208).
   nrec_per_point (may be NULL) receives each point's record count (the
   *FNum increment).  Returns TDF_ERR_CAPACITY with the needed sizes in
   *nrec / *npairs if the caller's arrays are too small. */
int tdf_search_points(tdf_engine *e, int npts, const int32_t *pm, const float *mm,
                      const float *nn, const float *sst,
                      tdf_record *recs, int64_t max_recs, int64_t *nrec,
                      float *pairs, int64_t max_pairs, int64_t *npairs,
                      int32_t *nrec_per_point);

/* Number of records tdf_search_points() would produce for these points (host
   arithmetic only, no device work): one per spindown of each point inside
   the sky ellipse (jobcore.c:248,427).  nrec_per_point may be NULL. */
int tdf_count_templates(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn,
                        const float *sst, int64_t *nrec, int32_t *nrec_per_point);

/* After tdf_search_points() returned TDF_ERR_CAPACITY the engine keeps the
   results; this copies them into larger arrays without running the search
   again.  Returns TDF_ERR_INVALID if no results are kept. */
int tdf_last_results(tdf_engine *e, tdf_record *recs, int64_t max_recs, int64_t *nrec,
                     float *pairs, int64_t max_pairs, int64_t *npairs, int32_t *nrec_per_point);

/* Device-only pass: same work as tdf_search_points() but the trigger list
   stays on the device; returns the record and trigger counts.  Used to time
   the kernels with inputs resident in HBM. */
int tdf_search_points_device(tdf_engine *e, int npts, const int32_t *pm, const float *mm,
                             const float *nn, const float *sst,
                             int64_t *nrec, int64_t *ntrig);

/* Several data segments of the same sizes resident on one engine.  The
   reference searches one segment per process (search/network/openmp/main.c;
   its spline keeps a static buffer sized for one N, auxi.c:97-99); here a
   run over many segments of one length keeps them all on the GPU.
   tdf_engine_add_segment() uploads another segment (sizes and detector count
   equal to the engine's; its grid matrix, ephemeris, noise levels and data
   may differ) and returns its slot (the engine's own segment is slot 0);
   tdf_engine_upload_segment() replaces a slot's inputs;
   tdf_engine_segment_count() gives the number of slots. */
int tdf_engine_add_segment(tdf_engine *e, const tdf_segment *seg, int32_t *slot);
int tdf_engine_upload_segment(tdf_engine *e, int32_t slot, const tdf_segment *seg);
int tdf_engine_segment_count(tdf_engine *e, int32_t *count);

/* Device-only pass over the points of several resident segments: segment
   slots[k] searches npts[k] points (pm, mm, nn hold them one segment after
   the other; spindowns from spndr[0]), the work of that many job_core()
   calls per segment (jobcore.c:193-630).  All template parameters are
   formed and uploaded first and the call's whole device work -- every
   batch's sky stage and spindown stage, segment after segment -- is one
   enqueue sequence with no host step between batches; the second call with
   the same batch list captures it into one CUDA graph, later calls replay
   it with a single launch.  Returns the record and trigger counts. */
int tdf_search_segments_device(tdf_engine *e, int32_t nseg, const int32_t *slots, const int32_t *npts,
                               const int32_t *pm, const float *mm, const float *nn,
                               int64_t *nrec, int64_t *ntrig);

/* The full F-statistic of one template (sky point, spindown ss) over bins
   [fr0, fr1], after the optional blocks_avg normalisation: F[k - fr0]
   (jobcore.c:481-515).  Returns TDF_ERR_INVALID if the point is outside the
   sky ellipse. */
int tdf_fstat_spectrum(tdf_engine *e, int32_t pm, float mm, float nn, float ss,
                       double *F, int64_t nF);

/* A continuous-wave signal to inject: the fields of the reference's signal
   file (read_signal_file, init.c:300-358) and the settings add_signal()
   reads (init.c:365-504). */
typedef struct tdf_signal {
     double h0;                /* GW amplitude (the 'amp' form); used when snr <= 0 */
     double snr;               /* > 0: h0 = snr / sqrt(sum_n sum_i s_n[i]^2 / sig2_n) */
     double freq, fdot;        /* [Hz], [Hz/s] in the reference segment */
     double ra, dec;           /* [rad] */
     double iota, psi, phase;  /* [rad] */
     double fpo, B;            /* band start and width [Hz] (sett->fpo, sett->B) */
     int32_t reffr;            /* reference segment of freq */
     int32_t seg;              /* this segment's number (opts->seg) */
} tdf_signal;

/* add_signal() (init.c:365-504) on the engine's resident data, replacing
   the host-side call main.c:101-104 makes before the search: h0*s_n[i] is
   added to detector n's xDat[i] wherever xDat[i] != 0; sig2 keeps the value
   of the data as read.  A signal outside [fpo, fpo + B] adds nothing
   (*in_band = 0), as in the reference.  *h0 (may be NULL) receives the
   amplitude used.  The reference's 'snr' form reads sig2 past the detector
   array (init.c:462-464); snr > 0 here is the network SNR above instead.
   tdf_engine_upload() replaces the data, injection included. */
int tdf_engine_add_signal(tdf_engine *e, const tdf_signal *sig, double *h0, int32_t *in_band);

/* h0*s_n[i], i < N, of the signal the last tdf_engine_add_signal() added to
   detector `det` (n >= N values): what the reference writes with
   mods=write_signal (init.c:475-497).  Held until the next search or upload
   (the engine reuses the memory); TDF_ERR_INVALID when no signal is held. */
int tdf_engine_get_signal(tdf_engine *e, int32_t det, double *out, int64_t n);

/* Copies detector det's resident xDat (the first n <= N floats, injections
   included) to the host. */
int tdf_engine_get_xdat(tdf_engine *e, int32_t det, float *xdat, int64_t n);

/* ---- coincidences between segments (coincidences/coincidences.c) ---- */

/* The options of the reference's [coincidences] INI section (io.c:86-154). */
typedef struct tdf_coinc_opts {
     int32_t refr;        /* reference segment: trigger frequencies are moved to it */
     double cthr;         /* F-statistic threshold */
     int32_t scalef;      /* cell size in frequency, in bins of pi/nfftf */
     int32_t scales, scalem, scalen;   /* cell sizes in grid steps */
     int32_t mincoin;     /* segments a coincidence needs (>= 1) */
     int32_t shift;       /* -1: the 16 cell shifts 0..15; else that one (bits m,n,s,f = 8,4,2,1) */
} tdf_coinc_opts;

/* One segment's search: what the reference reads from its trigger file.
   Every segment must hold the same templates in the same order (the same
   grid and search range); the template headers are taken from segment 0. */
typedef struct tdf_coinc_segment {
     int32_t seg;               /* segment number (opts.seg of that search) */
     int32_t N, nfftf;          /* sett.N, sett.nfftf (nfftf equal in all segments) */
     double dt, narrowdown;     /* sett.dt; opts.narrowdown [rad] */
     int32_t nlines;            /* veto intervals, [nlines][2] in units of f (0..pi) */
     const double *lines;
     int64_t nrec;              /* its records, as tdf_search_points() returns them */
     const tdf_record *recs;
     const float *pairs;
} tdf_coinc_segment;

typedef struct tdf_coincidence {
     int32_t shift;             /* 0..15, bits m,n,s,f = 8,4,2,1 (the reference's "mnsf" string) */
     int32_t w;                 /* segments in the coincidence */
     float avg_snr, avg_f, avg_fdot, avg_ra, avg_dec;
     int64_t member;            /* its w members start here in cseg[], trig[], ntrig[] */
} tdf_coincidence;

/* The coincidence search of coincidences.c:44-436 over nseg segments: per
   segment the triggers with F >= cthr inside the narrow-down window and
   outside the veto lines, moved to segment refr by their spindown
   (select_goodcands, :439-503); per shift the (m, n, s) cells of the
   templates, the loudest trigger per (cell, segment, frequency cell), and a
   coincidence wherever >= mincoin segments share a frequency cell.  Output,
   shift by shift in increasing order, each shift's coincidences in the
   reference's order (more segments first, then higher mean SNR): coi[] and
   their members (segment index cseg, template index trig, triggers in the
   cell ntrig); seginfo[nshift][nseg][3] = {segment number, selected
   triggers, unique triggers of the shift}.  If max_coi or max_members is too
   small nothing is written, *ncoi and *nmembers receive the sizes needed and
   the call returns TDF_ERR_CAPACITY.  Runs on the host; no device is needed.
   Extension of this library: the reference is a separate program reading
   HDF5 trigger files. */
int tdf_coincidences(const tdf_coinc_opts *opts, int32_t nseg, const tdf_coinc_segment *segs,
                     tdf_coincidence *coi, int64_t max_coi, int64_t *ncoi,
                     int16_t *cseg, int32_t *trig, int16_t *ntrig, int64_t max_members, int64_t *nmembers,
                     int32_t *seginfo);

/* F-statistic of one template of the split form from spindown operands that
   are already on the device, without allocating any memory.  No counterpart
   in the reference: it is for callers that must not allocate device memory
   once they run -- hosts whose memory is owned by another allocator or
   reserved up front, and code paths where the implicit synchronisation of
   cudaMalloc/cudaFree is not acceptable.  The caller owns every input and
   output buffer (DEVICE pointers):
     d_xab : float4 [nifo][Nal]  (xDatma/sig2 re, im, xDatmb/sig2 re, im)
     d_s2  : float  [nifo][Nal]  (float)(2 i shft[i])
     d_F   : float  [fr1 - fr0 + 1]  output, F over bins [fr0, fr1]
   het1, spnd: the template's phase coefficients (FP64); aa, bb: the network
   sums of the amplitude modulation (jobcore.c:373-386).  The intermediate
   spectra and FFT tables live in one static device array of the library
   (about 4.3 MB, held on every GPU that loads the library until the
   process exits), so nfftf is limited to 2^18 (4096 <= nfftf <= 2^18,
   power of two, N <= nfftf, 1 <= nifo <= 8); larger sizes are rejected with
   TDF_ERR_UNSUPPORTED.  The array holds the FFT tables of every supported
   nfftf.  The first call on a device (and the first after the device's
   context was reset) resolves the array's device address, writes all the
   tables on `stream` and waits for them there (a one-time synchronisation);
   it is refused with TDF_ERR_INVALID while `stream` is being captured, so
   make it outside any capture.  Later calls only read the tables.  All
   calls share the one array's spectra and parameters, which keep the last
   call's contents: calls whose work overlaps on the GPU (other streams,
   other host threads) race, so serialise them.  Work is enqueued on
   `stream` (cudaStream_t, NULL = default stream) and completes
   asynchronously. */
int tdf_fstat_operands_static(const void *d_xab, const float *d_s2, int32_t nifo, int32_t N, int32_t Nal,
                              int32_t nfftf, double het1, double spnd, float aa, float bb,
                              int32_t fr0, int32_t fr1, float *d_F, void *stream);

/* The CUDA stream the engine enqueues on (a cudaStream_t), and a way to make
   it enqueue on the caller's stream instead (NULL = the engine's own, which
   has the device's highest stream priority).  The sky stage of the next
   batch runs on an internal stream of the lowest priority, overlapping the
   spindown stage, only while the engine's stream has a higher priority than
   that; on a caller's stream of the default (lowest) priority it runs in
   line. */
int tdf_engine_get_stream(tdf_engine *e, void **stream);
int tdf_engine_set_stream(tdf_engine *e, void *stream);

/* Chooses the spindown stage's launch configuration by timing device-only
   passes over these points: the templates per chunk (one column-pass and
   one row-pass launch each; 6..96), then the lanes (concurrent streams with
   their own buffers; 2..6), then the templates per resolve group (the
   trigger-selection launch's share; 32, 64, 128), each at the best of the
   previous choices, and keeps the fastest in the engine; *best (may be
   NULL) receives the templates per chunk, tdf_engine_get_tuning() all
   three.  With the environment variable TDF_AUTOTUNE_CACHE=<file> the
   choice is appended to that file and picked up by engines created later
   for the same form, sizes, GPU, sky batch and F store. */
int tdf_engine_autotune(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn,
                        int32_t *best);
int tdf_engine_get_tuning(tdf_engine *e, int32_t *templates_per_chunk, int32_t *lanes, int32_t *group_templates);

/* Templates per chunk of the spindown stage (one column-pass and one
   row-pass launch each): get, and set to 1..96 (TDF_ERR_INVALID otherwise).
   tdf_engine_autotune() chooses it; a set value holds until the next
   autotune.  Extension of this library: job_core() has no chunking. */
int tdf_engine_get_templates_per_chunk(tdf_engine *e, int32_t *tc);
int tdf_engine_set_templates_per_chunk(tdf_engine *e, int32_t tc);

/* Kernel launches issued by the engine since creation (for accounting). */
int tdf_engine_launch_count(tdf_engine *e, int64_t *count);

/* Per-kernel device time, measured with CUDA events recorded on the
   engine's stream around each launch while timing is on. */
typedef struct tdf_kernel_times {
     double colpass_ms;          /* demodulation + first FFT pass (with the fused
                                    passes: the whole k_spinpass launch) */
     double rowpass_ms;          /* second FFT pass + F-statistic (0 when fused) */
     double threshold_ms;        /* local maxima, veto, trigger append */
     double sky_ms;              /* whole sky stage */
     int64_t colpass_launches, rowpass_launches, threshold_launches, sky_batches;
     int64_t colpass_templates;  /* templates processed by the timed column passes */
} tdf_kernel_times;

/* on != 0 starts timing (and clears the accumulators); 0 stops it. */
int tdf_engine_set_kernel_timing(tdf_engine *e, int on);
int tdf_engine_get_kernel_times(tdf_engine *e, tdf_kernel_times *out);

#ifdef __cplusplus
}
#endif

#endif
