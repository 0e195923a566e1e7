// refabi.cu -- job_core() with the reference's signature
// (search/network/openmp/jobcore.c:193-630), implemented as a client of the
// plain C ABI of tdfcuda.h.  See include/tdfcuda_refabi.h.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <vector>

#include "tdfcuda.h"
#include "tdfcuda_refabi.h"

// the host program's detector array (main.c:29); weak so that the library
// also loads into processes that do not define it
extern "C" __attribute__((weak)) tdf_ref_Detector_settings ifo[TDF_REF_MAX_DETECTORS];

namespace {

struct DropinState {
     tdf_engine *eng = nullptr;
     // what the engine was built from
     const void *key_ptrs[2 * TDF_REF_MAX_DETECTORS + 2] = {};
     int N = 0, nfftf = 0, nifo = 0, form = -1, bufsize = 0, numlines = 0, allsky = -1, blocks = -1;
     int fr0 = 0, fr1 = 0;
     double thr = 0.;
     float spndr1 = 0.f, sstep = 0.f;
     std::vector<tdf_record> recs;
     std::vector<float> pairs;
};

DropinState g_state;
std::mutex g_mu;

[[noreturn]] void die(const char *what, int st) {
     printf("\n[ERROR] %s: %s (%s)\n", what, tdf_status_string(st), tdf_last_error());
     printf("\nFAILURE\n");
     fflush(stdout);
     exit(EXIT_FAILURE);
}

int env_form() {
     const char *f = getenv("TDF_FORM");
     if (f && strcmp(f, "fp64") == 0) return TDF_FORM_FP64;
     return TDF_FORM_SPLIT;
}

}  // namespace

extern "C" {

size_t tdf_ref_struct_size(int which) {
     switch (which) {
     case 0: return sizeof(tdf_ref_Command_line_opts);
     case 1: return sizeof(tdf_ref_Signals);
     case 2: return sizeof(tdf_ref_Search_range);
     case 3: return sizeof(tdf_ref_Aux_arrays);
     case 4: return sizeof(tdf_ref_Search_settings);
     case 5: return sizeof(tdf_ref_Detector_settings);
     case 6: return sizeof(tdf_ref_Trigger);
     }
     return 0;
}

void tdf_job_core_release(void) {
     std::lock_guard<std::mutex> lk(g_mu);
     if (g_state.eng) tdf_engine_destroy(g_state.eng);
     g_state.eng = nullptr;
}

int tdf_job_core_ref(int pm, float mm, float nn, tdf_ref_Search_settings *sett, tdf_ref_Command_line_opts *opts,
                     tdf_ref_Search_range *s_range, void *plans, void *fftw_arr, tdf_ref_Aux_arrays *aux,
                     int *sgnlc, tdf_ref_Trigger *sgnlv, int *FNum) {
     (void)plans;
     (void)fftw_arr;
     std::lock_guard<std::mutex> lk(g_mu);
     if (&ifo[0] == nullptr) die("job_core: the host defines no ifo[] array", TDF_ERR_INVALID);
     const int nifo = sett->nifo;
     const int form = env_form();
     const int allsky = opts->gtype && strcmp(opts->gtype, "allsky") == 0;
     const int blocks = opts->fstat_norm && strcmp(opts->fstat_norm, "blocks_avg") == 0;
     DropinState &S = g_state;
     // (re)create the engine when the inputs or options change
     bool same = S.eng && S.N == sett->N && S.nfftf == sett->nfftf && S.nifo == nifo && S.form == form &&
                 S.bufsize == sett->bufsize && S.numlines == sett->numlines_band && S.allsky == allsky &&
                 S.blocks == blocks && S.fr0 == s_range->fr[0] && S.fr1 == s_range->fr[1] && S.thr == opts->thr &&
                 S.spndr1 == s_range->spndr[1] && S.sstep == s_range->sstep && S.key_ptrs[0] == aux->cosmodf &&
                 S.key_ptrs[1] == aux->sinmodf;
     for (int d = 0; same && d < nifo; d++)
          same = S.key_ptrs[2 + 2 * d] == ifo[d].sig.xDat && S.key_ptrs[3 + 2 * d] == ifo[d].sig.DetSSB;
     if (!same) {
          if (S.eng) tdf_engine_destroy(S.eng);
          S.eng = nullptr;
          tdf_segment seg;
          memset(&seg, 0, sizeof(seg));
          seg.N = sett->N;
          seg.nfft = sett->nfft;
          seg.nfftf = sett->nfftf;
          seg.Ninterp = sett->Ninterp;
          seg.interpftpad = sett->interpftpad;
          seg.nifo = nifo;
          seg.dt = sett->dt;
          seg.oms = sett->oms;
          seg.sepsm = sett->sepsm;
          seg.cepsm = sett->cepsm;
          seg.Smin = sett->Smin;
          seg.Smax = sett->Smax;
          memcpy(seg.M, sett->M, sizeof(seg.M));
          seg.cosmodf = aux->cosmodf;
          seg.sinmodf = aux->sinmodf;
          for (int d = 0; d < nifo; d++) {
               seg.det[d].xdat = ifo[d].sig.xDat;
               seg.det[d].detssb = ifo[d].sig.DetSSB;
               seg.det[d].sig2 = ifo[d].sig.sig2;
               seg.det[d].sphir = ifo[d].sig.sphir;
               seg.det[d].cphir = ifo[d].sig.cphir;
               const tdf_ref_Ampl_mod_coeff &a = ifo[d].amod;
               const double c[9] = {a.c1, a.c2, a.c3, a.c4, a.c5, a.c6, a.c7, a.c8, a.c9};
               memcpy(seg.det[d].amod, c, sizeof(c));
          }
          tdf_search_opts o;
          memset(&o, 0, sizeof(o));
          o.thr = opts->thr;
          o.fr[0] = s_range->fr[0];
          o.fr[1] = s_range->fr[1];
          o.allsky = allsky;
          o.blocks_avg = blocks;
          o.spndr[0] = s_range->spndr[0];
          o.spndr[1] = s_range->spndr[1];
          o.sstep = s_range->sstep;
          o.bufsize = sett->bufsize;
          o.numlines = sett->numlines_band;
          o.lines = &sett->lines[0][0];
          const char *dv = getenv("TDF_DEVICE");
          int st = tdf_engine_create(&seg, &o, form, dv ? atoi(dv) : 0, 1, &S.eng);
          if (st != TDF_OK) die("job_core: engine set-up", st);
          S.N = sett->N;
          S.nfftf = sett->nfftf;
          S.nifo = nifo;
          S.form = form;
          S.bufsize = sett->bufsize;
          S.numlines = sett->numlines_band;
          S.allsky = allsky;
          S.blocks = blocks;
          S.fr0 = s_range->fr[0];
          S.fr1 = s_range->fr[1];
          S.thr = opts->thr;
          S.spndr1 = s_range->spndr[1];
          S.sstep = s_range->sstep;
          S.key_ptrs[0] = aux->cosmodf;
          S.key_ptrs[1] = aux->sinmodf;
          for (int d = 0; d < nifo; d++) {
               S.key_ptrs[2 + 2 * d] = ifo[d].sig.xDat;
               S.key_ptrs[3 + 2 * d] = ifo[d].sig.DetSSB;
          }
     }
     // spindown range for the ">>" line (jobcore.c:399-414)
     const double *M = sett->M;
     float smin = s_range->sst, smax = s_range->spndr[1];
     const double al1 = nn * M[10] + mm * M[14], al2 = nn * M[11] + mm * M[15];
     if ((al1 * al1 + al2 * al2) / (sett->oms * sett->oms) > 1.) return 0;
     if (allsky) {
          smin = trunc((sett->Smin - nn * M[9] - mm * M[13]) / M[5]);
          smax = trunc(-(nn * M[9] + mm * M[13] + sett->Smax) / M[5]);
          if (smin > smax) {
               smin = smin + smax;
               smax = smin - smax;
               smin = smin - smax;
          }
     }
     printf("\n>>%d\t%g\t%g\t[%g..%g:%g]\n", *FNum, mm, nn, smin, smax, s_range->sstep);
     const int32_t p = pm;
     const float m = mm, n = nn, s0 = s_range->sst;
     int64_t nrec = 0, npairs = 0;
     struct timespec t0, t1;
     clock_gettime(CLOCK_MONOTONIC, &t0);
     int st = tdf_count_templates(S.eng, 1, &p, &m, &n, &s0, &nrec, nullptr);
     if (st != TDF_OK) die("job_core", st);
     if ((int64_t)S.recs.size() < nrec) S.recs.resize(nrec);
     st = tdf_search_points(S.eng, 1, &p, &m, &n, &s0, S.recs.data(), (int64_t)S.recs.size(), &nrec,
                            S.pairs.data(), (int64_t)S.pairs.size(), &npairs, nullptr);
     if (st == TDF_ERR_CAPACITY) {
          // the engine kept the results; fetch them into larger arrays
          S.recs.resize(nrec);
          S.pairs.resize(npairs);
          st = tdf_last_results(S.eng, S.recs.data(), nrec, &nrec, S.pairs.data(), npairs, &npairs, nullptr);
     }
     if (st == TDF_ERR_TRIGGER_OVERFLOW) {
          printf("\n[ERROR] Too many triggers! buffer_size=%d [triggers]\n", sett->bufsize / 2);
          printf("\nFAILURE\n");
          fflush(stdout);
          exit(EXIT_FAILURE);
     }
     if (st != TDF_OK) die("job_core", st);
     clock_gettime(CLOCK_MONOTONIC, &t1);
     int ntrig = 0, maxt = 0;
     for (int64_t r = 0; r < nrec; r++) {
          const tdf_record &R = S.recs[r];
          tdf_ref_Trigger &T = sgnlv[r];
          T.m = R.m;
          T.n = R.n;
          T.s = R.s;
          T.ra = R.ra;
          T.dec = R.dec;
          T.fdot = R.fdot;
          T.ffstat.len = R.len;
          if (T.ffstat.p == nullptr) {
               T.ffstat.p = malloc((size_t)sett->bufsize * sizeof(float));
               if (T.ffstat.p == nullptr) {
                    printf("[ERROR] Cannot allocate memory for triggers buffer of size %d\n", sett->bufsize);
                    exit(EXIT_FAILURE);
               }
          }
          if (R.len) memcpy(T.ffstat.p, S.pairs.data() + R.offset, R.len * sizeof(float));
          ntrig += (int)(R.len / 2);
          if ((int)(R.len / 2) > maxt) maxt = (int)(R.len / 2);
     }
     *FNum += (int)nrec;
     *sgnlc += ntrig;
     const int half = sett->bufsize / 2;
     printf("  ntrig=%d, buffer usage: [max=%d/%d=%.2f%%] [mean=%.2f%%]\n", *sgnlc, maxt, half,
            (float)maxt * 100 / half, nrec ? (float)(*sgnlc) * 100 / (half * (float)nrec) : 0.f);
     const double el = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
     printf("  [Perf] Spindown loop cputime: %e s, <cputime/ns>: %e s (ns: %lld)\n", el, nrec ? el / nrec : 0.,
            (long long)nrec);
     return 0;
}

int job_core(int pm, float mm, float nn, tdf_ref_Search_settings *sett, tdf_ref_Command_line_opts *opts,
             tdf_ref_Search_range *s_range, void *plans, void *fftw_arr, tdf_ref_Aux_arrays *aux, int *sgnlc,
             tdf_ref_Trigger *sgnlv, int *FNum) {
     return tdf_job_core_ref(pm, mm, nn, sett, opts, s_range, plans, fftw_arr, aux, sgnlc, sgnlv, FNum);
}

}  // extern "C"
