// coinc.cu -- tdf_coincidences(): the coincidence search between segments of
// coincidences/coincidences.c (host code).
//
// The reference scans, for every (m, n, s) cell, every frequency cell of
// the band (nfftf/scalef of them) in every segment (:291-362); here only the
// frequency cells the cell's triggers fall in are visited, in the same
// increasing order, which gives the same coincidences in the same order.
// Every expression keeps the reference's float/double evaluation (its build,
// coincidences/Makefile, contracts f + a*b into one fused multiply-add,
// which the segment shift below reproduces with std::fma).
//
// The 16 cell shifts are independent searches over the same selected
// triggers: they run on up to 16 host threads (TDF_COINC_THREADS, default
// the hardware threads), each with its own scratch, and their results are
// joined in shift order, so the output does not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "tdfcuda.h"

int tdf_internal_set_error(int code, const char *fmt, ...);

namespace {

struct Good {          // a selected trigger of one template in one segment
     float f, F;
};

// select_goodcands (coincidences.c:439-503) for one segment: per template
// the triggers kept, frequencies moved to segment refr
static int64_t select_good(const tdf_coinc_opts &o, const tdf_coinc_segment &s, std::vector<int64_t> &off,
                           std::vector<Good> &out) {
     off.assign(s.nrec + 1, 0);
     out.clear();
     int64_t nsel = 0;
     for (int64_t j = 0; j < s.nrec; j++) {
          off[j] = (int64_t)out.size();
          const tdf_record &r = s.recs[j];
          const float *p = s.pairs + r.offset;
          const float fdot_lin = (float)((double)r.fdot * M_PI * std::pow(s.dt, 2));
          for (uint32_t t = 0; t < r.len / 2; t++) {
               float f = p[2 * t];
               const float fstat = p[2 * t + 1];
               if (fstat < o.cthr) continue;
               if (((double)f <= M_PI_2 - s.narrowdown) || ((double)f >= M_PI_2 + s.narrowdown)) continue;
               bool isline = false;
               for (int il = 0; il < s.nlines; il++)
                    if ((double)f >= s.lines[2 * il] && (double)f <= s.lines[2 * il + 1]) {
                         isline = true;
                         break;
                    }
               if (isline) continue;
               // f = f + 2.*fdot_lin*(N)*(refr - seg), the last product and the
               // sum fused as the reference's build fuses them
               f = (float)std::fma(2. * (double)fdot_lin * (double)s.N, (double)(o.refr - s.seg), (double)f);
               if (((double)f < 0) || ((double)f > M_PI)) continue;
               out.push_back(Good{f, fstat});
               nsel++;
          }
     }
     off[s.nrec] = (int64_t)out.size();
     return nsel;
}

struct CellState {     // per (segment, frequency cell) of the current (m, n, s) cell
     float best_snr = 0.f, best_f = 0.f;
     int best = -1;
     int16_t ntrig = 0;
};

struct Coi {
     float avg_snr, avg_f, avg_fdot, avg_ra, avg_dec;
     int w;
     int64_t member;   // first member in the result's member arrays
};

struct ShiftInput {
     const tdf_coinc_opts *o;
     int nseg;
     const tdf_record *hdr;   // ctrigs take segment 0's headers (coincidences.c:80-91)
     int64_t nrec;
     int nfc;                 // frequency cells
     int nfftf;
     const std::vector<std::vector<int64_t>> *off;
     const std::vector<std::vector<Good>> *good;
};

struct ShiftScratch {
     struct Key { int mc, nc, sc; };
     std::vector<CellState> st;
     std::vector<int> dirty, fics;
     std::vector<int32_t> order;
     std::vector<Key> key;
};

struct ShiftResult {
     std::vector<Coi> coi;                  // in output order
     std::vector<int16_t> mem_seg, mem_n;
     std::vector<int32_t> mem_trig;
     std::vector<int32_t> uniq;             // per segment: coincidence members
};

// One cell shift ish (bits m, n, s, f = 8, 4, 2, 1): coincidences.c:196-367.
static void run_shift(const ShiftInput &in, int ish, ShiftScratch &sc, ShiftResult &r) {
     const tdf_coinc_opts *o = in.o;
     const int nseg = in.nseg, nfc = in.nfc, nfftf = in.nfftf;
     const int64_t nrec = in.nrec;
     const tdf_record *hdr = in.hdr;
     const auto &off = *in.off;
     const auto &good = *in.good;
     sc.st.assign((size_t)nseg * nfc, CellState());
     sc.order.resize(nrec);
     sc.key.resize(nrec);
     auto &st = sc.st;
     auto &order = sc.order;
     auto &key = sc.key;
     auto &dirty = sc.dirty;
     auto &fics = sc.fics;
     r.coi.clear();
     r.mem_seg.clear();
     r.mem_n.clear();
     r.mem_trig.clear();
     r.uniq.assign(nseg, 0);
     int32_t *un = r.uniq.data();
     auto &mem_seg = r.mem_seg;
     auto &mem_trig = r.mem_trig;
     auto &mem_n = r.mem_n;
     auto &shift_coi = r.coi;
     const float shm = ((ish >> 3) & 1) * 0.5f, shn = ((ish >> 2) & 1) * 0.5f;
     const float shs = ((ish >> 1) & 1) * 0.5f, shf = (ish & 1) * 0.5f;
     for (int64_t j = 0; j < nrec; j++) {
          key[j].mc = (int)floorf(hdr[j].m / o->scalem - shm);
          key[j].nc = (int)floorf(hdr[j].n / o->scalen - shn);
          key[j].sc = (int)floorf(hdr[j].s / o->scales - shs);
          order[j] = (int32_t)j;
     }
     // the reference's qsort (glibc: a merge sort, stable) by (mc, nc, sc)
     std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
          if (key[a].mc != key[b].mc) return key[a].mc < key[b].mc;
          if (key[a].nc != key[b].nc) return key[a].nc < key[b].nc;
          return key[a].sc < key[b].sc;
     });
     for (int64_t c0 = 0; c0 < nrec;) {
          int64_t c1 = c0 + 1;
          while (c1 < nrec && key[order[c1]].mc == key[order[c0]].mc && key[order[c1]].nc == key[order[c0]].nc &&
                 key[order[c1]].sc == key[order[c0]].sc)
               c1++;
          // pass 1 (:264-294): the loudest trigger per (segment, frequency cell)
          dirty.clear();
          for (int64_t jj = c0; jj < c1; jj++) {
               const int32_t cidx = order[jj];
               for (int s = 0; s < nseg; s++) {
                    for (int64_t k = off[s][cidx]; k < off[s][cidx + 1]; k++) {
                         const float f = good[s][k].f;
                         const float snr2 = (float)(2. * good[s][k].F - 4.);
                         const int fic = (int)floorf((float)((double)f / (M_PI / nfftf) / o->scalef - shf));
                         if ((unsigned)fic >= (unsigned)nfc) continue;
                         CellState &cs = st[(size_t)s * nfc + fic];
                         if (cs.best < 0 && cs.ntrig == 0) dirty.push_back(s * nfc + fic);
                         cs.ntrig++;
                         if (snr2 > cs.best_snr) {
                              cs.best_snr = snr2;
                              cs.best = cidx;
                              cs.best_f = f;
                         }
                    }
               }
          }
          // pass 2 (:296-362), over the frequency cells touched, increasing
          fics.clear();
          for (int d : dirty) fics.push_back(d % nfc);
          std::sort(fics.begin(), fics.end());
          fics.erase(std::unique(fics.begin(), fics.end()), fics.end());
          for (int fic : fics) {
               int w = 0;
               float sum_snr = 0.f, sum_f = 0.f, sum_fdot = 0.f, sum_ra = 0.f, sum_dec = 0.f;
               const size_t m0 = mem_seg.size();
               for (int s = 0; s < nseg; s++) {
                    const CellState &cs = st[(size_t)s * nfc + fic];
                    if (cs.best < 0) continue;
                    un[s]++;
                    mem_seg.push_back((int16_t)s);
                    mem_trig.push_back(cs.best);
                    mem_n.push_back(cs.ntrig);
                    sum_snr += cs.best_snr;
                    sum_f += cs.best_f;
                    sum_fdot += hdr[cs.best].fdot;
                    sum_ra += hdr[cs.best].ra;
                    sum_dec += hdr[cs.best].dec;
                    w++;
               }
               if (w < o->mincoin) {
                    mem_seg.resize(m0);
                    mem_trig.resize(m0);
                    mem_n.resize(m0);
                    continue;
               }
               shift_coi.push_back(Coi{sqrtf(sum_snr / w), sum_f / w, sum_fdot / w, sum_ra / w, sum_dec / w, w,
                                       (int64_t)m0});
          }
          for (int d : dirty) st[d] = CellState();
          c0 = c1;
     }
     // qsort(coi, cmp_coi) (:365): more segments first, then higher SNR; stable
     std::stable_sort(shift_coi.begin(), shift_coi.end(), [](const Coi &a, const Coi &b) {
          if (a.w != b.w) return a.w > b.w;
          return a.avg_snr > b.avg_snr;
     });
}

}  // namespace

extern "C" int tdf_coincidences(const tdf_coinc_opts *o, int32_t nseg, const tdf_coinc_segment *segs,
                                tdf_coincidence *coi, int64_t max_coi, int64_t *ncoi, int16_t *cseg, int32_t *trig,
                                int16_t *ntrig, int64_t max_members, int64_t *nmembers, int32_t *seginfo) {
     if (!o || !segs || nseg < 1 || !ncoi || !nmembers)
          return tdf_internal_set_error(TDF_ERR_INVALID, "null argument or no segment");
     if (o->scalef < 1 || o->scales < 1 || o->scalem < 1 || o->scalen < 1 || o->mincoin < 1 || o->shift < -1 ||
         o->shift > 15)
          return tdf_internal_set_error(TDF_ERR_INVALID, "cell scales and mincoin must be >= 1, shift -1..15");
     const int64_t nrec = segs[0].nrec;
     const int nfftf = segs[0].nfftf;
     for (int s = 0; s < nseg; s++) {
          if (segs[s].nrec != nrec)
               return tdf_internal_set_error(TDF_ERR_INVALID, "segment %d holds %lld records, segment 0 %lld", s,
                                             (long long)segs[s].nrec, (long long)nrec);
          if (segs[s].nfftf != nfftf) return tdf_internal_set_error(TDF_ERR_INVALID, "nfftf differs between segments");
          if (nrec > 0 && (!segs[s].recs || !segs[s].pairs))
               return tdf_internal_set_error(TDF_ERR_INVALID, "segment %d: null records", s);
          if (segs[s].nlines > 0 && !segs[s].lines) return tdf_internal_set_error(TDF_ERR_INVALID, "null lines");
     }
     if (nrec > INT32_MAX) return tdf_internal_set_error(TDF_ERR_UNSUPPORTED, "more than 2^31 templates");
     // selected triggers per segment
     std::vector<std::vector<int64_t>> off(nseg);
     std::vector<std::vector<Good>> good(nseg);
     std::vector<int32_t> nsel(nseg);
     for (int s = 0; s < nseg; s++) nsel[s] = (int32_t)select_good(*o, segs[s], off[s], good[s]);
     const int ish0 = o->shift < 0 ? 0 : o->shift, ish1 = o->shift < 0 ? 15 : o->shift;
     const int nsh = ish1 - ish0 + 1;
     std::vector<ShiftResult> res(nsh);
     const ShiftInput in{o, nseg, segs[0].recs, nrec, nfftf / o->scalef, nfftf, &off, &good};
     int nthr = (int)std::thread::hardware_concurrency();
     if (const char *ev = getenv("TDF_COINC_THREADS")) nthr = atoi(ev);
     nthr = std::max(1, std::min(nthr, nsh));
     std::vector<std::exception_ptr> fail(nthr);
     auto work = [&](int t) {
          try {
               ShiftScratch sc;
               for (int i = t; i < nsh; i += nthr) run_shift(in, ish0 + i, sc, res[i]);
          } catch (...) {
               fail[t] = std::current_exception();
          }
     };
     {
          // workers 1.. on threads (a worker whose thread cannot be started
          // runs here instead), worker 0 on this thread
          std::vector<std::thread> pool;
          std::vector<int> inline_workers;
          for (int t = 1; t < nthr; t++) {
               try {
                    pool.emplace_back(work, t);
               } catch (...) {
                    inline_workers.push_back(t);
               }
          }
          work(0);
          for (int t : inline_workers) work(t);
          for (auto &th : pool) th.join();
     }
     for (auto &f : fail)
          if (f) return tdf_internal_set_error(TDF_ERR_OUT_OF_MEMORY, "coincidence search: host allocation failed");
     // join in shift order
     std::vector<Coi> all;
     std::vector<int32_t> shifts;
     std::vector<int16_t> mem_seg, mem_n;
     std::vector<int32_t> mem_trig;
     for (int i = 0; i < nsh; i++) {
          for (Coi c : res[i].coi) {
               const int64_t m0 = (int64_t)mem_seg.size();
               for (int k = 0; k < c.w; k++) {
                    mem_seg.push_back(res[i].mem_seg[c.member + k]);
                    mem_trig.push_back(res[i].mem_trig[c.member + k]);
                    mem_n.push_back(res[i].mem_n[c.member + k]);
               }
               c.member = m0;
               all.push_back(c);
               shifts.push_back(ish0 + i);
          }
     }
     int64_t nm = 0;
     for (const Coi &c : all) nm += c.w;
     *ncoi = (int64_t)all.size();
     *nmembers = nm;
     if (seginfo) {
          for (int ish = ish0; ish <= ish1; ish++)
               for (int s = 0; s < nseg; s++) {
                    int32_t *si = seginfo + ((size_t)(ish - ish0) * nseg + s) * 3;
                    si[0] = segs[s].seg;
                    si[1] = nsel[s];
                    si[2] = res[ish - ish0].uniq[s];
               }
     }
     if ((int64_t)all.size() > max_coi || nm > max_members)
          return tdf_internal_set_error(TDF_ERR_CAPACITY, "need %lld coincidences and %lld members",
                                        (long long)all.size(), (long long)nm);
     if (!all.empty() && (!coi || !cseg || !trig || !ntrig))
          return tdf_internal_set_error(TDF_ERR_INVALID, "null output arrays");
     int64_t m = 0;
     for (size_t i = 0; i < all.size(); i++) {
          const Coi &c = all[i];
          coi[i].shift = shifts[i];
          coi[i].w = c.w;
          coi[i].avg_snr = c.avg_snr;
          coi[i].avg_f = c.avg_f;
          coi[i].avg_fdot = c.avg_fdot;
          coi[i].avg_ra = c.avg_ra;
          coi[i].avg_dec = c.avg_dec;
          coi[i].member = m;
          for (int k = 0; k < c.w; k++) {
               cseg[m + k] = mem_seg[c.member + k];
               trig[m + k] = mem_trig[c.member + k];
               ntrig[m + k] = mem_n[c.member + k];
          }
          m += c.w;
     }
     return TDF_OK;
}
