// engine.cu -- libtdfcuda: the B200 engine behind include/tdfcuda.h.
//
// One engine = one data segment resident on one GPU.  A call runs a list of
// sky points: the sky stage (FP64) for a batch of points, then every
// template (point, spindown) of the batch through
//   column pass  (demodulation fused into the first FFT pass)
//   row pass     (second FFT pass + F-statistic)
//   [block means](blocks_avg normalisation)
//   threshold    (MAX_ALG 3 local maxima, veto, trigger append)
// in chunks of templates.  Triggers are compacted on the device and sorted
// into the reference's record order on the host.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <cudaTypedefs.h>

#include "tdfcuda.h"
#include "tdf_kernels.cuh"

using namespace tdf;

// ------------------------------------------------------------------ errors

static thread_local std::string g_last_error;

static int set_error(int code, const char *fmt, ...) {
     char buf[1024];
     va_list ap;
     va_start(ap, fmt);
     vsnprintf(buf, sizeof(buf), fmt, ap);
     va_end(ap);
     g_last_error = buf;
     return code;
}

// the same for the library's other sources
int tdf_internal_set_error(int code, const char *fmt, ...) {
     char buf[1024];
     va_list ap;
     va_start(ap, fmt);
     vsnprintf(buf, sizeof(buf), fmt, ap);
     va_end(ap);
     g_last_error = buf;
     return code;
}

#define CUCHK(x)                                                                          \
     do {                                                                                 \
          cudaError_t e_ = (x);                                                           \
          if (e_ != cudaSuccess)                                                          \
               return set_error(e_ == cudaErrorMemoryAllocation ? TDF_ERR_OUT_OF_MEMORY   \
                                                                : TDF_ERR_CUDA,           \
                                "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__,   \
                                __LINE__);                                                \
     } while (0)

#define TRY(x)                        \
     do {                             \
          int s_ = (x);               \
          if (s_ != TDF_OK) return s_; \
     } while (0)

// ------------------------------------------------------------------ launch helpers

static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
static int ilog2i(int n) { int l = 0; while ((1 << l) < n) l++; return l; }

// kernel attributes already set, per (kernel, device): the largest dynamic
// shared memory asked for so far
static std::mutex g_attr_mu;
static std::vector<std::pair<std::pair<const void *, int>, size_t>> g_attr;

template <class K>
static int set_smem(K kern, size_t smem) {
     int dev = 0;
     CUCHK(cudaGetDevice(&dev));
     const std::pair<const void *, int> key((const void *)kern, dev);
     {
          std::lock_guard<std::mutex> lk(g_attr_mu);
          for (const auto &a : g_attr)
               if (a.first == key && a.second >= smem) return TDF_OK;
     }
     if (smem > 48 * 1024) CUCHK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
     // the FFT passes live in shared memory: ask for the largest carveout so
     // that more than one CTA fits per SM
     CUCHK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
     std::lock_guard<std::mutex> lk(g_attr_mu);
     for (auto &a : g_attr)
          if (a.first == key) {
               a.second = std::max(a.second, smem);
               return TDF_OK;
          }
     g_attr.push_back({key, smem});
     return TDF_OK;
}

// Kernels of the sky stage (the FP64 interpolation passes run with one
// array, NA = 1; the spindown passes with two).  A captured graph holding
// both gets the sky stage's kernel nodes at the low stream priority and the
// others at the high one, as the two streams have them when launched
// directly (set_graph_priorities).
static std::mutex g_sky_mu;
static std::vector<const void *> g_sky_kernels;

static void register_sky_kernel(const void *k) {
     std::lock_guard<std::mutex> lk(g_sky_mu);
     if (std::find(g_sky_kernels.begin(), g_sky_kernels.end(), k) == g_sky_kernels.end()) g_sky_kernels.push_back(k);
}

static bool is_sky_kernel(const void *k) {
     std::lock_guard<std::mutex> lk(g_sky_mu);
     return std::find(g_sky_kernels.begin(), g_sky_kernels.end(), k) != g_sky_kernels.end();
}

template <typename T, int L, int SIGN, int NA, class Pro, class Epi>
static int launch_col_L(dim3 grid, const Pro &pro, const Epi &epi_in, const cx<T> *tw, cudaStream_t st) {
     size_t smem = pass_smem_bytes<T, L, NA>();
     if constexpr (is_staged<Pro>::value) smem = pro.smem;
     Epi epi = epi_in;
     if constexpr (has_tables<Epi>::value) {
          // the epilogue's tables go after everything else
          smem = (smem + 15) / 16 * 16;
          epi.tab_off = (unsigned)smem;
          smem += Epi::template table_bytes<L>(epi.N2);
     }
     auto kern = k_colpass<T, L, SIGN, NA, Pro, Epi>;
     if constexpr (NA == 1) register_sky_kernel((const void *)kern);
     TRY(set_smem(kern, smem));
     kern<<<grid, pass_threads<L>(), smem, st>>>(pro, epi, tw);
     CUCHK(cudaGetLastError());
     return TDF_OK;
}

template <typename T, int L, int SIGN, int NA, class Src, class Epi>
static int launch_row_L(dim3 grid, const Src &src_in, const Epi &epi, const cx<T> *tw, cudaStream_t st) {
     size_t smem = pass_smem_bytes<T, L, NA>();
     Src src = src_in;
     if constexpr (is_bulk<Src>::value) {
          // the copies' barrier after the line buffers
          smem = (smem + 15) / 16 * 16;
          src.bar_off = (unsigned)smem;
          smem += 16;
     }
     auto kern = k_rowpass<T, L, SIGN, NA, Src, Epi>;
     if constexpr (NA == 1) register_sky_kernel((const void *)kern);
     TRY(set_smem(kern, smem));
     kern<<<grid, pass_threads<L>(), smem, st>>>(src, epi, tw);
     CUCHK(cudaGetLastError());
     return TDF_OK;
}

template <typename T, int SIGN, int NA, class Pro, class Epi>
static int launch_col(int L, dim3 grid, const Pro &pro, const Epi &epi, const cx<T> *tw, cudaStream_t st) {
     switch (L) {
     case 64: return launch_col_L<T, 64, SIGN, NA>(grid, pro, epi, tw, st);
     case 128: return launch_col_L<T, 128, SIGN, NA>(grid, pro, epi, tw, st);
     case 256: return launch_col_L<T, 256, SIGN, NA>(grid, pro, epi, tw, st);
     case 512: return launch_col_L<T, 512, SIGN, NA>(grid, pro, epi, tw, st);
     case 1024:
          if constexpr (pass_smem_bytes<T, 1024, NA>() <= 227 * 1024)
               return launch_col_L<T, 1024, SIGN, NA>(grid, pro, epi, tw, st);
          else
               return set_error(TDF_ERR_UNSUPPORTED, "column FFT of 1024 points not built for this form");
     }
     return set_error(TDF_ERR_UNSUPPORTED, "column FFT length %d", L);
}

template <typename T, int SIGN, int NA, class Src, class Epi>
static int launch_row(int L, dim3 grid, const Src &src, const Epi &epi, const cx<T> *tw, cudaStream_t st) {
     switch (L) {
     case 64: return launch_row_L<T, 64, SIGN, NA>(grid, src, epi, tw, st);
     case 128: return launch_row_L<T, 128, SIGN, NA>(grid, src, epi, tw, st);
     case 256: return launch_row_L<T, 256, SIGN, NA>(grid, src, epi, tw, st);
     case 512: return launch_row_L<T, 512, SIGN, NA>(grid, src, epi, tw, st);
     case 1024:
          if constexpr (pass_smem_bytes<T, 1024, NA>() <= 227 * 1024)
               return launch_row_L<T, 1024, SIGN, NA>(grid, src, epi, tw, st);
          else
               return set_error(TDF_ERR_UNSUPPORTED, "row FFT of 1024 points not built for this form");
     }
     return set_error(TDF_ERR_UNSUPPORTED, "row FFT length %d", L);
}

// ------------------------------------------------------------------ device buffers

struct DevBuf {
     void *p = nullptr;
     size_t bytes = 0;
     int alloc(size_t n) {
          if (n <= bytes && p) return TDF_OK;
          if (p) cudaFree(p);
          p = nullptr;
          bytes = 0;
          if (n == 0) n = 16;
          CUCHK(cudaMalloc(&p, n));
          bytes = n;
          return TDF_OK;
     }
     void release() {
          if (p) cudaFree(p);
          p = nullptr;
          bytes = 0;
     }
     template <typename X> X *as() const { return reinterpret_cast<X *>(p); }
};

// twiddle tables of one four-step size N = N1*N2 in one precision
template <typename T>
struct FFTTables {
     int N = 0, N1 = 0, N2 = 0;
     DevBuf line1, line2, hi, lo, base, step;
     int build(int n) {
          N = n;
          int l = ilog2i(n);
          N1 = 1 << ((l + 1) / 2);
          N2 = n / N1;
          if (N1 < 64 || N2 < 64 || N1 > 1024 || N2 > 1024)
               return set_error(TDF_ERR_UNSUPPORTED, "FFT length %d outside 2^12..2^20", n);
          TRY(fill(line1, N1, N1));
          TRY(fill(line2, N2, N2));
          int nhi = std::max(1, n / 1024);
          std::vector<cx<T>> h(nhi), o(1024);
          for (int j = 0; j < nhi; j++) h[j] = tw((long)j * 1024, n);
          for (int j = 0; j < 1024; j++) o[j] = tw(j, n);
          TRY(hi.alloc(nhi * sizeof(cx<T>)));
          TRY(lo.alloc(1024 * sizeof(cx<T>)));
          CUCHK(cudaMemcpy(hi.p, h.data(), nhi * sizeof(cx<T>), cudaMemcpyHostToDevice));
          CUCHK(cudaMemcpy(lo.p, o.data(), 1024 * sizeof(cx<T>), cudaMemcpyHostToDevice));
          return TDF_OK;
     }
     // per-thread base twiddles of the column-pass epilogue (StoreFourstepG):
     // base[t*N2 + n2] = W^(n2*t), t < N1/8, and step[n2] = W^(n2*N1/8)
     int build_base() {
          const int R = N1 / 8;
          std::vector<cx<T>> b((size_t)R * N2), st(N2);
          for (int t = 0; t < R; t++)
               for (int n2 = 0; n2 < N2; n2++) b[(size_t)t * N2 + n2] = tw((long)n2 * t, N);
          for (int n2 = 0; n2 < N2; n2++) st[n2] = tw((long)n2 * R, N);
          TRY(base.alloc(b.size() * sizeof(cx<T>)));
          TRY(step.alloc(st.size() * sizeof(cx<T>)));
          CUCHK(cudaMemcpy(base.p, b.data(), b.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
          CUCHK(cudaMemcpy(step.p, st.data(), st.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
          return TDF_OK;
     }
     static cx<T> tw(long m, long n) {
          // e^{-2 pi i m/n}; m/n exact for power-of-two n
          double a = -2.0 * M_PI * ((double)(m % n) / (double)n);
          cx<T> r;
          r.x = (T)std::cos(a);
          r.y = (T)std::sin(a);
          return r;
     }
     int fill(DevBuf &b, int L, int n) {
          std::vector<cx<T>> v(L);
          for (int m = 0; m < L; m++) v[m] = tw(m, n);
          TRY(b.alloc(L * sizeof(cx<T>)));
          CUCHK(cudaMemcpy(b.p, v.data(), L * sizeof(cx<T>), cudaMemcpyHostToDevice));
          return TDF_OK;
     }
     void release() { line1.release(); line2.release(); hi.release(); lo.release(); base.release(); step.release(); }
     const cx<T> *l1() const { return line1.as<cx<T>>(); }
     const cx<T> *l2() const { return line2.as<cx<T>>(); }
     const cx<T> *h() const { return hi.as<cx<T>>(); }
     const cx<T> *o() const { return lo.as<cx<T>>(); }
};


// host view of one template
struct HostTmpl {
     int pt;         // index of the point in the call
     float ss;
     double spnd, het1;
     double sgnl0;
};

struct HostPoint {
     int inside = 0;
     SkyParam sp;
     float ra = 0, dec = 0;
     float smin = 0;
     int iss_size = 0;
     int first_tmpl = 0;
};

// The inputs of one data segment resident on the engine's GPU: the host
// scalars the per-point set-up reads and the device copies the sky stage
// reads.  Slot 0 is the segment the engine was created with; further
// segments of the same sizes may be added (tdf_engine_add_segment).
struct SegData {
     tdf_segment seg{};
     std::vector<DetParam> dets;
     DevBuf xdat, detssb, cosm, sinm, detp;
     void release() { xdat.release(); detssb.release(); cosm.release(); sinm.release(); detp.release(); }
};

struct tdf_engine {
     int dev = 0, form = TDF_FORM_SPLIT;
     cudaStream_t own = nullptr, stream = nullptr;
     // The sky stage of the next batch runs on sky_stream, created at the
     // lowest stream priority while the engine's own stream and the lanes
     // get the highest: its CTAs take the SMs the spindown passes leave
     // free in their tails instead of competing with them (TDF_SKY_OVERLAP=0:
     // sky stage on the engine stream, serialised with the spindown stage).
     cudaStream_t sky_stream = nullptr;
     bool overlap = true;
     // the last injected signal s_n[i] (tdf_engine_add_signal) stays in the
     // sky work buffer B0 until the next sky stage or upload overwrites it
     double signal_h0 = 0.;
     bool signal_valid = false;
     int prio_low = 0, prio_high = 0;     // the device's stream priority range (low >= high numerically)
     bool stream_outranks_sky = true;     // the engine stream has a higher priority than sky_stream
     cudaEvent_t sky_done[2] = {nullptr, nullptr}, spin_done[2] = {nullptr, nullptr};
     std::vector<SegData> sdv;   // resident segments; the work being enqueued reads sdv[act]
     int act = 0;
     SegData &S() { return sdv[act]; }
     const SegData &S() const { return sdv[act]; }
     tdf_search_opts opts{};
     std::vector<double> lines;
     int N = 0, nfft = 0, nfftf = 0, Ninterp = 0, nifo = 0, Nal = 0, n2N = 0;
     int nF = 0, nblk_mu = 0;
     int Bs = 8;        // sky points per batch
     int Tc = 16;       // templates per chunk (intermediate spectra sized for L2)
     int TcMax = 32;    // buffers are sized for chunks up to this size
     int Gt = 64;       // templates per resolve group at most (whole chunks; TDF_GROUP_TEMPLATES)
     static constexpr int kGtMax = 128;   // buffers are sized for groups up to this size
     int64_t launches = 0;
     FFTTables<double> t_nfft, t_ninterp, t_f64;
     FFTTables<float> t_f32;
     // inputs
     DevBuf pco, gco;
     // sky stage
     DevBuf skyp[2], B0, B1, B2, shftf, partial, aabb[2];
     // operands
     DevBuf xab[2], s2[2], xa64[2], xb64[2], t1[2];   // per batch slot
     // TMA staging of the split-form operands in the column pass
     bool staged = false;
     CUtensorMap tm_x[2], tm_s[2];   // xab[k], s2[k]
     int stg_groups = 0, stg_stages = 0;
     unsigned stg_bar_off = 0, stg_smem = 0;
     // spindown stage: consecutive resolve groups alternate between lanes,
     // each with its own stream and buffers, so that one lane's kernel tails
     // and trigger resolution overlap the other lane's passes
     struct Lane {
          DevBuf Ybuf;    // four-step intermediate of a chunk
          DevBuf Fbuf;    // F ring of a resolve group
          DevBuf mubuf;   // blocks_avg means of a resolve group
          DevBuf tcnt;    // per-template trigger counts + candidate count
          DevBuf cand;    // candidate bins of a resolve group (uint2), or the sparse store's records (uint4)
          DevBuf Ebuf;    // sparse F store: edge ring of a resolve group (split form)
          DevBuf ctl;     // fused pass order: tickets, finished CTAs, column blocks done per template
     };
     static constexpr int kMaxLanes = 6;
     Lane ln[kMaxLanes];
     int lanes_alloc = kMaxLanes;   // lanes with buffers and streams (TDF_LANES fixes it to that count)
     int nlanes = 3;                                  // TDF_LANES=n (1..4)
     cudaStream_t lane_own[kMaxLanes] = {};          // streams of lanes 1.. (lane 0 runs on `stream`)
     cudaEvent_t fork_ev = nullptr, join_ev[kMaxLanes] = {};
     DevBuf tparam, linesd;
     unsigned cand_cap = 0;
     // two batch slots: while the host drains one slot's triggers the
     // device runs the other slot's batch
     DevBuf trig[2], counters[2];
     unsigned long long trig_cap = 0;
     SkyParam *h_sky[2] = {nullptr, nullptr};     // pinned staging per slot
     TmplParam *h_tp[2] = {nullptr, nullptr};
     size_t h_tp_cap = 0;
     unsigned long long *h_cnt = nullptr;         // pinned [slot][count, error flags]
     cudaEvent_t done[2] = {nullptr, nullptr};
     int cur = 0;                                 // slot the kernels write to
     std::vector<Trig> h_trig;
     // results of the last search kept after a TDF_ERR_CAPACITY return
     bool kept = false;
     std::vector<tdf_record> last_recs;
     std::vector<float> last_pairs;
     std::vector<int32_t> last_per;
     // CUDA graphs of the spindown stage of a batch, keyed by everything the
     // captured launches bake in; captured on the second sighting of a key
     struct GraphKey {
          int slot, nt, Tc, Gt, lanes;
          bool sparse;
          const void *tp, *trig;
          unsigned long long trig_cap;
          bool operator==(const GraphKey &o) const {
               return slot == o.slot && nt == o.nt && Tc == o.Tc && Gt == o.Gt && lanes == o.lanes &&
                      sparse == o.sparse && tp == o.tp &&
                      trig == o.trig && trig_cap == o.trig_cap;
          }
     };
     struct GraphEntry {
          GraphKey key;
          int seen = 0;
          cudaGraphExec_t exec = nullptr;
          int64_t launches = 0;   // kernels per replay
          uint64_t last = 0;
     };
     static constexpr size_t kMaxGraphs = 8;
     std::vector<GraphEntry> graphs;
     // whole-call plans (tdf_search_segments_device): every batch's sky and
     // template parameters on the device at once, the call's work captured
     // as one graph, keyed by a hash of its batch list and configuration
     DevBuf plan_sky, plan_tp, plan_pts;
     int plan_npts = 0;
     cudaEvent_t plan_ev = nullptr;
     struct PlanGraph {
          uint64_t key = 0;
          int seen = 0;
          cudaGraphExec_t exec = nullptr;
          int64_t launches = 0;
          uint64_t last = 0;
     };
     std::vector<PlanGraph> plan_graphs;
     uint64_t graph_tick = 0;
     bool use_graphs = true;   // TDF_GRAPHS=0 launches every kernel from the host
     bool graph_prio = true;   // TDF_GRAPH_PRIORITY=0 leaves captured kernel nodes at their default priority
     bool row_bulk = true;     // row passes fetch their rows by bulk copies (TDF_ROW_BULK=0: per thread)
     // split form, N1 = N2: TDF_FUSED_PASSES=1 runs the column and row
     // passes of a chunk as one ordered launch of persistent CTAs
     // (k_spinpass), a template's rows fuse_lag templates behind its
     // columns (TDF_FUSE_LAG=n).  Off by default: its spectra stay in L2,
     // but each row block's wait and the publishing fences sit on the CTA's
     // critical path, and it measured ~10% slower than the two launches.
     bool fused = false;
     int fuse_lag = 3;
     // split form: the row pass keeps F on the chip and hands over only the
     // candidates and the edge bins of its runs (TDF_FULL_F=1: full F ring);
     // blocks_avg, and a batch that needs more of the spectrum, use the full
     // store.  sparse_now is the store the current search uses.
     bool sparse_f = true;
     bool sparse_now = false;
     // optional per-kernel event timing
     bool timing = false;
     tdf_kernel_times kt{};
     std::vector<cudaEvent_t> evpool;
     std::vector<size_t> evfree;
     struct Pending { int kind; size_t ev; int64_t templates; };
     std::vector<Pending> pending;
};

enum { KT_COL = 0, KT_ROW = 1, KT_THR = 2, KT_SKY = 3 };

// records the opening event of a timed region; returns the index of an
// event pair in the pool (pairs are recycled once collected)
static size_t timing_begin(tdf_engine *e, cudaStream_t st = nullptr) {
     if (e->evfree.empty()) {
          cudaEvent_t a, b;
          if (cudaEventCreate(&a) != cudaSuccess) return (size_t)-1;
          if (cudaEventCreate(&b) != cudaSuccess) {
               cudaEventDestroy(a);
               return (size_t)-1;
          }
          e->evpool.push_back(a);
          e->evpool.push_back(b);
          e->evfree.push_back(e->evpool.size() - 2);
     }
     size_t i = e->evfree.back();
     e->evfree.pop_back();
     cudaEventRecord(e->evpool[i], st ? st : e->stream);
     return i;
}

static void timing_end(tdf_engine *e, size_t i, int kind, int64_t templates, cudaStream_t st = nullptr) {
     if (i == (size_t)-1) return;
     cudaEventRecord(e->evpool[i + 1], st ? st : e->stream);
     e->pending.push_back({kind, i, templates});
}

// folds the completed pairs (in recording order) into kt
static void timing_collect(tdf_engine *e) {
     size_t k = 0;
     for (; k < e->pending.size(); k++) {
          const auto &p = e->pending[k];
          if (cudaEventQuery(e->evpool[p.ev + 1]) != cudaSuccess) break;
          float ms = 0.f;
          if (cudaEventElapsedTime(&ms, e->evpool[p.ev], e->evpool[p.ev + 1]) == cudaSuccess) {
               switch (p.kind) {
               case KT_COL: e->kt.colpass_ms += ms; e->kt.colpass_launches++; e->kt.colpass_templates += p.templates; break;
               case KT_ROW: e->kt.rowpass_ms += ms; e->kt.rowpass_launches++; break;
               case KT_THR: e->kt.threshold_ms += ms; e->kt.threshold_launches++; break;
               case KT_SKY: e->kt.sky_ms += ms; e->kt.sky_batches++; break;
               }
          }
          e->evfree.push_back(p.ev);
     }
     cudaGetLastError();   // a not-ready query leaves no sticky error, clear it anyway
     e->pending.erase(e->pending.begin(), e->pending.begin() + k);
}

static size_t Wstride(const tdf_engine *e) { return (size_t)e->Ninterp; }

// ------------------------------------------------------------------ setup

static int validate(const tdf_segment *s, const tdf_search_opts *o) {
     if (!s || !o) return set_error(TDF_ERR_INVALID, "null segment or options");
     if (s->nifo < 1 || s->nifo > TDF_MAX_DETECTORS) return set_error(TDF_ERR_INVALID, "nifo=%d", s->nifo);
     if (s->N < 2) return set_error(TDF_ERR_INVALID, "N=%d", s->N);
     if (!pow2(s->nfft) || !pow2(s->nfftf) || !pow2(s->Ninterp))
          return set_error(TDF_ERR_INVALID, "nfft/nfftf/Ninterp must be powers of two");
     if (s->N > s->nfft || s->nfftf < s->nfft || s->Ninterp != s->interpftpad * s->nfft)
          return set_error(TDF_ERR_INVALID, "inconsistent sizes N=%d nfft=%d nfftf=%d Ninterp=%d", s->N, s->nfft,
                           s->nfftf, s->Ninterp);
     if (s->interpftpad * s->N > s->Ninterp) return set_error(TDF_ERR_INVALID, "interpftpad*N > Ninterp");
     if (s->nfft < 4096 || s->Ninterp > (1 << 20) || s->nfftf > (1 << 20))
          return set_error(TDF_ERR_UNSUPPORTED, "FFT lengths must lie in 2^12..2^20");
     if (o->fr[0] < 0 || o->fr[1] < o->fr[0] || o->fr[1] >= s->nfftf)
          return set_error(TDF_ERR_INVALID, "fr range [%d, %d] outside [0, nfftf)", o->fr[0], o->fr[1]);
     if (o->numlines < 0 || o->numlines > TDF_MAX_LINES || (o->numlines > 0 && !o->lines))
          return set_error(TDF_ERR_INVALID, "numlines=%d", o->numlines);
     if (!o->allsky && !(o->sstep > 0)) return set_error(TDF_ERR_INVALID, "sstep must be > 0");
     if (o->bufsize < 2) return set_error(TDF_ERR_INVALID, "bufsize=%d", o->bufsize);
     if (!s->cosmodf || !s->sinmodf) return set_error(TDF_ERR_INVALID, "null aux arrays");
     for (int d = 0; d < s->nifo; d++)
          if (!s->det[d].xdat || !s->det[d].detssb || !(s->det[d].sig2 > 0))
               return set_error(TDF_ERR_INVALID, "detector %d: null input or sig2 <= 0", d);
     return TDF_OK;
}

static int upload_inputs(tdf_engine *e, const tdf_segment *s) {
     const int N = e->N, nifo = e->nifo;
     for (int d = 0; d < nifo; d++) {
          CUCHK(cudaMemcpyAsync(e->S().xdat.as<float>() + (size_t)d * e->Nal, s->det[d].xdat, N * sizeof(float),
                                cudaMemcpyHostToDevice, e->stream));
          CUCHK(cudaMemcpyAsync(e->S().detssb.as<double>() + (size_t)d * 3 * N, s->det[d].detssb, 3 * (size_t)N * sizeof(double),
                                cudaMemcpyHostToDevice, e->stream));
          DetParam &D = e->S().dets[d];
          for (int k = 0; k < 9; k++) D.amod[k] = s->det[d].amod[k];
          D.cphir = s->det[d].cphir;
          D.sphir = s->det[d].sphir;
          D.sig2 = s->det[d].sig2;
     }
     CUCHK(cudaMemcpyAsync(e->S().cosm.p, s->cosmodf, N * sizeof(double), cudaMemcpyHostToDevice, e->stream));
     CUCHK(cudaMemcpyAsync(e->S().sinm.p, s->sinmodf, N * sizeof(double), cudaMemcpyHostToDevice, e->stream));
     CUCHK(cudaMemcpyAsync(e->S().detp.p, e->S().dets.data(), nifo * sizeof(DetParam), cudaMemcpyHostToDevice, e->stream));
     e->S().seg = *s;
     return TDF_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); null when the driver does not provide it
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
     static std::once_flag once;
     static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
     std::call_once(once, [] {
          void *p = nullptr;
          cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
          if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
              q == cudaDriverEntryPointSuccess)
               fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
     });
     return fn;
}

template <int L>
static void col_geometry(size_t *smem, int *blocks) {
     *smem = pass_smem_bytes<float, L, 2>();
     *blocks = pass_min_blocks<float, L>();
}

// Sizes the TMA ring of the split-form column pass (DemodSplitStaged) and
// encodes the operand tensor maps of both batch slots.  The ring takes as
// many row groups as fit in the shared memory a CTA may use at the pass's
// occupancy (228 KB per SM, 1 KB reserved per CTA).  Used with
// TDF_STAGED_OPERANDS=1; by default the column pass loads its operands per
// thread (DemodSplit), which measured as fast with the operands L2-resident.
static int staged_setup(tdf_engine *e) {
     e->staged = false;
     if (e->form != TDF_FORM_SPLIT) return TDF_OK;
     const char *env = getenv("TDF_STAGED_OPERANDS");
     if (!env || env[0] != '1') return TDF_OK;
     const int L = e->t_f32.N1, N2 = e->t_f32.N2, R = L / 8, nifo = e->nifo;
     if (e->Nal % N2 != 0) return TDF_OK;
     size_t pass_smem = 0;
     int blocks = 1;
     switch (L) {
     case 64: col_geometry<64>(&pass_smem, &blocks); break;
     case 128: col_geometry<128>(&pass_smem, &blocks); break;
     case 256: col_geometry<256>(&pass_smem, &blocks); break;
     case 512: col_geometry<512>(&pass_smem, &blocks); break;
     case 1024: col_geometry<1024>(&pass_smem, &blocks); break;
     default: return TDF_OK;
     }
     const size_t tw = (size_t)L * sizeof(float2);
     const size_t lines = pass_smem - tw;
     const size_t slot = (size_t)nifo * R * LINES * (sizeof(float4) + sizeof(float));
     const size_t bars = 8 * sizeof(uint64_t);
     const int rows = (e->N + N2 - 1) / N2;
     const int groups = std::min(8, (rows + R - 1) / R);
     // less the epilogue's twiddle tables (StoreFourstep), which follow the ring
     const size_t tables = sizeof(float2) * ((size_t)L * N2 / 1024 + 1024) + 16;
     const size_t budget = std::min<size_t>(227 * 1024, 233472 / blocks - 1024) - tables;
     if (budget < tw + bars + slot) return TDF_OK;
     const int stages = (int)std::min<size_t>((size_t)groups, (budget - tw - bars) / slot);
     const size_t area = std::max(lines, (size_t)stages * slot);
     PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
     if (!encode) return TDF_OK;
     for (int k = 0; k < 2; k++) {
          // interleaved operands: sample i, detector d at word (slot*Nal + i)*nifo + d
          const cuuint64_t rowsx = (cuuint64_t)(e->Nal / N2);
          const cuuint64_t dx[3] = {(cuuint64_t)4 * nifo * N2, rowsx, (cuuint64_t)e->Bs};
          const cuuint64_t sx[2] = {(cuuint64_t)nifo * N2 * 16, (cuuint64_t)e->Nal * nifo * 16};
          const cuuint32_t bx[3] = {(cuuint32_t)(4 * nifo * LINES), (cuuint32_t)R, 1};
          const cuuint64_t ds[3] = {(cuuint64_t)nifo * N2, rowsx, (cuuint64_t)e->Bs};
          const cuuint64_t ss[2] = {(cuuint64_t)nifo * N2 * 4, (cuuint64_t)e->Nal * nifo * 4};
          const cuuint32_t bs[3] = {(cuuint32_t)(nifo * LINES), (cuuint32_t)R, 1};
          const cuuint32_t one[3] = {1, 1, 1};
          CUresult r = encode(&e->tm_x[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, e->xab[k].p, dx, sx, bx, one,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
          if (r != CUDA_SUCCESS) return set_error(TDF_ERR_CUDA, "cuTensorMapEncodeTiled (operands xab): %d", (int)r);
          r = encode(&e->tm_s[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, e->s2[k].p, ds, ss, bs, one,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
          if (r != CUDA_SUCCESS) return set_error(TDF_ERR_CUDA, "cuTensorMapEncodeTiled (operands s2): %d", (int)r);
     }
     e->stg_groups = groups;
     e->stg_stages = stages;
     e->stg_bar_off = (unsigned)(tw + area);
     e->stg_smem = (unsigned)(tw + area + bars);
     e->staged = true;
     return TDF_OK;
}

// device inputs of one resident segment (xDat rows padded to Nal with zeros)
static int seg_alloc(const tdf_engine *e, SegData &d) {
     const int nifo = e->nifo;
     d.dets.resize(nifo);
     TRY(d.xdat.alloc((size_t)nifo * e->Nal * sizeof(float)));
     CUCHK(cudaMemset(d.xdat.p, 0, d.xdat.bytes));
     TRY(d.detssb.alloc((size_t)nifo * 3 * e->N * sizeof(double)));
     TRY(d.cosm.alloc(e->N * sizeof(double)));
     TRY(d.sinm.alloc(e->N * sizeof(double)));
     TRY(d.detp.alloc(nifo * sizeof(DetParam)));
     return TDF_OK;
}

static int engine_alloc(tdf_engine *e) {
     const int nifo = e->nifo, Bs = e->Bs, Tc = e->TcMax;
     const size_t Q = (size_t)Bs * nifo;
     TRY(seg_alloc(e, e->sdv[0]));
     // spline recurrence factors (auxi.c:102-108): invp[i] = 2/(g[i-1]+4), g[i] = -0.5 invp[i]
     {
          const int n = e->n2N;
          std::vector<double> p(n, 0.), g(n, 0.);
          for (int i = 1; i < n - 1; i++) {
               p[i] = 2. / (g[i - 1] + 4.);
               g[i] = -.5 * p[i];
          }
          TRY(e->pco.alloc(n * sizeof(double)));
          TRY(e->gco.alloc(n * sizeof(double)));
          CUCHK(cudaMemcpy(e->pco.p, p.data(), n * sizeof(double), cudaMemcpyHostToDevice));
          CUCHK(cudaMemcpy(e->gco.p, g.data(), n * sizeof(double), cudaMemcpyHostToDevice));
     }
     for (int k = 0; k < 2; k++) TRY(e->skyp[k].alloc(Bs * sizeof(SkyParam)));
     const size_t ws = Wstride(e);
     TRY(e->B0.alloc(Q * 2 * ws * sizeof(double2)));
     TRY(e->B1.alloc(Q * 2 * ws * sizeof(double2)));
     TRY(e->B2.alloc(Q * 2 * ws * sizeof(double2)));
     TRY(e->shftf.alloc(Q * e->Nal * sizeof(double)));
     TRY(e->partial.alloc(Q * (e->nfft / 256) * 2 * sizeof(double)));
     for (int k = 0; k < 2; k++) TRY(e->aabb[k].alloc(Bs * sizeof(AaBb)));
     const size_t ops = Q * e->Nal;
     if (e->form == TDF_FORM_SPLIT) {
          for (int k = 0; k < 2; k++) {
               TRY(e->xab[k].alloc(ops * sizeof(float4)));
               TRY(e->s2[k].alloc(ops * sizeof(float)));
          }
     } else {
          for (int k = 0; k < 2; k++) {
               TRY(e->xa64[k].alloc(ops * sizeof(double2)));
               TRY(e->xb64[k].alloc(ops * sizeof(double2)));
               TRY(e->t1[k].alloc(ops * sizeof(double)));
          }
     }
     const size_t csz = e->form == TDF_FORM_SPLIT ? sizeof(float2) : sizeof(double2);
     const size_t rsz = e->form == TDF_FORM_SPLIT ? sizeof(float) : sizeof(double);
     const size_t G = (size_t)std::max(tdf_engine::kGtMax, Tc);   // templates per resolve group at most
     e->cand_cap = (unsigned)G * 4096u;
     for (int l = 0; l < e->lanes_alloc; l++) {   // every lane the autotuner may use
          tdf_engine::Lane &L = e->ln[l];
          TRY(L.Ybuf.alloc((size_t)Tc * 2 * e->nfftf * csz));
          TRY(L.Fbuf.alloc(G * e->nF * rsz));
          TRY(L.mubuf.alloc(G * std::max(1, e->nblk_mu) * rsz));
          TRY(L.tcnt.alloc((G + 1) * sizeof(unsigned)));
          CUCHK(cudaMemset(L.tcnt.p, 0, L.tcnt.bytes));
          TRY(L.cand.alloc(e->cand_cap * sizeof(uint4)));
          // edge ring: 2 floats per (template, row CTA, k2) = nfftf bytes per template
          if (e->form == TDF_FORM_SPLIT) TRY(L.Ebuf.alloc(G * (size_t)e->nfftf));
          TRY(L.ctl.alloc((2 + (size_t)Tc) * sizeof(unsigned)));
          CUCHK(cudaMemset(L.ctl.p, 0, L.ctl.bytes));
     }
     TRY(e->linesd.alloc(std::max<size_t>(1, e->lines.size()) * sizeof(double)));
     if (!e->lines.empty())
          CUCHK(cudaMemcpy(e->linesd.p, e->lines.data(), e->lines.size() * sizeof(double), cudaMemcpyHostToDevice));
     e->trig_cap = 1ull << 21;
     for (int s = 0; s < 2; s++) {
          TRY(e->counters[s].alloc(2 * sizeof(unsigned long long)));
          CUCHK(cudaMemset(e->counters[s].p, 0, 2 * sizeof(unsigned long long)));
          TRY(e->trig[s].alloc(e->trig_cap * sizeof(Trig)));
          CUCHK(cudaMallocHost((void **)&e->h_sky[s], Bs * sizeof(SkyParam)));
          CUCHK(cudaEventCreateWithFlags(&e->done[s], cudaEventDisableTiming));
     }
     CUCHK(cudaMallocHost((void **)&e->h_cnt, 4 * sizeof(unsigned long long)));
     TRY(e->t_nfft.build(e->nfft));
     TRY(e->t_ninterp.build(e->Ninterp));
     if (e->form == TDF_FORM_SPLIT) {
          TRY(e->t_f32.build(e->nfftf));
          TRY(e->t_f32.build_base());
     }
     else TRY(e->t_f64.build(e->nfftf));
     TRY(staged_setup(e));
     return TDF_OK;
}

static void graphs_clear(tdf_engine *e) {
     for (auto &g : e->graphs)
          if (g.exec) cudaGraphExecDestroy(g.exec);
     e->graphs.clear();
     for (auto &g : e->plan_graphs)
          if (g.exec) cudaGraphExecDestroy(g.exec);
     e->plan_graphs.clear();
}

static void engine_free(tdf_engine *e) {
     graphs_clear(e);
     for (SegData &d : e->sdv) d.release();
     DevBuf *bufs[] = {&e->pco, &e->gco, &e->plan_sky, &e->plan_tp, &e->plan_pts, &e->skyp[0],
                       &e->skyp[1], &e->B0, &e->B1, &e->B2, &e->shftf, &e->partial, &e->aabb[0], &e->aabb[1],
                       &e->xab[0], &e->xab[1], &e->s2[0], &e->s2[1], &e->xa64[0], &e->xa64[1], &e->xb64[0],
                       &e->xb64[1], &e->t1[0], &e->t1[1], &e->tparam, &e->trig[0], &e->trig[1],
                       &e->counters[0], &e->counters[1], &e->linesd};
     for (DevBuf *b : bufs) b->release();
     for (tdf_engine::Lane &L : e->ln) {
          L.Ybuf.release();
          L.Fbuf.release();
          L.mubuf.release();
          L.tcnt.release();
          L.cand.release();
          L.Ebuf.release();
     }
     e->t_nfft.release();
     e->t_ninterp.release();
     e->t_f32.release();
     e->t_f64.release();
     for (int s = 0; s < 2; s++) {
          if (e->h_sky[s]) cudaFreeHost(e->h_sky[s]);
          if (e->h_tp[s]) cudaFreeHost(e->h_tp[s]);
          if (e->done[s]) cudaEventDestroy(e->done[s]);
          e->h_sky[s] = nullptr;
          e->h_tp[s] = nullptr;
          e->done[s] = nullptr;
     }
     if (e->h_cnt) cudaFreeHost(e->h_cnt);
     e->h_cnt = nullptr;
     for (cudaEvent_t ev : e->evpool) cudaEventDestroy(ev);
     e->evpool.clear();
     e->evfree.clear();
     e->pending.clear();
     for (int k = 0; k < 2; k++) {
          if (e->sky_done[k]) cudaEventDestroy(e->sky_done[k]);
          if (e->spin_done[k]) cudaEventDestroy(e->spin_done[k]);
          e->sky_done[k] = e->spin_done[k] = nullptr;
     }
     if (e->fork_ev) cudaEventDestroy(e->fork_ev);
     e->fork_ev = nullptr;
     if (e->plan_ev) cudaEventDestroy(e->plan_ev);
     e->plan_ev = nullptr;
     for (int l = 0; l < tdf_engine::kMaxLanes; l++) {
          if (e->join_ev[l]) cudaEventDestroy(e->join_ev[l]);
          if (e->lane_own[l]) cudaStreamDestroy(e->lane_own[l]);
          e->join_ev[l] = nullptr;
          e->lane_own[l] = nullptr;
     }
     if (e->sky_stream) cudaStreamDestroy(e->sky_stream);
     e->sky_stream = nullptr;
     if (e->own) cudaStreamDestroy(e->own);
     e->own = nullptr;
}

// ------------------------------------------------------------------ host-side per-point math

// jobcore.c:243-262 (sky geometry) and 399-430 (spindown range), with the
// reference's float/double types; `flt` selects FLOAT_TYPE = float.
static void point_setup(const tdf_engine *e, int pm, float mm, float nn, float sst, HostPoint &P) {
     const double *M = e->S().seg.M;
     double al1 = nn * M[10] + mm * M[14];
     double al2 = nn * M[11] + mm * M[15];
     double cof = e->S().seg.oms;
     P.inside = !(((al1 * al1) + (al2 * al2)) / (cof * cof) > 1.);
     if (!P.inside) return;
     double be1 = al1 / cof, be2 = al2 / cof;
     double sindel = be1 * e->S().seg.sepsm - (2 * pm - 3) * std::sqrt(1. - be1 * be1 - be2 * be2) * e->S().seg.cepsm;
     double cosdel = std::sqrt(1. - sindel * sindel);
     double sinal = (be1 - e->S().seg.sepsm * sindel) / (e->S().seg.cepsm * cosdel);
     double cosal = be2 / cosdel;
     SkyParam &S = P.sp;
     S.sinalt = sinal;
     S.cosalt = cosal;
     S.sindelt = sindel;
     S.cosdelt = cosdel;
     S.het0 = std::fmod(nn * M[8] + mm * M[12], M[0]);
     S.nS0 = cosal * cosdel;
     S.nS1 = sinal * cosdel;
     S.nS2 = sindel;
     // sgnlt[2..3] (FLOAT_TYPE) then the float record fields: one rounding
     P.dec = (float)std::asin(sindel);
     P.ra = (float)std::fmod(std::atan2(sinal, cosal) + 2. * M_PI, 2. * M_PI);
     float smin = sst, smax = e->opts.spndr[1];
     if (e->opts.allsky) {
          smin = std::trunc((e->S().seg.Smin - nn * M[9] - mm * M[13]) / M[5]);
          smax = std::trunc(-(nn * M[9] + mm * M[13] + e->S().seg.Smax) / M[5]);
          if (smin > smax) {
               smin = smin + smax;
               smax = smin - smax;
               smin = smin - smax;
          }
     }
     float sstep = e->opts.sstep;
     if (e->opts.allsky && !(sstep > 0)) sstep = 1.f;
     P.smin = smin;
     int iss = (int)((smax - smin) / sstep + 1);
     P.iss_size = iss > 0 ? iss : 0;
}

static void tmpl_setup(const tdf_engine *e, const HostPoint &P, float mm, float nn, float ss, HostTmpl &T) {
     const double *M = e->S().seg.M;
     T.ss = ss;
     T.spnd = ss * M[5] + nn * M[9] + mm * M[13];
     double het1 = std::fmod(ss * M[4], M[0]);
     if (het1 < 0) het1 += M[0];
     T.het1 = het1;
     if (e->form == TDF_FORM_SPLIT) {
          // FLOAT build: het1 and sgnl0 are float (jobcore.c:458-468)
          float h1 = (float)std::fmod(ss * M[4], M[0]);
          if (h1 < 0) h1 += M[0];
          float s0 = P.sp.het0 + h1;
          T.sgnl0 = (double)s0;
     } else {
          T.sgnl0 = P.sp.het0 + het1;
     }
}

// fdot of the record (jobcore.c:439,447): sgnlt[1] is FLOAT_TYPE
static float rec_fdot(const tdf_engine *e, double spnd) {
     if (e->form == TDF_FORM_SPLIT) return (float)((double)(float)spnd / (M_PI * e->S().seg.dt * e->S().seg.dt));
     return (float)(spnd / (M_PI * e->S().seg.dt * e->S().seg.dt));
}

// ------------------------------------------------------------------ device pipeline

// The stream of the sky stage: its own one when it overlaps the spindown
// stage, the engine stream otherwise and while kernels are being timed (the
// per-kernel event times are then those of kernels running alone).
// A caller's stream of the lowest priority would compete with the sky
// stream on equal terms, which measured slower than running the sky stage
// in line, so the overlap then stays off.
static cudaStream_t sky_stream_of(const tdf_engine *e) {
     return e->overlap && !e->timing && e->stream_outranks_sky ? e->sky_stream : e->stream;
}

// Sky stage of npts points into batch slot e->cur, on the sky stream: it
// first waits until the slot's previous spindown work released the slot's
// operands, and records sky_done[slot] for the spindown work to wait on.
// dsky: the points' sky parameters already on the device (else the slot's
// pinned staging is copied); wait_on: the event the sky stream waits for
// before it overwrites the slot (default: the slot's previous spindown work).
static int run_sky_stage(tdf_engine *e, int npts, const SkyParam *dsky = nullptr, cudaEvent_t wait_on = nullptr) {
     e->signal_valid = false;   // B0 is the sky stage's work buffer
     cudaStream_t st = sky_stream_of(e);
     CUCHK(cudaStreamWaitEvent(st, wait_on ? wait_on : e->spin_done[e->cur], 0));
     const int nifo = e->nifo, Q = npts * nifo;
     const size_t ws = Wstride(e);
     const int sl = e->cur;
     if (!dsky) {
          CUCHK(cudaMemcpyAsync(e->skyp[sl].p, e->h_sky[sl], npts * sizeof(SkyParam), cudaMemcpyHostToDevice, st));
          dsky = e->skyp[sl].as<SkyParam>();
     }
     const int nblk = e->nfft / 256;
     const bool split = e->form == TDF_FORM_SPLIT;
     k_sky_prep<<<dim3(nblk, Q), 256, 0, st>>>(
          e->S().xdat.as<float>(), e->S().detssb.as<double>(), e->S().cosm.as<double>(), e->S().sinm.as<double>(),
          dsky, e->S().detp.as<DetParam>(), nifo, e->N, e->nfft, e->Nal, e->S().seg.oms,
          e->B0.as<double2>(), ws, e->shftf.as<double>(), split ? e->s2[sl].as<float>() : nullptr,
          split ? nullptr : e->t1[sl].as<double>(), e->partial.as<double>());
     CUCHK(cudaGetLastError());
     k_sky_sums<<<npts, 256, 0, st>>>(e->partial.as<double>(), nblk, e->S().detp.as<DetParam>(), nifo,
                                       e->aabb[sl].as<AaBb>());
     CUCHK(cudaGetLastError());
     e->launches += 2;
     // forward FFT (nfft) of every (point, detector, a|b): B0 -> B1 -> B2
     {
          const FFTTables<double> &t = e->t_nfft;
          LoadNatural<double> pro{e->B0.as<double2>(), t.N2, (int)ws};
          StoreFourstep<double, -1, 1> epi{e->B1.as<double2>(), t.h(), t.o(), t.N2, (int)ws};
          TRY((launch_col<double, -1, 1>(t.N1, dim3(t.N2 / LINES, 2 * Q), pro, epi, t.l1(), st)));
          RowsY<double, 1> src{e->B1.as<double2>(), (int)ws, t.N2};
          StoreNatural<double> epi2{e->B2.as<double2>(), t.N1, (int)ws, e->nfft, 1.0};
          TRY((launch_row<double, -1, 1>(t.N2, dim3(t.N1 / LINES, 2 * Q), src, epi2, t.l2(), st)));
     }
     // inverse FFT (Ninterp) of the spread spectrum, scaled by interpftpad/Ninterp:
     // B2 -> B1 -> B0 (first interpftpad*N samples kept)
     {
          const FFTTables<double> &t = e->t_ninterp;
          LoadShuffled<double> pro{e->B2.as<double2>(), t.N2, (int)ws, e->nfft, e->Ninterp};
          StoreFourstep<double, +1, 1> epi{e->B1.as<double2>(), t.h(), t.o(), t.N2, (int)ws};
          TRY((launch_col<double, +1, 1>(t.N1, dim3(t.N2 / LINES, 2 * Q), pro, epi, t.l1(), st)));
          RowsY<double, 1> src{e->B1.as<double2>(), (int)ws, t.N2};
          const double ft = (double)e->S().seg.interpftpad / e->Ninterp;
          StoreNatural<double> epi2{e->B0.as<double2>(), t.N1, (int)ws, e->n2N, ft};
          TRY((launch_row<double, +1, 1>(t.N2, dim3(t.N1 / LINES, 2 * Q), src, epi2, t.l2(), st)));
     }
     e->launches += 4;
     // spline: B0 (samples) -> B1 (u) -> B2 (second derivatives)
     {
          dim3 g((e->n2N + SPL_TILE - 1) / SPL_TILE, 2 * Q);
          k_spline_fwd<<<g, SPL_T, 0, st>>>(e->B0.as<double2>(), e->B1.as<double2>(), ws, e->pco.as<double>(), e->n2N);
          CUCHK(cudaGetLastError());
          k_spline_bwd<<<g, SPL_T, 0, st>>>(e->B1.as<double2>(), e->B2.as<double2>(), ws, e->gco.as<double>(), e->n2N);
          CUCHK(cudaGetLastError());
     }
     k_splint<<<dim3((e->N + 255) / 256, Q), 256, 0, st>>>(
          e->B0.as<double2>(), e->B2.as<double2>(), ws, e->shftf.as<double>(), e->Nal, e->N, e->n2N,
          e->S().seg.interpftpad, e->S().detp.as<DetParam>(), nifo, split ? e->xab[sl].as<float4>() : nullptr,
          split ? nullptr : e->xa64[sl].as<double2>(), split ? nullptr : e->xb64[sl].as<double2>());
     CUCHK(cudaGetLastError());
     e->launches += 3;
     CUCHK(cudaEventRecord(e->sky_done[sl], st));
     return TDF_OK;
}

// Spindown stage, FFT part, for chunk `ci` of a resolve group whose templates
// start at dtp: the column pass (demodulation + first FFT pass) and the row
// pass (second FFT pass + F + candidate bins) for nt templates.
static cudaStream_t lane_stream(const tdf_engine *e, int l) { return l == 0 ? e->stream : e->lane_own[l]; }

// templates whose F spectra share one trigger-selection launch: whole chunks,
// at most Gt templates (one chunk when a chunk is larger)
static int group_templates(const tdf_engine *e) { return std::max(1, e->Gt / e->Tc) * e->Tc; }

// Split-form spindown passes with the four-step geometry fixed at compile
// time for the transform lengths of the benchmark sizes (nfftf 2^15 .. 2^18,
// two detectors); every other case takes the same policies with the
// geometry read at run time.
template <int L, int N2C>
static int launch_split_col_c(dim3 grid, const DemodSplitIL &p, const StoreFourstepG<0> &g, const float2 *tw,
                              cudaStream_t st) {
     DemodSplitILT<N2C, 2> pro{p.xab, p.s2, p.tp, p.N, p.N2, p.Nal, p.nifo};
     StoreFourstepG<N2C> epi{g.y, g.w0, g.ws, g.N2, g.N};
     return launch_col_L<float, L, -1, 2>(grid, pro, epi, tw, st);
}

static int launch_split_col(int nifo, int N1, int N2, dim3 grid, const DemodSplitIL &pro, const StoreFourstepG<0> &epi,
                            const float2 *tw, cudaStream_t st) {
     if (nifo == 2) {
          if (N1 == 512 && N2 == 512) return launch_split_col_c<512, 512>(grid, pro, epi, tw, st);
          if (N1 == 512 && N2 == 256) return launch_split_col_c<512, 256>(grid, pro, epi, tw, st);
          if (N1 == 256 && N2 == 256) return launch_split_col_c<256, 256>(grid, pro, epi, tw, st);
          if (N1 == 256 && N2 == 128) return launch_split_col_c<256, 128>(grid, pro, epi, tw, st);
     }
     return launch_col<float, -1, 2>(N1, grid, pro, epi, tw, st);
}

template <int L, int N1C, bool HALF>
static int launch_split_row_c(dim3 grid, const RowsYBulk<float> &src, const StoreFstatT<0, false> &f,
                              const float2 *tw, cudaStream_t st) {
     StoreFstatT<N1C, HALF> epi{f.F, f.tp, f.ab, f.nF, f.fr0, f.fr1, f.N1, f.thr, f.cand, f.cand_cnt, f.cand_cap, f.boff,
                                f.E, f.scand};
     return launch_row_L<float, L, -1, 2>(grid, src, epi, tw, st);
}

template <int L, int N1C>
static int launch_split_row_h(bool half, dim3 grid, const RowsYBulk<float> &src, const StoreFstatT<0, false> &f,
                              const float2 *tw, cudaStream_t st) {
     return half ? launch_split_row_c<L, N1C, true>(grid, src, f, tw, st)
                 : launch_split_row_c<L, N1C, false>(grid, src, f, tw, st);
}

// the row pass keeps only bins <= fr1; with fr1 < nfftf/2 = N1*N2/2 every
// kept output has k2 < N2/2
static int launch_split_row(int N1, int N2, int fr1, dim3 grid, const RowsYBulk<float> &src,
                            const StoreFstatT<0, false> &epi, const float2 *tw, cudaStream_t st) {
     const bool half = (int64_t)fr1 < (int64_t)N1 * N2 / 2;
     if (N2 == 512 && N1 == 512) return launch_split_row_h<512, 512>(half, grid, src, epi, tw, st);
     if (N2 == 256 && N1 == 512) return launch_split_row_h<256, 512>(half, grid, src, epi, tw, st);
     if (N2 == 256 && N1 == 256) return launch_split_row_h<256, 256>(half, grid, src, epi, tw, st);
     if (N2 == 128 && N1 == 256) return launch_split_row_h<128, 256>(half, grid, src, epi, tw, st);
     return launch_row<float, -1, 2>(N2, grid, src, epi, tw, st);
}

// The two split-form passes of nt templates as one ordered launch of
// persistent CTAs (k_spinpass), for N1 = N2 = L (nfftf 2^16, 2^18) and two
// detectors; ctl (2 + nt words) is zeroed first, on the same stream.
template <int L, bool HALF>
static int launch_spin_c(int nt, int lag, const DemodSplitIL &p, const StoreFourstepG<0> &g, const RowsYBulk<float> &s,
                         const StoreFstatT<0, false> &f, const float2 *tw, unsigned *ctl, unsigned *err,
                         cudaStream_t st) {
     DemodSplitILT<L, 2> pro{p.xab, p.s2, p.tp, p.N, p.N2, p.Nal, p.nifo};
     StoreFourstepG<L> epic{g.y, g.w0, g.ws, g.N2, g.N};
     StoreFstatT<L, HALF> epir{f.F, f.tp, f.ab, f.nF, f.fr0, f.fr1, f.N1, f.thr, f.cand, f.cand_cnt, f.cand_cap, f.boff,
                               f.E, f.scand};
     RowsYBulk<float> src = s;
     size_t smem = pass_smem_bytes<float, L, 2>();
     smem = (smem + 15) / 16 * 16;
     src.bar_off = (unsigned)smem;
     smem += 16;
     SpinOrder o{ctl, err, nt, L / LINES, L / LINES, std::max(1, std::min(lag, nt)), 1 << 20};
     auto kern = k_spinpass<L, DemodSplitILT<L, 2>, StoreFourstepG<L>, RowsYBulk<float>, StoreFstatT<L, HALF>>;
     TRY(set_smem(kern, smem));
     // as many CTAs as are resident at once (queried once per device and variant)
     static std::mutex mu;
     static int resident[64] = {};
     int dev = 0;
     CUCHK(cudaGetDevice(&dev));
     int nres;
     {
          std::lock_guard<std::mutex> lk(mu);
          if (dev < 64 && resident[dev] > 0) {
               nres = resident[dev];
          } else {
               int per_sm = 0, nsm = 0;
               CUCHK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, pass_threads<L>(), smem));
               CUCHK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
               nres = std::max(1, per_sm) * std::max(1, nsm);
               if (dev < 64) resident[dev] = nres;
          }
     }
     const unsigned items = (unsigned)nt * (unsigned)(o.C + o.R);
     CUCHK(cudaMemsetAsync(ctl, 0, (2 + (size_t)nt) * sizeof(unsigned), st));
     kern<<<std::min(items, (unsigned)nres), pass_threads<L>(), smem, st>>>(pro, epic, src, epir, tw, o);
     CUCHK(cudaGetLastError());
     return TDF_OK;
}

// whether the chunk passes of this engine run as one ordered launch
static bool spin_fused(const tdf_engine *e, int N1, int N2) {
     return e->fused && !e->staged && e->row_bulk && e->nifo == 2 && N1 == N2 && (N1 == 512 || N1 == 256);
}

template <typename T>
static int run_chunk(tdf_engine *e, int l, const TmplParam *dtp, int ci, int nt) {
     cudaStream_t st = lane_stream(e, l);
     tdf_engine::Lane &Ln = e->ln[l];
     const FFTTables<T> *tb;
     if constexpr (std::is_same<T, float>::value) tb = &e->t_f32;
     else tb = &e->t_f64;
     const FFTTables<T> &t = *tb;
     const int boff = ci * e->Tc;
     const TmplParam *ctp = dtp + boff;
     const unsigned G = (unsigned)group_templates(e);
     unsigned *tcnt = Ln.tcnt.as<unsigned>();
     size_t tev = e->timing ? timing_begin(e, st) : (size_t)-1;
     if constexpr (std::is_same<T, float>::value) {
          if (spin_fused(e, t.N1, t.N2)) {
               StoreFourstepG<0> epi{Ln.Ybuf.as<float2>(), t.base.template as<float2>(), t.step.template as<float2>(),
                                     t.N2, e->nfftf};
               DemodSplitIL pro{e->xab[e->cur].as<float4>(), e->s2[e->cur].as<float>(), ctp, e->N, t.N2, e->Nal,
                                e->nifo};
               unsigned *errw = reinterpret_cast<unsigned *>(e->counters[e->cur].as<unsigned long long>() + 1);
               const bool blocks = e->opts.blocks_avg && e->nblk_mu > 0;
               StoreFstatT<0, false> epi2{Ln.Fbuf.as<float>() + (size_t)boff * e->nF, ctp, e->aabb[e->cur].as<AaBb>(),
                                          e->nF, e->opts.fr[0], e->opts.fr[1], t.N1, e->opts.thr,
                                          blocks ? nullptr : Ln.cand.as<uint2>(), tcnt + G, e->cand_cap, boff};
               if (e->sparse_now) {
                    epi2.cand = nullptr;
                    epi2.E = Ln.Ebuf.as<float>();
                    epi2.scand = Ln.cand.as<uint4>();
               }
               RowsYBulk<float> src{Ln.Ybuf.as<float2>(), e->nfftf, t.N2, errw};
               const bool half = (int64_t)e->opts.fr[1] < (int64_t)t.N1 * t.N2 / 2;
               unsigned *ctl = Ln.ctl.as<unsigned>();
               const float2 *tw = t.l1();   // N1 = N2: the row pass's line table is the same
               int rc;
               if (t.N1 == 512)
                    rc = half ? launch_spin_c<512, true>(nt, e->fuse_lag, pro, epi, src, epi2, tw, ctl, errw, st)
                              : launch_spin_c<512, false>(nt, e->fuse_lag, pro, epi, src, epi2, tw, ctl, errw, st);
               else
                    rc = half ? launch_spin_c<256, true>(nt, e->fuse_lag, pro, epi, src, epi2, tw, ctl, errw, st)
                              : launch_spin_c<256, false>(nt, e->fuse_lag, pro, epi, src, epi2, tw, ctl, errw, st);
               TRY(rc);
               if (e->timing) timing_end(e, tev, KT_COL, nt, st);
               e->launches += 1;   // the memset before it is not a kernel
               return TDF_OK;
          }
          StoreFourstepG<0> epi{Ln.Ybuf.as<float2>(), t.base.template as<float2>(), t.step.template as<float2>(), t.N2,
                                e->nfftf};
          if (e->staged) {
               DemodSplitStaged pro;
               pro.mx = e->tm_x[e->cur];
               pro.ms = e->tm_s[e->cur];
               pro.tp = ctp;
               pro.err = reinterpret_cast<unsigned *>(e->counters[e->cur].as<unsigned long long>() + 1);
               pro.N = e->N;
               pro.N2 = t.N2;
               pro.nifo = e->nifo;
               pro.groups = e->stg_groups;
               pro.stages = e->stg_stages;
               pro.bar_off = e->stg_bar_off;
               pro.smem = e->stg_smem;
               TRY((launch_col<T, -1, 2>(t.N1, dim3(t.N2 / LINES, nt), pro, epi, t.l1(), st)));
          } else {
               DemodSplitIL pro{e->xab[e->cur].as<float4>(), e->s2[e->cur].as<float>(), ctp, e->N, t.N2, e->Nal,
                                e->nifo};
               TRY(launch_split_col(e->nifo, t.N1, t.N2, dim3(t.N2 / LINES, nt), pro, epi, t.l1(), st));
          }
     } else {
          StoreFourstep<T, -1, 2> epi{Ln.Ybuf.as<cx<T>>(), t.h(), t.o(), t.N2, e->nfftf};
          DemodFP64 pro{e->xa64[e->cur].as<double2>(), e->xb64[e->cur].as<double2>(), e->t1[e->cur].as<double>(), ctp,
                        e->N, t.N2, e->Nal, e->nifo};
          TRY((launch_col<T, -1, 2>(t.N1, dim3(t.N2 / LINES, nt), pro, epi, t.l1(), st)));
     }
     if (e->timing) timing_end(e, tev, KT_COL, nt, st);
     const bool blocks = e->opts.blocks_avg && e->nblk_mu > 0;
     tev = e->timing ? timing_begin(e, st) : (size_t)-1;
     unsigned *errw = reinterpret_cast<unsigned *>(e->counters[e->cur].as<unsigned long long>() + 1);
     if constexpr (std::is_same<T, float>::value) {
          StoreFstatT<0, false> epi2{Ln.Fbuf.as<float>() + (size_t)boff * e->nF, ctp, e->aabb[e->cur].as<AaBb>(), e->nF,
                                     e->opts.fr[0], e->opts.fr[1], t.N1, e->opts.thr,
                                     blocks ? nullptr : Ln.cand.as<uint2>(), tcnt + G, e->cand_cap, boff};
          if (e->sparse_now) {
               epi2.cand = nullptr;
               epi2.E = Ln.Ebuf.as<float>();
               epi2.scand = Ln.cand.as<uint4>();
          }
          if (e->row_bulk) {
               RowsYBulk<float> src{Ln.Ybuf.as<float2>(), e->nfftf, t.N2, errw};
               TRY(launch_split_row(t.N1, t.N2, e->opts.fr[1], dim3(t.N1 / LINES, nt), src, epi2, t.l2(), st));
          } else {
               RowsY<float, 2> src{Ln.Ybuf.as<float2>(), e->nfftf, t.N2};
               TRY((launch_row<float, -1, 2>(t.N2, dim3(t.N1 / LINES, nt), src, epi2, t.l2(), st)));
          }
     } else {
          StoreFstat<T> epi2{Ln.Fbuf.as<T>() + (size_t)boff * e->nF, ctp, e->aabb[e->cur].as<AaBb>(), e->nF,
                             e->opts.fr[0], e->opts.fr[1], t.N1, e->opts.thr,
                             blocks ? nullptr : Ln.cand.as<uint2>(), tcnt + G, e->cand_cap, boff};
          if (e->row_bulk) {
               RowsYBulk<T> src{Ln.Ybuf.as<cx<T>>(), e->nfftf, t.N2, errw};
               TRY((launch_row<T, -1, 2>(t.N2, dim3(t.N1 / LINES, nt), src, epi2, t.l2(), st)));
          } else {
               RowsY<T, 2> src{Ln.Ybuf.as<cx<T>>(), e->nfftf, t.N2};
               TRY((launch_row<T, -1, 2>(t.N2, dim3(t.N1 / LINES, nt), src, epi2, t.l2(), st)));
          }
     }
     if (e->timing) timing_end(e, tev, KT_ROW, nt, st);
     e->launches += 2;
     return TDF_OK;
}

// Trigger selection for the ntg templates of a resolve group (starting at
// dtp; their F spectra fill the F ring in order): the candidate bins the row
// passes collected, or, with blocks_avg, block means and a scan of every bin.
template <typename T>
static int run_resolve(tdf_engine *e, int l, const TmplParam *dtp, int ntg) {
     cudaStream_t st = lane_stream(e, l);
     tdf_engine::Lane &Ln = e->ln[l];
     const bool split = std::is_same<T, float>::value;
     const unsigned G = (unsigned)group_templates(e);
     unsigned *tcnt = Ln.tcnt.as<unsigned>();
     const bool blocks = e->opts.blocks_avg && e->nblk_mu > 0;
     unsigned long long *cnt = e->counters[e->cur].as<unsigned long long>();
     ThrArgs A;
     A.nF = e->nF;
     A.fr0 = e->opts.fr[0];
     A.fr1 = e->opts.fr[1];
     A.thr = e->opts.thr;
     A.nblk = blocks ? e->nblk_mu : 0;
     A.tp = dtp;
     A.nfftf = e->nfftf;
     A.lines = e->linesd.as<double>();
     A.numlines = e->opts.numlines;
     A.bufhalf = (unsigned)(e->opts.bufsize / 2);
     A.trig = e->trig[e->cur].as<Trig>();
     A.cap = e->trig_cap;
     A.cnt = cnt;
     A.tcnt = tcnt;
     A.err = reinterpret_cast<unsigned *>(cnt + 1);
     size_t tev = e->timing ? timing_begin(e, st) : (size_t)-1;
     if (blocks) {
          k_block_means<T><<<dim3(e->nblk_mu, ntg), 256, 0, st>>>(Ln.Fbuf.as<T>(), e->nF, e->nblk_mu, Ln.mubuf.as<T>());
          CUCHK(cudaGetLastError());
          dim3 g((e->nF + 255) / 256, ntg);
          if (split) k_threshold<T, false><<<g, 256, 0, st>>>(Ln.Fbuf.as<T>(), Ln.mubuf.as<T>(), A);
          else k_threshold<T, true><<<g, 256, 0, st>>>(Ln.Fbuf.as<T>(), Ln.mubuf.as<T>(), A);
          e->launches += 2;
     } else if (split && e->sparse_now) {
          SparseArgs S{Ln.Ebuf.as<float>(), Ln.cand.as<uint4>(), tcnt + G, e->cand_cap, e->t_f32.N1, e->t_f32.N2};
          k_resolve_sparse<<<64, 256, 0, st>>>(A, S);
          e->launches++;
     } else {
          if (split) k_resolve<T, false><<<64, 256, 0, st>>>(Ln.Fbuf.as<T>(), A, Ln.cand.as<uint2>(), tcnt + G, e->cand_cap, ntg);
          else k_resolve<T, true><<<64, 256, 0, st>>>(Ln.Fbuf.as<T>(), A, Ln.cand.as<uint2>(), tcnt + G, e->cand_cap, ntg);
          e->launches++;
     }
     CUCHK(cudaGetLastError());
     if (e->timing) timing_end(e, tev, KT_THR, ntg, st);
     // ready for the next group: trigger counters and candidate count
     CUCHK(cudaMemsetAsync(tcnt, 0, (G + 1) * sizeof(unsigned), st));
     return TDF_OK;
}

// The spindown stage of nt templates starting at dtp: resolve groups of
// chunks, group k on lane k % nlanes.  Lanes 1.. start after everything
// queued on the engine stream so far (sky stage, template upload) and the
// engine stream waits for them at the end, so callers see one ordered stream.
static int run_templates(tdf_engine *e, const TmplParam *dtp, int nt) {
     const int G = group_templates(e);
     const int ngroups = (nt + G - 1) / G;
     // per-kernel event timing measures kernels one after another: one lane
     const int lanes = e->timing ? 1 : std::min(e->nlanes, ngroups);
     if (lanes > 1) {
          CUCHK(cudaEventRecord(e->fork_ev, e->stream));
          for (int l = 1; l < lanes; l++) CUCHK(cudaStreamWaitEvent(e->lane_own[l], e->fork_ev, 0));
     }
     for (int gi = 0; gi < ngroups; gi++) {
          const int g0 = gi * G;
          const int l = gi % lanes;
          const int ntg = std::min(G, nt - g0);
          for (int ci = 0; ci * e->Tc < ntg; ci++) {
               const int n = std::min(e->Tc, ntg - ci * e->Tc);
               if (e->form == TDF_FORM_SPLIT) TRY(run_chunk<float>(e, l, dtp + g0, ci, n));
               else TRY(run_chunk<double>(e, l, dtp + g0, ci, n));
          }
          if (e->form == TDF_FORM_SPLIT) TRY(run_resolve<float>(e, l, dtp + g0, ntg));
          else TRY(run_resolve<double>(e, l, dtp + g0, ntg));
     }
     for (int l = 1; l < lanes; l++) {
          CUCHK(cudaEventRecord(e->join_ev[l], e->lane_own[l]));
          CUCHK(cudaStreamWaitEvent(e->stream, e->join_ev[l], 0));
     }
     return TDF_OK;
}

static int set_graph_priorities(const tdf_engine *e, cudaGraph_t g) {
     if (!e->overlap || !e->stream_outranks_sky || !e->graph_prio) return TDF_OK;
     {
          // the sky kernels launched with <<<>>> (the passes register themselves)
          static std::once_flag once;
          std::call_once(once, [] {
               register_sky_kernel((const void *)k_sky_prep);
               register_sky_kernel((const void *)k_sky_sums);
               register_sky_kernel((const void *)k_spline_fwd);
               register_sky_kernel((const void *)k_spline_bwd);
               register_sky_kernel((const void *)k_splint);
          });
     }
     size_t n = 0;
     CUCHK(cudaGraphGetNodes(g, nullptr, &n));
     std::vector<cudaGraphNode_t> nodes(n);
     CUCHK(cudaGraphGetNodes(g, nodes.data(), &n));
     for (cudaGraphNode_t nd : nodes) {
          cudaGraphNodeType ty;
          CUCHK(cudaGraphNodeGetType(nd, &ty));
          if (ty != cudaGraphNodeTypeKernel) continue;
          cudaKernelNodeParams kp;
          CUCHK(cudaGraphKernelNodeGetParams(nd, &kp));
          cudaKernelNodeAttrValue v;
          memset(&v, 0, sizeof(v));
          v.priority = is_sky_kernel(kp.func) ? e->prio_low : e->prio_high;
          CUCHK(cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributePriority, &v));
     }
     return TDF_OK;
}

// The spindown stage of the current batch (nt templates uploaded to tparam):
// the first time a configuration is seen its kernels are launched one by one;
// the second time they are captured (all lanes) into a graph, which later
// batches with the same configuration replay with one launch.
static int run_templates_batch(tdf_engine *e, int nt) {
     const TmplParam *dtp = e->tparam.as<TmplParam>();
     if (!e->use_graphs || e->timing) return run_templates(e, dtp, nt);
     const tdf_engine::GraphKey k{e->cur, nt, e->Tc, e->Gt, e->nlanes, e->sparse_now, e->tparam.p, e->trig[e->cur].p,
                                  e->trig_cap};
     size_t gi = e->graphs.size();
     for (size_t i = 0; i < e->graphs.size(); i++)
          if (e->graphs[i].key == k) gi = i;
     if (gi == e->graphs.size()) {
          if (e->graphs.size() >= tdf_engine::kMaxGraphs) {
               size_t old = 0;
               for (size_t i = 1; i < e->graphs.size(); i++)
                    if (e->graphs[i].last < e->graphs[old].last) old = i;
               if (e->graphs[old].exec) cudaGraphExecDestroy(e->graphs[old].exec);
               e->graphs.erase(e->graphs.begin() + old);
          }
          e->graphs.push_back(tdf_engine::GraphEntry());
          gi = e->graphs.size() - 1;
          e->graphs[gi].key = k;
     }
     tdf_engine::GraphEntry &g = e->graphs[gi];
     g.last = ++e->graph_tick;
     if (!g.exec && ++g.seen < 2) return run_templates(e, dtp, nt);
     if (!g.exec) {
          if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
               // e.g. the legacy default stream: no capture, plain launches from now on
               cudaGetLastError();
               e->use_graphs = false;
               return run_templates(e, dtp, nt);
          }
          const int64_t l0 = e->launches;
          const int st = run_templates(e, dtp, nt);
          cudaGraph_t graph = nullptr;
          const cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
          if (st != TDF_OK || ce != cudaSuccess) {
               if (graph) cudaGraphDestroy(graph);
               e->launches = l0;
               return st != TDF_OK ? st : set_error(TDF_ERR_CUDA, "stream capture: %s", cudaGetErrorString(ce));
          }
          const int ps = set_graph_priorities(e, graph);
          if (ps != TDF_OK) {
               cudaGraphDestroy(graph);
               e->launches = l0;
               return ps;
          }
          const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
          cudaGraphDestroy(graph);
          if (ie != cudaSuccess) {
               g.exec = nullptr;
               e->launches = l0;
               return set_error(TDF_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ie));
          }
          g.launches = e->launches - l0;
          e->launches = l0;
     }
     CUCHK(cudaGraphLaunch(g.exec, e->stream));
     e->launches += g.launches;
     return TDF_OK;
}

static int ensure_tparam(tdf_engine *e, size_t n) {
     if (n > e->h_tp_cap) {
          CUCHK(cudaStreamSynchronize(e->stream));
          size_t cap = std::max<size_t>(n, 4096);
          for (int s = 0; s < 2; s++) {
               if (e->h_tp[s]) cudaFreeHost(e->h_tp[s]);
               e->h_tp[s] = nullptr;
               CUCHK(cudaMallocHost((void **)&e->h_tp[s], cap * sizeof(TmplParam)));
          }
          e->h_tp_cap = cap;
          TRY(e->tparam.alloc(cap * sizeof(TmplParam)));
     }
     return TDF_OK;
}

// the error of a kernel error word whose bounded waits gave up, else TDF_OK
static int wait_error(unsigned errf) {
     if (errf & ERR_STAGE_TIMEOUT)
          return set_error(TDF_ERR_CUDA, "spindown stage: an asynchronous copy did not complete within its wait limit");
     if (errf & ERR_ORDER_TIMEOUT)
          return set_error(TDF_ERR_CUDA, "spindown stage: a row block's wait for its column blocks gave up");
     return TDF_OK;
}

// Waits for the batch last run in `slot`, checks its flags and collects its
// triggers; *over is set when the trigger buffer was too small.
static int finish_slot(tdf_engine *e, int slot, bool collect, int64_t *ntrig_total, bool *over, bool *need_full) {
     CUCHK(cudaEventSynchronize(e->done[slot]));
     if (e->timing) timing_collect(e);
     const unsigned long long nfound = e->h_cnt[2 * slot];
     const unsigned errf = (unsigned)(e->h_cnt[2 * slot + 1] & 0xffffffffu);
     if (errf & ERR_OVERFLOW)
          return set_error(TDF_ERR_TRIGGER_OVERFLOW, "Too many triggers! buffer_size=%d [triggers]", e->opts.bufsize / 2);
     TRY(wait_error(errf));
     if (errf & ERR_NEED_FULL_F) {
          *need_full = true;
          return TDF_OK;
     }
     if (nfound > e->trig_cap) {
          *over = true;
          e->h_cnt[2 * slot] = nfound;   // keep the needed size visible
          return TDF_OK;
     }
     *ntrig_total += (int64_t)nfound;
     if (collect && nfound) {
          size_t o = e->h_trig.size();
          e->h_trig.resize(o + nfound);
          // the batch is complete (event above); the engine stream may run on
          CUCHK(cudaMemcpy(e->h_trig.data() + o, e->trig[slot].p, nfound * sizeof(Trig), cudaMemcpyDeviceToHost));
     }
     CUCHK(cudaMemsetAsync(e->counters[slot].p, 0, 2 * sizeof(unsigned long long), e->stream));
     return TDF_OK;
}

// The whole search over npts points.  Fills host-side templates (and
// optionally collects triggers).  On return *ntrig_total holds the trigger
// count; triggers are appended to e->h_trig when `collect`.
static int search_core(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn, const float *sst,
                       std::vector<HostPoint> &pts, std::vector<HostTmpl> &tm, bool collect, int64_t *ntrig_total) {
     if (npts < 0) return set_error(TDF_ERR_INVALID, "npts < 0");
     if (npts > 0 && (!pm || !mm || !nn)) return set_error(TDF_ERR_INVALID, "null sky point arrays");
     pts.assign(npts, HostPoint());
     // the point geometry up front (cheap); the per-template scalars are made
     // batch by batch below, while the device runs the previous batch
     int64_t ntm = 0;
     for (int i = 0; i < npts; i++) {
          if (pm[i] != 1 && pm[i] != 2) return set_error(TDF_ERR_INVALID, "pm[%d]=%d (must be 1 or 2)", i, pm[i]);
          float s0 = sst ? sst[i] : e->opts.spndr[0];
          point_setup(e, pm[i], mm[i], nn[i], s0, pts[i]);
          if (!pts[i].inside) continue;
          pts[i].first_tmpl = (int)ntm;
          ntm += pts[i].iss_size;
     }
     if (ntm > (int64_t)UINT32_MAX) return set_error(TDF_ERR_UNSUPPORTED, "more than 2^32 templates in one call");
     tm.resize(ntm);
     // sky batches of consecutive inside points
     std::vector<int> inside;
     for (int i = 0; i < npts; i++)
          if (pts[i].inside && pts[i].iss_size > 0) inside.push_back(i);
     size_t maxnt = 0;
     for (size_t b0 = 0; b0 < inside.size(); b0 += e->Bs) {
          size_t nt = 0;
          for (size_t k = b0; k < std::min(inside.size(), b0 + e->Bs); k++) nt += pts[inside[k]].iss_size;
          maxnt = std::max(maxnt, nt);
     }
     TRY(ensure_tparam(e, maxnt));
     e->sparse_now = e->sparse_f && e->form == TDF_FORM_SPLIT && !(e->opts.blocks_avg && e->nblk_mu > 0);
     for (int grown = 0;;) {
          e->h_trig.clear();
          *ntrig_total = 0;
          CUCHK(cudaStreamSynchronize(e->sky_stream));
          CUCHK(cudaStreamSynchronize(e->stream));
          for (int s = 0; s < 2; s++) CUCHK(cudaMemsetAsync(e->counters[s].p, 0, 2 * sizeof(unsigned long long), e->stream));
          for (int l = 0; l < e->lanes_alloc; l++) CUCHK(cudaMemsetAsync(e->ln[l].tcnt.p, 0, e->ln[l].tcnt.bytes, e->stream));
          int pending[2] = {0, 0};
          bool over = false, need_full = false;
          size_t b = 0;
          for (size_t b0 = 0; b0 < inside.size(); b0 += e->Bs, b++) {
               const int slot = (int)(b & 1);
               // the slot's previous batch must be drained before its staging
               // and trigger buffer are reused; the other slot keeps running
               if (pending[slot]) {
                    TRY(finish_slot(e, slot, collect, ntrig_total, &over, &need_full));
                    pending[slot] = 0;
                    if (over || need_full) break;
               }
               e->cur = slot;
               const int nb = (int)std::min<size_t>(e->Bs, inside.size() - b0);
               int nt = 0;
               for (int k = 0; k < nb; k++) {
                    const HostPoint &P = pts[inside[b0 + k]];
                    e->h_sky[slot][k] = P.sp;
                    nt += P.iss_size;
               }
               int w = 0;
               for (int k = 0; k < nb; k++) {
                    const int ip = inside[b0 + k];
                    const HostPoint &P = pts[ip];
                    for (int s = 0; s < P.iss_size; s++) {
                         HostTmpl &T = tm[P.first_tmpl + s];
                         T.pt = ip;
                         tmpl_setup(e, P, mm[ip], nn[ip], P.smin + s * e->opts.sstep, T);
                         TmplParam &q = e->h_tp[slot][w++];
                         q.het1 = T.het1;
                         q.spnd = T.spnd;
                         q.sgnl0 = T.sgnl0;
                         q.slot = k;
                         q.id = (uint32_t)(P.first_tmpl + s);
                    }
               }
               cudaStream_t sst = sky_stream_of(e);
               size_t sev = e->timing ? timing_begin(e, sst) : (size_t)-1;
               TRY(run_sky_stage(e, nb));
               if (e->timing) timing_end(e, sev, KT_SKY, nb, sst);
               CUCHK(cudaStreamWaitEvent(e->stream, e->sky_done[slot], 0));
               CUCHK(cudaMemcpyAsync(e->tparam.p, e->h_tp[slot], nt * sizeof(TmplParam), cudaMemcpyHostToDevice, e->stream));
               TRY(run_templates_batch(e, nt));
               CUCHK(cudaEventRecord(e->spin_done[slot], e->stream));
               CUCHK(cudaMemcpyAsync(e->h_cnt + 2 * slot, e->counters[slot].p, 2 * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, e->stream));
               CUCHK(cudaEventRecord(e->done[slot], e->stream));
               pending[slot] = 1;
          }
          // drain in batch order: the slot of the second-to-last batch first
          for (int k = 0; k < 2 && !over && !need_full; k++) {
               const int slot = (int)((b + k) & 1);
               if (pending[slot]) {
                    TRY(finish_slot(e, slot, collect, ntrig_total, &over, &need_full));
                    pending[slot] = 0;
               }
          }
          CUCHK(cudaStreamSynchronize(e->stream));
          if (need_full) {
               // a MAX_ALG 3 tie or more candidates than the list holds: the
               // whole search again with the full F store
               if (!e->sparse_now) return set_error(TDF_ERR_CUDA, "trigger selection asked for the full F store twice");
               e->sparse_now = false;
               continue;
          }
          if (!over) break;
          if (++grown > 3) return set_error(TDF_ERR_CAPACITY, "trigger buffer could not be sized");
          // a batch found more triggers than the buffer holds: grow and rerun
          unsigned long long need = std::max(e->h_cnt[0], e->h_cnt[2]);
          e->trig_cap = std::max<unsigned long long>(need + (need >> 2), e->trig_cap * 2);
          for (int s = 0; s < 2; s++) {
               e->trig[s].release();
               TRY(e->trig[s].alloc(e->trig_cap * sizeof(Trig)));
          }
     }
     return TDF_OK;
}

// ------------------------------------------------------------------ autotuning
//
// The templates per chunk (Tc) set how many CTAs a column/row pass launches
// (32*Tc and 64*Tc for nfftf = 2^17) against the SM count, and how much of
// L2 the intermediate spectra take.  tdf_engine_autotune() times candidates
// on the caller's points; with TDF_AUTOTUNE_CACHE=<file> the choice is kept
// per (form, N, nfftf, nifo, SM count, sky batch) and reused by later
// engines.

static int sm_count(int dev) {
     int n = 0;
     if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
          cudaGetLastError();
          return 0;
     }
     return n;
}

// the cache key: form, sizes, GPU (SM count), sky batch and F store; the
// value: templates per chunk, lanes, templates per resolve group
static std::string autotune_key(const tdf_engine *e) {
     char k[256];
     snprintf(k, sizeof(k), "tune %d %d %d %d %d %d %d", e->form, e->N, e->nfftf, e->nifo, sm_count(e->dev), e->Bs,
              e->sparse_f ? 1 : 0);
     return k;
}

static void autotune_cache_lookup(tdf_engine *e) {
     const char *path = getenv("TDF_AUTOTUNE_CACHE");
     if (!path || !*path || getenv("TDF_TEMPLATES_PER_CHUNK")) return;
     FILE *f = fopen(path, "r");
     if (!f) return;
     const std::string key = autotune_key(e);
     char line[512];
     while (fgets(line, sizeof(line), f)) {
          if (strncmp(line, key.c_str(), key.size()) == 0 && line[key.size()] == ' ') {
               int tc = 0, lanes = 0, gt = 0;
               if (sscanf(line + key.size() + 1, "%d %d %d", &tc, &lanes, &gt) == 3 && tc > 0 && tc <= e->TcMax &&
                   lanes >= 1 && lanes <= e->lanes_alloc && gt >= 1 && gt <= tdf_engine::kGtMax) {
                    e->Tc = tc;
                    e->nlanes = lanes;
                    e->Gt = gt;
               }
          }
     }
     fclose(f);
}

static void autotune_cache_store(const tdf_engine *e) {
     const char *path = getenv("TDF_AUTOTUNE_CACHE");
     if (!path || !*path) return;
     FILE *f = fopen(path, "a");
     if (!f) return;
     fprintf(f, "%s %d %d %d\n", autotune_key(e).c_str(), e->Tc, e->nlanes, e->Gt);
     fclose(f);
}

// One warp waits on an mbarrier that announces 16 bytes of transactions no
// copy will deliver: the bounded wait of the pipeline kernels gives up after
// `probes` probes and the kernel reports ERR_STAGE_TIMEOUT, as a pass whose
// bulk copies never completed would.  No copy is issued, so nothing is in
// flight when the kernel returns.  Then lane 0 waits, as a fused pass's row
// block does for its column blocks, on a count (err[1], zero) that nothing
// raises, and reports ERR_ORDER_TIMEOUT when that wait gives up.
__global__ void k_wait_probe(unsigned *err, int probes) {
     __shared__ __align__(8) uint64_t bar;
     if (threadIdx.x == 0) {
          mbar_init(&bar, 1);
          mbar_fence_init();
     }
     __syncthreads();
     if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);
     const bool done = mbar_wait(&bar, 0u, probes);
     if (!done && threadIdx.x == 0) atomicOr(err, ERR_STAGE_TIMEOUT);
     if (threadIdx.x == 0 && !wait_count(err + 1, 1u, probes)) atomicOr(err, ERR_ORDER_TIMEOUT);
}

// ------------------------------------------------------------------ whole-call plans
//
// tdf_search_segments_device(): the points of several resident segments
// searched by one enqueue sequence -- every batch's sky stage and spindown
// stage, segment after segment, with no host work between batches -- which
// the second call with the same batch list captures into one CUDA graph and
// later calls replay with a single launch.  Trigger counts accumulate in the
// two batch slots' counters and are read once at the end.

struct PlanBatch {
     int slot, nb, nt;
     size_t sky_off, tp_off;
};

// One sky point of a plan: what tmpl_setup() needs to form its templates
// (the segment's grid-matrix entries travel with it, segments differ).
struct PlanPoint {
     double het0, M0, M4, M5, M9, M13;
     float mm, nn, smin, sstep;
     int32_t iss, slot;     // spindowns; the point's index in its sky batch
     uint32_t id0, tp0;     // template number and plan index of its first spindown
};

// tmpl_setup() on the device, one CTA per point: the same IEEE operations in
// the same order (no contraction), so the parameters equal the host's bit
// for bit.  grid (points), 128 threads
__global__ void __launch_bounds__(128) k_plan_templates(const PlanPoint *__restrict__ pts, TmplParam *__restrict__ tp,
                                                        int split)
{
     const PlanPoint P = pts[blockIdx.x];
     for (int s = threadIdx.x; s < P.iss; s += blockDim.x) {
          const float ss = __fadd_rn(P.smin, __fmul_rn((float)s, P.sstep));
          TmplParam q;
          q.spnd = __dadd_rn(__dadd_rn(__dmul_rn((double)ss, P.M5), __dmul_rn((double)P.nn, P.M9)),
                             __dmul_rn((double)P.mm, P.M13));
          const double r = fmod(__dmul_rn((double)ss, P.M4), P.M0);
          q.het1 = r < 0 ? __dadd_rn(r, P.M0) : r;
          if (split) {
               float h1 = (float)r;
               if (h1 < 0) h1 = (float)__dadd_rn((double)h1, P.M0);
               q.sgnl0 = (double)(float)__dadd_rn(P.het0, (double)h1);
          } else {
               q.sgnl0 = __dadd_rn(P.het0, q.het1);
          }
          q.slot = P.slot;
          q.id = P.id0 + (uint32_t)s;
          tp[P.tp0 + s] = q;
     }
}

static uint64_t fnv1a(uint64_t h, const void *p, size_t n) {
     const unsigned char *c = (const unsigned char *)p;
     for (size_t i = 0; i < n; i++) {
          h ^= c[i];
          h *= 1099511628211ull;
     }
     return h;
}

static int enqueue_plan(tdf_engine *e, const std::vector<PlanBatch> &pb) {
     const SkyParam *dsky = e->plan_sky.as<SkyParam>();
     const TmplParam *dtp = e->plan_tp.as<TmplParam>();
     k_plan_templates<<<e->plan_npts, 128, 0, e->stream>>>(e->plan_pts.as<PlanPoint>(), e->plan_tp.as<TmplParam>(),
                                                            e->form == TDF_FORM_SPLIT);
     CUCHK(cudaGetLastError());
     e->launches++;
     for (int s = 0; s < 2; s++) CUCHK(cudaMemsetAsync(e->counters[s].p, 0, 2 * sizeof(unsigned long long), e->stream));
     for (int l = 0; l < e->lanes_alloc; l++) CUCHK(cudaMemsetAsync(e->ln[l].tcnt.p, 0, e->ln[l].tcnt.bytes, e->stream));
     // the sky stream's first work of the plan follows this point of the engine stream
     CUCHK(cudaEventRecord(e->plan_ev, e->stream));
     for (size_t i = 0; i < pb.size(); i++) {
          e->cur = (int)(i & 1);
          e->act = pb[i].slot;
          const int st = run_sky_stage(e, pb[i].nb, dsky + pb[i].sky_off, i < 2 ? e->plan_ev : nullptr);
          e->act = 0;
          TRY(st);
          CUCHK(cudaStreamWaitEvent(e->stream, e->sky_done[e->cur], 0));
          TRY(run_templates(e, dtp + pb[i].tp_off, pb[i].nt));
          CUCHK(cudaEventRecord(e->spin_done[e->cur], e->stream));
     }
     for (int s = 0; s < 2; s++)
          CUCHK(cudaMemcpyAsync(e->h_cnt + 2 * s, e->counters[s].p, 2 * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, e->stream));
     return TDF_OK;
}

// runs the plan once: the captured graph when one exists for `key`, else
// plain launches (the first sighting) or a capture (the second)
static int run_plan(tdf_engine *e, const std::vector<PlanBatch> &pb, uint64_t key) {
     if (!e->use_graphs || e->timing) return enqueue_plan(e, pb);
     size_t gi = e->plan_graphs.size();
     for (size_t i = 0; i < e->plan_graphs.size(); i++)
          if (e->plan_graphs[i].key == key) gi = i;
     if (gi == e->plan_graphs.size()) {
          if (e->plan_graphs.size() >= tdf_engine::kMaxGraphs) {
               size_t old = 0;
               for (size_t i = 1; i < e->plan_graphs.size(); i++)
                    if (e->plan_graphs[i].last < e->plan_graphs[old].last) old = i;
               if (e->plan_graphs[old].exec) cudaGraphExecDestroy(e->plan_graphs[old].exec);
               e->plan_graphs.erase(e->plan_graphs.begin() + old);
          }
          e->plan_graphs.push_back(tdf_engine::PlanGraph());
          gi = e->plan_graphs.size() - 1;
          e->plan_graphs[gi].key = key;
     }
     tdf_engine::PlanGraph &g = e->plan_graphs[gi];
     g.last = ++e->graph_tick;
     if (!g.exec && ++g.seen < 2) return enqueue_plan(e, pb);
     if (!g.exec) {
          if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
               cudaGetLastError();
               e->use_graphs = false;
               return enqueue_plan(e, pb);
          }
          const int64_t l0 = e->launches;
          const int st = enqueue_plan(e, pb);
          cudaGraph_t graph = nullptr;
          const cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
          if (st != TDF_OK || ce != cudaSuccess) {
               if (graph) cudaGraphDestroy(graph);
               e->launches = l0;
               return st != TDF_OK ? st : set_error(TDF_ERR_CUDA, "stream capture: %s", cudaGetErrorString(ce));
          }
          const int ps = set_graph_priorities(e, graph);
          if (ps != TDF_OK) {
               cudaGraphDestroy(graph);
               e->launches = l0;
               return ps;
          }
          const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
          cudaGraphDestroy(graph);
          if (ie != cudaSuccess) {
               g.exec = nullptr;
               e->launches = l0;
               return set_error(TDF_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ie));
          }
          g.launches = e->launches - l0;
          e->launches = l0;
     }
     CUCHK(cudaGraphLaunch(g.exec, e->stream));
     e->launches += g.launches;
     return TDF_OK;
}

// TDF_CHECK_PLAN=1: the templates the device formed for a plan, compared bit
// for bit with tmpl_setup() on the host for the same points (a self-check of
// k_plan_templates; the search's own path never reads them back).  seg[i]
// is the segment slot of plan point i.
static int plan_check(tdf_engine *e, const std::vector<PlanPoint> &hp, const std::vector<int> &seg, int64_t ntm) {
     std::vector<TmplParam> dev((size_t)ntm);
     CUCHK(cudaMemcpy(dev.data(), e->plan_tp.p, (size_t)ntm * sizeof(TmplParam), cudaMemcpyDeviceToHost));
     for (size_t i = 0; i < hp.size(); i++) {
          const PlanPoint &P = hp[i];
          HostPoint H;
          H.sp.het0 = P.het0;
          e->act = seg[i];
          for (int s2 = 0; s2 < P.iss; s2++) {
               HostTmpl T;
               tmpl_setup(e, H, P.mm, P.nn, P.smin + s2 * P.sstep, T);
               const TmplParam &d = dev[P.tp0 + s2];
               if (memcmp(&d.spnd, &T.spnd, 8) || memcmp(&d.het1, &T.het1, 8) || memcmp(&d.sgnl0, &T.sgnl0, 8) ||
                   d.slot != P.slot || d.id != P.id0 + (uint32_t)s2) {
                    e->act = 0;
                    return set_error(TDF_ERR_CUDA, "plan self-check: template %d of plan point %zu differs from "
                                     "the host's", s2, i);
               }
          }
     }
     e->act = 0;
     return TDF_OK;
}

// ------------------------------------------------------------------ C ABI

extern "C" {

int tdf_spin_order_item(int32_t nt, int32_t blocks, int32_t lag, uint32_t ticket, int32_t *tmpl, int32_t *block,
                        int32_t *row) {
     if (!tmpl || !block || !row || nt < 1 || blocks < 1 || lag < 1 ||
         (int64_t)nt * blocks * 2 > (int64_t)UINT32_MAX || (int64_t)ticket >= (int64_t)nt * blocks * 2)
          return set_error(TDF_ERR_INVALID, "outputs must be non-null, nt, blocks, lag >= 1 and ticket < 2*nt*blocks");
     // the launcher's order: C = R = blocks per template, lag clamped to [1, nt]
     SpinOrder o{nullptr, nullptr, nt, blocks, blocks, std::max(1, std::min(lag, nt)), 0};
     int b = 0, blk = 0;
     bool r = false;
     spin_item(o, ticket, b, blk, r);
     *tmpl = b;
     *block = blk;
     *row = r ? 1 : 0;
     return TDF_OK;
}

int tdf_check_bounded_wait(int device, int32_t probes, uint32_t *status) {
     if (!status || probes < 1 || probes > (1 << 20))
          return set_error(TDF_ERR_INVALID, "status must be non-null and probes in 1..2^20");
     int ndev = 0;
     if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
          cudaGetLastError();
          return set_error(TDF_ERR_NO_DEVICE, "no CUDA device");
     }
     if (device < 0 || device >= ndev) return set_error(TDF_ERR_INVALID, "device %d of %d", device, ndev);
     CUCHK(cudaSetDevice(device));
     unsigned *d = nullptr;
     CUCHK(cudaMalloc((void **)&d, 2 * sizeof(unsigned)));
     cudaError_t ce = cudaMemset(d, 0, 2 * sizeof(unsigned));
     if (ce == cudaSuccess) {
          k_wait_probe<<<1, 32>>>(d, probes);
          ce = cudaGetLastError();
     }
     unsigned h = 0;
     if (ce == cudaSuccess) ce = cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost);
     cudaFree(d);
     if (ce != cudaSuccess) return set_error(TDF_ERR_CUDA, "bounded-wait check: %s", cudaGetErrorString(ce));
     *status = h;
     return TDF_OK;
}

const char *tdf_status_string(int status) {
     switch (status) {
     case TDF_OK: return "ok";
     case TDF_ERR_INVALID: return "invalid argument";
     case TDF_ERR_CUDA: return "CUDA error";
     case TDF_ERR_TRIGGER_OVERFLOW: return "too many triggers in one spindown";
     case TDF_ERR_OUT_OF_MEMORY: return "out of device memory";
     case TDF_ERR_CAPACITY: return "output arrays too small";
     case TDF_ERR_UNSUPPORTED: return "unsupported size or option";
     case TDF_ERR_NO_DEVICE: return "no CUDA device";
     case TDF_ERR_NOT_BUILT: return "not available in this build";
     }
     return "unknown status";
}

const char *tdf_last_error(void) { return g_last_error.c_str(); }

int tdf_device_count(int *count) {
     if (!count) return set_error(TDF_ERR_INVALID, "null count");
     int n = 0;
     cudaError_t e = cudaGetDeviceCount(&n);
     if (e != cudaSuccess) {
          *count = 0;
          cudaGetLastError();
          return set_error(TDF_ERR_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
     }
     *count = n;
     return TDF_OK;
}

int tdf_engine_create(const tdf_segment *seg, const tdf_search_opts *opts, int form, int device, int max_sky_batch,
                      tdf_engine **out) {
     if (!out) return set_error(TDF_ERR_INVALID, "null out");
     *out = nullptr;
     TRY(validate(seg, opts));
     if (form != TDF_FORM_SPLIT && form != TDF_FORM_FP64) return set_error(TDF_ERR_INVALID, "form=%d", form);
     if (form == TDF_FORM_FP64 && seg->nfftf > (1 << 18))
          return set_error(TDF_ERR_UNSUPPORTED, "FP64 form supports nfftf <= 2^18");
     int ndev = 0;
     if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
          cudaGetLastError();
          return set_error(TDF_ERR_NO_DEVICE, "no CUDA device");
     }
     if (device < 0 || device >= ndev) return set_error(TDF_ERR_INVALID, "device %d of %d", device, ndev);
     CUCHK(cudaSetDevice(device));
     tdf_engine *e = new tdf_engine();
     e->dev = device;
     e->form = form;
     e->sdv.resize(1);
     e->act = 0;
     e->S().seg = *seg;
     e->opts = *opts;
     e->N = seg->N;
     e->nfft = seg->nfft;
     e->nfftf = seg->nfftf;
     e->Ninterp = seg->Ninterp;
     e->nifo = seg->nifo;
     // a multiple of every row length N2 <= 1024 of the four-step split, so
     // that the operand arrays view as whole rows for the TMA boxes
     e->Nal = (seg->N + 1023) / 1024 * 1024;
     e->n2N = seg->interpftpad * seg->N;
     e->nF = opts->fr[1] - opts->fr[0] + 1;
     e->nblk_mu = opts->blocks_avg ? (opts->fr[1] - opts->fr[0]) / TDF_NAVFSTAT : 0;
     if (max_sky_batch > 0) e->Bs = max_sky_batch;
     const char *tc = getenv("TDF_TEMPLATES_PER_CHUNK");
     if (tc && atoi(tc) > 0) e->Tc = atoi(tc);
     // buffers for chunks up to 96 templates (the autotuner's range), or for
     // exactly the fixed chunk size TDF_TEMPLATES_PER_CHUNK asks for
     e->TcMax = (tc && atoi(tc) > 0) ? e->Tc : std::max(96, e->Tc);
     const char *ov = getenv("TDF_SKY_OVERLAP");
     if (ov && ov[0] == '0') e->overlap = false;
     const char *nl = getenv("TDF_LANES");
     if (nl && atoi(nl) > 0) {
          // a fixed lane count: buffers and streams for that many only
          e->nlanes = std::min(atoi(nl), (int)tdf_engine::kMaxLanes);
          e->lanes_alloc = e->nlanes;
     }
     const char *gr = getenv("TDF_GRAPHS");
     if (gr && gr[0] == '0') e->use_graphs = false;
     const char *gp = getenv("TDF_GRAPH_PRIORITY");
     if (gp && gp[0] == '0') e->graph_prio = false;
     const char *ff = getenv("TDF_FULL_F");
     if (ff && ff[0] == '1') e->sparse_f = false;
     const char *rb = getenv("TDF_ROW_BULK");
     if (rb && rb[0] == '0') e->row_bulk = false;
     const char *fp = getenv("TDF_FUSED_PASSES");
     if (fp && fp[0] == '1') e->fused = true;
     const char *fl = getenv("TDF_FUSE_LAG");
     if (fl && atoi(fl) > 0) e->fuse_lag = atoi(fl);
     const char *gt = getenv("TDF_GROUP_TEMPLATES");
     if (gt && atoi(gt) > 0) e->Gt = std::min(atoi(gt), (int)tdf_engine::kGtMax);
     autotune_cache_lookup(e);
     e->lines.assign(opts->lines, opts->lines + 2 * (size_t)opts->numlines);
     e->opts.lines = nullptr;
     e->S().dets.resize(seg->nifo);
     int st = TDF_OK;
     int &prio_low = e->prio_low, &prio_high = e->prio_high;
     cudaError_t ce = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
     e->stream_outranks_sky = prio_high < prio_low;
     if (ce == cudaSuccess) ce = cudaStreamCreateWithPriority(&e->own, cudaStreamNonBlocking, prio_high);
     if (ce == cudaSuccess) ce = cudaStreamCreateWithPriority(&e->sky_stream, cudaStreamNonBlocking, prio_low);
     if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->fork_ev, cudaEventDisableTiming);
     if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->plan_ev, cudaEventDisableTiming);
     for (int l = 1; l < e->lanes_alloc && ce == cudaSuccess; l++) {
          ce = cudaStreamCreateWithPriority(&e->lane_own[l], cudaStreamNonBlocking, prio_high);
          if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->join_ev[l], cudaEventDisableTiming);
     }
     for (int k = 0; k < 2 && ce == cudaSuccess; k++) {
          ce = cudaEventCreateWithFlags(&e->sky_done[k], cudaEventDisableTiming);
          if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->spin_done[k], cudaEventDisableTiming);
     }
     if (ce != cudaSuccess) st = set_error(TDF_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(ce));
     e->stream = e->own;
     if (st == TDF_OK) st = engine_alloc(e);
     if (st == TDF_OK) st = upload_inputs(e, seg);
     if (st == TDF_OK) {
          ce = cudaStreamSynchronize(e->stream);
          if (ce != cudaSuccess) st = set_error(TDF_ERR_CUDA, "upload: %s", cudaGetErrorString(ce));
     }
     if (st != TDF_OK) {
          engine_free(e);
          delete e;
          return st;
     }
     *out = e;
     return TDF_OK;
}

int tdf_engine_upload(tdf_engine *e, const tdf_segment *seg) {
     if (!e || !seg) return set_error(TDF_ERR_INVALID, "null engine or segment");
     tdf_search_opts o = e->opts;
     o.lines = e->lines.data();
     TRY(validate(seg, &o));
     e->signal_valid = false;
     if (seg->N != e->N || seg->nfft != e->nfft || seg->nfftf != e->nfftf || seg->Ninterp != e->Ninterp ||
         seg->nifo != e->nifo)
          return set_error(TDF_ERR_INVALID, "segment sizes differ from the engine's");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->sky_stream));
     TRY(upload_inputs(e, seg));
     CUCHK(cudaStreamSynchronize(e->stream));
     return TDF_OK;
}

int tdf_engine_destroy(tdf_engine *e) {
     if (!e) return TDF_OK;
     cudaSetDevice(e->dev);
     if (e->sky_stream) cudaStreamSynchronize(e->sky_stream);
     for (cudaStream_t ls : e->lane_own)
          if (ls) cudaStreamSynchronize(ls);
     if (e->stream) cudaStreamSynchronize(e->stream);
     engine_free(e);
     delete e;
     return TDF_OK;
}

int tdf_search_points(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn, const float *sst,
                      tdf_record *recs, int64_t max_recs, int64_t *nrec, float *pairs, int64_t max_pairs,
                      int64_t *npairs, int32_t *nrec_per_point) {
     if (!e || !nrec || !npairs) return set_error(TDF_ERR_INVALID, "null engine or count pointers");
     CUCHK(cudaSetDevice(e->dev));
     std::vector<HostPoint> pts;
     std::vector<HostTmpl> tm;
     int64_t ntrig = 0;
     e->kept = false;
     TRY(search_core(e, npts, pm, mm, nn, sst, pts, tm, true, &ntrig));
     // sort triggers into (template, bin) order: the reference's order
     std::vector<Trig> &tg = e->h_trig;
     std::sort(tg.begin(), tg.end(), [](const Trig &a, const Trig &b) {
          return a.id != b.id ? a.id < b.id : a.bin < b.bin;
     });
     const int64_t need_recs = (int64_t)tm.size(), need_pairs = 2 * (int64_t)tg.size();
     *nrec = need_recs;
     *npairs = need_pairs;
     if (nrec_per_point)
          for (int i = 0; i < npts; i++) nrec_per_point[i] = pts[i].inside ? pts[i].iss_size : 0;
     const bool fits = !(need_recs > max_recs || need_pairs > max_pairs || (need_recs && !recs) || (need_pairs && !pairs));
     if (!fits) {
          // keep the results for tdf_last_results()
          e->last_recs.resize(need_recs);
          e->last_pairs.resize(need_pairs);
          e->last_per.assign(npts, 0);
          for (int i = 0; i < npts; i++) e->last_per[i] = pts[i].inside ? pts[i].iss_size : 0;
          recs = e->last_recs.data();
          pairs = e->last_pairs.data();
     }
     size_t k = 0;
     int64_t off = 0;
     for (size_t t = 0; t < tm.size(); t++) {
          const HostTmpl &T = tm[t];
          const HostPoint &P = pts[T.pt];
          tdf_record &r = recs[t];
          r.m = mm[T.pt];
          r.n = nn[T.pt];
          r.s = T.ss;
          r.ra = P.ra;
          r.dec = P.dec;
          r.fdot = rec_fdot(e, T.spnd);
          r.pad = 0;
          r.offset = off;
          uint32_t len = 0;
          while (k < tg.size() && tg[k].id == (uint32_t)t) {
               pairs[off++] = tg[k].f;
               pairs[off++] = tg[k].F;
               len += 2;
               k++;
          }
          r.len = len;
     }
     if (!fits) {
          e->kept = true;
          return set_error(TDF_ERR_CAPACITY, "need %lld records and %lld floats", (long long)need_recs,
                           (long long)need_pairs);
     }
     return TDF_OK;
}

int tdf_last_results(tdf_engine *e, tdf_record *recs, int64_t max_recs, int64_t *nrec, float *pairs,
                     int64_t max_pairs, int64_t *npairs, int32_t *nrec_per_point) {
     if (!e || !nrec || !npairs) return set_error(TDF_ERR_INVALID, "null engine or count pointers");
     if (!e->kept) return set_error(TDF_ERR_INVALID, "no results kept from a previous tdf_search_points() call");
     *nrec = (int64_t)e->last_recs.size();
     *npairs = (int64_t)e->last_pairs.size();
     if (*nrec > max_recs || *npairs > max_pairs || (*nrec && !recs) || (*npairs && !pairs))
          return set_error(TDF_ERR_CAPACITY, "need %lld records and %lld floats", (long long)*nrec, (long long)*npairs);
     if (*nrec) memcpy(recs, e->last_recs.data(), *nrec * sizeof(tdf_record));
     if (*npairs) memcpy(pairs, e->last_pairs.data(), *npairs * sizeof(float));
     if (nrec_per_point && !e->last_per.empty())
          memcpy(nrec_per_point, e->last_per.data(), e->last_per.size() * sizeof(int32_t));
     return TDF_OK;
}

int tdf_count_templates(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn,
                        const float *sst, int64_t *nrec, int32_t *nrec_per_point) {
     if (!e || !nrec) return set_error(TDF_ERR_INVALID, "null engine or count pointer");
     if (npts < 0 || (npts > 0 && (!pm || !mm || !nn))) return set_error(TDF_ERR_INVALID, "bad sky point arrays");
     int64_t n = 0;
     for (int i = 0; i < npts; i++) {
          if (pm[i] != 1 && pm[i] != 2) return set_error(TDF_ERR_INVALID, "pm[%d]=%d (must be 1 or 2)", i, pm[i]);
          HostPoint P;
          point_setup(e, pm[i], mm[i], nn[i], sst ? sst[i] : e->opts.spndr[0], P);
          const int c = P.inside ? P.iss_size : 0;
          if (nrec_per_point) nrec_per_point[i] = c;
          n += c;
     }
     *nrec = n;
     return TDF_OK;
}

int tdf_search_points_device(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn,
                             const float *sst, int64_t *nrec, int64_t *ntrig) {
     if (!e || !nrec || !ntrig) return set_error(TDF_ERR_INVALID, "null engine or count pointers");
     CUCHK(cudaSetDevice(e->dev));
     std::vector<HostPoint> pts;
     std::vector<HostTmpl> tm;
     TRY(search_core(e, npts, pm, mm, nn, sst, pts, tm, false, ntrig));
     *nrec = (int64_t)tm.size();
     return TDF_OK;
}

int tdf_engine_add_segment(tdf_engine *e, const tdf_segment *seg, int32_t *slot) {
     if (!e || !seg || !slot) return set_error(TDF_ERR_INVALID, "null engine, segment or slot");
     tdf_search_opts o = e->opts;
     o.lines = e->lines.data();
     TRY(validate(seg, &o));
     if (seg->N != e->N || seg->nfft != e->nfft || seg->nfftf != e->nfftf || seg->Ninterp != e->Ninterp ||
         seg->nifo != e->nifo || seg->interpftpad != e->S().seg.interpftpad)
          return set_error(TDF_ERR_INVALID, "segment sizes differ from the engine's");
     if (e->sdv.size() >= 4096) return set_error(TDF_ERR_UNSUPPORTED, "at most 4096 resident segments");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->sky_stream));
     CUCHK(cudaStreamSynchronize(e->stream));
     e->sdv.emplace_back();
     const int k = (int)e->sdv.size() - 1;
     int st = seg_alloc(e, e->sdv[k]);
     if (st == TDF_OK) {
          e->act = k;
          st = upload_inputs(e, seg);
          e->act = 0;
     }
     if (st == TDF_OK) {
          const cudaError_t ce = cudaStreamSynchronize(e->stream);
          if (ce != cudaSuccess) st = set_error(TDF_ERR_CUDA, "segment upload: %s", cudaGetErrorString(ce));
     }
     if (st != TDF_OK) {
          e->sdv[k].release();
          e->sdv.pop_back();
          return st;
     }
     *slot = k;
     return TDF_OK;
}

int tdf_engine_upload_segment(tdf_engine *e, int32_t slot, const tdf_segment *seg) {
     if (!e || !seg) return set_error(TDF_ERR_INVALID, "null engine or segment");
     if (slot < 0 || slot >= (int)e->sdv.size()) return set_error(TDF_ERR_INVALID, "segment slot %d of %d", slot, (int)e->sdv.size());
     tdf_search_opts o = e->opts;
     o.lines = e->lines.data();
     TRY(validate(seg, &o));
     if (seg->N != e->N || seg->nfft != e->nfft || seg->nfftf != e->nfftf || seg->Ninterp != e->Ninterp ||
         seg->nifo != e->nifo)
          return set_error(TDF_ERR_INVALID, "segment sizes differ from the engine's");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->sky_stream));
     CUCHK(cudaStreamSynchronize(e->stream));
     if (slot == 0) e->signal_valid = false;
     e->act = slot;
     const int st = upload_inputs(e, seg);
     e->act = 0;
     TRY(st);
     CUCHK(cudaStreamSynchronize(e->stream));
     return TDF_OK;
}

int tdf_engine_segment_count(tdf_engine *e, int32_t *count) {
     if (!e || !count) return set_error(TDF_ERR_INVALID, "null argument");
     *count = (int32_t)e->sdv.size();
     return TDF_OK;
}

int tdf_search_segments_device(tdf_engine *e, int32_t nseg, const int32_t *slots, const int32_t *npts,
                               const int32_t *pm, const float *mm, const float *nn, int64_t *nrec, int64_t *ntrig) {
     if (!e || !nrec || !ntrig) return set_error(TDF_ERR_INVALID, "null engine or count pointers");
     if (nseg < 0 || (nseg > 0 && (!slots || !npts))) return set_error(TDF_ERR_INVALID, "bad segment arrays");
     int64_t tot = 0;
     for (int k = 0; k < nseg; k++) {
          if (slots[k] < 0 || slots[k] >= (int)e->sdv.size())
               return set_error(TDF_ERR_INVALID, "segment slot %d of %d", slots[k], (int)e->sdv.size());
          if (npts[k] < 0) return set_error(TDF_ERR_INVALID, "npts[%d] < 0", k);
          tot += npts[k];
     }
     if (tot > 0 && (!pm || !mm || !nn)) return set_error(TDF_ERR_INVALID, "null sky point arrays");
     CUCHK(cudaSetDevice(e->dev));
     // the batch list: each segment's inside points in batches of Bs, with
     // the sky and template parameters as search_core forms them
     std::vector<PlanBatch> pb;
     std::vector<SkyParam> hs;
     std::vector<PlanPoint> hp;
     std::vector<int> hp_seg;   // segment slot of each plan point
     int64_t ntm = 0;
     size_t off = 0;
     for (int k = 0; k < nseg; k++) {
          e->act = slots[k];
          std::vector<HostPoint> pts(npts[k]);
          std::vector<int> inside;
          for (int i = 0; i < npts[k]; i++) {
               const size_t q = off + i;
               if (pm[q] != 1 && pm[q] != 2) {
                    e->act = 0;
                    return set_error(TDF_ERR_INVALID, "pm[%lld]=%d (must be 1 or 2)", (long long)q, pm[q]);
               }
               point_setup(e, pm[q], mm[q], nn[q], e->opts.spndr[0], pts[i]);
               if (pts[i].inside && pts[i].iss_size > 0) inside.push_back(i);
          }
          for (size_t b0 = 0; b0 < inside.size(); b0 += e->Bs) {
               PlanBatch B;
               B.slot = slots[k];
               B.nb = (int)std::min<size_t>(e->Bs, inside.size() - b0);
               B.sky_off = hs.size();
               B.tp_off = (size_t)ntm;
               B.nt = 0;
               const double *M = e->S().seg.M;
               for (int j = 0; j < B.nb; j++) {
                    const int ip = inside[b0 + j];
                    const HostPoint &P = pts[ip];
                    hs.push_back(P.sp);
                    PlanPoint q;
                    q.het0 = P.sp.het0;
                    q.M0 = M[0];
                    q.M4 = M[4];
                    q.M5 = M[5];
                    q.M9 = M[9];
                    q.M13 = M[13];
                    q.mm = mm[off + ip];
                    q.nn = nn[off + ip];
                    q.smin = P.smin;
                    q.sstep = e->opts.sstep;
                    q.iss = P.iss_size;
                    q.slot = j;
                    q.id0 = (uint32_t)ntm;
                    q.tp0 = (uint32_t)ntm;
                    hp.push_back(q);
                    hp_seg.push_back(slots[k]);
                    ntm += P.iss_size;
                    B.nt += P.iss_size;
               }
               pb.push_back(B);
          }
          off += npts[k];
     }
     e->act = 0;
     if (ntm > (int64_t)UINT32_MAX) return set_error(TDF_ERR_UNSUPPORTED, "more than 2^32 templates in one call");
     *nrec = ntm;
     *ntrig = 0;
     if (pb.empty()) return TDF_OK;
     CUCHK(cudaStreamSynchronize(e->sky_stream));
     CUCHK(cudaStreamSynchronize(e->stream));
     TRY(e->plan_sky.alloc(std::max<size_t>(e->plan_sky.bytes, hs.size() * sizeof(SkyParam))));
     TRY(e->plan_pts.alloc(std::max<size_t>(e->plan_pts.bytes, hp.size() * sizeof(PlanPoint))));
     TRY(e->plan_tp.alloc(std::max<size_t>(e->plan_tp.bytes, (size_t)ntm * sizeof(TmplParam))));
     CUCHK(cudaMemcpy(e->plan_sky.p, hs.data(), hs.size() * sizeof(SkyParam), cudaMemcpyHostToDevice));
     CUCHK(cudaMemcpy(e->plan_pts.p, hp.data(), hp.size() * sizeof(PlanPoint), cudaMemcpyHostToDevice));
     e->plan_npts = (int)hp.size();
     e->sparse_now = e->sparse_f && e->form == TDF_FORM_SPLIT && !(e->opts.blocks_avg && e->nblk_mu > 0);
     const char *cp = getenv("TDF_CHECK_PLAN");
     const bool check_plan = cp && cp[0] == '1';
     for (int pass = 0; pass < 2; pass++) {
          uint64_t key = 1469598103934665603ull;
          for (const PlanBatch &B : pb) {
               const uint64_t f[] = {(uint64_t)B.slot, (uint64_t)B.nb, (uint64_t)B.nt, (uint64_t)B.sky_off,
                                     (uint64_t)B.tp_off};
               key = fnv1a(key, f, sizeof(f));
          }
          const uintptr_t cfg[] = {(uintptr_t)e->Tc, (uintptr_t)e->Gt, (uintptr_t)e->nlanes, (uintptr_t)e->sparse_now,
                                   (uintptr_t)e->plan_sky.p, (uintptr_t)e->plan_tp.p, (uintptr_t)e->plan_pts.p,
                                   (uintptr_t)e->plan_npts, (uintptr_t)e->trig[0].p,
                                   (uintptr_t)e->trig[1].p, (uintptr_t)e->trig_cap};
          key = fnv1a(key, cfg, sizeof(cfg));
          TRY(run_plan(e, pb, key));
          CUCHK(cudaStreamSynchronize(e->stream));
          if (check_plan) TRY(plan_check(e, hp, hp_seg, ntm));
          const unsigned errf = (unsigned)((e->h_cnt[1] | e->h_cnt[3]) & 0xffffffffu);
          if (errf & ERR_OVERFLOW)
               return set_error(TDF_ERR_TRIGGER_OVERFLOW, "Too many triggers! buffer_size=%d [triggers]", e->opts.bufsize / 2);
          TRY(wait_error(errf));
          if ((errf & ERR_NEED_FULL_F) && e->sparse_now) {
               e->sparse_now = false;   // once more with the full F store
               continue;
          }
          if (errf & ERR_NEED_FULL_F) return set_error(TDF_ERR_CUDA, "trigger selection asked for the full F store twice");
          *ntrig = (int64_t)(e->h_cnt[0] + e->h_cnt[2]);
          return TDF_OK;
     }
     return set_error(TDF_ERR_CUDA, "plan did not complete");
}

// add_signal (init.c:365-504) on the resident xDat.  The constants are
// formed here as the reference forms them; k_signal computes s_n[i] into the
// sky-stage scratch B0 (idle between searches), k_add_signal adds h0 s_n[i].
int tdf_engine_add_signal(tdf_engine *e, const tdf_signal *sig, double *h0_out, int32_t *in_band) {
     if (!e || !sig) return set_error(TDF_ERR_INVALID, "null engine or signal");
     if (in_band) *in_band = 0;
     CUCHK(cudaSetDevice(e->dev));
     const int N = e->N, nifo = e->nifo;
     const double dt = e->S().seg.dt;
     const int dseg = sig->seg - sig->reffr;
     double freqo0 = 2 * M_PI * sig->freq * dt;
     const double freqo1 = M_PI * sig->fdot * dt * dt;
     freqo0 += 2. * freqo1 * N * dseg;
     e->signal_valid = false;
     if (freqo0 / (2 * M_PI * dt) < sig->fpo || freqo0 / (2 * M_PI * dt) > sig->fpo + sig->B) return TDF_OK;
     SignalParam P;
     P.sinal = std::sin(sig->ra);
     P.cosal = std::cos(sig->ra);
     P.sindel = std::sin(sig->dec);
     P.cosdel = std::cos(sig->dec);
     const double cosi = std::cos(sig->iota), psi = sig->psi, phi = sig->phase;
     const double cosip = (1. + cosi * cosi) / 2.;
     P.amp[0] = std::cos(2. * psi) * cosip * std::cos(phi) - std::sin(2. * psi) * cosi * std::sin(phi);
     P.amp[1] = std::sin(2. * psi) * cosip * std::cos(phi) + std::cos(2. * psi) * cosi * std::sin(phi);
     P.amp[2] = -std::cos(2. * psi) * cosip * std::sin(phi) - std::sin(2. * psi) * cosi * std::cos(phi);
     P.amp[3] = -std::sin(2. * psi) * cosip * std::sin(phi) + std::cos(2. * psi) * cosi * std::cos(phi);
     P.nS0 = P.cosal * P.cosdel;
     P.nS1 = P.sinal * P.cosdel;
     P.nS2 = P.sindel;
     P.freqo0 = freqo0;
     P.freqo1 = freqo1;
     P.phaseshift = freqo0 * N * dseg - freqo1 * std::pow((double)(N * dseg), 2);
     P.dephase = 2 * M_PI * dt * sig->fpo;
     const int nblk = (N + 255) / 256;
     if (e->B0.bytes < (size_t)nifo * N * sizeof(double) || e->partial.bytes < (size_t)nifo * nblk * sizeof(double))
          return set_error(TDF_ERR_UNSUPPORTED, "injection scratch too small");
     CUCHK(cudaStreamSynchronize(e->sky_stream));
     cudaStream_t st = e->stream;
     double *s = e->B0.as<double>();
     double *part = e->partial.as<double>();
     k_signal<<<dim3(nblk, nifo), 256, 0, st>>>(e->S().xdat.as<float>(), e->S().detssb.as<double>(), e->S().cosm.as<double>(),
                                                e->S().sinm.as<double>(), e->S().detp.as<DetParam>(), N, e->Nal, P, s, part);
     CUCHK(cudaGetLastError());
     double h0 = sig->h0;
     if (sig->snr > 0.) {
          std::vector<double> ps((size_t)nifo * nblk);
          CUCHK(cudaMemcpyAsync(ps.data(), part, ps.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
          CUCHK(cudaStreamSynchronize(st));
          double net = 0.;
          for (int n = 0; n < nifo; n++) {
               double sum = 0.;
               for (int b = 0; b < nblk; b++) sum += ps[(size_t)n * nblk + b];
               net += sum / e->S().dets[n].sig2;
          }
          if (!(net > 0.)) return set_error(TDF_ERR_INVALID, "signal has no power in the data (snr form)");
          h0 = sig->snr / std::sqrt(net);
     }
     k_add_signal<<<dim3(nblk, nifo), 256, 0, st>>>(e->S().xdat.as<float>(), s, N, e->Nal, h0);
     CUCHK(cudaGetLastError());
     CUCHK(cudaStreamSynchronize(st));
     e->launches += 2;
     if (h0_out) *h0_out = h0;
     if (in_band) *in_band = 1;
     e->signal_h0 = h0;
     e->signal_valid = true;
     return TDF_OK;
}

int tdf_engine_get_signal(tdf_engine *e, int32_t det, double *out, int64_t n) {
     if (!e || !out) return set_error(TDF_ERR_INVALID, "null engine or output");
     if (det < 0 || det >= e->nifo) return set_error(TDF_ERR_INVALID, "detector %d of %d", det, e->nifo);
     if (n < e->N) return set_error(TDF_ERR_CAPACITY, "need %d values", e->N);
     if (!e->signal_valid)
          return set_error(TDF_ERR_INVALID, "no injected signal held (none added since the last search or upload)");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaMemcpy(out, e->B0.as<double>() + (size_t)det * e->N, (size_t)e->N * sizeof(double),
                      cudaMemcpyDeviceToHost));
     for (int i = 0; i < e->N; i++) out[i] = e->signal_h0 * out[i];   // h0*signadd (init.c:491)
     return TDF_OK;
}

int tdf_engine_get_xdat(tdf_engine *e, int32_t det, float *xdat, int64_t n) {
     if (!e || !xdat) return set_error(TDF_ERR_INVALID, "null argument");
     if (det < 0 || det >= e->nifo || n < 0 || n > e->N)
          return set_error(TDF_ERR_INVALID, "detector %d of %d, %lld samples of %d", det, e->nifo, (long long)n, e->N);
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->stream));
     CUCHK(cudaMemcpy(xdat, e->S().xdat.as<float>() + (size_t)det * e->Nal, n * sizeof(float), cudaMemcpyDeviceToHost));
     return TDF_OK;
}

int tdf_fstat_spectrum(tdf_engine *e, int32_t pm, float mm, float nn, float ss, double *F, int64_t nF) {
     if (!e || !F) return set_error(TDF_ERR_INVALID, "null engine or output");
     if (nF < e->nF) return set_error(TDF_ERR_CAPACITY, "need %d values", e->nF);
     if (pm != 1 && pm != 2) return set_error(TDF_ERR_INVALID, "pm=%d", pm);
     CUCHK(cudaSetDevice(e->dev));
     HostPoint P;
     point_setup(e, pm, mm, nn, e->opts.spndr[0], P);
     if (!P.inside) return set_error(TDF_ERR_INVALID, "sky point outside the grid ellipse");
     HostTmpl T;
     tmpl_setup(e, P, mm, nn, ss, T);
     CUCHK(cudaStreamSynchronize(e->sky_stream));
     CUCHK(cudaStreamSynchronize(e->stream));
     TRY(ensure_tparam(e, 1));
     e->cur = 0;
     e->h_sky[0][0] = P.sp;
     TmplParam &q = e->h_tp[0][0];
     q.het1 = T.het1;
     q.spnd = T.spnd;
     q.sgnl0 = T.sgnl0;
     q.slot = 0;
     q.id = 0;
     TRY(run_sky_stage(e, 1));
     CUCHK(cudaStreamWaitEvent(e->stream, e->sky_done[0], 0));
     CUCHK(cudaMemcpyAsync(e->tparam.p, e->h_tp[0], sizeof(TmplParam), cudaMemcpyHostToDevice, e->stream));
     CUCHK(cudaMemsetAsync(e->counters[0].p, 0, 2 * sizeof(unsigned long long), e->stream));
     for (int l = 0; l < e->lanes_alloc; l++) CUCHK(cudaMemsetAsync(e->ln[l].tcnt.p, 0, e->ln[l].tcnt.bytes, e->stream));
     e->sparse_now = false;   // the spectrum itself is the output: the full F store
     TRY(run_templates(e, e->tparam.as<TmplParam>(), 1));
     CUCHK(cudaMemcpyAsync(e->h_cnt, e->counters[0].p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, e->stream));
     CUCHK(cudaStreamSynchronize(e->stream));
     TRY(wait_error((unsigned)(e->h_cnt[1] & 0xffffffffu)));
     const int n = e->nF;
     if (e->form == TDF_FORM_SPLIT) {
          std::vector<float> f(n), mu(std::max(1, e->nblk_mu));
          CUCHK(cudaMemcpyAsync(f.data(), e->ln[0].Fbuf.p, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
          if (e->nblk_mu)
               CUCHK(cudaMemcpyAsync(mu.data(), e->ln[0].mubuf.p, e->nblk_mu * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
          CUCHK(cudaStreamSynchronize(e->stream));
          for (int i = 0; i < n; i++) F[i] = (i < e->nblk_mu * TDF_NAVFSTAT) ? (double)(f[i] / mu[i >> 12]) : (double)f[i];
     } else {
          std::vector<double> mu(std::max(1, e->nblk_mu));
          CUCHK(cudaMemcpyAsync(F, e->ln[0].Fbuf.p, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
          if (e->nblk_mu)
               CUCHK(cudaMemcpyAsync(mu.data(), e->ln[0].mubuf.p, e->nblk_mu * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
          CUCHK(cudaStreamSynchronize(e->stream));
          for (int i = 0; i < n && i < e->nblk_mu * TDF_NAVFSTAT; i++) F[i] = F[i] / mu[i >> 12];
     }
     return TDF_OK;
}

int tdf_engine_get_stream(tdf_engine *e, void **stream) {
     if (!e || !stream) return set_error(TDF_ERR_INVALID, "null argument");
     *stream = (void *)e->stream;
     return TDF_OK;
}

int tdf_engine_set_stream(tdf_engine *e, void *stream) {
     if (!e) return set_error(TDF_ERR_INVALID, "null engine");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->stream));
     e->stream = stream ? (cudaStream_t)stream : e->own;
     int p = e->prio_low;
     CUCHK(cudaStreamGetPriority(e->stream, &p));
     e->stream_outranks_sky = p < e->prio_low;
     return TDF_OK;
}

// Times device-only searches of the caller's points (the fastest of plain
// launches, capture and replay when graphs are on) for one setting.
static int autotune_time(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn, cudaEvent_t a,
                         cudaEvent_t b, float *best_ms) {
     std::vector<HostPoint> pts;
     std::vector<HostTmpl> tm;
     int64_t ntrig = 0;
     float m2 = 1e30f;
     const int reps = e->use_graphs ? 3 : 2;
     for (int rep = 0; rep < reps; rep++) {
          CUCHK(cudaEventRecord(a, e->stream));
          TRY(search_core(e, npts, pm, mm, nn, nullptr, pts, tm, false, &ntrig));
          CUCHK(cudaEventRecord(b, e->stream));
          CUCHK(cudaEventSynchronize(b));
          float ms = 0.f;
          CUCHK(cudaEventElapsedTime(&ms, a, b));
          m2 = std::min(m2, ms);
     }
     *best_ms = m2;
     return TDF_OK;
}

// Coordinate search: the templates per chunk (6..96) at the current lanes and
// group size, then the lanes (2..6) at the best chunk size, then the
// templates per resolve group (32, 64, 128).
int tdf_engine_autotune(tdf_engine *e, int npts, const int32_t *pm, const float *mm, const float *nn,
                        int32_t *best) {
     if (!e) return set_error(TDF_ERR_INVALID, "null engine");
     CUCHK(cudaSetDevice(e->dev));
     static const int tcs[] = {6, 8, 10, 12, 14, 16, 20, 24, 28, 32, 37, 41, 48, 64, 80, 96};
     static const int lanes[] = {2, 3, 4, 5, 6};
     static const int gts[] = {32, 64, 128};
     cudaEvent_t a, b;
     CUCHK(cudaEventCreate(&a));
     CUCHK(cudaEventCreate(&b));
     const int keep_tc = e->Tc, keep_l = e->nlanes, keep_g = e->Gt;
     int st = TDF_OK;
     float best_ms = 1e30f, ms = 0.f;
     int btc = keep_tc, bl = keep_l, bg = keep_g;
     for (int c : tcs) {
          if (c > e->TcMax || st != TDF_OK) continue;
          e->Tc = c;
          st = autotune_time(e, npts, pm, mm, nn, a, b, &ms);
          if (st == TDF_OK && ms < best_ms) {
               best_ms = ms;
               btc = c;
          }
     }
     e->Tc = btc;
     for (int l : lanes) {
          if (st != TDF_OK || l == bl || l > e->lanes_alloc) continue;
          e->nlanes = l;
          st = autotune_time(e, npts, pm, mm, nn, a, b, &ms);
          if (st == TDF_OK && ms < best_ms) {
               best_ms = ms;
               bl = l;
          }
     }
     e->nlanes = bl;
     for (int g : gts) {
          if (st != TDF_OK || g == bg) continue;
          e->Gt = g;
          st = autotune_time(e, npts, pm, mm, nn, a, b, &ms);
          if (st == TDF_OK && ms < best_ms) {
               best_ms = ms;
               bg = g;
          }
     }
     e->Gt = bg;
     cudaEventDestroy(a);
     cudaEventDestroy(b);
     if (st != TDF_OK) {
          e->Tc = keep_tc;
          e->nlanes = keep_l;
          e->Gt = keep_g;
          return st;
     }
     graphs_clear(e);   // the candidates' graphs
     autotune_cache_store(e);
     if (best) *best = btc;
     return TDF_OK;
}

int tdf_engine_get_tuning(tdf_engine *e, int32_t *templates_per_chunk, int32_t *lanes, int32_t *group_templates) {
     if (!e) return set_error(TDF_ERR_INVALID, "null engine");
     if (templates_per_chunk) *templates_per_chunk = e->Tc;
     if (lanes) *lanes = e->nlanes;
     if (group_templates) *group_templates = e->Gt;
     return TDF_OK;
}

int tdf_engine_get_templates_per_chunk(tdf_engine *e, int32_t *tc) {
     if (!e || !tc) return set_error(TDF_ERR_INVALID, "null argument");
     *tc = e->Tc;
     return TDF_OK;
}

int tdf_engine_set_templates_per_chunk(tdf_engine *e, int32_t tc) {
     if (!e) return set_error(TDF_ERR_INVALID, "null engine");
     if (tc < 1 || tc > e->TcMax) return set_error(TDF_ERR_INVALID, "templates per chunk %d outside 1..%d", tc, e->TcMax);
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->stream));
     e->Tc = tc;
     return TDF_OK;
}

int tdf_engine_launch_count(tdf_engine *e, int64_t *count) {
     if (!e || !count) return set_error(TDF_ERR_INVALID, "null argument");
     *count = e->launches;
     return TDF_OK;
}

int tdf_engine_set_kernel_timing(tdf_engine *e, int on) {
     if (!e) return set_error(TDF_ERR_INVALID, "null engine");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->stream));
     if (e->timing) timing_collect(e);
     e->timing = on != 0;
     if (on) e->kt = tdf_kernel_times{};
     return TDF_OK;
}

int tdf_engine_get_kernel_times(tdf_engine *e, tdf_kernel_times *out) {
     if (!e || !out) return set_error(TDF_ERR_INVALID, "null argument");
     CUCHK(cudaSetDevice(e->dev));
     CUCHK(cudaStreamSynchronize(e->stream));
     timing_collect(e);
     *out = e->kt;
     return TDF_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ allocation-free entry point
//
// tdf_fstat_operands_static(): the spindown-stage kernels (column pass with
// the demodulation, row pass with the F-statistic) of one split-form template
// on caller-owned device operands.  Its scratch -- the intermediate spectra,
// the FFT twiddle tables and the template parameters -- is the static array
// below, so a call allocates nothing.  Host code must not pass the array's
// name to a kernel (on the host it is only a stand-in); the device address is
// resolved with cudaGetSymbolAddress, once per device context.
//
// The array holds one set of twiddle tables for every supported transform
// length (2^12 .. 2^18), all written once when a device context is first
// seen, so no later call rewrites state that earlier enqueued work (or a
// replayed graph) reads.

namespace {

constexpr int kStaticMinLog2 = 12;
constexpr int kStaticMaxLog2 = 18;                                  // nfftf <= 2^18
constexpr size_t kStaticY = 2ull * (1ull << kStaticMaxLog2) * sizeof(float2);   // two spectra

// float2 entries of the tables of a 2^l transform: line tables of N1 and N2
// points, four-step hi (2^l / 1024) and lo (1024)
constexpr int static_n1(int l) { return 1 << ((l + 1) / 2); }
constexpr int static_n2(int l) { return 1 << (l / 2); }
constexpr int static_nhi(int l) { return l >= 10 ? 1 << (l - 10) : 1; }
constexpr size_t static_tab_entries(int l) { return (size_t)static_n1(l) + static_n2(l) + static_nhi(l) + 1024; }
constexpr size_t static_tab_offset(int l) {   // float2 entries before the tables of 2^l
     return l <= kStaticMinLog2 ? 0 : static_tab_offset(l - 1) + static_tab_entries(l - 1);
}
constexpr size_t kStaticTab = static_tab_offset(kStaticMaxLog2 + 1) * sizeof(float2);
constexpr size_t kStaticPar = 256;                                  // TmplParam + AaBb
constexpr size_t kStaticBytes = kStaticY + kStaticTab + kStaticPar;
static_assert(kStaticTab % 16 == 0, "parameter block alignment");

struct StaticDevState {
     unsigned long long ctx = 0;      // id of the device context the state below belongs to (0: none yet)
     unsigned char *base = nullptr;   // device address of g_static_scratch in that context
};
constexpr int kStaticMaxDevices = 64;
StaticDevState g_static_dev[kStaticMaxDevices];
std::mutex g_static_mu;

// id of the calling thread's current CUDA context (cuCtxGetId, through the
// runtime's driver entry points); 0 when it cannot be read
unsigned long long current_context_id() {
     static std::once_flag once;
     static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
     static PFN_cuCtxGetId_v12000 get_id = nullptr;
     std::call_once(once, [] {
          void *p = nullptr;
          cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
          if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
              q == cudaDriverEntryPointSuccess)
               get_cur = (PFN_cuCtxGetCurrent_v4000)p;
          p = nullptr;
          if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
              q == cudaDriverEntryPointSuccess)
               get_id = (PFN_cuCtxGetId_v12000)p;
     });
     if (!get_cur || !get_id) return 0;
     CUcontext c = nullptr;
     unsigned long long id = 0;
     if (get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
     return id;
}

}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

// twiddle tables of an N = N1*N2 transform (forward sign), as FFTTables
// builds them: line tables of N1 and N2 points, four-step hi/lo tables
__global__ void k_static_tables(float2 *line1, int N1, float2 *line2, int N2, float2 *hi, float2 *lo, int N)
{
     const int i = blockIdx.x * blockDim.x + threadIdx.x;
     double s, c;
     if (i < N1) { sincospi(-2.0 * i / N1, &s, &c); line1[i] = make_float2((float)c, (float)s); }
     if (i < N2) { sincospi(-2.0 * i / N2, &s, &c); line2[i] = make_float2((float)c, (float)s); }
     if (i < (N >= 1024 ? N / 1024 : 1)) { sincospi(-2.0 * ((double)i * 1024 / N), &s, &c); hi[i] = make_float2((float)c, (float)s); }
     if (i < 1024) { sincospi(-2.0 * ((double)i / N), &s, &c); lo[i] = make_float2((float)c, (float)s); }
}

__global__ void k_static_params(TmplParam *tp, AaBb *ab, TmplParam t, AaBb a)
{
     if (threadIdx.x == 0 && blockIdx.x == 0) {
          *tp = t;
          *ab = a;
     }
}

extern "C" int tdf_fstat_operands_static(const void *d_xab, const float *d_s2, int32_t nifo, int32_t N, int32_t Nal,
                                         int32_t nfftf, double het1, double spnd, float aa, float bb,
                                         int32_t fr0, int32_t fr1, float *d_F, void *stream)
{
     if (!d_xab || !d_s2 || !d_F) return set_error(TDF_ERR_INVALID, "null device pointer");
     if (nifo < 1 || nifo > TDF_MAX_DETECTORS) return set_error(TDF_ERR_INVALID, "nifo=%d", nifo);
     if (!pow2(nfftf) || nfftf < (1 << kStaticMinLog2))
          return set_error(TDF_ERR_INVALID, "nfftf=%d must be a power of two >= 4096", nfftf);
     if (nfftf > (1 << kStaticMaxLog2))
          return set_error(TDF_ERR_UNSUPPORTED, "nfftf=%d exceeds the static scratch limit 2^%d of tdf_fstat_operands_static",
                           nfftf, kStaticMaxLog2);
     if (N < 1 || N > nfftf || Nal < N) return set_error(TDF_ERR_INVALID, "N=%d, Nal=%d, nfftf=%d", N, Nal, nfftf);
     if (fr0 < 0 || fr1 < fr0 || fr1 >= nfftf) return set_error(TDF_ERR_INVALID, "fr range [%d, %d]", fr0, fr1);
     if (!(aa > 0.f) || !(bb > 0.f)) return set_error(TDF_ERR_INVALID, "aa, bb must be > 0");
     int dev = 0;
     CUCHK(cudaGetDevice(&dev));
     if (dev < 0 || dev >= kStaticMaxDevices) return set_error(TDF_ERR_UNSUPPORTED, "device %d", dev);
     cudaStream_t st = (cudaStream_t)stream;
     const int l = ilog2i(nfftf);
     const int N1 = static_n1(l), N2 = static_n2(l);
     unsigned char *base;
     {
          std::lock_guard<std::mutex> lk(g_static_mu);
          StaticDevState &S = g_static_dev[dev];
          // the symbol's address in the current context (this also makes
          // the runtime set the context up), then that context's id: a new
          // context (first call, or after cudaDeviceReset) gets its array's
          // tables written before anything reads them
          void *p = nullptr;
          CUCHK(cudaGetSymbolAddress(&p, g_static_scratch));
          const unsigned long long ctx = current_context_id();
          if (!ctx || ctx != S.ctx || (unsigned char *)p != S.base) {
               cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
               CUCHK(cudaStreamIsCapturing(st, &cs));
               if (cs != cudaStreamCaptureStatusNone)
                    return set_error(TDF_ERR_INVALID, "tdf_fstat_operands_static: the first call on a device (which "
                                     "writes the FFT tables) must not be made while its stream is being captured");
               float2 *tabs = (float2 *)((unsigned char *)p + kStaticY);
               for (int k = kStaticMinLog2; k <= kStaticMaxLog2; k++) {
                    float2 *t = tabs + static_tab_offset(k);
                    const int n1 = static_n1(k), n2 = static_n2(k);
                    k_static_tables<<<(1024 + 255) / 256, 256, 0, st>>>(t, n1, t + n1, n2, t + n1 + n2,
                                                                         t + n1 + n2 + static_nhi(k), 1 << k);
                    CUCHK(cudaGetLastError());
               }
               // later calls may come on other streams: the tables are complete first
               CUCHK(cudaStreamSynchronize(st));
               S.base = (unsigned char *)p;
               S.ctx = ctx;
          }
          base = S.base;
     }
     float2 *Y = (float2 *)base;
     const float2 *tab = (const float2 *)(base + kStaticY) + static_tab_offset(l);
     const float2 *line1 = tab, *line2 = tab + N1, *hi = tab + N1 + N2, *lo = tab + N1 + N2 + static_nhi(l);
     TmplParam *tp = (TmplParam *)(base + kStaticY + kStaticTab);
     AaBb *ab = (AaBb *)(base + kStaticY + kStaticTab + 128);
     TmplParam t;
     t.het1 = het1;
     t.spnd = spnd;
     t.sgnl0 = 0.;
     t.slot = 0;
     t.id = 0;
     AaBb a;
     a.aa = aa;
     a.bb = bb;
     a.aaf = aa;
     a.bbf = bb;
     k_static_params<<<1, 32, 0, st>>>(tp, ab, t, a);
     CUCHK(cudaGetLastError());
     DemodSplit pro{(const float4 *)d_xab, d_s2, tp, N, N2, Nal, nifo};
     StoreFourstep<float, -1, 2> epi{Y, hi, lo, N2, nfftf};
     TRY((launch_col<float, -1, 2>(N1, dim3(N2 / LINES, 1), pro, epi, line1, st)));
     RowsY<float, 2> src{Y, nfftf, N2};
     StoreFstat<float> epi2{d_F, tp, ab, fr1 - fr0 + 1, fr0, fr1, N1, 0.0, nullptr, nullptr, 0u, 0};
     TRY((launch_row<float, -1, 2>(N2, dim3(N1 / LINES, 1), src, epi2, line2, st)));
     return TDF_OK;
}
