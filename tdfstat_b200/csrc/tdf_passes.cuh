// tdf_passes.cuh -- the two four-step pass kernels (see tdf_fft.cuh) and the
// prologue/epilogue policies fused into them.
//
//   k_colpass<T, L, SIGN, NA, Pro, Epi>: CTA = LINES columns n2 of an
//     N = L*N2 transform, L threads; Pro::load fills the first-pass inputs
//     x[N2*n1 + n2] straight into registers (coalesced across the 8 columns),
//     Epi::store consumes the outputs k1 = t + m*L/8.
//   k_rowpass<T, L, SIGN, NA, Src, Epi>: CTA = LINES rows k1 of an
//     N = N1*L transform, L threads; the first-pass inputs are loaded from
//     the rows straight into registers, Epi::store consumes X[k1 + N1*k2].
//   k_spinpass<L, ...>: both passes of the FP32 spindown transform (N1 = N2
//     = L) as one launch of persistent CTAs taking column and row blocks in
//     ticket order (opt-in; see the comment above its definition).
#pragma once

#include <type_traits>

#include "tdf_bulk.cuh"
#include "tdf_fft.cuh"

namespace tdf {

// threads of a pass CTA: L/8 per line, LINES lines
template <int L>
constexpr int pass_threads() { return L / 8 * LINES; }

template <typename T, int L, int NA>
constexpr size_t pass_smem_bytes() {
     return sizeof(cx<T>) * (L + (size_t)NA * LINES * LineGeom<T, L>::STRIDE);
}

// resident CTAs per SM the FP32 passes are compiled for (register cap):
// column passes, and row passes (which hold no demodulation operands and fit
// 64 registers at L <= 256 without spilling)
template <typename T, int L>
constexpr int pass_min_blocks() {
     return sizeof(T) == 4 ? (L <= 256 ? 3 : (L == 512 ? 2 : 1)) : 1;
}
template <typename T, int L>
constexpr int row_min_blocks() {
     return sizeof(T) == 4 ? (L <= 256 ? 4 : (L == 512 ? 2 : 1)) : 1;
}

// A prologue with `static constexpr bool kStaged = true` stages its operands
// through shared memory itself: load_staged() gets the line-buffer area (free
// until the first pass stores) and its barriers at byte offset pro.bar_off.
template <class P, class = void>
struct is_staged : std::false_type {};
template <class P>
struct is_staged<P, std::void_t<decltype(P::kStaged)>> : std::integral_constant<bool, P::kStaged> {};

// An epilogue with `static constexpr bool kTables = true` keeps tables in
// dynamic shared memory at byte offset tab_off: load_tables<L>() fills them
// before the first barrier and store() gets the shared memory base.
// A row-pass source with `static constexpr bool kBulk = true` brings the
// CTA's rows into shared memory itself: load_bulk() gets the line-buffer
// area (free until the first pass stores) and its barrier at pro.bar_off,
// and loads the line twiddle table on the way.
template <class P, class = void>
struct is_bulk : std::false_type {};
template <class P>
struct is_bulk<P, std::void_t<decltype(P::kBulk)>> : std::integral_constant<bool, P::kBulk> {};

template <class P, class = void>
struct has_tables : std::false_type {};
template <class P>
struct has_tables<P, std::void_t<decltype(P::kTables)>> : std::integral_constant<bool, P::kTables> {};

// The column pass of CTA (blk, b): columns n2 = blk*LINES + c of batch b.
// twline == nullptr: the line table is in shared memory already.
template <typename T, int L, int SIGN, int NA, class Pro, class Epi>
__device__ __forceinline__ void col_body(const Pro &pro, const Epi &epi, const cx<T> *__restrict__ twline, int blk,
                                         int b, unsigned char *smem_raw) {
     using G = LineGeom<T, L>;
     cx<T> *tw = reinterpret_cast<cx<T> *>(smem_raw);
     cx<T> *lines = tw + L;
     if (twline) load_table<T>(tw, twline, L);
     if constexpr (has_tables<Epi>::value) epi.template load_tables<L>(smem_raw);
     const int tid = threadIdx.x;
     const int c = tid % LINES, t = tid / LINES;
     const int n2 = blk * LINES + c;
     cx<T> v[NA][8];
     if constexpr (is_staged<Pro>::value)
          pro.template load_staged<L>(v, b, n2, t, reinterpret_cast<unsigned char *>(lines),
                                      reinterpret_cast<uint64_t *>(smem_raw + pro.bar_off));
     else
          pro.template load<L>(v, b, n2, t);
     cx<T> *s[NA];
#pragma unroll
     for (int a = 0; a < NA; a++) s[a] = lines + (a * LINES + c) * G::STRIDE;
     __syncthreads();
     line_fft<T, L, SIGN, NA>(v, s, tw, t);
     if constexpr (has_tables<Epi>::value)
          epi.template store<L>(v, b, n2, t, smem_raw);
     else
          epi.template store<L>(v, b, n2, t);
}

// The row pass of CTA (blk, b): rows k1 = blk*LINES + c of batch b.
// twline == nullptr: the line table is in shared memory already.  A bulk
// source initialises its barrier itself (bar_init) or finds it initialised
// and waits for the phase of `parity`.
template <typename T, int L, int SIGN, int NA, class Src, class Epi>
__device__ __forceinline__ void row_body(const Src &src, const Epi &epi, const cx<T> *__restrict__ twline, int blk,
                                         int b, unsigned char *smem_raw, bool bar_init = true,
                                         unsigned parity = 0u) {
     using G = LineGeom<T, L>;
     cx<T> *tw = reinterpret_cast<cx<T> *>(smem_raw);
     cx<T> *lines = tw + L;
     const int tid = threadIdx.x;
     const int k1b = blk * LINES;
     const int c = tid % LINES, t = tid / LINES;
     cx<T> v[NA][8];
     cx<T> *s[NA];
     if constexpr (is_bulk<Src>::value) {
          src.template load_bulk<L>(v, b, k1b, c, t, reinterpret_cast<unsigned char *>(lines),
                                    reinterpret_cast<uint64_t *>(smem_raw + src.bar_off), tw, twline, bar_init,
                                    parity);
     } else {
          // first-pass inputs straight from the rows into registers: per load
          // instruction a warp reads 4 consecutive elements of each of 8 rows
          src.template load<L>(v, b, k1b + c, t);
          if (twline) load_table<T>(tw, twline, L);
     }
#pragma unroll
     for (int a = 0; a < NA; a++) s[a] = lines + (a * LINES + c) * G::STRIDE;
     __syncthreads();
     line_fft<T, L, SIGN, NA>(v, s, tw, t);
     epi.template store<L>(v, b, k1b + c, t);
}

template <typename T, int L, int SIGN, int NA, class Pro, class Epi>
__global__ void __launch_bounds__(pass_threads<L>(), (pass_min_blocks<T, L>()))
k_colpass(const __grid_constant__ Pro pro, Epi epi, const cx<T> *__restrict__ twline) {
     extern __shared__ __align__(128) unsigned char smem_raw[];
     col_body<T, L, SIGN, NA>(pro, epi, twline, blockIdx.x, blockIdx.y, smem_raw);
}

template <typename T, int L, int SIGN, int NA, class Src, class Epi>
__global__ void __launch_bounds__(pass_threads<L>(), (row_min_blocks<T, L>())) k_rowpass(Src src, Epi epi, const cx<T> *__restrict__ twline) {
     extern __shared__ __align__(128) unsigned char smem_raw[];
     row_body<T, L, SIGN, NA>(src, epi, twline, blockIdx.x, blockIdx.y, smem_raw);
}

// ------------------------------------------------------------------ fused pass order
//
// k_spinpass runs the column pass and the row pass of nt templates (FP32, two
// arrays, N1 = N2 = L) as one launch of persistent CTAs (as many as are
// resident at once).  C = R = L/LINES blocks per template and pass; the
// items are handed out by tickets (ctl[0]) in the order
//   col(0) .. col(D-1), then for b = 0 .. nt-D-1: col(b+D), row(b),
//   then row(nt-D) .. row(nt-1)
// (col(b) = the C column blocks of template b, row(b) its R row blocks), so
// that a template's rows follow its columns by about D templates while its
// spectra Y are still in L2.  A CTA takes its next ticket while it works on
// the current item.  When a CTA starts the item after a column block of
// template b, its thread 0 publishes that block (device-scope fence, then
// ctl[2+b] += 1): the fence overlaps the new item instead of holding the
// CTA.  A row block of template b waits until ctl[2+b] == C (bounded: on
// time-out ERR_ORDER_TIMEOUT goes to *err and the block goes on).
// No deadlock: a CTA publishes before it waits, and waits only for items of
// smaller tickets; the waiting CTA whose current ticket is smallest depends
// on items that are finished, current in CTAs that wait on nothing, or next
// in CTAs whose current item has a smaller ticket and so is not waiting.
// ctl is zeroed (memset) before each launch.
constexpr unsigned ERR_ORDER_TIMEOUT = 8u;

struct SpinOrder {
     unsigned *ctl;   // [0] tickets, [1] unused, [2 + b] column blocks done of template b
     unsigned *err;
     int nt, C, R, D;
     int limit;       // probes of a row block's wait
};

__host__ __device__ __forceinline__ void spin_item(const SpinOrder &o, unsigned k, int &b, int &blk, bool &row) {
     const unsigned C = (unsigned)o.C, R = (unsigned)o.R, D = (unsigned)o.D;
     const unsigned head = D * C;
     if (k < head) {
          row = false;
          b = (int)(k / C);
          blk = (int)(k % C);
          return;
     }
     k -= head;
     const unsigned mid = (unsigned)(o.nt - o.D) * (C + R);
     if (k < mid) {
          const unsigned g = k / (C + R), r = k % (C + R);
          row = r >= C;
          b = (int)(row ? g : g + D);
          blk = (int)(row ? r - C : r);
          return;
     }
     k -= mid;
     row = true;
     b = (int)((unsigned)(o.nt - o.D) + k / R);
     blk = (int)(k % R);
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
     unsigned v;
     asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
     return v;
}

// orders this thread's generic-proxy accesses (and those it has observed)
// before the bulk copies it issues next, in global and shared memory
__device__ __forceinline__ void fence_proxy_async() {
     asm volatile("fence.proxy.async;" ::: "memory");
}

// Waits until *p >= target, giving up after `limit` probes; returns false
// when it gave up.
__device__ __forceinline__ bool wait_count(const unsigned *p, unsigned target, int limit) {
     for (int it = 0; it < limit; it++) {
          if (ld_acquire_gpu(p) >= target) return true;
          __nanosleep(64);
     }
     return ld_acquire_gpu(p) >= target;
}

template <int L, class Pro, class EpiC, class Src, class EpiR>
__global__ void __launch_bounds__(pass_threads<L>(), (L <= 256 ? 4 : 2))
k_spinpass(const __grid_constant__ Pro pro, const __grid_constant__ EpiC epic, const __grid_constant__ Src src,
           const __grid_constant__ EpiR epir, const float2 *__restrict__ twline, const __grid_constant__ SpinOrder o) {
     extern __shared__ __align__(128) unsigned char smem_raw[];
     __shared__ unsigned s_tk[2];
     uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + src.bar_off);
     const unsigned total = (unsigned)o.nt * (unsigned)(o.C + o.R);
     if (threadIdx.x == 0) {
          s_tk[0] = atomicAdd(&o.ctl[0], 1u);
          mbar_init(bar, 1);
          mbar_fence_init();
     }
     // one line table serves both passes (N1 = N2)
     load_table<float>(reinterpret_cast<float2 *>(smem_raw), twline, L);
     __syncthreads();
     int pend = -1;         // template of the column block finished last, not yet published
     unsigned nrow = 0;     // row items done (barrier phase)
     for (int it = 0;; it++) {
          const unsigned k = s_tk[it & 1];
          if (threadIdx.x == 0) {
               if (pend >= 0) {
                    __threadfence();
                    atomicAdd(&o.ctl[2 + pend], 1u);
               }
               if (k < total) s_tk[(it + 1) & 1] = atomicAdd(&o.ctl[0], 1u);
          }
          pend = -1;
          if (k >= total) break;
          int b, blk;
          bool row;
          spin_item(o, k, b, blk, row);
          if (!row) {
               col_body<float, L, -1, 2>(pro, epic, (const float2 *)nullptr, blk, b, smem_raw);
               pend = b;
          } else {
               if (threadIdx.x == 0) {
                    if (!wait_count(&o.ctl[2 + b], (unsigned)o.C, o.limit)) atomicOr(o.err, ERR_ORDER_TIMEOUT);
                    fence_proxy_async();
               }
               __syncthreads();
               row_body<float, L, -1, 2>(src, epir, (const float2 *)nullptr, blk, b, smem_raw, false, nrow & 1u);
               nrow++;
          }
          __syncthreads();   // the item's shared memory is free; the next ticket is visible
     }
}

// ------------------------------------------------------------------ policies

// Column-pass epilogue: multiply by W_N^(n2*k1) and store Y[k1*N2 + n2].
// Batch b's arrays are interleaved element by element: array a of element e
// lives at y[((size_t)b*N + e)*NA + a], so both arrays of a sample move in one
// access (16 bytes for two float2).
// The twiddle tables hi[L*N2/1024] = W^(1024 i), lo[1024] = W^j are copied
// into dynamic shared memory at byte offset tab_off (set by the launcher) when
// the kernel starts, in the same batch of loads as the line table.  FP32
// passes form a thread's eight twiddles W^(n2 (t + m L/8)) by recurrence from
// W^(n2 t) and W^(n2 L/8) (relative error below 1e-6); FP64 passes look each
// one up.
template <typename T, int SIGN, int NA>
struct StoreFourstep {
     cx<T> *y;
     const cx<T> *hi, *lo;
     int N2;
     int N;                 // array stride
     unsigned tab_off = 0;  // byte offset of the shared copies of hi, lo
     static constexpr bool kTables = true;

     template <int L>
     __host__ __device__ static constexpr int nhi(int N2) { return L * N2 / 1024; }
     template <int L>
     __host__ __device__ static size_t table_bytes(int N2) { return sizeof(cx<T>) * (size_t)(nhi<L>(N2) + 1024); }

     template <int L>
     __device__ __forceinline__ void load_tables(unsigned char *smem) const {
          cx<T> *s = reinterpret_cast<cx<T> *>(smem + tab_off);
          const int nh = nhi<L>(N2);
          for (int i = threadIdx.x; i < nh + 1024; i += blockDim.x) s[i] = i < nh ? __ldg(&hi[i]) : __ldg(&lo[i - nh]);
     }

     template <int L>
     __device__ __forceinline__ void store(const cx<T> (&v)[NA][8], int b, int n2, int t, unsigned char *smem) const {
          const cx<T> *hs = reinterpret_cast<const cx<T> *>(smem + tab_off);
          const cx<T> *ls = hs + nhi<L>(N2);
          cx<T> w = twsign<SIGN>(fourstep_twiddle_smem<T>(hs, ls, n2 * t));
          cx<T> st = w;
          if constexpr (sizeof(T) == 4) st = twsign<SIGN>(fourstep_twiddle_smem<T>(hs, ls, n2 * (L / 8)));
#pragma unroll
          for (int m = 0; m < 8; m++) {
               const int k1 = t + m * (L / 8);
               if constexpr (sizeof(T) == 4) {
                    if (m > 0) w = cmul(w, st);
               } else {
                    w = twsign<SIGN>(fourstep_twiddle_smem<T>(hs, ls, n2 * k1));
               }
               cx<T> *dst = y + ((size_t)b * N + n2 + (size_t)k1 * N2) * NA;
               if constexpr (NA == 2 && sizeof(T) == 4) {
                    const cx<T> p = cmul(v[0][m], w), q = cmul(v[1][m], w);
                    *reinterpret_cast<float4 *>(dst) = make_float4(p.x, p.y, q.x, q.y);
               } else {
#pragma unroll
                    for (int a = 0; a < NA; a++) dst[a] = cmul(v[a][m], w);
               }
          }
     }
};

// StoreFourstep for the FP32 spindown transform (two arrays) with the row
// length N2 fixed at compile time (CN2 > 0, else the struct's N2) and the
// thread's base twiddles read from global tables instead of shared copies:
// w0[t*N2 + n2] = W^(n2*t) (t < L/8) and ws[n2] = W^(n2*L/8), forward sign,
// formed in FP64 and rounded once.  The eight twiddles W^(n2*(t + m*L/8))
// then follow by the same recurrence as StoreFourstep's FP32 path.
template <int CN2 = 0>
struct StoreFourstepG {
     float2 *y;
     const float2 *w0, *ws;
     int N2;
     int N;   // array stride (nfftf)

     template <int L>
     __device__ __forceinline__ void store(const float2 (&v)[2][8], int b, int n2, int t) const {
          const int n2s = CN2 > 0 ? CN2 : N2;
          float2 w = __ldg(&w0[t * n2s + n2]);
          const float2 st = __ldg(&ws[n2]);
          float4 *dst = reinterpret_cast<float4 *>(y) + ((size_t)b * N + n2 + (size_t)t * n2s);
          const int step = (L / 8) * n2s;   // elements between the thread's outputs
#pragma unroll
          for (int m = 0; m < 8; m++) {
               if (m > 0) w = cmul(w, st);
               const float2 p = cmul(v[0][m], w), q = cmul(v[1][m], w);
               dst[(size_t)m * step] = make_float4(p.x, p.y, q.x, q.y);
          }
     }
};

// Row-pass source: rows of Y laid out as in StoreFourstep.  load() fills the
// first-pass inputs v[a][m] = row k1 element t + m*L/8 of every array.
template <typename T, int NA>
struct RowsY {
     const cx<T> *y;
     int N;          // N1*N2
     int rowstride;  // N2
     template <int L>
     __device__ __forceinline__ void load(cx<T> (&v)[NA][8], int b, int k1, int t) const {
          const cx<T> *r = y + ((size_t)b * N + (size_t)k1 * rowstride) * NA;
#pragma unroll
          for (int m = 0; m < 8; m++) {
               const cx<T> *e = r + (size_t)(t + m * (L / 8)) * NA;
               if constexpr (NA == 2 && sizeof(T) == 4) {
                    const float4 q = *reinterpret_cast<const float4 *>(e);
                    v[0][m] = make_float2(q.x, q.y);
                    v[1][m] = make_float2(q.z, q.w);
               } else {
#pragma unroll
                    for (int a = 0; a < NA; a++) v[a][m] = e[a];
               }
          }
     }
};

// RowsY<T, 2> with the CTA's LINES rows brought in by bulk copies: row r
// (N2 elements of 2 cx<T>, both arrays) goes to shared offset
// r * (EB*N2 + 16).  A 16-byte load is served 8 lanes at a time, here the 8
// rows at one element; the 16-byte pad puts those on 8 different 16-byte
// bank groups (EB*N2 is a multiple of 128).  The slots alias the line
// buffers, which the first
// pass only writes after k_rowpass's barrier that follows the reads.  Thread
// 0 issues the copies; everyone waits on one mbarrier (bounded: on time-out
// ERR_STAGE_TIMEOUT is or-ed into *err).
template <typename T>
struct RowsYBulk {
     const cx<T> *y;
     int N;            // N1*N2
     int rowstride;    // N2
     unsigned *err;
     unsigned bar_off = 0;   // byte offset of the barrier in dynamic shared memory (set by the launcher)
     static constexpr bool kBulk = true;
     static constexpr unsigned kPad = 16;
     static constexpr unsigned EB = 2 * sizeof(cx<T>);   // bytes of an element, both arrays

     template <int L>
     __host__ __device__ static constexpr size_t stage_bytes() { return (size_t)LINES * (EB * L + kPad); }

     template <int L>
     __device__ __forceinline__ void load_bulk(cx<T> (&v)[2][8], int b, int k1b, int c, int t, unsigned char *stage,
                                               uint64_t *bar, cx<T> *tw, const cx<T> *twline, bool init = true,
                                               unsigned parity = 0u) const {
          constexpr unsigned RB = EB * L;   // bytes of a row
          static_assert(stage_bytes<L>() <= sizeof(cx<T>) * 2 * LINES * LineGeom<T, L>::STRIDE,
                        "row slots must fit in the line buffers");
          if (init) {
               if (threadIdx.x == 0) {
                    mbar_init(bar, 1);
                    mbar_fence_init();
               }
               __syncthreads();   // the barrier is initialised before anyone waits on it
          }
          if (threadIdx.x == 0) {
               mbar_expect_tx(bar, LINES * RB);
               const cx<T> *r0 = y + ((size_t)b * N + (size_t)k1b * rowstride) * 2;
#pragma unroll
               for (int r = 0; r < LINES; r++)
                    bulk_load(stage + r * (RB + kPad), r0 + (size_t)r * rowstride * 2, RB, bar);
          }
          if (twline) load_table<T>(tw, twline, L);
          const bool ok = mbar_wait(bar, parity);
          const unsigned char *row = stage + c * (RB + kPad);
#pragma unroll
          for (int m = 0; m < 8; m++) {
               const int e = t + m * (L / 8);
               if constexpr (sizeof(T) == 4) {
                    const float4 q = reinterpret_cast<const float4 *>(row)[e];
                    v[0][m] = make_float2(q.x, q.y);
                    v[1][m] = make_float2(q.z, q.w);
               } else {
                    v[0][m] = reinterpret_cast<const cx<T> *>(row)[2 * e];
                    v[1][m] = reinterpret_cast<const cx<T> *>(row)[2 * e + 1];
               }
          }
          if (!ok) atomicOr(err, ERR_STAGE_TIMEOUT);
          // k_rowpass's barrier after this call keeps the first pass's stores
          // (the slots alias the line buffers) behind every thread's reads
     }
};

// Row-pass epilogue: natural-order output X[k1 + N1*k2] * scale for k < nkeep.
template <typename T>
struct StoreNatural {
     cx<T> *x;
     int N1;
     int N;          // array stride
     int nkeep;
     T scale;
     template <int L>
     __device__ __forceinline__ void store(const cx<T> (&v)[1][8], int b, int k1, int t) const {
          cx<T> *dst = x + (size_t)b * N;
#pragma unroll
          for (int m = 0; m < 8; m++) {
               int k = k1 + N1 * (t + m * (L / 8));
               if (k < nkeep) dst[k] = cscale(v[0][m], scale);
          }
     }
};

// Column-pass prologue: plain load of x[N2*n1 + n2] from natural-order arrays
// of stride N (arrays already zero-padded to N).
template <typename T>
struct LoadNatural {
     const cx<T> *x;
     int N2;
     int N;
     template <int L>
     __device__ __forceinline__ void load(cx<T> (&v)[1][8], int b, int n2, int t) const {
          const cx<T> *src = x + (size_t)b * N + n2;
#pragma unroll
          for (int m = 0; m < 8; m++) v[0][m] = src[(size_t)N2 * (t + m * (L / 8))];
     }
};

// Column-pass prologue of the interpolation inverse FFT: the spectrum of
// length nfft is spread to Ninterp = ratio*nfft, moving bins [nyqst, nfft)
// to the top and zeroing the middle (jobcore.c:336-350).
template <typename T>
struct LoadShuffled {
     const cx<T> *x;  // forward spectra (nfft values each), arrays `stride` apart
     int N2;          // of the Ninterp transform
     int stride;
     int nfft;
     int Ninterp;
     template <int L>
     __device__ __forceinline__ void load(cx<T> (&v)[1][8], int b, int n2, int t) const {
          const cx<T> *src = x + (size_t)b * stride;
          const int nyqst = nfft / 2 + 1;
          const int gap = Ninterp - nfft;
#pragma unroll
          for (int m = 0; m < 8; m++) {
               int k = N2 * (t + m * (L / 8)) + n2;
               cx<T> z;
               z.x = 0;
               z.y = 0;
               if (k < nyqst) z = src[k];
               else if (k >= nyqst + gap) z = src[k - gap];
               v[0][m] = z;
          }
     }
};

}  // namespace tdf
