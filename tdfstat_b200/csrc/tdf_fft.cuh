// tdf_fft.cuh -- shared-memory FFT building blocks for sm_100a.
//
// Long power-of-two transforms (N = 2^12 .. 2^20) are done as four-step
// FFTs, N = N1 * N2 (input index n = N2*n1 + n2, output k = k1 + N1*k2):
//   column pass: for each n2, an N1-point FFT over n1, then the twiddle
//                W_N^(n2*k1); result Y[k1*N2 + n2]
//   row pass:    for each k1, an N2-point FFT over n2 of the row Y[k1][.];
//                result X[k1 + N1*k2]
// Each pass is one kernel.  A CTA owns LINES = 8 columns (or rows); a line of
// length L is transformed by L/8 threads with radix-8 Stockham passes (a
// radix-4 or radix-2 pass last when L is not a power of 8), data exchanged
// through shared memory between passes.  The first pass takes its inputs
// from registers and the last pass leaves its outputs in registers, so that
// kernels fuse their own prologue (e.g. the spindown demodulation) and
// epilogue (e.g. the F-statistic) around the transform.
//
// Register convention of a line transform: thread t of a line holds
// v[m] = x[t + m*L/8] on entry and v[m] = X[t + m*L/8] on exit (m < 8).
//
// Shared-memory layout: element p of a line sits at pad(p) = p + p/8 inside
// the line, lines are STRIDE elements apart.  Lane l of a warp works on line
// l % 8 at position t = l / 8.  64-bit accesses are serviced per half-warp
// (8 lines x 2 consecutive t) and 128-bit accesses per quarter-warp (8 lines,
// one t), so STRIDE = 2 (mod 16) for float2 and odd for double2 puts the
// lanes of each phase on distinct banks for every load/store pattern of the
// Stockham passes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tdf {

template <typename T> struct CxT;
template <> struct CxT<float> { using type = float2; };
template <> struct CxT<double> { using type = double2; };
template <typename T> using cx = typename CxT<T>::type;

template <typename V> __device__ __forceinline__ V cmake(decltype(V::x) a, decltype(V::x) b) { V r; r.x = a; r.y = b; return r; }
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
     V r;
     r.x = a.x * b.x - a.y * b.y;
     r.y = a.x * b.y + a.y * b.x;
     return r;
}
template <typename V> __device__ __forceinline__ V cscale(V a, decltype(V::x) s) { V r; r.x = a.x * s; r.y = a.y * s; return r; }
template <typename V> __device__ __forceinline__ decltype(V::x) cnorm(V a) { return a.x * a.x + a.y * a.y; }

// multiply by SIGN*i (SIGN = -1: forward transform convention)
template <int SIGN, typename V> __device__ __forceinline__ V mul_si(V a) {
     V r;
     if (SIGN < 0) { r.x = a.y; r.y = -a.x; }
     else { r.x = -a.y; r.y = a.x; }
     return r;
}
// twiddle tables hold forward (e^{-i...}) factors; the inverse uses conjugates
template <int SIGN, typename V> __device__ __forceinline__ V twsign(V w) {
     if (SIGN > 0) w.y = -w.y;
     return w;
}

template <int SIGN, typename V> __device__ __forceinline__ void dft2(V &a, V &b) {
     V t = a;
     a = cadd(t, b);
     b = csub(t, b);
}

// 4-point DFT in place, natural-order outputs
template <int SIGN, typename V> __device__ __forceinline__ void dft4(V &y0, V &y1, V &y2, V &y3) {
     V c0 = cadd(y0, y2), c1 = csub(y0, y2), c2 = cadd(y1, y3);
     V c3 = mul_si<SIGN>(csub(y1, y3));
     y0 = cadd(c0, c2);
     y2 = csub(c0, c2);
     y1 = cadd(c1, c3);
     y3 = csub(c1, c3);
}

// 8-point DFT of v[o], v[o+st], ..., v[o+7*st]; natural-order outputs
template <int SIGN, typename V, int ST>
__device__ __forceinline__ void dft8s(V *v) {
     using R = decltype(V::x);
     const R h = (R)0.70710678118654752440;
     V a0 = cadd(v[0], v[4 * ST]), b0 = csub(v[0], v[4 * ST]);
     V a1 = cadd(v[ST], v[5 * ST]), b1 = csub(v[ST], v[5 * ST]);
     V a2 = cadd(v[2 * ST], v[6 * ST]), b2 = csub(v[2 * ST], v[6 * ST]);
     V a3 = cadd(v[3 * ST], v[7 * ST]), b3 = csub(v[3 * ST], v[7 * ST]);
     // b1 *= W8, b2 *= W8^2 = SIGN*i, b3 *= W8^3 = SIGN*i*W8;  W8 = h(1 + SIGN i)
     V w1;
     w1.x = h * (b1.x - (R)SIGN * b1.y);
     w1.y = h * ((R)SIGN * b1.x + b1.y);
     b1 = w1;
     b2 = mul_si<SIGN>(b2);
     V w3;
     w3.x = h * (b3.x - (R)SIGN * b3.y);
     w3.y = h * ((R)SIGN * b3.x + b3.y);
     b3 = mul_si<SIGN>(w3);
     dft4<SIGN>(a0, a1, a2, a3);
     dft4<SIGN>(b0, b1, b2, b3);
     v[0] = a0; v[ST] = b0; v[2 * ST] = a1; v[3 * ST] = b1;
     v[4 * ST] = a2; v[5 * ST] = b2; v[6 * ST] = a3; v[7 * ST] = b3;
}

__host__ __device__ constexpr int ilog8(int L) { return L >= 512 ? 3 : (L >= 64 ? 2 : (L >= 8 ? 1 : 0)); }
__host__ __device__ constexpr int ipow8(int p) { return p == 0 ? 1 : 8 * ipow8(p - 1); }
__device__ __forceinline__ int pad8(int p) { return p + (p >> 3); }

template <typename T, int L> struct LineGeom {
     static constexpr int LP = L + L / 8;   // padded line length
     // bank-spreading line stride: == 2 (mod 16) for 8-byte, odd for 16-byte elements
     static constexpr int STRIDE = sizeof(cx<T>) == 8 ? LP + ((2 - LP % 16) + 16) % 16 : LP + (LP % 2 == 0 ? 1 : 0);
     static constexpr int NT = L / 8;       // threads per line
     static constexpr int P8 = ilog8(L);    // radix-8 passes
     static constexpr int RL = L / ipow8(ilog8(L));   // last radix (1 = none)
};

constexpr int LINES = 8;   // lines (columns or rows) per CTA

// Apply the Stockham twiddles of a pass (radix R, span NS) to the butterflies
// a thread owns, for all NA lines it holds (the twiddles depend only on the
// butterfly, so they are formed once).  tw[m] = e^{-2 pi i m / L}, m < L
// (shared memory).  Powers 1, 2, 4 come from the table, the others as
// products of two of them.
template <typename T, int L, int R, int SIGN, int NA>
__device__ __forceinline__ void pass_twiddle(cx<T> (&v)[NA][8], const cx<T> *tw, int t, int NS) {
#pragma unroll
     for (int q = 0; q < 8 / R; q++) {
          int j = t + q * (L / 8);
          int jm = j % NS;
          int step = jm * (L / (NS * R));
          cx<T> w[8];
          w[1] = twsign<SIGN>(tw[step]);
          if (R >= 4) {
               w[2] = twsign<SIGN>(tw[2 * step]);
               w[3] = cmul(w[1], w[2]);
          }
          if (R == 8) {
               w[4] = twsign<SIGN>(tw[4 * step]);
               w[5] = cmul(w[1], w[4]);
               w[6] = cmul(w[2], w[4]);
               w[7] = cmul(w[3], w[4]);
          }
#pragma unroll
          for (int a = 0; a < NA; a++) {
#pragma unroll
               for (int r = 1; r < R; r++) v[a][q + r * (8 / R)] = cmul(v[a][q + r * (8 / R)], w[r]);
          }
     }
}

template <int R, int SIGN, typename V>
__device__ __forceinline__ void pass_dft(V (&v)[8]) {
     if (R == 8) {
          dft8s<SIGN, V, 1>(v);
     } else if (R == 4) {
          dft4<SIGN>(v[0], v[2], v[4], v[6]);
          dft4<SIGN>(v[1], v[3], v[5], v[7]);
     } else if (R == 2) {
          dft2<SIGN>(v[0], v[4]);
          dft2<SIGN>(v[1], v[5]);
          dft2<SIGN>(v[2], v[6]);
          dft2<SIGN>(v[3], v[7]);
     }
}

// Output r of butterfly j of a pass of span NS goes to line position
// base + r*NS, base = (j/NS)*NS*R + j%NS, stored at pad8(position).  The
// padded addresses are formed from one per-thread offset: with NS = 1 and
// R = 8 the outputs are 8j .. 8j+7, i.e. pad8 = 9j + r; with NS a multiple
// of 8, pad8(base + r*NS) = pad8(base) + r*9*NS/8.  (NS is a constant once
// line_fft's pass loop is unrolled.)
template <typename T, int L, int R>
__device__ __forceinline__ void pass_store(const cx<T> (&v)[8], cx<T> *s, int t, int NS) {
#pragma unroll
     for (int q = 0; q < 8 / R; q++) {
          const int j = t + q * (L / 8);
          if (NS == 1 && R == 8) {
               cx<T> *d = s + 9 * j;
#pragma unroll
               for (int r = 0; r < R; r++) d[r] = v[q + r * (8 / R)];
          } else if (NS % 8 == 0) {
               cx<T> *d = s + pad8((j / NS) * NS * R + (j % NS));
#pragma unroll
               for (int r = 0; r < R; r++) d[r * (NS + NS / 8)] = v[q + r * (8 / R)];
          } else {
               const int base = (j / NS) * NS * R + (j % NS);
#pragma unroll
               for (int r = 0; r < R; r++) s[pad8(base + r * NS)] = v[q + r * (8 / R)];
          }
     }
}

// Input r of butterfly j of the next pass is line position j + r*L/R; L/R is
// a multiple of 8, so pad8(j + r*L/R) = pad8(j) + r*9*(L/R)/8.
template <typename T, int L, int R>
__device__ __forceinline__ void pass_load(cx<T> (&v)[8], const cx<T> *s, int t) {
     static_assert((L / R) % 8 == 0, "line length per radix must be a multiple of 8");
#pragma unroll
     for (int q = 0; q < 8 / R; q++) {
          const cx<T> *d = s + pad8(t + q * (L / 8));
#pragma unroll
          for (int r = 0; r < R; r++) v[q + r * (8 / R)] = d[r * ((L / R) + (L / R) / 8)];
     }
}

// Full L-point transform of NA lines that share a thread: v[a] in/out as in
// the register convention above; s[a] = the line's shared memory; tw = line
// twiddle table (shared).  All threads of the CTA must call it (barriers).
template <typename T, int L, int SIGN, int NA>
__device__ __forceinline__ void line_fft(cx<T> (&v)[NA][8], cx<T> *const (&s)[NA], const cx<T> *tw, int t) {
     using G = LineGeom<T, L>;
     int NS = 1;
#pragma unroll
     for (int p = 0; p < G::P8; p++) {
          if (p > 0) pass_twiddle<T, L, 8, SIGN, NA>(v, tw, t, NS);
#pragma unroll
          for (int a = 0; a < NA; a++) pass_dft<8, SIGN>(v[a]);
          const bool last = (p == G::P8 - 1) && (G::RL == 1);
          if (!last) {
#pragma unroll
               for (int a = 0; a < NA; a++) pass_store<T, L, 8>(v[a], s[a], t, NS);
               __syncthreads();
               constexpr int RN = 8;   // next pass radix (8, or the last radix)
               if (p + 1 < G::P8) {
#pragma unroll
                    for (int a = 0; a < NA; a++) pass_load<T, L, RN>(v[a], s[a], t);
               } else {
#pragma unroll
                    for (int a = 0; a < NA; a++) pass_load<T, L, (G::RL > 1 ? G::RL : 8)>(v[a], s[a], t);
               }
               __syncthreads();
          }
          NS *= 8;
     }
     if (G::RL > 1) {
          constexpr int RR = G::RL > 1 ? G::RL : 2;
          pass_twiddle<T, L, RR, SIGN, NA>(v, tw, t, NS);
#pragma unroll
          for (int a = 0; a < NA; a++) pass_dft<RR, SIGN>(v[a]);
     }
}

// Copy a line twiddle table (L entries) from global to shared memory.
template <typename T>
__device__ __forceinline__ void load_table(cx<T> *dst, const cx<T> *__restrict__ src, int n) {
     for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Four-step twiddle W_N^m (forward sign), m < N <= 2^20, from two tables:
// hi[m >> 10] * lo[m & 1023].
template <typename T>
__device__ __forceinline__ cx<T> fourstep_twiddle(const cx<T> *__restrict__ hi, const cx<T> *__restrict__ lo, int m) {
     cx<T> a = __ldg(&hi[m >> 10]);
     cx<T> b = __ldg(&lo[m & 1023]);
     return cmul(a, b);
}

// the same from copies of the tables in shared memory
template <typename T>
__device__ __forceinline__ cx<T> fourstep_twiddle_smem(const cx<T> *hi, const cx<T> *lo, int m) {
     return cmul(hi[m >> 10], lo[m & 1023]);
}

}  // namespace tdf
