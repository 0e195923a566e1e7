// tdf_kernels.cuh -- the hot-path kernels of the job_core() chain
// (search/network/openmp/jobcore.c:193-630) other than the FFT passes:
//
//   sky stage (FP64, once per sky point and detector)
//     k_sky_prep      modvir + barycentric shift + phase modulation
//                     (settings.c:254-294, jobcore.c:283-312), zero padding,
//                     partial sums of aa^2, bb^2 (jobcore.c:373-391)
//     k_sky_sums      aa, bb network sums (FLOAT_TYPE emulation per form)
//     k_spline_fwd /
//     k_spline_bwd    natural cubic spline second derivatives (auxi.c:93-117)
//                     as blocked recurrences with warm-up
//     k_splint        spline evaluation at 2(i - shftf[i]) (auxi.c:120-169),
//                     division by sig2, conversion to the spindown operands
//   spindown stage (once per template)
//     DemodSplit /
//     DemodSplitStaged /
//     DemodFP64       column-pass prologues: spindown_modulation
//                     (spinmod.c:490-514) fused into the first FFT pass
//     StoreFstat      row-pass epilogue: F = |Fa|^2/aa + |Fb|^2/bb
//                     (jobcore.c:481-484)
//     k_block_means   FStat blocks_avg means (auxi.c:336-363)
//     k_threshold     MAX_ALG 3 local maxima, veto, trigger append
//                     (jobcore.c:552-603)
#pragma once

#include <float.h>
#include "tdf_bulk.cuh"
#include "tdf_passes.cuh"

namespace tdf {

struct SkyParam {
     double sinalt, cosalt, sindelt, cosdelt, het0;
     double nS0, nS1, nS2;
};

struct DetParam {
     double amod[9];
     double cphir, sphir, sig2;
};

// one template: (sky slot, spindown)
struct TmplParam {
     double het1;     // fmod(ss*M[4], M[0]) (+M[0] if negative), FP64
     double spnd;     // ss*M[5] + nn*M[9] + mm*M[13], FP64
     double sgnl0;    // het0 + het1 as the emulated build rounds it (trigger frequency)
     int32_t slot;    // operand slot of the sky point
     uint32_t id;     // template number within the call
};

struct AaBb {
     double aa, bb;
     float aaf, bbf;
};

struct Trig {
     uint32_t id, bin;
     float f, F;
};

constexpr unsigned ERR_OVERFLOW = 1u;
constexpr double TWO_PI = 6.283185307179586476925286766559;
constexpr double INV_TWO_PI = 0.15915494309189533576888376337251;
constexpr double M_PI_D = 3.14159265358979323846;

// ------------------------------------------------------------------ sky stage

// modvir (settings.c:254-294) at one sample: the amplitude modulations
// a(t), b(t) of detector D for a source at (alpha, delta), 0 where
// |xDat[t]| <= DBL_MIN
__device__ __forceinline__ void modvir_at(const DetParam &D, double sinal, double cosal, double sindel, double cosdel,
                                          double cosm, double sinm, float x, double &aa, double &bb) {
     aa = 0.;
     bb = 0.;
     if (fabs((double)x) > DBL_MIN) {
          const double cosalfr = cosal * D.cphir + sinal * D.sphir;
          const double sinalfr = sinal * D.cphir - cosal * D.sphir;
          const double c2d = cosdel * cosdel, c2sd = sindel * cosdel;
          const double c = cosalfr * cosm + sinalfr * sinm;
          const double s = sinalfr * cosm - cosalfr * sinm;
          const double c2s = 2. * c * c, cs = c * s;
          aa = D.amod[0] * (2. - c2d) * c2s + D.amod[1] * (2. - c2d) * 2. * cs +
               D.amod[2] * c2sd * c + D.amod[3] * c2sd * s - D.amod[0] * (2. - c2d) + D.amod[4] * c2d;
          bb = D.amod[5] * sindel * c2s + D.amod[6] * sindel * 2. * cs +
               D.amod[7] * cosdel * c + D.amod[8] * cosdel * s - D.amod[5] * sindel;
     }
}

// grid (ceil(nfft/256), Q = npts*nifo), 256 threads
__global__ void __launch_bounds__(256) k_sky_prep(
     const float *__restrict__ xdat, const double *__restrict__ detssb,
     const double *__restrict__ cosm, const double *__restrict__ sinm,
     const SkyParam *__restrict__ sp, const DetParam *__restrict__ dp,
     int nifo, int N, int nfft, int Nal, double oms,
     double2 *__restrict__ W, size_t Wstride, double *__restrict__ shftf,
     float *__restrict__ s2, double *__restrict__ t1, double *__restrict__ partial)
{
     const int q = blockIdx.y, p = q / nifo, d = q % nifo;
     const int i = blockIdx.x * 256 + threadIdx.x;
     double a2 = 0., b2 = 0.;
     if (i < nfft) {
          double2 xa = make_double2(0., 0.), xb = make_double2(0., 0.);
          if (i < N) {
               const SkyParam S = sp[p];
               const DetParam &D = dp[d];
               const float x = xdat[(size_t)d * Nal + i];
               double aa, bb;
               modvir_at(D, S.sinalt, S.cosalt, S.sindelt, S.cosdelt, cosm[i], sinm[i], x, aa, bb);
               const double *e = detssb + (size_t)d * 3 * N;
               // shift and phase without FMA contraction: the phase reaches
               // ~1e5 rad, so its rounding must follow the reference's
               const double sh = __dadd_rn(__dadd_rn(__dmul_rn(S.nS0, e[3 * (size_t)i]), __dmul_rn(S.nS1, e[3 * (size_t)i + 1])),
                                           __dmul_rn(S.nS2, e[3 * (size_t)i + 2]));
               const double sh1 = __dadd_rn(__dadd_rn(__dmul_rn(S.nS0, e[0]), __dmul_rn(S.nS1, e[1])), __dmul_rn(S.nS2, e[2]));
               shftf[(size_t)q * Nal + i] = __dsub_rn(sh, sh1);
               const size_t o = ((size_t)p * nifo + d) * Nal + i;      // planar (FP64 operands)
               const size_t oi = ((size_t)p * Nal + i) * nifo + d;     // interleaved by detector (split)
               const double di = (double)i;
               if (s2) s2[oi] = (float)__dmul_rn((double)(2 * i), sh);
               if (t1) t1[o] = __dadd_rn(__dmul_rn(di, di), __dmul_rn((double)(2 * i), sh));
               const double phase = __dadd_rn(__dmul_rn(S.het0, di), __dmul_rn(oms, sh));
               double sn, cn;
               sincos(phase, &sn, &cn);
               const double ra = (double)x * aa, rb = (double)x * bb;
               xa = make_double2(ra * cn, ra * -sn);
               xb = make_double2(rb * cn, rb * -sn);
               a2 = aa * aa;
               b2 = bb * bb;
          }
          W[((size_t)q * 2 + 0) * Wstride + i] = xa;
          W[((size_t)q * 2 + 1) * Wstride + i] = xb;
     }
     // block partial sums of aa^2, bb^2
     __shared__ double ra_[8], rb_[8];
#pragma unroll
     for (int o = 16; o > 0; o >>= 1) {
          a2 += __shfl_down_sync(0xffffffffu, a2, o);
          b2 += __shfl_down_sync(0xffffffffu, b2, o);
     }
     const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
     if (l == 0) { ra_[w] = a2; rb_[w] = b2; }
     __syncthreads();
     if (threadIdx.x == 0) {
          double sa = 0., sb = 0.;
          for (int k = 0; k < 8; k++) { sa += ra_[k]; sb += rb_[k]; }
          partial[((size_t)q * gridDim.x + blockIdx.x) * 2 + 0] = sa;
          partial[((size_t)q * gridDim.x + blockIdx.x) * 2 + 1] = sb;
     }
}

// ------------------------------------------------------------------ injection

// add_signal (init.c:365-504) constants, formed on the host in the
// reference's evaluation order
struct SignalParam {
     double sinal, cosal, sindel, cosdel;   // of the source
     double nS0, nS1, nS2;                  // cos a cos d, sin a cos d, sin d
     double amp[4];                         // amplit[] (init.c:411-414)
     double freqo0, freqo1, phaseshift;     // init.c:382-386, 417-418
     double dephase;                        // 2 pi dt fpo (init.c:447)
};

// grid (ceil(N/256), nifo), 256 threads: the signal s_n[i] of detector n
// (init.c:428-456) into s[n*N + i], and per-block sums of s^2 into
// partial[n*gridDim.x + block].  Products and sums are not contracted, as
// in the reference's DOUBLE build (the phase reaches ~1e8 rad).
__global__ void __launch_bounds__(256) k_signal(
     const float *__restrict__ xdat, const double *__restrict__ detssb, const double *__restrict__ cosm,
     const double *__restrict__ sinm, const DetParam *__restrict__ dp, int N, int Nal, SignalParam P,
     double *__restrict__ s, double *__restrict__ partial)
{
     const int d = blockIdx.y;
     const int i = blockIdx.x * 256 + threadIdx.x;
     double v = 0.;
     if (i < N) {
          const DetParam &D = dp[d];
          double aa, bb;
          modvir_at(D, P.sinal, P.cosal, P.sindel, P.cosdel, cosm[i], sinm[i], xdat[(size_t)d * Nal + i], aa, bb);
          const double *e = detssb + (size_t)d * 3 * N + 3 * (size_t)i;
          const double sh = __dadd_rn(__dadd_rn(__dmul_rn(P.nS0, e[0]), __dmul_rn(P.nS1, e[1])), __dmul_rn(P.nS2, e[2]));
          const double di = (double)i;
          // freqo0*(i + sh) + freqo1*(2 sh i + i^2 + sh^2) + phaseshift - dephase*i
          const double q = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(2., sh), di), __dmul_rn(di, di)), __dmul_rn(sh, sh));
          double ph = __dadd_rn(__dadd_rn(__dmul_rn(P.freqo0, __dadd_rn(di, sh)), __dmul_rn(P.freqo1, q)), P.phaseshift);
          ph = __dsub_rn(ph, __dmul_rn(P.dephase, di));
          double sn, cn;
          sincos(ph, &sn, &cn);
          v = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(P.amp[0], aa), cn), __dmul_rn(__dmul_rn(P.amp[1], bb), cn)),
                                  __dmul_rn(__dmul_rn(P.amp[2], aa), sn)),
                        __dmul_rn(__dmul_rn(P.amp[3], bb), sn));
          s[(size_t)d * N + i] = v;
     }
     double v2 = v * v;
#pragma unroll
     for (int o = 16; o > 0; o >>= 1) v2 += __shfl_down_sync(0xffffffffu, v2, o);
     __shared__ double red[8];
     if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v2;
     __syncthreads();
     if (threadIdx.x == 0) {
          double t = 0.;
          for (int k = 0; k < 8; k++) t += red[k];
          partial[(size_t)d * gridDim.x + blockIdx.x] = t;
     }
}

// grid (ceil(N/256), nifo), 256 threads: xDat[i] += h0 s_n[i] where xDat[i]
// != 0, the sum in FP64 and rounded to float once (init.c:468-473)
__global__ void __launch_bounds__(256) k_add_signal(float *__restrict__ xdat, const double *__restrict__ s, int N,
                                                    int Nal, double h0)
{
     const int d = blockIdx.y;
     const int i = blockIdx.x * 256 + threadIdx.x;
     if (i >= N) return;
     float *x = xdat + (size_t)d * Nal + i;
     if (*x != 0.f) *x = (float)__dadd_rn((double)*x, __dmul_rn(h0, s[(size_t)d * N + i]));
}

// one CTA per sky point: aa = sum_n sum_i aa_n^2/sig2_n (jobcore.c:373-386);
// each detector's partials reduced by a fixed tree (reproducible), then
// accumulated over detectors into FLOAT_TYPE as the reference build does.
// grid (npts), 256 threads
__global__ void __launch_bounds__(256) k_sky_sums(const double *__restrict__ partial, int nblk,
                                                  const DetParam *__restrict__ dp, int nifo, AaBb *__restrict__ out)
{
     const int p = blockIdx.x;
     __shared__ double ra[256], rb[256];
     double aa = 0., bb = 0.;
     float aaf = 0.f, bbf = 0.f;
     for (int d = 0; d < nifo; d++) {
          const double *pp = partial + (size_t)(p * nifo + d) * nblk * 2;
          double sa = 0., sb = 0.;
          for (int k = threadIdx.x; k < nblk; k += 256) { sa += pp[2 * k]; sb += pp[2 * k + 1]; }
          ra[threadIdx.x] = sa;
          rb[threadIdx.x] = sb;
          __syncthreads();
          for (int o = 128; o > 0; o >>= 1) {
               if (threadIdx.x < o) {
                    ra[threadIdx.x] += ra[threadIdx.x + o];
                    rb[threadIdx.x] += rb[threadIdx.x + o];
               }
               __syncthreads();
          }
          sa = ra[0];
          sb = rb[0];
          __syncthreads();
          aa += sa / dp[d].sig2;
          bb += sb / dp[d].sig2;
          aaf = (float)((double)aaf + sa / dp[d].sig2);
          bbf = (float)((double)bbf + sb / dp[d].sig2);
     }
     if (threadIdx.x == 0) {
          out[p].aa = aa;
          out[p].bb = bb;
          out[p].aaf = aaf;
          out[p].bbf = bbf;
     }
}

// The natural-spline sweeps (auxi.c:102-115) as blocked recurrences: a
// thread computes a chunk of SPL_K consecutive indices, started SPL_W indices
// early from zero -- both recurrences contract by |0.5*invp| ~ 0.27 per step,
// so the start-up error is below 1e-27 of the values after 48 steps and the
// results are those of one sequential sweep.  A CTA of SPL_T threads stages
// its tile of the inputs (and the warm-up margin) in shared memory with
// per-thread asynchronous copies (all in flight at once); lane j then reads
// index j*SPL_K + r, and one pad word per 16 elements puts the lanes of a
// wavefront on distinct banks.  A thread keeps its SPL_K outputs in
// registers until the whole CTA is done reading the staged inputs, writes
// them over the tile's part of the staging buffer, and the CTA stores the
// tile with consecutive lanes on consecutive indices.
constexpr int SPL_T = 64;                  // threads per CTA
constexpr int SPL_K = 16;                  // indices per thread
constexpr int SPL_W = 48;                  // warm-up steps
constexpr int SPL_TILE = SPL_T * SPL_K;    // indices per CTA
__device__ __forceinline__ int spl_pad(int s) { return s + (s >> 4); }

// Forward sweep (auxi.c:102-111), u[i] for i in [1, n-2] (u[0] = 0).
// grid (ceil(n/SPL_TILE), 2*Q), SPL_T threads
__global__ void __launch_bounds__(SPL_T) k_spline_fwd(const double2 *__restrict__ Z, double2 *__restrict__ U,
                                                      size_t stride, const double *__restrict__ pco, int n)
{
     constexpr int S = SPL_TILE + SPL_W + 2;   // staged samples: [tile0 - W - 1, tile0 + TILE + 1)
     constexpr int P = SPL_TILE + SPL_W;       // staged factors:  [tile0 - W, tile0 + TILE)
     __shared__ __align__(16) double2 ys[S + S / 16 + 1];
     __shared__ __align__(16) double ps[P + P / 16 + 1];
     const int arr = blockIdx.y;
     const double2 *y = Z + (size_t)arr * stride;
     double2 *u = U + (size_t)arr * stride;
     const int tile0 = blockIdx.x * SPL_TILE;
     const int yb = tile0 - SPL_W - 1, pb = tile0 - SPL_W;
     for (int k = threadIdx.x; k < S; k += SPL_T) {
          const int i = yb + k;
          if (i >= 0 && i < n) cp_async16(&ys[spl_pad(k)], &y[i]);
     }
     for (int k = threadIdx.x; k < P; k += SPL_T) {
          const int i = pb + k;
          if (i >= 0 && i < n) cp_async8(&ps[spl_pad(k)], &pco[i]);
     }
     cp_async_wait_all();
     __syncthreads();
     const int lo = tile0 + threadIdx.x * SPL_K;
     const int hi = min(n - 1, lo + SPL_K);
     double2 out[SPL_K];
     if (lo < n) {
          const int i0 = max(1, lo - SPL_W);
          double ur = 0., ui = 0.;
          double2 ym = ys[spl_pad(i0 - 1 - yb)], y0 = ys[spl_pad(i0 - yb)];
          auto step = [&](int i) {
               const double2 yp = ys[spl_pad(i + 1 - yb)];
               const double p = ps[spl_pad(i - pb)];
               const double dr = ym.x - 2. * y0.x + yp.x;
               const double dI = ym.y - 2. * y0.y + yp.y;
               ur = (-.5 * ur + 3. * dr) * p;
               ui = (-.5 * ui + 3. * dI) * p;
               ym = y0;
               y0 = yp;
          };
          for (int i = i0; i < lo; i++) step(i);   // warm-up
#pragma unroll
          for (int r = 0; r < SPL_K; r++) {
               const int i = lo + r;
               out[r] = make_double2(0., 0.);      // u[0] = 0
               if (i >= i0 && i < hi) {
                    step(i);
                    out[r] = make_double2(ur, ui);
               }
          }
     }
     __syncthreads();   // every thread is done with the staged samples
     if (lo < n) {
#pragma unroll
          for (int r = 0; r < SPL_K; r++)
               if (lo + r < hi || lo + r == 0) ys[spl_pad(lo + r - yb)] = out[r];
     }
     __syncthreads();
     for (int k = threadIdx.x; k < SPL_TILE; k += SPL_T) {
          const int i = tile0 + k;
          if (i < n - 1) u[i] = ys[spl_pad(k + SPL_W + 1)];
     }
}

// Back substitution (auxi.c:112-115): y2[n-1] = 0, y2[k] = g[k]*y2[k+1] + u[k];
// a thread's chunk is started SPL_W indices late from y2 = 0.
// grid (ceil(n/SPL_TILE), 2*Q), SPL_T threads
__global__ void __launch_bounds__(SPL_T) k_spline_bwd(const double2 *__restrict__ U, double2 *__restrict__ Y2,
                                                      size_t stride, const double *__restrict__ gco, int n)
{
     constexpr int S = SPL_TILE + SPL_W;       // staged: [tile0, tile0 + TILE + W)
     __shared__ __align__(16) double2 us[S + S / 16 + 1];
     __shared__ __align__(16) double gs[S + S / 16 + 1];
     const int arr = blockIdx.y;
     const double2 *u = U + (size_t)arr * stride;
     double2 *y2 = Y2 + (size_t)arr * stride;
     const int tile0 = blockIdx.x * SPL_TILE;
     for (int k = threadIdx.x; k < S; k += SPL_T) {
          const int i = tile0 + k;
          if (i < n) {
               cp_async16(&us[spl_pad(k)], &u[i]);
               cp_async8(&gs[spl_pad(k)], &gco[i]);
          }
     }
     cp_async_wait_all();
     __syncthreads();
     const int lo = tile0 + threadIdx.x * SPL_K;
     const int hi = min(n, lo + SPL_K);
     double2 out[SPL_K];
     if (lo < n) {
          const int ks = min(n - 1, hi + SPL_W);
          double yr = 0., yi = 0.;
          auto step = [&](int k) {
               const double g = gs[spl_pad(k - tile0)];
               const double2 uk = us[spl_pad(k - tile0)];
               yr = g * yr + uk.x;
               yi = g * yi + uk.y;
          };
          for (int k = ks - 1; k >= hi; k--) step(k);   // warm-up
#pragma unroll
          for (int r = SPL_K - 1; r >= 0; r--) {
               const int k = lo + r;
               out[r] = make_double2(0., 0.);      // y2[n-1] = 0
               if (k < hi && k < ks) {
                    step(k);
                    out[r] = make_double2(yr, yi);
               }
          }
     }
     __syncthreads();   // every thread is done with the staged inputs
     if (lo < n) {
#pragma unroll
          for (int r = 0; r < SPL_K; r++)
               if (lo + r < hi) us[spl_pad(lo + r - tile0)] = out[r];
     }
     __syncthreads();
     for (int k = threadIdx.x; k < SPL_TILE; k += SPL_T) {
          const int i = tile0 + k;
          if (i < n) y2[i] = us[spl_pad(k)];
     }
}

__device__ __forceinline__ double2 splint_eval(const double2 *__restrict__ ya, const double2 *__restrict__ y2a, int n, double x)
{
     if (x < 0 || x > n - 1) return make_double2(0., 0.);
     const int klo = (int)floor(x);
     const int khi = klo + 1;
     const double a = khi - x, b = x - klo;
     const double2 yl = ya[klo], sl = y2a[klo];
     const double2 yh = khi < n ? ya[khi] : make_double2(0., 0.);
     const double2 sh = khi < n ? y2a[khi] : make_double2(0., 0.);
     const double ca = a * a * a - a, cb = b * b * b - b;
     return make_double2(a * yl.x + b * yh.x + (ca * sl.x + cb * sh.x) / 6.0,
                         a * yl.y + b * yh.y + (ca * sl.y + cb * sh.y) / 6.0);
}

// grid (ceil(N/256), Q), 256 threads: xDatm{a,b}[i] = splint(...)/sig2 as
// split (float4 xa.re, xa.im, xb.re, xb.im, interleaved by detector:
// [slot][i][det]) or FP64 (two double2, planar: [slot][det][i]) operands
__global__ void __launch_bounds__(256) k_splint(
     const double2 *__restrict__ Z, const double2 *__restrict__ Y2, size_t stride,
     const double *__restrict__ shftf, int Nal, int N, int n, int interpftpad,
     const DetParam *__restrict__ dp, int nifo,
     float4 *__restrict__ xab, double2 *__restrict__ xa64, double2 *__restrict__ xb64)
{
     const int q = blockIdx.y, p = q / nifo, d = q % nifo;
     const int i = blockIdx.x * 256 + threadIdx.x;
     if (i >= N) return;
     const double x = interpftpad * (i - shftf[(size_t)q * Nal + i]);
     const double2 va = splint_eval(Z + ((size_t)q * 2) * stride, Y2 + ((size_t)q * 2) * stride, n, x);
     const double2 vb = splint_eval(Z + ((size_t)q * 2 + 1) * stride, Y2 + ((size_t)q * 2 + 1) * stride, n, x);
     const double s2 = dp[d].sig2;
     const double2 a = make_double2(va.x / s2, va.y / s2), b = make_double2(vb.x / s2, vb.y / s2);
     if (xab) xab[((size_t)p * Nal + i) * nifo + d] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
     if (xa64) {
          const size_t o = ((size_t)p * nifo + d) * Nal + i;
          xa64[o] = a;
          xb64[o] = b;
     }
}

// ------------------------------------------------------------------ spindown stage

// Neumaier-compensated accumulation of the detector-network sum
struct CompSum {
     float s, c;
     __device__ __forceinline__ void init(float v) { s = v; c = 0.f; }
     __device__ __forceinline__ void add(float x) {
          float t = s + x;
          c += (fabsf(s) >= fabsf(x)) ? ((s - t) + x) : ((x - t) + s);
          s = t;
     }
     __device__ __forceinline__ float value() const { return s + c; }
};

// Split form: phase = het1*i + spnd*i^2 formed and reduced mod 2 pi in FP64,
// plus spnd*(2 i shft_n[i]) in FP32 per detector; FP32 sincos and products.
// The detector-network sum is compensated (Neumaier) for three or more
// detectors; for one or two it is a single rounded addition, which the
// compensation would not change.  Operands planar by detector,
// xab[(slot*nifo + d)*Nal + i] (the layout tdf_fstat_operands_static takes).
struct DemodSplit {
     const float4 *xab;
     const float *s2;
     const TmplParam *tp;
     int N, N2, Nal, nifo;
     static constexpr int kQ = 1;   // elements whose operand loads are issued together

     // x * (cs - i sn) for the two arrays of an operand x = (a.re, a.im, b.re, b.im)
     static __device__ __forceinline__ void rot(const float4 x, float phf, float2 &pa, float2 &pb) {
          float sn, cs;
          __sincosf(phf, &sn, &cs);
          pa = make_float2(fmaf(x.x, cs, x.y * sn), fmaf(x.y, cs, -x.x * sn));
          pb = make_float2(fmaf(x.z, cs, x.w * sn), fmaf(x.w, cs, -x.z * sn));
     }

     template <int L>
     __device__ __forceinline__ void load(float2 (&v)[2][8], int b, int n2, int t) const {
          const TmplParam P = tp[b];
          const float spf = (float)P.spnd;
          const size_t base = (size_t)P.slot * nifo * Nal;
#pragma unroll
          for (int h = 0; h < 8 / kQ; h++) {
               int ii[kQ];
               float pr[kQ];
#pragma unroll
               for (int q = 0; q < kQ; q++) ii[q] = N2 * (t + (kQ * h + q) * (L / 8)) + n2;
               float2 fa[kQ], fb[kQ];
               if (ii[0] >= N) {
                    // zero padding beyond N: the whole group (the tail rows of
                    // every column, uniform across the warp)
#pragma unroll
                    for (int q = 0; q < kQ; q++) {
                         v[0][kQ * h + q] = make_float2(0.f, 0.f);
                         v[1][kQ * h + q] = make_float2(0.f, 0.f);
                    }
                    continue;
               }
#pragma unroll
               for (int q = 0; q < kQ; q++) {
                    const double di = (double)ii[q];
                    const double ph = fma(P.spnd, di * di, P.het1 * di);
                    const double kk = rint(ph * INV_TWO_PI);
                    pr[q] = (float)fma(-kk, TWO_PI, ph);
               }
               if (nifo <= 2) {
                    float4 x0[kQ], x1[kQ];
                    float s0[kQ], s1[kQ];
#pragma unroll
                    for (int q = 0; q < kQ; q++) {
                         const bool ok = ii[q] < N;
                         const size_t o = base + ii[q];
                         x0[q] = ok ? __ldg(&xab[o]) : make_float4(0.f, 0.f, 0.f, 0.f);
                         s0[q] = ok ? __ldg(&s2[o]) : 0.f;
                         const bool ok1 = ok && nifo == 2;
                         x1[q] = ok1 ? __ldg(&xab[o + Nal]) : make_float4(0.f, 0.f, 0.f, 0.f);
                         s1[q] = ok1 ? __ldg(&s2[o + Nal]) : 0.f;
                    }
#pragma unroll
                    for (int q = 0; q < kQ; q++) {
                         if (ii[q] >= N) {
                              fa[q] = make_float2(0.f, 0.f);
                              fb[q] = make_float2(0.f, 0.f);
                              continue;
                         }
                         rot(x0[q], fmaf(spf, s0[q], pr[q]), fa[q], fb[q]);
                         if (nifo == 2) {
                              float2 pa, pb;
                              rot(x1[q], fmaf(spf, s1[q], pr[q]), pa, pb);
                              fa[q] = cadd(fa[q], pa);
                              fb[q] = cadd(fb[q], pb);
                         }
                    }
               } else {
#pragma unroll
                    for (int q = 0; q < kQ; q++) {
                         fa[q] = make_float2(0.f, 0.f);
                         fb[q] = make_float2(0.f, 0.f);
                         if (ii[q] >= N) continue;
                         CompSum ar, ai, br, bi;
                         for (int d = 0; d < nifo; d++) {
                              const size_t o = base + (size_t)d * Nal + ii[q];
                              float2 pa, pb;
                              rot(__ldg(&xab[o]), fmaf(spf, __ldg(&s2[o]), pr[q]), pa, pb);
                              if (d == 0) { ar.init(pa.x); ai.init(pa.y); br.init(pb.x); bi.init(pb.y); }
                              else { ar.add(pa.x); ai.add(pa.y); br.add(pb.x); bi.add(pb.y); }
                         }
                         fa[q] = make_float2(ar.value(), ai.value());
                         fb[q] = make_float2(br.value(), bi.value());
                    }
               }
#pragma unroll
               for (int q = 0; q < kQ; q++) {
                    v[0][kQ * h + q] = fa[q];
                    v[1][kQ * h + q] = fb[q];
               }
          }
     }
};

// Two detectors' demodulated operands summed in one chain of fused
// multiply-adds per component: fa + i... = x0 (c0 - i s0) + x1 (c1 - i s1)
// for the two arrays of x = (a.re, a.im, b.re, b.im).
__device__ __forceinline__ void demod2(const float4 x0, const float4 x1, float ph0, float ph1, float2 &fa,
                                       float2 &fb) {
     float s0, c0, s1, c1;
     __sincosf(ph0, &s0, &c0);
     __sincosf(ph1, &s1, &c1);
     fa.x = fmaf(x0.x, c0, fmaf(x0.y, s0, fmaf(x1.x, c1, x1.y * s1)));
     fa.y = fmaf(x0.y, c0, fmaf(-x0.x, s0, fmaf(x1.y, c1, -x1.x * s1)));
     fb.x = fmaf(x0.z, c0, fmaf(x0.w, s0, fmaf(x1.z, c1, x1.w * s1)));
     fb.y = fmaf(x0.w, c0, fmaf(-x0.z, s0, fmaf(x1.w, c1, -x1.z * s1)));
}

// DemodSplit over operands interleaved by detector, xab[(slot*Nal + i)*nifo
// + d] and s2 likewise (the engine's layout): with two detectors a sample's
// operands are two adjacent 16-byte words and one 8-byte word, each read
// from one address, and one pointer per operand array steps through the
// thread's samples.  Same arithmetic, in the same order, as DemodSplit.
// CN2 / CNIFO > 0 fix the row length N2 and the detector count at compile
// time (the thread's eight samples are then constant offsets from one
// pointer); 0 reads them from the struct.
template <int CN2 = 0, int CNIFO = 0>
struct DemodSplitILT {
     const float4 *xab;
     const float *s2;
     const TmplParam *tp;
     int N, N2, Nal, nifo;

     template <int L>
     __device__ __forceinline__ void load(float2 (&v)[2][8], int b, int n2, int t) const {
          const int n2s = CN2 > 0 ? CN2 : N2;
          const int nf = CNIFO > 0 ? CNIFO : nifo;
          const TmplParam P = tp[b];
          const float spf = (float)P.spnd;
          const int i0 = n2s * t + n2;
          const int di = n2s * (L / 8);   // samples between the thread's elements
          const int de = di * nf;         // operand words between them
          const size_t e0 = ((size_t)P.slot * Nal + i0) * nf;
          const float4 *xp = xab + e0;
          const float *sp = s2 + e0;
#pragma unroll
          for (int m = 0; m < 8; m++) {
               const int i = i0 + m * di;
               float2 fa = make_float2(0.f, 0.f), fb = make_float2(0.f, 0.f);
               if (i < N) {
                    const double dd = (double)i;
                    const double ph = fma(P.spnd, dd * dd, P.het1 * dd);
                    const double kk = rint(ph * INV_TWO_PI);
                    const float pr = (float)fma(-kk, TWO_PI, ph);
                    const float4 *x = xp + m * de;
                    const float *s = sp + m * de;
                    if (nf == 2) {
                         // both detectors' rotated operands summed in one
                         // chain of fused multiply-adds per component
                         const float2 ss = __ldg(reinterpret_cast<const float2 *>(s));
                         demod2(__ldg(x), __ldg(x + 1), fmaf(spf, ss.x, pr), fmaf(spf, ss.y, pr), fa, fb);
                    } else if (nf == 1) {
                         DemodSplit::rot(__ldg(x), fmaf(spf, __ldg(s), pr), fa, fb);
                    } else {
                         CompSum ar, ai, br, bi;
                         for (int d = 0; d < nf; d++) {
                              float2 pa, pb;
                              DemodSplit::rot(__ldg(x + d), fmaf(spf, __ldg(s + d), pr), pa, pb);
                              if (d == 0) { ar.init(pa.x); ai.init(pa.y); br.init(pb.x); bi.init(pb.y); }
                              else { ar.add(pa.x); ai.add(pa.y); br.add(pb.x); bi.add(pb.y); }
                         }
                         fa = make_float2(ar.value(), ai.value());
                         fb = make_float2(br.value(), bi.value());
                    }
               }
               v[0][m] = fa;
               v[1][m] = fb;
          }
     }
};
using DemodSplitIL = DemodSplitILT<0, 0>;

// DemodSplitIL with its operands brought in by TMA.  Thread (c, t) of the CTA
// needs, for element m, the samples of row n1 = t + m*R (R = L/8) of column
// n2 = x0 + c, so the rows of a group m of the CTA's LINES columns, every
// detector, form one box of each operand tensor (interleaved layout):
//   xab as floats {4*nifo*N2, rows, slots}, box {4*nifo*LINES, R, 1}
//   s2            {nifo*N2,   rows, slots}, box {nifo*LINES,   R, 1}
// (rows = Nal/N2, Nal a multiple of N2).  The groups holding samples < N go
// through a ring of `stages` shared-memory slots that aliases the line
// buffers (unused until the first FFT pass stores), each slot completing on
// its own mbarrier; all copies of the ring are in flight while the threads
// demodulate, instead of one element's loads per thread at a time.
// The arithmetic per element is DemodSplit's, in the same order.
// Opt-in (TDF_STAGED_OPERANDS=1): with the operands L2-resident it measured
// slower than DemodSplitIL's per-thread loads.
struct DemodSplitStaged {
     CUtensorMap mx;    // xab
     CUtensorMap ms;    // s2
     const TmplParam *tp;
     unsigned *err;     // ERR_STAGE_TIMEOUT is or-ed in when a wait gives up
     int N, N2, nifo;
     int groups;        // row groups holding samples < N (<= 8)
     int stages;        // ring slots (>= 1)
     unsigned bar_off;  // byte offset of the ring's mbarriers in dynamic shared memory
     unsigned smem;     // dynamic shared memory of the launch
     static constexpr bool kStaged = true;

     template <int L>
     __device__ __forceinline__ void issue(int g, int s, unsigned char *ring, uint64_t *bars, unsigned slot_bytes,
                                           unsigned xbytes, int x0, int w) const {
          unsigned char *dst = ring + (size_t)s * slot_bytes;
          mbar_expect_tx(&bars[s], slot_bytes);
          tma_load_3d(dst, &mx, 4 * nifo * x0, g * (L / 8), w, &bars[s]);
          tma_load_3d(dst + xbytes, &ms, nifo * x0, g * (L / 8), w, &bars[s]);
     }

     template <int L>
     __device__ __forceinline__ void load_staged(float2 (&v)[2][8], int b, int n2, int t, unsigned char *ring,
                                                 uint64_t *bars) const {
          constexpr int R = L / 8;
          const TmplParam P = tp[b];
          const float spf = (float)P.spnd;
          const unsigned xbytes = (unsigned)nifo * R * LINES * 16;
          const unsigned slot_bytes = xbytes + (unsigned)nifo * R * LINES * 4;
          const int x0 = blockIdx.x * LINES;
          const int c = threadIdx.x % LINES;
          if (threadIdx.x == 0) {
               for (int s = 0; s < stages; s++) mbar_init(&bars[s], 1);
               mbar_fence_init();
          }
          __syncthreads();
          if (threadIdx.x == 0)
               for (int g = 0; g < stages; g++) issue<L>(g, g, ring, bars, slot_bytes, xbytes, x0, (int)P.slot);
          bool waited = true;
          int s = 0;            // ring slot of group m
          unsigned par = 0u;    // phase parity of that slot's barrier
#pragma unroll
          for (int m = 0; m < 8; m++) {
               float2 fa = make_float2(0.f, 0.f), fb = make_float2(0.f, 0.f);
               if (m < groups) {
                    waited &= mbar_wait(&bars[s], par);
                    const unsigned char *sl = ring + (size_t)s * slot_bytes;
                    const float4 *X = reinterpret_cast<const float4 *>(sl);
                    const float *S2 = reinterpret_cast<const float *>(sl + xbytes);
                    const int i = N2 * (t + m * R) + n2;
                    if (i < N) {
                         const double di = (double)i;
                         const double ph = fma(P.spnd, di * di, P.het1 * di);
                         const double kk = rint(ph * INV_TWO_PI);
                         const float pr = (float)fma(-kk, TWO_PI, ph);
                         const int e0 = (t * LINES + c) * nifo;
                         if (nifo == 2) {
                              demod2(X[e0], X[e0 + 1], fmaf(spf, S2[e0], pr), fmaf(spf, S2[e0 + 1], pr), fa, fb);
                         } else if (nifo == 1) {
                              DemodSplit::rot(X[e0], fmaf(spf, S2[e0], pr), fa, fb);
                         } else {
                              CompSum ar, ai, br, bi;
                              for (int d = 0; d < nifo; d++) {
                                   const int ed = e0 + d;
                                   float2 pa, pb;
                                   DemodSplit::rot(X[ed], fmaf(spf, S2[ed], pr), pa, pb);
                                   if (d == 0) { ar.init(pa.x); ai.init(pa.y); br.init(pb.x); bi.init(pb.y); }
                                   else { ar.add(pa.x); ai.add(pa.y); br.add(pb.x); bi.add(pb.y); }
                              }
                              fa = make_float2(ar.value(), ai.value());
                              fb = make_float2(br.value(), bi.value());
                         }
                    }
                    if (m + stages < groups) {
                         // every thread is done with slot s: refill it
                         __syncthreads();
                         if (threadIdx.x == 0)
                              issue<L>(m + stages, s, ring, bars, slot_bytes, xbytes, x0, (int)P.slot);
                    }
                    if (++s == stages) {
                         s = 0;
                         par ^= 1u;
                    }
               }
               v[0][m] = fa;
               v[1][m] = fb;
          }
          if (!waited) atomicOr(err, ERR_STAGE_TIMEOUT);
     }
};

// Plain FP64 form: the reference's DOUBLE-build spindown_modulation.
struct DemodFP64 {
     const double2 *xa, *xb;
     const double *t1;
     const TmplParam *tp;
     int N, N2, Nal, nifo;
     template <int L>
     __device__ __forceinline__ void load(double2 (&v)[2][8], int b, int n2, int t) const {
          const TmplParam P = tp[b];
          const size_t base = (size_t)P.slot * nifo * Nal;
#pragma unroll
          for (int m = 0; m < 8; m++) {
               const int i = N2 * (t + m * (L / 8)) + n2;
               double2 fa = make_double2(0., 0.), fb = make_double2(0., 0.);
               if (i < N) {
                    for (int d = 0; d < nifo; d++) {
                         const size_t o = base + (size_t)d * Nal + i;
                         const double phase = __dadd_rn(__dmul_rn(P.het1, (double)i), __dmul_rn(P.spnd, __ldg(&t1[o])));
                         double sn, cs;
                         sincos(phase, &sn, &cs);
                         const double2 x = __ldg(&xa[o]), y = __ldg(&xb[o]);
                         const double er = cs, ei = -sn;
                         fa.x += x.x * er - x.y * ei;
                         fa.y += x.x * ei + x.y * er;
                         fb.x += y.x * er - y.y * ei;
                         fb.y += y.x * ei + y.y * er;
                    }
               }
               v[0][m] = fa;
               v[1][m] = fb;
          }
     }
};

template <typename T> __device__ __forceinline__ T aa_of(const AaBb &ab);
template <> __device__ __forceinline__ float aa_of<float>(const AaBb &ab) { return ab.aaf; }
template <> __device__ __forceinline__ double aa_of<double>(const AaBb &ab) { return ab.aa; }
template <typename T> __device__ __forceinline__ T bb_of(const AaBb &ab);
template <> __device__ __forceinline__ float bb_of<float>(const AaBb &ab) { return ab.bbf; }
template <> __device__ __forceinline__ double bb_of<double>(const AaBb &ab) { return ab.bb; }

// Row-pass epilogue of the spindown FFT: F[k] over [fr0, fr1].  With a
// candidate list (cand != nullptr) it also appends every bin of the MAX_ALG 3
// loop range [fr0+1, fr1-2] whose F passes the threshold test, so that the
// local-maximum rule only has to look at those bins afterwards.
template <typename T>
struct StoreFstat {
     T *F;
     const TmplParam *tp;
     const AaBb *ab;
     int nF, fr0, fr1, N1;
     double thr;
     uint2 *cand;
     unsigned *cand_cnt;
     unsigned cand_cap;
     int boff;        // index of this chunk's first template within its resolve group
     template <int L>
     __device__ __forceinline__ void store(const cx<T> (&v)[2][8], int b, int k1, int t) const {
          const AaBb s = ab[tp[b].slot];
          const T aa = aa_of<T>(s), bb = bb_of<T>(s);
          T *dst = F + (size_t)b * nF - fr0;
#pragma unroll
          for (int m = 0; m < 8; m++) {
               const int k = k1 + N1 * (t + m * (L / 8));
               if (k >= fr0 && k <= fr1) {
                    const T f = cnorm(v[0][m]) / aa + cnorm(v[1][m]) / bb;
                    dst[k] = f;
                    if (cand && !(f < thr) && k >= fr0 + 1 && k < fr1 - 1) {
                         const unsigned c = atomicAdd(cand_cnt, 1u);
                         if (c < cand_cap) cand[c] = make_uint2((unsigned)(b + boff), (unsigned)k);
                    }
               }
          }
     }
};

// Candidate records of the sparse F store (16 bytes): template (within the
// resolve group) | kind << 24, bin, F[bin], and one neighbour's F.
constexpr unsigned CAND_LOCAL = 0u;   // a local maximum decided in the row pass; no tie with bin-1
constexpr unsigned CAND_LEFT = 1u;    // first bin of a CTA's run of 8: F[bin-1] is in the edge ring (nb = F[bin+1])
constexpr unsigned CAND_RIGHT = 2u;   // last bin of a run: F[bin+1] is in the edge ring (nb = F[bin-1])
constexpr unsigned CAND_TIE = 3u;     // F[bin-1] == F[bin]: the MAX_ALG 3 run needs F[bin-2]
constexpr unsigned ERR_NEED_FULL_F = 4u;   // a batch needs the full F spectra (tie or candidate overflow)

// StoreFstat for the split form with the four-step column count N1 fixed at
// compile time (CN1 > 0, else the struct's N1) and, when HALF, only the
// outputs k2 < L/2 of each row formed: every bin the search keeps lies below
// nfftf/2 (fr1 < N1*L/2), so the upper half of the row transform's last
// pass is never computed (its outputs are dead).  F = |Fa|^2 * (1/aa) +
// |Fb|^2 * (1/bb), the reciprocals formed once per thread.
//
// Two ways to hand F to the trigger selection:
//   full (E == nullptr): the whole spectrum [fr0, fr1] goes to the F ring
//     and the bins passing the threshold test to the candidate list (uint2
//     {template, bin}); used with blocks_avg and as the fallback.
//   sparse (E != nullptr): no spectrum leaves the SM.  The 8 lanes c of a
//     thread group hold the consecutive bins k1b + c + N1*k2 of one k2, so a
//     bin's neighbours are one shuffle away except at the run's ends: the
//     row pass decides the local-maximum test itself for c = 1..6 and
//     writes candidate records (uint4, kinds above) for bins passing the
//     threshold; only the end bins c = 0 and 7 of every run go to the edge
//     ring E[((b*NJ + j)*L + k2)*2 + (c == 7)] (j = CTA index) for the
//     neighbours of the other CTAs' end-bin candidates.
template <int CN1, bool HALF>
struct StoreFstatT {
     float *F;
     const TmplParam *tp;
     const AaBb *ab;
     int nF, fr0, fr1, N1;
     double thr;
     uint2 *cand;
     unsigned *cand_cnt;
     unsigned cand_cap;
     int boff;        // index of this chunk's first template within its resolve group
     float *E = nullptr;       // sparse form: edge ring of the resolve group
     uint4 *scand = nullptr;   // sparse form: candidate records
     template <int L>
     __device__ __forceinline__ void store(const float2 (&v)[2][8], int b, int k1, int t) const {
          const AaBb s = ab[tp[b].slot];
          const float ia = 1.f / s.aaf, ib = 1.f / s.bbf;
          const float thrf = (float)thr;
          const bool exact_thr = (double)thrf == thr;   // then f < thr compares the same in float
          const int n1 = CN1 > 0 ? CN1 : N1;
          if (E == nullptr) {
               float *dst = F + (size_t)b * nF - fr0;
#pragma unroll
               for (int m = 0; m < (HALF ? 4 : 8); m++) {
                    const int k = k1 + n1 * (t + m * (L / 8));
                    if (k >= fr0 && k <= fr1) {
                         const float f = fmaf(cnorm(v[0][m]), ia, cnorm(v[1][m]) * ib);
                         dst[k] = f;
                         const bool pass = exact_thr ? !(f < thrf) : !((double)f < thr);
                         if (cand && pass && k >= fr0 + 1 && k < fr1 - 1) {
                              const unsigned c = atomicAdd(cand_cnt, 1u);
                              if (c < cand_cap) cand[c] = make_uint2((unsigned)(b + boff), (unsigned)k);
                         }
                    }
               }
               return;
          }
          const int c = k1 & (LINES - 1);
          const int nj = n1 / LINES;
          const unsigned bg = (unsigned)(b + boff);
          float *ej = E + ((size_t)bg * nj + (k1 >> 3)) * (2 * L) + (c == LINES - 1 ? 1 : 0);
#pragma unroll
          for (int m = 0; m < (HALF ? 4 : 8); m++) {
               const int k2 = t + m * (L / 8);
               const int k = k1 + n1 * k2;
               const float f = fmaf(cnorm(v[0][m]), ia, cnorm(v[1][m]) * ib);
               // neighbours within the run of 8 (lanes c-1, c+1 of the same k2)
               const float fm = __shfl_up_sync(0xffffffffu, f, 1, LINES);
               const float fp = __shfl_down_sync(0xffffffffu, f, 1, LINES);
               if (k >= fr0 && k <= fr1) {
                    if (c == 0 || c == LINES - 1) ej[2 * k2] = f;
                    const bool pass = exact_thr ? !(f < thrf) : !((double)f < thr);
                    if (pass && k >= fr0 + 1 && k < fr1 - 1) {
                         unsigned kind;
                         float nb = 0.f;
                         bool keep = true;
                         if (c == 0) {
                              kind = CAND_LEFT;
                              nb = fp;
                         } else if (c == LINES - 1) {
                              kind = CAND_RIGHT;
                              nb = fm;
                         } else {
                              keep = !(fm > f || f < fp);   // a local maximum
                              kind = fm == f ? CAND_TIE : CAND_LOCAL;
                         }
                         if (keep) {
                              const unsigned q = atomicAdd(cand_cnt, 1u);
                              if (q < cand_cap)
                                   scand[q] = make_uint4(bg | (kind << 24), (unsigned)k, __float_as_uint(f),
                                                         __float_as_uint(nb));
                         }
                    }
               }
          }
     }
};

// blocks_avg means (auxi.c:349-355): mu_j = sum of the j-th block of NAV
// values of F[fr0..] / (2 NAV).  grid (nblk, ntmpl), 256 threads
template <typename T>
__global__ void k_block_means(const T *__restrict__ F, int nF, int nblk, T *__restrict__ mu)
{
     const int j = blockIdx.x, b = blockIdx.y;
     const T *src = F + (size_t)b * nF + (size_t)j * 4096;
     T s = 0;
     for (int k = threadIdx.x; k < 4096; k += 256) s += src[k];
     __shared__ T red[256];
     red[threadIdx.x] = s;
     __syncthreads();
     for (int o = 128; o > 0; o >>= 1) {
          if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
          __syncthreads();
     }
     if (threadIdx.x == 0) mu[(size_t)b * nblk + j] = (T)(red[0] / (2. * 4096));
}

template <typename T>
__device__ __forceinline__ T fval(const T *Fb, const T *mub, int k, int fr0, int nblk) {
     T f = Fb[k];
     if (mub) {
          const int r = k - fr0;
          if (r < nblk * 4096) f = f / mub[r >> 12];
     }
     return f;
}

template <typename T>
__device__ __forceinline__ bool is_peak(const T *Fb, const T *mub, int k, int fr0, int nblk, double thr) {
     const T f = fval(Fb, mub, k, fr0, nblk);
     return !(f < thr || fval(Fb, mub, k - 1, fr0, nblk) > f || f < fval(Fb, mub, k + 1, fr0, nblk));
}

struct ThrArgs {
     int nF, fr0, fr1;
     double thr;
     int nblk;
     const TmplParam *tp;
     int nfftf;
     const double *lines;
     int numlines;
     unsigned bufhalf;
     Trig *trig;
     unsigned long long cap;
     unsigned long long *cnt;
     unsigned *tcnt;
     unsigned *err;
};

// Appends the trigger at bin i of template b (group-relative) with F value
// Fc: its frequency (jobcore.c:571) in the emulated build's arithmetic, the
// veto intervals (jobcore.c:575-583), the per-template count against
// bufsize/2 (jobcore.c:586-590), then the compacted trigger list.
template <bool FP64>
__device__ __forceinline__ void emit_trigger(const ThrArgs &A, int b, int i, double Fc)
{
     const TmplParam P = A.tp[b];
     double fcmp;
     float ff;
     if (FP64) {
          // FLOAT_TYPE = double: f_ = (double)(2ic)/(double)nfftf*M_PI + sgnl0
          const double f_ = __dadd_rn(__dmul_rn(__ddiv_rn((double)(2 * i), (double)A.nfftf), M_PI_D), P.sgnl0);
          fcmp = f_;
          ff = (float)f_;
     } else {
          // FLOAT_TYPE = float: the quotient in float, the product and sum in
          // double, stored to float
          const float qf = __fdiv_rn((float)(2 * i), (float)A.nfftf);
          ff = (float)__dadd_rn(__dmul_rn((double)qf, M_PI_D), P.sgnl0);
          fcmp = (double)ff;
     }
     for (int k = 0; k < A.numlines; k++)
          if (fcmp >= A.lines[2 * k] && fcmp <= A.lines[2 * k + 1]) return;
     const unsigned c = atomicAdd(&A.tcnt[b], 1u);
     if (c >= A.bufhalf) {
          atomicOr(A.err, ERR_OVERFLOW);
          return;
     }
     const unsigned long long g = atomicAdd(A.cnt, 1ull);
     if (g < A.cap) {
          Trig r;
          r.id = P.id;
          r.bin = (uint32_t)i;
          r.f = ff;
          r.F = (float)Fc;
          A.trig[g] = r;
     }
}

// MAX_ALG 3 (jobcore.c:556-603) as the single-threaded loop executes it:
// bin i (fr0 < i < fr1-1) is a trigger when it is a local maximum >= thr
// and the previous accepted bin is not i-1 (the loop's "i++" skip), i.e.
// when the run of consecutive local-maximum bins ending at i-1 has even
// length.  Then the veto intervals are checked and the trigger appended.
template <typename T, bool FP64>
__device__ __forceinline__ void threshold_bin(const T *__restrict__ F, const T *__restrict__ mu, const ThrArgs &A,
                                              int b, int i)
{
     const int fr0 = A.fr0, nblk = A.nblk;
     const double thr = A.thr;
     const T *Fb = F + (size_t)b * A.nF - fr0;
     const T *mub = mu ? mu + (size_t)b * nblk : nullptr;
     if (!is_peak(Fb, mub, i, fr0, nblk, thr)) return;
     int run = 0;
     for (int k = i - 1; k >= fr0 + 1 && is_peak(Fb, mub, k, fr0, nblk, thr); k--) run++;
     if (run & 1) return;
     emit_trigger<FP64>(A, b, i, (double)fval(Fb, mub, i, fr0, nblk));
}

// The candidates the row pass collected; when the list overflowed, every
// bin of the chunk (grid-stride).  grid (G), 256 threads
template <typename T, bool FP64>
__global__ void __launch_bounds__(256) k_resolve(const T *__restrict__ F, ThrArgs A, const uint2 *__restrict__ cand,
                                                 const unsigned *__restrict__ cand_cnt, unsigned cand_cap, int nt)
{
     const unsigned n = *cand_cnt;
     const unsigned gs = gridDim.x * blockDim.x;
     const unsigned g0 = blockIdx.x * blockDim.x + threadIdx.x;
     if (n <= cand_cap) {
          for (unsigned c = g0; c < n; c += gs) {
               const uint2 q = cand[c];
               threshold_bin<T, FP64>(F, nullptr, A, (int)q.x, (int)q.y);
          }
     } else {
          const unsigned nb = (unsigned)(A.fr1 - A.fr0 - 2 > 0 ? A.fr1 - A.fr0 - 2 : 0);   // bins fr0+1 .. fr1-2
          for (unsigned long long x = g0; x < (unsigned long long)nt * nb; x += gs)
               threshold_bin<T, FP64>(F, nullptr, A, (int)(x / nb), A.fr0 + 1 + (int)(x % nb));
     }
}

// Trigger selection from the sparse F store's candidate records: the
// missing neighbour of a run's end bin from the edge ring, the local-maximum
// test, and the trigger append.  A record whose MAX_ALG 3 run needs more of
// the spectrum (a tie with the previous bin), or a candidate list that
// overflowed, sets ERR_NEED_FULL_F: the host then reruns the batch with the
// full F store.  grid (G), 256 threads
struct SparseArgs {
     const float *E;
     const uint4 *cand;
     const unsigned *cand_cnt;
     unsigned cand_cap;
     int N1, L;       // four-step column count and row length
};

__global__ void __launch_bounds__(256) k_resolve_sparse(ThrArgs A, SparseArgs S)
{
     const unsigned n = *S.cand_cnt;
     if (n > S.cand_cap) {
          if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(A.err, ERR_NEED_FULL_F);
          return;
     }
     const unsigned gs = gridDim.x * blockDim.x;
     const int nj = S.N1 / LINES;
     for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gs) {
          const uint4 r = S.cand[i];
          const int b = (int)(r.x & 0xffffffu);
          const unsigned kind = r.x >> 24;
          const int k = (int)r.y;
          const float f = __uint_as_float(r.z);
          if (kind == CAND_TIE) {
               atomicOr(A.err, ERR_NEED_FULL_F);
               continue;
          }
          if (kind != CAND_LOCAL) {
               const int k1 = k % S.N1, k2 = k / S.N1, j = k1 / LINES;
               const float *Eb = S.E + (size_t)b * nj * (2 * S.L);
               float fm, fp;
               if (kind == CAND_LEFT) {
                    // bin k-1: the last bin of the previous CTA's run (or of the last CTA's at k2-1)
                    fm = j > 0 ? Eb[((size_t)(j - 1) * S.L + k2) * 2 + 1] : Eb[((size_t)(nj - 1) * S.L + (k2 - 1)) * 2 + 1];
                    fp = __uint_as_float(r.w);
               } else {
                    // bin k+1: the first bin of the next CTA's run (or of the first CTA's at k2+1)
                    fp = j < nj - 1 ? Eb[((size_t)(j + 1) * S.L + k2) * 2] : Eb[((size_t)k2 + 1) * 2];
                    fm = __uint_as_float(r.w);
               }
               if (fm > f || f < fp) continue;   // not a local maximum
               if (fm == f) {
                    atomicOr(A.err, ERR_NEED_FULL_F);
                    continue;
               }
          }
          emit_trigger<false>(A, b, k, (double)f);
     }
}

// Full scan of every bin (used with the blocks_avg normalisation).
// grid (ceil((fr1-fr0+1)/256), ntmpl), 256 threads
template <typename T, bool FP64>
__global__ void __launch_bounds__(256) k_threshold(const T *__restrict__ F, const T *__restrict__ mu, ThrArgs A)
{
     const int b = blockIdx.y;
     const int i = A.fr0 + blockIdx.x * 256 + threadIdx.x;
     if (i < A.fr0 + 1 || i >= A.fr1 - 1) return;
     threshold_bin<T, FP64>(F, mu, A, b, i);
}

}  // namespace tdf
