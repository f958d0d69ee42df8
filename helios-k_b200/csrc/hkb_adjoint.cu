// hkb_adjoint.cu -- vector-Jacobian product of the opacity (sm_100a).
//
// Given one state (T, P) and a seed u_i = dLoss/dK_i on the grid, computes
//   dLoss/dT, dLoss/dP, and per line dLoss/dlog S_l and dLoss/dgammaL_l
// (gammaL: the line's Lorentz half-width at the state).  No counterpart in
// the reference, which has no derivatives; the forward it differentiates is
// the Voigt sum of voigt.h:1177-1816 (regions A, B, C) as restated by the
// forward kernels of this library.
//
// A line contributes c_li = (S^/sqrt(pi)) V^(x_li, y_l) to K_i, with
// S^ = S(T) / alphaD (LineState.S), x = (nu_i - nu_l) / alphaD,
// y = gammaL / alphaD and V^ the region's shape (region C: Algorithm 916;
// B: y/sqrt(pi) GH2; A: y/sqrt(pi) / (x^2 + y^2); profiles 2-4 are their
// region-A shape over the whole window: Lorentz, Doppler, binned Gaussian,
// the last two in the FP64 form whatever the precision asked for).  Pass 1 recomputes the forward per (grid
// tile, line) -- nothing of the forward is stored -- and reduces four sums
// per line:
//   G_S = sum_i u_i c_li,         G_y = sum_i u_i dc/dy,
//   G_x = sum_i u_i dc/dx x_li,   G_n = sum_i u_i dc/dx,
// so that dLoss/dlog S^ = G_S, dLoss/dy = G_y, dLoss/d(1/alphaD) at fixed y
// = G_x alphaD and dLoss/dnu_l = -G_n / alphaD.  Pass 2 (adjoint_line_kernel)
// applies the chain rule of the line scaling (prep_line) to T and P.
// Plain form: pass 1 is adjoint_tile_kernel, FP64 for all regions.  Mixed
// form: pass 1 is adjoint_ab_kernel (regions A and B in FP32, x from the
// FP64 offset, the far field as per-block series), then adjoint_c_kernel
// takes region C in FP32 (voigt_c_grad_f: the asymptotic series of w and
// dw/dz, the differentiated Algorithm-916 series) before pass 2; the sums
// are FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "hkb_device.cuh"
#include "hkb_kernels.h"

namespace hkb {

constexpr int AD_THREADS = 256;
constexpr int AD_WARPS = AD_THREADS / 32;
constexpr int AD_G = 2048;  // grid points per tile

// first index in [0, n) with a[idx] >= v (n if none); all 32 lanes call it
__device__ int64_t ad_lower_bound_warp(const double *__restrict__ a, int64_t n, double v) {
  const int lane = threadIdx.x & 31;
  int64_t lo = 0, hi = n;
  while (hi - lo > 32) {
    const int64_t span = hi - lo;
    const int64_t pos = lo + ((int64_t)(lane + 1) * span) / 33;
    const unsigned m = __ballot_sync(0xffffffffu, a[pos] >= v);
    if (m == 0u) {
      lo = lo + (32 * span) / 33 + 1;
    } else {
      const int f = __ffs(m) - 1;
      const int64_t nh = lo + ((int64_t)(f + 1) * span) / 33;
      const int64_t nl = (f == 0) ? lo : lo + ((int64_t)f * span) / 33 + 1;
      lo = nl;
      hi = nh;
    }
  }
  const int64_t pos = lo + lane;
  const unsigned m = __ballot_sync(0xffffffffu, (pos < hi) && (a[pos] < v));
  return lo + __popc(m);
}

// Per (line, point): dc/dx and dc/dy (and c) for regions A and B in the
// working precision F, with Sp = S^/pi.
template <class F>
__device__ __forceinline__ void ab_terms(bool regionB, F x, F y, double Sp, double &c,
                                         double &cx, double &cy) {
  const F s = x * x, Y = y * y;
  F t, ts, tY;
  if (regionB) {
    gh2_grad<F>(s, Y, t, ts, tY);
  } else {
    t = F(1) / (s + Y);
    ts = -t * t;
    tY = ts;
  }
  // c = Sp y t;  dc/dx = Sp y t_s 2x;  dc/dy = Sp (t + y t_Y 2y)
  c = Sp * (double)(y * t);
  cx = Sp * (double)(y * ts * F(2) * x);
  cy = Sp * (double)(t + F(2) * Y * tY);
}

// Profiles 3-4 (region A only, FP64): the shape with its S1 and dc/dx,
// dc/dvb (vb = dnu iad, the grid step in Doppler units).  Doppler: S1
// e^{-x^2}.  Binned Gaussian: S1 (erf(x+h) - erf(x-h)) / (2 vb), h = vb/2; its
// two exponentials come from the larger one, e^{-(|x|-h)^2}, so neither their
// difference nor their sum cancels or overflows.
__device__ __forceinline__ void profile34_grad_d(int profile, double x, double S1, double vb,
                                                 double &c, double &cx, double &cvb) {
  if (profile == 3) {
    c = S1 * exp(-(x * x));
    cx = -2.0 * x * c;
    cvb = 0.0;
    return;
  }
  const double isp = 0.56418958354775628695;  // 1/sqrt(pi)
  const double h = 0.5 * vb, ax = fabs(x), sx = x < 0.0 ? -1.0 : 1.0;
  const double D = erf_diff(x + h, x - h);
  const double Eb = exp(-(ax - h) * (ax - h));
  const double dE = sx * Eb * expm1(-4.0 * ax * h);    // e^{-(x+h)^2} - e^{-(x-h)^2}
  const double sE = Eb * (1.0 + exp(-4.0 * ax * h));   // e^{-(x+h)^2} + e^{-(x-h)^2}
  const double k = S1 / (2.0 * vb);
  c = k * D;
  cx = k * (2.0 * isp) * dE;
  cvb = k * (sE * isp - D / vb);
}

// Region B of the mixed form in FP32: the GH2 shape t and dt/ds, dt/dY with
// one reciprocal (gh2_grad divides three times).  Region A needs no helper:
// t = 1/(s + Y), dt/ds = dt/dY = -t^2.
__device__ __forceinline__ void gh2_grad_f(float s, float Y, float &t, float &ts, float &tY) {
  const float u = s + Y;
  const float a1 = u + 1.5f;
  const float c4 = (float)(4.0 / CUDART_PI), c6 = (float)(6.0 / CUDART_PI);
  const float num = fmaf(a1, u + 1.0f, -c4 * s);
  const float q = fmaf(a1, a1, -c6 * s);
  const float rden = rcp_fast(u * q);
  t = num * rden;
  const float num_s = (u + 1.0f) + a1 - c4, num_Y = (u + 1.0f) + a1;
  const float den_s = fmaf(u, 2.0f * a1 - c6, q), den_Y = fmaf(u, 2.0f * a1, q);
  ts = fmaf(-t, den_s, num_s) * rden;
  tY = fmaf(-t, den_Y, num_Y) * rden;
}

// Plain form, FP64 throughout.  Tickets are (tile, part): a tile's line
// range is cut into nsplit parts so that a grid of a few hundred tiles
// still fills the GPU; the per-line sums go to G through FP64 atomics.
__global__ void __launch_bounds__(AD_THREADS, 2)
adjoint_tile_kernel(const LinePrep *__restrict__ P, const double *__restrict__ nu0, int64_t nlines,
                    GridDev g, const StateDev *__restrict__ states, int ntiles, int nsplit,
                    unsigned *__restrict__ ticket, const double *__restrict__ u,
                    double *__restrict__ G) {
  __shared__ double su[AD_G];
  __shared__ int s_t;
  __shared__ long long s_L0, s_L1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const StateDev &st = states[0];
  const double isp = 0.56418958354775628695;  // 1/sqrt(pi)
  const int ntickets = ntiles * nsplit;
  for (;;) {
    if (tid == 0) s_t = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int t = s_t;
    if (t >= ntickets) break;
    const int tile = t / nsplit, part = t - tile * nsplit;
    const int64_t g0 = (int64_t)tile * AD_G;
    const int64_t g1 = min(g0 + (int64_t)AD_G, g.nx);
    for (int k = tid; k < AD_G; k += AD_THREADS) su[k] = (g0 + k < g1) ? u[g0 + k] : 0.0;
    if (warp == 0) {
      const double W = st.wmax + st.shift + 2.0 * g.dnu;
      const double xlo = grid_x(g, g0) - W, xhi = grid_x(g, g1 - 1) + W;
      const double pad = 1e-12 * (fabs(xlo) + fabs(xhi)) + 1e-300;
      const int64_t L0 = ad_lower_bound_warp(nu0, nlines, xlo - pad);
      const int64_t L1 = ad_lower_bound_warp(nu0, nlines, xhi + pad);
      if (lane == 0) {
        s_L0 = L0 + (L1 - L0) * part / nsplit;
        s_L1 = L0 + (L1 - L0) * (part + 1) / nsplit;
      }
    }
    __syncthreads();
    const int64_t L0 = s_L0, L1 = s_L1;
    for (int64_t l = L0 + warp; l < L1; l += AD_WARPS) {
      const LinePrep lp = P[l];
      const int64_t lo = max((int64_t)lp.i0, g0), hi = min((int64_t)lp.i1, g1);
      if (lo >= hi || lp.Sc == 0.0) continue;
      const double Sp = lp.Sc * isp;  // S^/pi
      double gS = 0.0, gy = 0.0, gx = 0.0, gn = 0.0;
      const double vbl = g.dnu * lp.iad;
      for (int64_t k = lo + lane; k < hi; k += 32) {
        const double uk = su[k - g0];
        const double xd = __dmul_rn(__dsub_rn(grid_x(g, k), lp.nu), lp.iad);
        if (g.profile >= 3) {
          // no y dependence; the shape depends on iad through x and vb
          double c, cx, cvb;
          profile34_grad_d(g.profile, xd, lp.S1, vbl, c, cx, cvb);
          gS = fma(uk, c, gS);
          gx = fma(uk, fma(cx, xd, cvb * vbl), gx);
          gn = fma(uk, cx, gn);
          continue;
        }
        double c, cx, cy;
        if (k >= lp.c0 && k < lp.c1) {
          const VDer d = voigt916_dd(xd, lp.vy, lp.ey);
          c = lp.Sc * d.v;
          cx = lp.Sc * d.vx;
          cy = lp.Sc * d.vy;
        } else {
          ab_terms<double>(k >= lp.b0 && k < lp.b1, xd, lp.vy, Sp, c, cx, cy);
        }
        gS = fma(uk, c, gS);
        gy = fma(uk, cy, gy);
        gx = fma(uk * cx, xd, gx);
        gn = fma(uk, cx, gn);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        gS += __shfl_xor_sync(0xffffffffu, gS, o);
        gy += __shfl_xor_sync(0xffffffffu, gy, o);
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
        gn += __shfl_xor_sync(0xffffffffu, gn, o);
      }
      if (lane == 0) {
        atomicAdd(&G[l], gS);
        atomicAdd(&G[nlines + l], gy);
        atomicAdd(&G[2 * nlines + l], gx);
        atomicAdd(&G[3 * nlines + l], gn);
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ mixed form
constexpr int AB_G = 8192;  // grid points per tile of the mixed A/B pass

// Warp sum of four values per lane with six shuffles: the first two levels
// halve the values each lane carries, so value q's total ends in lanes
// 8q .. 8q+7.
template <class F>
__device__ __forceinline__ F warp_sum4(F v0, F v1, F v2, F v3, int lane) {
  const bool h4 = lane & 16, h3 = lane & 8;
  const F w0 = (h4 ? v2 : v0) + __shfl_xor_sync(0xffffffffu, h4 ? v0 : v2, 16);
  const F w1 = (h4 ? v3 : v1) + __shfl_xor_sync(0xffffffffu, h4 ? v1 : v3, 16);
  F z = (h3 ? w1 : w0) + __shfl_xor_sync(0xffffffffu, h3 ? w0 : w1, 8);
  z += __shfl_xor_sync(0xffffffffu, z, 4);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}

// The four per-lane sums of one line over tile points [k0, k1) of one
// region (B or A), x_k = (k + kf0) vb + fr in FP32 with k + kf0 exact:
//   fS = sum u t,  fY = sum u dt/dY,  fn = sum u dt/ds x,  fx = sum u dt/ds x^2
// (s = x^2; region A: t = 1/(s+Y), dt/ds = dt/dY = -t^2).  U and A are the
// types of u and of the sums: FP32 for tiles staged in FP32, FP64 for the
// others.
template <bool REGION_B, class U, class A>
__device__ __forceinline__ void ab_seg(const U *__restrict__ us, int k0, int k1, int lane, float kf0,
                                       float vbf, float frf, float Y, A &fS, A &fY, A &fn, A &fx) {
  float kf = (float)(k0 + lane) + kf0;
#pragma unroll 4
  for (int k = k0 + lane; k < k1; k += 32, kf += 32.0f) {
    const A uk = (A)us[k];
    const float x = fmaf(kf, vbf, frf);
    if (REGION_B) {
      float t, ts, tY;
      gh2_grad_f(x * x, Y, t, ts, tY);
      const A bsx = uk * (A)(ts * x);
      fS = fma(uk, (A)t, fS);
      fY = fma(uk, (A)tY, fY);
      fn += bsx;
      fx = fma(bsx, (A)x, fx);
    } else {
      const float t = rcp_fast(fmaf(x, x, Y));
      const A a = uk * (A)t;
      const A p = a * (A)t, px = p * (A)x;
      fS += a;
      fY -= p;
      fn -= px;
      fx = fma(-px, (A)x, fx);
    }
  }
}

template <class U, class A>
__device__ __forceinline__ void ab_line(const U *__restrict__ us, int a0, int rb0, int rc0, int rc1,
                                        int rb1, int a1, int lane, float kf0, float vbf, float frf,
                                        float Y, A &fS, A &fY, A &fn, A &fx) {
  ab_seg<false>(us, a0, rb0, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  ab_seg<true>(us, rb0, rc0, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  ab_seg<true>(us, rc1, rb1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  ab_seg<false>(us, rb1, a1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
}

// ------------------------------------------------------- far field
// As in the forward sum: over a 64-point block whose centre is at least
// AF_DK grid steps from the line centre, inside one region segment (A or B,
// which lie on one side of the centre), the shape t is a Taylor series in
// j = k - (block centre), and so is dt/dY.  The block's four sums are then
// the series' coefficients dotted with the block's moments M_n = sum_j u_j
// j^n of the staged u, computed once per tile:
//   fS = sum q_n M_n,  fY = sum dq_n M_n,  fn = sum c_n M_n,
//   fx = sum (x0 c_n + vb c_(n-1)) M_n,  c_n = (n + 1) q_(n+1) / (2 vb)
// ((dt/ds) x = (1/2) dt/dx and (dt/ds) x^2 = (x/2) dt/dx).  Region A:
// t = 1/(s + Y), q_n = -(b q_(n-1) + c q_(n-2)) / d0, dt/dY = -t^2 (the
// square of the series).  Region B: GH2 = N(s)/D(s) with N and D as
// polynomials in j, the quotient series and its derivative in Y
// (forward mode through the recursion, N and D's coefficients depend on Y).
// The remainder is about 1e-7 of the term (ratio 31.5 / 315 and a near
// double pole for small y); float32 prototypes of all four sums against
// FP64 with random signed u: <= 3.8e-7 of sum |u f|.
constexpr int AF_FB = 64, AF_NC = 8;
constexpr int AF_NB = AB_G / AF_FB;
constexpr float AF_DK = 315.5f;

// far block range [fl, fh) of a one-sided segment [k0, k1) (tile-local
// points, line centre at the tile point kc): blocks wholly inside it whose
// centre is at least AF_DK from kc (empty if the segment holds the centre)
__device__ __forceinline__ void af_range(int k0, int k1, float kc, int &fl, int &fh) {
  const int bl = (k0 + AF_FB - 1) / AF_FB, bh = k1 / AF_FB;
  const int nb0 = (int)floorf((kc - AF_DK - 31.5f) * (1.0f / AF_FB)) + 1;
  const int nb1 = (int)ceilf((kc + AF_DK - 31.5f) * (1.0f / AF_FB));
  fl = fh = 0;
  if (bh <= nb0 || bl >= nb1) {
    fl = bl;
    fh = bh;
  } else if (bl < nb0 && bh <= nb1) {
    fl = bl;
    fh = nb0;
  } else if (bl >= nb0 && bh > nb1) {
    fl = nb1;
    fh = bh;
  }
  if (fh <= fl) fl = fh = 0;
}

template <bool REGION_B>
__device__ __forceinline__ void af_seg(const float *__restrict__ mom, int fl, int fh, int lane, float kf0,
                                       float vbf, float frf, float Y, float &fS, float &fY, float &fn,
                                       float &fx) {
  const float ih = 0.5f * rcp_fast(vbf);
  for (int b = fl + lane; b < fh; b += 32) {
    const float x0 = fmaf((float)(b * AF_FB) + 31.5f + kf0, vbf, frf);
    const float bb = 2.0f * x0 * vbf, cc = vbf * vbf;
    float q[AF_NC + 1], dq[AF_NC];
    if (REGION_B) {
      const float c4 = (float)(4.0 / CUDART_PI), c6 = (float)(6.0 / CUDART_PI);
      const float A1 = fmaf(2.0f, Y, 2.5f - c4), B1 = (Y + 1.5f) * (Y + 1.0f);
      const float A2 = fmaf(2.0f, Y, 3.0f - c6), B2 = (Y + 1.5f) * (Y + 1.5f);
      const float E2 = A2 + Y, E1 = fmaf(A2, Y, B2), E0 = B2 * Y;
      const float dB1 = fmaf(2.0f, Y, 2.5f), dE1 = fmaf(2.0f, Y + 1.5f, fmaf(2.0f, Y, A2));
      const float dE0 = fmaf(2.0f * (Y + 1.5f), Y, B2);
      const float s0 = x0 * x0;
      // s, s^2, s^3 as polynomials in j
      const float S1[3] = {s0, bb, cc};
      const float S2[5] = {s0 * s0, 2.0f * s0 * bb, fmaf(bb, bb, 2.0f * s0 * cc), 2.0f * bb * cc, cc * cc};
      float S3[7];
#pragma unroll
      for (int n = 0; n < 7; ++n) S3[n] = 0.f;
#pragma unroll
      for (int i = 0; i < 5; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) S3[i + k] = fmaf(S2[i], S1[k], S3[i + k]);
      float N[5], D[7], dN[3], dD[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) N[n] = S2[n] + (n < 3 ? A1 * S1[n] : 0.f);
      N[0] += B1;
#pragma unroll
      for (int n = 0; n < 3; ++n) dN[n] = 2.0f * S1[n];
      dN[0] += dB1;
#pragma unroll
      for (int n = 0; n < 7; ++n) D[n] = S3[n] + (n < 5 ? E2 * S2[n] : 0.f) + (n < 3 ? E1 * S1[n] : 0.f);
      D[0] += E0;
#pragma unroll
      for (int n = 0; n < 5; ++n) dD[n] = 3.0f * S2[n] + (n < 3 ? dE1 * S1[n] : 0.f);
      dD[0] += dE0;
      const float iD = rcp_fast(D[0]);
#pragma unroll
      for (int n = 0; n <= AF_NC; ++n) {
        float a = n < 5 ? N[n] : 0.f;
#pragma unroll
        for (int i = 1; i <= 6; ++i)
          if (i <= n) a = fmaf(-D[i], q[n - i], a);
        q[n] = a * iD;
      }
#pragma unroll
      for (int n = 0; n < AF_NC; ++n) {
        float a = fmaf(-dD[0], q[n], n < 3 ? dN[n] : 0.f);
#pragma unroll
        for (int i = 1; i <= 6; ++i)
          if (i <= n) a = fmaf(-D[i], dq[n - i], i < 5 ? fmaf(-dD[i], q[n - i], a) : a);
        dq[n] = a * iD;
      }
    } else {
      const float iD = rcp_fast(fmaf(x0, x0, Y));
      q[0] = iD;
      q[1] = -(bb * q[0]) * iD;
#pragma unroll
      for (int n = 2; n <= AF_NC; ++n) q[n] = -fmaf(bb, q[n - 1], cc * q[n - 2]) * iD;
#pragma unroll
      for (int n = 0; n < AF_NC; ++n) {
        float a = 0.f;
#pragma unroll
        for (int i = 0; i <= n; ++i) a = fmaf(q[i], q[n - i], a);
        dq[n] = -a;
      }
    }
    float cprev = 0.f;
#pragma unroll
    for (int n = 0; n < AF_NC; ++n) {
      const float m = mom[n * AF_NB + b];
      const float cn = (float)(n + 1) * q[n + 1] * ih;
      fS = fmaf(q[n], m, fS);
      fY = fmaf(dq[n], m, fY);
      fn = fmaf(cn, m, fn);
      fx = fmaf(fmaf(x0, cn, vbf * cprev), m, fx);
      cprev = cn;
    }
  }
}

// one region segment: the direct sweep outside its far blocks, the far
// field inside them
template <bool REGION_B>
__device__ __forceinline__ void ab_seg_far(const float *__restrict__ us, const float *__restrict__ mom,
                                           int k0, int k1, int lane, float kf0, float vbf, float frf,
                                           float Y, float &fS, float &fY, float &fn, float &fx) {
  int fl = 0, fh = 0;
  if (k1 - k0 >= AF_FB && fabsf(kf0) < 2097152.0f) af_range(k0, k1, -kf0, fl, fh);
  if (fl < fh) {
    ab_seg<REGION_B>(us, k0, fl * AF_FB, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
    af_seg<REGION_B>(mom, fl, fh, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
    ab_seg<REGION_B>(us, fh * AF_FB, k1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  } else {
    ab_seg<REGION_B>(us, k0, k1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  }
}

__device__ __forceinline__ void ab_line_far(const float *__restrict__ us, const float *__restrict__ mom,
                                            int a0, int rb0, int rc0, int rc1, int rb1, int a1, int lane,
                                            float kf0, float vbf, float frf, float Y, float &fS, float &fY,
                                            float &fn, float &fx) {
  ab_seg_far<false>(us, mom, a0, rb0, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  ab_seg_far<true>(us, mom, rb0, rc0, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  ab_seg_far<true>(us, mom, rc1, rb1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
  ab_seg_far<false>(us, mom, rb1, a1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
}

// Regions A and B of the mixed form.  Per line, the offset at the tile's
// first point is formed in FP64 once and x_k = (k - kc) vb + fr follows in
// FP32 as in the forward (k - kc exact, |fr| <= vb/2); the shape terms are
// FP32 with one reciprocal.  u is staged in shared memory as FP32 scaled by
// 2^-e (e from the tile's largest |u|), so the per-lane products and sums
// are FP32 with the line strength and 2^e factored out; lane sums are
// reduced in FP32 and added to G in FP64.  A tile whose nonzero |u| span
// more than 2^64, or that holds a non-finite u, keeps u and the sums in
// FP64 (u read from global memory).  Region C is left to adjoint_c_kernel.
__global__ void __launch_bounds__(AD_THREADS, 4)
adjoint_ab_kernel(const LinePrep *__restrict__ P, const double *__restrict__ nu0, int64_t nlines,
                  GridDev g, const StateDev *__restrict__ states, int ntiles, int nsplit,
                  unsigned *__restrict__ ticket, const double *__restrict__ u,
                  double *__restrict__ G) {
  __shared__ float suf[AB_G];
  __shared__ float s_mom[AF_NC * AF_NB];  // far field: block moments of the staged u
  __shared__ double s_max[AD_WARPS], s_min[AD_WARPS];
  __shared__ int s_bad[AD_WARPS];
  __shared__ int s_t;
  __shared__ long long s_L0, s_L1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const StateDev &st = states[0];
  const double isp = 0.56418958354775628695;  // 1/sqrt(pi)
  const double idnu = 1.0 / g.dnu;
  const int ntickets = ntiles * nsplit;
  for (;;) {
    if (tid == 0) s_t = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int t = s_t;
    if (t >= ntickets) break;
    const int tile = t / nsplit, part = t - tile * nsplit;
    const int64_t g0 = (int64_t)tile * AB_G;
    const int64_t g1 = min(g0 + (int64_t)AB_G, g.nx);
    const int gi0 = (int)g0, gn = (int)(g1 - g0);
    // the tile's range of |u|
    {
      double amax = 0.0, amin = CUDART_INF;
      int bad = 0;
      for (int k = tid; k < gn; k += AD_THREADS) {
        const double v = fabs(u[g0 + k]);
        bad |= !(v <= DBL_MAX);
        amax = fmax(amax, v);
        if (v > 0.0) amin = fmin(amin, v);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        amin = fmin(amin, __shfl_xor_sync(0xffffffffu, amin, o));
      }
      bad = __any_sync(0xffffffffu, bad);
      if (lane == 0) {
        s_max[warp] = amax;
        s_min[warp] = amin;
        s_bad[warp] = bad;
      }
    }
    if (warp == 0) {
      const double W = st.wmax + st.shift + 2.0 * g.dnu;
      const double xlo = grid_x(g, g0) - W, xhi = grid_x(g, g1 - 1) + W;
      const double pad = 1e-12 * (fabs(xlo) + fabs(xhi)) + 1e-300;
      const int64_t L0 = ad_lower_bound_warp(nu0, nlines, xlo - pad);
      const int64_t L1 = ad_lower_bound_warp(nu0, nlines, xhi + pad);
      if (lane == 0) {
        s_L0 = L0 + (L1 - L0) * part / nsplit;
        s_L1 = L0 + (L1 - L0) * (part + 1) / nsplit;
      }
    }
    __syncthreads();
    double amax = 0.0, amin = CUDART_INF;
    int bad = 0;
#pragma unroll
    for (int w = 0; w < AD_WARPS; ++w) {
      amax = fmax(amax, s_max[w]);
      amin = fmin(amin, s_min[w]);
      bad |= s_bad[w];
    }
    const int e = amax > 0.0 ? ilogb(amax) + 1 : 0;
    const bool f32 = !bad && e > -1000 && e < 1000 && (amax == 0.0 || amin >= ldexp(amax, -64));
    const double su_scale = f32 ? ldexp(1.0, e) : 1.0;  // u = su_scale * staged value
    if (f32) {
      const double inv = ldexp(1.0, -e);
      for (int k = tid; k < AB_G; k += AD_THREADS) suf[k] = k < gn ? (float)(u[g0 + k] * inv) : 0.f;
    }
    __syncthreads();
    if (f32) {
      // moments M_n = sum_j u j^n of each 64-point block (j = -31.5 .. 31.5)
      for (int b = tid; b < AF_NB; b += AD_THREADS) {
        float m[AF_NC];
#pragma unroll
        for (int n = 0; n < AF_NC; ++n) m[n] = 0.f;
        for (int i = 0; i < AF_FB; ++i) {
          const float jj = (float)i - 31.5f;
          float p = suf[b * AF_FB + i];
#pragma unroll
          for (int n = 0; n < AF_NC; ++n) {
            m[n] += p;
            p *= jj;
          }
        }
#pragma unroll
        for (int n = 0; n < AF_NC; ++n) s_mom[n * AF_NB + b] = m[n];
      }
      __syncthreads();
    }
    const int64_t L0 = s_L0, L1 = s_L1;
    const double xg0 = grid_x(g, g0);
    for (int64_t l = L0 + warp; l < L1; l += AD_WARPS) {
      const LinePrep &lp = P[l];
      const int a0 = max(lp.i0 - gi0, 0), a1 = min(lp.i1 - gi0, gn);
      const double Sc = lp.Sc;
      if (a0 >= a1 || Sc == 0.0) continue;
      // tile-relative bounds: A [a0, rb0), B [rb0, rc0), C [rc0, rc1),
      // B [rc1, rb1), A [rb1, a1)
      const int rb0 = min(max(lp.b0 - gi0, a0), a1), rc0 = min(max(lp.c0 - gi0, a0), a1);
      const int rc1 = min(max(lp.c1 - gi0, a0), a1), rb1 = min(max(lp.b1 - gi0, a0), a1);
      const double nu = lp.nu, iad = lp.iad, vy = lp.vy;
      const double D0 = __dmul_rn(__dsub_rn(xg0, nu), iad);
      const double vb = __dmul_rn(g.dnu, iad);
      const double kc = fmin(fmax(rint((nu - xg0) * idnu), -8388608.0), 8388608.0);
      const float vbf = (float)vb, frf = (float)(D0 + kc * vb), kf0 = (float)(-kc);
      const double Yd = vy * vy;
      const float Y = (float)Yd;
      // Lorentz lines with y^2 < 2^-40 would square t = 1/(x^2 + y^2) past
      // the FP32 range at the centre: their sums stay in FP64
      const bool f32l = f32 && !(g.profile == 2 && Yd < 0x1p-40);
      double z, zS;
      if (f32l) {
        float fS = 0.f, fY = 0.f, fn = 0.f, fx = 0.f;
        ab_line_far(suf, s_mom, a0, rb0, rc0, rc1, rb1, a1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
        const float zf = warp_sum4(fS, fY, fn, fx, lane);
        z = (double)zf;
        zS = (double)__shfl_sync(0xffffffffu, zf, 0);
      } else {
        double fS = 0.0, fY = 0.0, fn = 0.0, fx = 0.0;
        ab_line(u + g0, a0, rb0, rc0, rc1, rb1, a1, lane, kf0, vbf, frf, Y, fS, fY, fn, fx);
        z = warp_sum4(fS, fY, fn, fx, lane);
        zS = __shfl_sync(0xffffffffu, z, 0);
      }
      // value q = lane / 8: 0 fS, 1 fY, 2 fn, 3 fx.
      //   G_S = S^/pi y fS, G_y = S^/pi (fS + 2Y fY), G_x = 2 S^/pi y fx,
      //   G_n = 2 S^/pi y fn  (times the staging scale)
      if ((lane & 7) == 0) {
        const int q = lane >> 3;
        const double Sp = Sc * isp * (f32l ? su_scale : 1.0), Spy = Sp * vy;
        const double v = q == 0 ? Spy * zS : q == 1 ? Sp * fma(2.0 * Yd, z, zS) : 2.0 * Spy * z;
        const int64_t dst = q == 0 ? 0 : q == 1 ? 1 : q == 2 ? 3 : 2;
        atomicAdd(&G[dst * nlines + l], v);
      }
    }
    __syncthreads();
  }
}

// Region C of the mixed form in FP32 (voigt_c_grad_f; FP64 for y = 0),
// after the A/B pass.  Each warp takes 32 consecutive lines and walks the
// concatenation of their [c0, c1) windows, one (line, point) pair per lane,
// so lanes stay busy whatever the windows' widths (a few points per line);
// the owner of pair j is found by a binary search over the warp's prefix
// sums of the widths.  Pair terms are summed per line by a segmented
// shuffle scan, and the last lane of each line's run adds to G.
__global__ void __launch_bounds__(AD_THREADS)
adjoint_c_kernel(const LinePrep *__restrict__ P, int64_t nlines, GridDev g,
                 const double *__restrict__ u, double *__restrict__ G) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * AD_THREADS + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * AD_THREADS) >> 5;
  for (int64_t base = w0 * 32; base < nlines; base += nw * 32) {
    const int64_t lme = base + lane;
    int c0 = 0, wd = 0;
    if (lme < nlines) {
      const LinePrep &lp = P[lme];
      if (lp.Sc != 0.0 && lp.c1 > lp.c0) {
        c0 = lp.c0;
        wd = lp.c1 - lp.c0;
      }
    }
    int incl = wd;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    for (int j0 = 0; j0 < total; j0 += 32) {
      const int j = j0 + lane;
      // q = number of lanes whose inclusive sum is <= j: the owner of pair j
      int q = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int v = __shfl_sync(FULL, incl, q + step - 1);
        if (v <= j) q += step;
      }
      const bool act = j < total;
      if (!act) q = 31;
      const int qc0 = __shfl_sync(FULL, c0, q);
      const int qincl = __shfl_sync(FULL, incl, q), qwd = __shfl_sync(FULL, wd, q);
      double gS = 0.0, gy = 0.0, gx = 0.0, gn = 0.0;
      if (act) {
        const LinePrep &lp = P[base + q];
        const int64_t k = (int64_t)qc0 + (j - (qincl - qwd));
        const double xd = __dmul_rn(__dsub_rn(grid_x(g, k), lp.nu), lp.iad);
        const double uk = u[k];
        const double Sc = lp.Sc;
        // FP32 values and derivatives (lines without Lorentz width: FP64)
        VDer d;
        if (lp.vy > 0.0) {
          const VDerF f = voigt_c_grad_f((float)xd, (float)lp.vy, (float)lp.ey, lp.sig1, lp.dsig1);
          d.v = f.v;
          d.vx = f.vx;
          d.vy = f.vy;
        } else {
          d = voigt916_dd(xd, lp.vy, lp.ey);
        }
        const double cx = Sc * d.vx;
        gS = uk * (Sc * d.v);
        gy = uk * (Sc * d.vy);
        gx = uk * cx * xd;
        gn = uk * cx;
      }
      // segmented inclusive scan over lanes of equal q (q ascends with lane)
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int qo = __shfl_up_sync(FULL, q, o);
        const double a = __shfl_up_sync(FULL, gS, o), b = __shfl_up_sync(FULL, gy, o);
        const double c = __shfl_up_sync(FULL, gx, o), d = __shfl_up_sync(FULL, gn, o);
        if (lane >= o && qo == q) {
          gS += a;
          gy += b;
          gx += c;
          gn += d;
        }
      }
      const int qn = __shfl_down_sync(FULL, q, 1);
      const bool actn = __shfl_down_sync(FULL, (int)act, 1);
      if (act && (lane == 31 || qn != q || !actn)) {
        const int64_t l = base + q;
        atomicAdd(&G[l], gS);
        atomicAdd(&G[nlines + l], gy);
        atomicAdd(&G[2 * nlines + l], gx);
        atomicAdd(&G[3 * nlines + l], gn);
      }
    }
  }
}

// Chain rule of the line scaling (prep_line) per line, in FP64.
//   HITRAN: S = Sf/Q(T) ab ss exp(c E''(1/T0 - 1/T)) (1 - e^{-c nu/T}) /
//           (1 - e^{-c nu/T0}) / alphaD,  nu = nu0 + delta P,  c = hc/k;
//   ExoMol: S = Sf ab ss / Q(T) e^{-c1 E''} (1 - e^{-c1 nu}) / alphaD,
//           c1 = hc/(kT);
//   gammaL = g_l (gam (P/P0) (T0/T)^n + A/(4 pi c)),  1/alphaD = iad0(T)/nu,
//   iad0 ~ T^-1/2,  y = gammaL/alphaD.
__global__ void __launch_bounds__(256)
adjoint_line_kernel(LinesDev L, StateDev st, const double *__restrict__ G,
                    const int64_t *__restrict__ order, double *__restrict__ dlogS,
                    double *__restrict__ dgam, int log_gamma, double *__restrict__ dTP) {
  __shared__ double sT[8], sP[8];
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double vT = 0.0, vP = 0.0;
  if (l < L.n) {
    const LineState ls = prep_line(L, st, l);
    const double gS = G[l], gy = G[L.n + l], gx = G[2 * L.n + l], gn = G[3 * L.n + l];
    const int j = L.iso ? (int)L.iso[l] : 0;
    const double T = st.T;
    const double el = L.EL ? L.EL[l] : L.EL_c;
    const double gam = L.gam ? L.gam[l] : L.gam_c;
    const double ne = L.nexp ? L.nexp[l] : L.nexp_c;
    const double At = L.Aterm ? L.Aterm[l] : L.Aterm_c;
    const double gs = L.gscale ? L.gscale[l] : 1.0;
    const double nu = ls.nu, iad = ls.iad;
    double dlS_dT, dlS_dnu = 0.0, delta = 0.0;
    if (L.database == HK_DB_HITRAN) {
      delta = L.delta ? L.delta[l] : L.delta_c;
      const double c = HK_H * HK_C / HK_KB;
      const double e1 = exp(-c * nu / T), e0 = exp(-c * nu / HK_T0);
      dlS_dT = -st.dlnQ[j] + c * el / (T * T) - (c * nu / (T * T)) * e1 / (1.0 - e1) - 0.5 / T;
      dlS_dnu = (c / T) * e1 / (1.0 - e1) - (c / HK_T0) * e0 / (1.0 - e0) - 1.0 / nu;
    } else {
      const double e2 = exp(-st.c1 * nu);
      dlS_dT = -st.dlnQ[j] + st.c1 * el / T - (st.c1 * nu / T) * e2 / (1.0 - e2) - 0.5 / T;
    }
    const double pb = pow(st.powbase, ne);
    const double aLc = gs * gam * st.PoverP0 * pb;  // collisional part
    const double aL = gs * (gam * st.PoverP0 * pb + At);
    const double P0 = (L.database == HK_DB_HITRAN) ? HK_PO_ATM : HK_PO_BAR;
    const double daL_dT = -ne * aLc / T;
    const double daL_dP = gs * gam * pb / P0;
    const double diad_dT = -0.5 * iad / T;
    const double diad_dP = -iad * delta / nu;
    const double dy_dT = daL_dT * iad + aL * diad_dT;
    const double dy_dP = daL_dP * iad + aL * diad_dP;
    if (ls.S != 0.0 && iad > 0.0) {
      // dLoss/d(1/alphaD) at fixed y: G_x alphaD;  dLoss/dnu_l = -G_n / alphaD
      const double gI = gx / iad, gN = -gn * iad;
      vT = gS * dlS_dT + gy * dy_dT + gI * diad_dT;
      vP = gS * dlS_dnu * delta + gy * dy_dP + gI * diad_dP + gN * delta;
    }
    const int64_t o = order ? order[l] : l;
    if (dlogS) dlogS[o] = gS;
    // dLoss/dgammaL = G_y / alphaD; per log gammaL: times gammaL
    if (dgam) dgam[o] = log_gamma ? gy * iad * aL : gy * iad;
  }
  for (int off = 16; off > 0; off >>= 1) {
    vT += __shfl_xor_sync(0xffffffffu, vT, off);
    vP += __shfl_xor_sync(0xffffffffu, vP, off);
  }
  if ((threadIdx.x & 31) == 0) {
    sT[threadIdx.x >> 5] = vT;
    sP[threadIdx.x >> 5] = vP;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += sT[w];
      b += sP[w];
    }
    atomicAdd(&dTP[0], a);
    atomicAdd(&dTP[1], b);
  }
}

cudaError_t launch_opacity_vjp(bool mixed, const LinesDev &L, const GridDev &g,
                               const StateDev *state_d, const StateDev &state_h,
                               const LinePrep *prep_d, const double *u_d, unsigned *ticket_d,
                               double *G_d, const int64_t *order_d, double *dlogS_d,
                               double *dgam_d, int log_gamma, double *dTP_d, cudaStream_t stream) {
  mixed = mixed && g.profile <= 2;  // Doppler and binned Gaussian: the FP64 form
  cudaError_t e = cudaMemsetAsync(G_d, 0, 4 * sizeof(double) * (size_t)L.n, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dTP_d, 0, 2 * sizeof(double), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ticket_d, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  if (L.n == 0 || g.nx == 0) return cudaSuccess;
  const int tpts = mixed ? AB_G : AD_G;
  const int ntiles = (int)((g.nx + tpts - 1) / tpts);
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (mixed)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_ab_kernel, AD_THREADS, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_tile_kernel, AD_THREADS, 0);
  const int resident = nsm * (per_sm < 1 ? 1 : per_sm);
  // about 8 tickets per resident CTA, at most 64 parts of a tile's lines
  const int nsplit = (int)std::min<int64_t>(64, std::max<int64_t>(1, (8LL * resident + ntiles - 1) / ntiles));
  const int ctas = (int)std::min<int64_t>((int64_t)ntiles * nsplit, resident);
  if (mixed) {
    adjoint_ab_kernel<<<ctas, AD_THREADS, 0, stream>>>(prep_d, L.nu0, L.n, g, state_d, ntiles, nsplit,
                                                       ticket_d, u_d, G_d);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    adjoint_c_kernel<<<nsm * 8, AD_THREADS, 0, stream>>>(prep_d, L.n, g, u_d, G_d);
  } else {
    adjoint_tile_kernel<<<ctas, AD_THREADS, 0, stream>>>(prep_d, L.nu0, L.n, g, state_d, ntiles, nsplit,
                                                         ticket_d, u_d, G_d);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  adjoint_line_kernel<<<(unsigned)((L.n + 255) / 256), 256, 0, stream>>>(L, state_h, G_d, order_d,
                                                                         dlogS_d, dgam_d, log_gamma,
                                                                         dTP_d);
  return cudaGetLastError();
}

}  // namespace hkb
