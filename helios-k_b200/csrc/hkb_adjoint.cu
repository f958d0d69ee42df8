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
// B: y/sqrt(pi) GH2; A: y/sqrt(pi) / (x^2 + y^2)).  Pass 1 (adjoint_tile_kernel)
// recomputes the forward per (grid tile, line) -- nothing of the forward is
// stored -- and reduces four sums per line:
//   G_S = sum_i u_i c_li,         G_y = sum_i u_i dc/dy,
//   G_x = sum_i u_i dc/dx x_li,   G_n = sum_i u_i dc/dx,
// so that dLoss/dlog S^ = G_S, dLoss/dy = G_y, dLoss/d(1/alphaD) at fixed y
// = G_x alphaD and dLoss/dnu_l = -G_n / alphaD.  Pass 2 (adjoint_line_kernel)
// applies the chain rule of the line scaling (prep_line) to T and P.
// Mixed form: regions A and B in FP32 (x from the FP64 offset) in pass 1,
// region C in FP64 (the differentiated Algorithm-916 series) in its own
// per-line pass (adjoint_c_kernel) between the two; the sums are FP64.
#include <cuda_runtime.h>

#include <algorithm>

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

// Regions A and B of the mixed form in FP32: t, dt/ds, dt/dY of the shape
// with one reciprocal (gh2_grad divides three times).
__device__ __forceinline__ void ab_grad_f(bool regionB, float s, float Y, float &t, float &ts,
                                          float &tY) {
  const float u = s + Y;
  if (!regionB) {
    t = rcp_fast(u);
    ts = -t * t;
    tY = ts;
    return;
  }
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

// Tickets are (tile, part): a tile's line range is cut into nsplit parts so
// that a grid of a few hundred tiles still fills the GPU; the per-line sums
// go to G through FP64 atomics either way.
// Mixed form: per line, the offset at the tile's first point of the window
// is formed in FP64 once, x_k = (k - kc) vb + fr in FP32 as in the forward
// (k - kc exact, |fr| <= vb/2); regions A and B accumulate per lane in FP32
// with the line strength factored out and the lane sums are reduced in FP64;
// region C is left to adjoint_c_kernel.
template <bool MIXED>
__global__ void __launch_bounds__(AD_THREADS, MIXED ? 4 : 2)
adjoint_tile_kernel(const LinePrep *__restrict__ P, const double *__restrict__ nu0, int64_t nlines,
                    GridDev g, const StateDev *__restrict__ states, int ntiles, int nsplit,
                    unsigned *__restrict__ ticket, const double *__restrict__ u,
                    double *__restrict__ G) {
  __shared__ double su[AD_G];  // u of the tile (FP32 in the first half for MIXED)
  float *suf = reinterpret_cast<float *>(su);
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
    const int64_t g0 = (int64_t)tile * AD_G;
    const int64_t g1 = min(g0 + (int64_t)AD_G, g.nx);
    for (int k = tid; k < AD_G; k += AD_THREADS) {
      const double v = (g0 + k < g1) ? u[g0 + k] : 0.0;
      if (MIXED)
        suf[k] = (float)v;
      else
        su[k] = v;
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
    const int64_t L0 = s_L0, L1 = s_L1;
    for (int64_t l = L0 + warp; l < L1; l += AD_WARPS) {
      const LinePrep lp = P[l];
      const int64_t lo = max((int64_t)lp.i0, g0), hi = min((int64_t)lp.i1, g1);
      if (lo >= hi || lp.Sc == 0.0) continue;
      const double Sp = lp.Sc * isp;  // S^/pi
      double gS = 0.0, gy = 0.0, gx = 0.0, gn = 0.0;
      if (MIXED) {
        // tile-relative int32 bounds: the A/B points [a0, c0) and [c1, a1),
        // region B within [rb0, rb1), region C [c0, c1)
        const int a0 = (int)(lo - g0), a1 = (int)(hi - g0);
        const int rc0 = (int)min(max((int64_t)lp.c0, lo), hi) - (int)g0;
        const int rc1 = (int)min(max((int64_t)lp.c1, lo), hi) - (int)g0;
        const int rb0 = (int)min(max((int64_t)lp.b0, lo), hi) - (int)g0;
        const int rb1 = (int)min(max((int64_t)lp.b1, lo), hi) - (int)g0;
        const double D0 = __dmul_rn(__dsub_rn(grid_x(g, g0), lp.nu), lp.iad);
        const double vb = __dmul_rn(g.dnu, lp.iad);
        const double kc = fmin(fmax(rint((lp.nu - grid_x(g, g0)) * idnu), -8388608.0), 8388608.0);
        const float vbf = (float)vb, frf = (float)(D0 + kc * vb), nkc = (float)(-kc);
        const float Y = (float)(lp.vy * lp.vy);
        // per lane: fS = sum u t, fY = sum u dt/dY, fn = sum u dt/ds x,
        // fx = sum u dt/ds x^2 (s = x^2)
        float fS = 0.f, fY = 0.f, fn = 0.f, fx = 0.f;
        auto ab_seg = [&](int k0, int k1) {
          float kf = (float)(k0 + lane) + nkc;
          for (int k = k0 + lane; k < k1; k += 32, kf += 32.0f) {
            const float uk = suf[k];
            const float x = fmaf(kf, vbf, frf);
            float tt, ts, tY;
            ab_grad_f(k >= rb0 && k < rb1, x * x, Y, tt, ts, tY);
            const float bs = uk * ts, bsx = bs * x;
            fS = fmaf(uk, tt, fS);
            fY = fmaf(uk, tY, fY);
            fn += bsx;
            fx = fmaf(bsx, x, fx);
          }
        };
        ab_seg(a0, rc0);
        ab_seg(rc1, a1);
        // S^/pi y t, S^/pi (t + 2Y dt/dY), S^/pi 2y x dt/ds (times x for gx)
        const double Spy = Sp * lp.vy;
        gS = fma(Spy, (double)fS, gS);
        gy = fma(Sp, fma(2.0 * lp.vy * lp.vy, (double)fY, (double)fS), gy);
        gx = fma(2.0 * Spy, (double)fx, gx);
        gn = fma(2.0 * Spy, (double)fn, gn);
      } else {
        for (int64_t k = lo + lane; k < hi; k += 32) {
          const double uk = su[k - g0];
          const double xd = __dmul_rn(__dsub_rn(grid_x(g, k), lp.nu), lp.iad);
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

// Region C of the mixed form: one warp per line over its whole [c0, c1)
// window in FP64 (Algorithm 916 with derivatives), added to the line's sums
// after the tile pass.  Kept out of the tile kernel, whose FP32 loop would
// otherwise carry the FP64 call's registers.  One warp owns each line, and
// the tile pass has finished on the stream, so the adds need no atomics.
__global__ void __launch_bounds__(AD_THREADS)
adjoint_c_kernel(const LinePrep *__restrict__ P, int64_t nlines, GridDev g,
                 const double *__restrict__ u, double *__restrict__ G) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * AD_THREADS + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * AD_THREADS) >> 5;
  for (int64_t l = w0; l < nlines; l += nw) {
    const LinePrep &lp = P[l];
    if (lp.c0 >= lp.c1 || lp.Sc == 0.0) continue;
    const double Sc = lp.Sc, nu = lp.nu, iad = lp.iad, vy = lp.vy, ey = lp.ey;
    double gS = 0.0, gy = 0.0, gx = 0.0, gn = 0.0;
    for (int64_t k = lp.c0 + lane; k < lp.c1; k += 32) {
      const double xd = __dmul_rn(__dsub_rn(grid_x(g, k), nu), iad);
      const double uk = u[k];
      const VDer d = voigt916_dd(xd, vy, ey);
      const double cx = Sc * d.vx;
      gS = fma(uk, Sc * d.v, gS);
      gy = fma(uk, Sc * d.vy, gy);
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
      G[l] += gS;
      G[nlines + l] += gy;
      G[2 * nlines + l] += gx;
      G[3 * nlines + l] += gn;
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
                    double *__restrict__ dgam, double *__restrict__ dTP) {
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
    if (dgam) dgam[o] = gy * iad;
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
                               double *dgam_d, double *dTP_d, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(G_d, 0, 4 * sizeof(double) * (size_t)L.n, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dTP_d, 0, 2 * sizeof(double), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ticket_d, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  if (L.n == 0 || g.nx == 0) return cudaSuccess;
  const int ntiles = (int)((g.nx + AD_G - 1) / AD_G);
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (mixed)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_tile_kernel<true>, AD_THREADS, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_tile_kernel<false>, AD_THREADS, 0);
  const int resident = nsm * (per_sm < 1 ? 1 : per_sm);
  // about 8 tickets per resident CTA, at most 32 parts of a tile's lines
  const int nsplit = (int)std::min<int64_t>(32, std::max<int64_t>(1, (8LL * resident + ntiles - 1) / ntiles));
  const int ctas = (int)std::min<int64_t>((int64_t)ntiles * nsplit, resident);
  if (mixed)
    adjoint_tile_kernel<true><<<ctas, AD_THREADS, 0, stream>>>(prep_d, L.nu0, L.n, g, state_d, ntiles,
                                                               nsplit, ticket_d, u_d, G_d);
  else
    adjoint_tile_kernel<false><<<ctas, AD_THREADS, 0, stream>>>(prep_d, L.nu0, L.n, g, state_d, ntiles,
                                                                nsplit, ticket_d, u_d, G_d);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (mixed) {
    adjoint_c_kernel<<<nsm * 8, AD_THREADS, 0, stream>>>(prep_d, L.n, g, u_d, G_d);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  adjoint_line_kernel<<<(unsigned)((L.n + 255) / 256), 256, 0, stream>>>(L, state_h, G_d, order_d,
                                                                         dlogS_d, dgam_d, dTP_d);
  return cudaGetLastError();
}

}  // namespace hkb
