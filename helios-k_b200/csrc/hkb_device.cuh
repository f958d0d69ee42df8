// hkb_device.cuh -- device-side math of the opacity path (sm_100a).
//
// Line scaling to a (T, P) state, the exact FP64 index-window rule, and the
// piecewise Voigt profile in FP64 (plain form) and FP32 (mixed form).
// Reference citations are file:line in the HELIOS-K source tree.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "hkb_types.h"

namespace hkb {

// ----------------------------------------------------------------- grid
// voigt.h:751-768 (setX_kernel): x_d[id] = numin + id * dnu, contracted to
// one FMA by nvcc; reproduced exactly with __fma_rn.
__device__ __forceinline__ double grid_x(const GridDev &g, int64_t i) {
  return __fma_rn((double)i, g.dnu, g.numin);
}

// ------------------------------------------------------------ line prep
struct LineState {
  double nu;   // line centre after the pressure shift
  double S;    // integrated strength scaled to (T, P), times 1/alphaD
  double iad;  // 1 / alphaD
  double vy;   // gammaL / alphaD
};

// HITRAN: host.h:598-649 (readFile) + voigt.h:331-363 (S2_kernel).
// ExoMol: voigt.h:484-504 (L_kernelExomol) + voigt.h:365-397 (Sf_kernel).
// The state-independent parts (combined width gam, A/(4 pi c)) were formed
// on the host at load time with the reference's expressions.
__device__ __forceinline__ LineState prep_line(const LinesDev &L,
                                               const StateDev &st,
                                               int64_t l) {
  LineState o;
  const int j = L.iso ? (int)L.iso[l] : 0;
  const double nu0 = L.nu0[l];
  const double Sf = L.Sfile[l];
  const double el = L.EL ? L.EL[l] : L.EL_c;
  const double gam = L.gam ? L.gam[l] : L.gam_c;
  const double ne = L.nexp ? L.nexp[l] : L.nexp_c;
  const double At = L.Aterm ? L.Aterm[l] : L.Aterm_c;
  double nu, S, iad;
  if (L.database == HK_DB_HITRAN) {
    const double de = L.delta ? L.delta[l] : L.delta_c;
    const double c = HK_H * HK_C / HK_KB;
    nu = __fma_rn(de, st.P, nu0);
    iad = __ddiv_rn(st.iad0[j], nu);
    S = __dmul_rn(__dmul_rn(__ddiv_rn(Sf, st.Q[j]), st.ab[j]), st.ss[j]);
    const double earg = __dadd_rn(__ddiv_rn(__dmul_rn(-el, c), st.T),
                                  __ddiv_rn(__dmul_rn(el, c), HK_T0));
    const double e1 = exp(__ddiv_rn(__dmul_rn(-c, nu), st.T));
    const double e0 = exp(__ddiv_rn(__dmul_rn(-c, nu), HK_T0));
    const double f = __dmul_rn(
        __ddiv_rn(__dmul_rn(exp(earg), __dsub_rn(1.0, e1)), __dsub_rn(1.0, e0)),
        iad);
    S = __dmul_rn(S, f);
  } else {
    // ExoMol: no pressure shift; S = S_file * Ab * Sscale / Q first
    nu = nu0;
    iad = __ddiv_rn(st.iad0[j], nu);
    S = __ddiv_rn(__dmul_rn(__dmul_rn(Sf, st.ab[j]), st.ss[j]), st.Q[j]);
    const double e1 = exp(__dmul_rn(-st.c1, el));
    const double e2 = exp(__dmul_rn(-st.c1, nu));
    S = __dmul_rn(S, __dmul_rn(__dmul_rn(e1, __dsub_rn(1.0, e2)), iad));
  }
  double aL = __dmul_rn(gam, __dmul_rn(st.PoverP0, pow(st.powbase, ne)));
  aL = __dadd_rn(aL, At);
  if (L.sscale) S = __dmul_rn(S, L.sscale[l]);
  if (L.gscale) aL = __dmul_rn(aL, L.gscale[l]);
  double vy = __dmul_rn(aL, iad);
  if (nu == 0.0) {
    S = 0.0;
    iad = 0.0;
    vy = 0.0;
  }
  o.nu = nu;
  o.S = S;
  o.iad = iad;
  o.vy = vy;
  return o;
}

// -------------------------------------------------------- index windows
// The region classes of nuLimits_kernel (voigt.h:2205-2341) and the
// per-pair tests of Line6fA/B/C (voigt.h:1223, 1481, 1662), as exact FP64
// index ranges (same predicates as the oracle, evaluated with explicit
// IEEE-rounded intrinsics so no FMA contraction changes a bit):
//   cut window [i0, i1): |x_i - nu| < w ;  B or C [b0, b1): r2 < 1e6 ;
//   C [c0, c1): r2 < 100 ;  r2 = (dnu_i * iad)^2 + vy^2.
struct WinCtx {
  double numin, dnu, nu, iad, vy2, w;
};

enum { HK_P_LEFT_CUT = 0, HK_P_RIGHT_CUT, HK_P_CENTER, HK_P_LEFT_R, HK_P_RIGHT_R };

__device__ __forceinline__ double win_d(const WinCtx &c, int64_t i) {
  return __dsub_rn(__fma_rn((double)i, c.dnu, c.numin), c.nu);
}

__device__ __forceinline__ bool win_pred(const WinCtx &c, int kind, int64_t i,
                                         double R) {
  const double d = win_d(c, i);
  switch (kind) {
  case HK_P_LEFT_CUT: return d > -c.w;
  case HK_P_RIGHT_CUT: return d >= c.w;
  case HK_P_CENTER: return d >= 0.0;
  default: {
    const double x = __dmul_rn(d, c.iad);
    const double r2 = __dadd_rn(__dmul_rn(x, x), c.vy2);
    return (kind == HK_P_LEFT_R) ? (r2 < R) : (r2 >= R);
  }
  }
}

// First index in [lo, hi) where the monotone predicate holds (hi if none).
// The answer does not depend on the estimate e (galloping + bisection).
static __device__ __noinline__ int64_t first_true(const WinCtx &c, int kind, double R,
                                           int64_t lo, int64_t hi, int64_t e) {
  if (lo >= hi) return lo;
  if (e < lo) e = lo;
  if (e > hi) e = hi;
  int64_t a, b;
  if (e >= hi || win_pred(c, kind, e, R)) {
    b = e;
    int64_t step = 1;
    while (true) {
      const int64_t t = b - step;
      if (t < lo) { a = lo; break; }
      if (!win_pred(c, kind, t, R)) { a = t + 1; break; }
      b = t;
      step *= 2;
    }
  } else {
    a = e + 1;
    int64_t step = 1;
    while (true) {
      const int64_t t = a - 1 + step;
      if (t >= hi) { b = hi; break; }
      if (win_pred(c, kind, t, R)) { b = t; break; }
      a = t + 1;
      step *= 2;
    }
  }
  while (a < b) {
    const int64_t m = a + (b - a) / 2;
    if (win_pred(c, kind, m, R)) b = m;
    else a = m + 1;
  }
  return a;
}

// A starting index for first_true (any value gives the same answer; a
// close one saves steps): idnu = 1 / dnu.
__device__ __forceinline__ int64_t est_index(double edge, const GridDev &g,
                                             int64_t hi, double idnu) {
  const double e = ceil((edge - g.numin) * idnu);
  if (!(e > -1.0)) return 0;
  if (e > (double)hi) return hi;
  return (int64_t)e;
}

// Profiles 2-4 have no regions B and C: the whole cut window is region A
// (nuLimits_kernel voigt.h:2250, "profile != 1"; only Line6A runs for them).
// Window boundaries of one line restricted to grid indices [g0, g1):
// out[0..5] = i0, b0, c0, c1, b1, i1 (absolute indices, each clipped to
// [g0, g1]).  Equals clip(oracle window) because every predicate is
// monotone on the range it is searched over.
__device__ __forceinline__ void line_windows(const GridDev &g, const StateDev &st,
                                             const LineState &ls, int64_t g0,
                                             int64_t g1, int64_t out[6]) {
  if (ls.S == 0.0 || !(ls.iad > 0.0)) {
    for (int k = 0; k < 6; ++k) out[k] = g0;
    return;
  }
  WinCtx c;
  c.numin = g.numin;
  c.dnu = g.dnu;
  c.nu = ls.nu;
  c.iad = ls.iad;
  c.vy2 = __dmul_rn(ls.vy, ls.vy);
  double w;
  if (g.cutMode == 1) w = __ddiv_rn(__dmul_rn(g.cut, ls.vy), ls.iad);
  else if (g.cutMode == 2) w = __ddiv_rn(g.cut, ls.iad);
  else w = g.cut;
  c.w = w;
  // the searches' starting points need no exact arithmetic (FP64 division
  // and square root are slow on this part)
  const double idnu = 1.0 / g.dnu;
  const int64_t i0 = first_true(c, HK_P_LEFT_CUT, 0.0, g0, g1, est_index(ls.nu - w, g, g1, idnu));
  const int64_t i1 = first_true(c, HK_P_RIGHT_CUT, 0.0, i0, g1, est_index(ls.nu + w, g, g1, idnu));
  if (i1 <= i0) {
    for (int k = 0; k < 6; ++k) out[k] = i0;
    return;
  }
  const int64_t ic = first_true(c, HK_P_CENTER, 0.0, i0, i1, est_index(ls.nu, g, g1, idnu));
  const double Rs[2] = {1.0e6, 100.0};
  int64_t lohi[2][2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const double R = Rs[r];
    const double h2 = R - c.vy2;
    if (g.profile == 1 && h2 > 0.0) {  // regions B and C are the Voigt profile's
      const double h = (double)(sqrtf((float)h2) / (float)c.iad);
      lohi[r][0] = first_true(c, HK_P_LEFT_R, R, i0, ic, est_index(ls.nu - h, g, g1, idnu));
      lohi[r][1] = first_true(c, HK_P_RIGHT_R, R, ic, i1, est_index(ls.nu + h, g, g1, idnu));
    } else {
      lohi[r][0] = ic;
      lohi[r][1] = ic;
    }
  }
  out[0] = i0;
  out[1] = lohi[0][0];
  out[2] = lohi[1][0];
  out[3] = lohi[1][1];
  out[4] = lohi[0][1];
  out[5] = i1;
}

// -------------------------------------------------------------- profile
// Region B rational (voigt.h:1481-1490), rewritten with u = r2, s = x^2:
//   t4 = [(u+1.5)(u+1) - (4/pi) s] / [u ((u+1.5)^2 - (6/pi) s)]
// which is the reference's (t3(2t2+r2) - 2t1) / (3 r2 (t3 t2 - t1)) with
// numerator and denominator divided by 3 pi.
__device__ __forceinline__ double gh2_d(double x, double y2) {
  const double s = x * x;
  const double u = s + y2;
  const double a1 = u + 1.5;
  const double num = a1 * (u + 1.0) - (4.0 / CUDART_PI) * s;
  const double den = u * (a1 * a1 - (6.0 / CUDART_PI) * s);
  return num / den;
}

// Zaghloul & Ali, Algorithm 916 in FP64: restates voigt.h:165-216 (Sigmab)
// and voigt.h:278-300 (voigt_916) with def_TOL; ey = erfcx(y) per line.
static __device__ __noinline__ double voigt916_d(double x, double y, double ey) {
  const double a = HK_A916_D;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const double ax = fabs(x);
  const double ex2 = exp(-ax * ax);
  if (ax != 0.0 && y != 0.0) {
    double o1 = 0.0, o2 = 0.0, o3 = 0.0;
    const double yy = y * y;
    const int n0 = (int)ceil(ax / a);
    bool st1 = false, st2 = false, st3 = false;
    for (int n = 1; n < 100; ++n) {
      const int n3p = n0 + n - 1, n3n = n0 - n;
      const double an = a * n, an3p = a * n3p, an3n = a * n3n;
      const double f = 1.0 / (an * an + yy);
      const double f3p = 1.0 / (an3p * an3p + yy);
      const double f3n = 1.0 / (an3n * an3n + yy);
      s1 += f * exp(-(an * an + ax * ax));
      s2 += f * exp(-(an + ax) * (an + ax));
      s3 += f3p * exp(-(an3p - ax) * (an3p - ax));
      if (n3n >= 1) s3 += f3n * exp(-(an3n - ax) * (an3n - ax));
      if (fabs(s1 - o1) < HK_TOL) st1 = true;
      if (fabs(s2 - o2) < HK_TOL) st2 = true;
      if (fabs(s3 - o3) < HK_TOL) st3 = true;
      if (st1 && st2 && st3) break;
      o1 = s1;
      o2 = s2;
      o3 = s3;
    }
  }
  const double xy = ax * y;
  const double cos2xy = cos(2.0 * xy);
  const double sinxy = sin(xy);
  double t1 = ex2 * ey * cos2xy;
  if (ax != 0.0 && y != 0.0) {
    const double a2ipi = 2.0 * a / CUDART_PI;
    t1 += a2ipi * sinxy * ex2 * sinxy / y;
    t1 += a2ipi * y * (-cos2xy * s1 + 0.5 * (s2 + s3));
  }
  if (ax == 0.0) t1 = ey;
  if (y == 0.0) t1 = ex2;
  return t1;
}

// Profiles 2-4 at x (Doppler units) for a line with S1 as line_prep_kernel
// forms it per profile: Lorentz S1 / (x^2 + y^2) (S1 = S y / pi), Doppler
// S1 exp(-x^2) (S1 = S / sqrt(pi)), binned Gaussian S1 (erf(x + vb/2) -
// erf(x - vb/2)) / (2 vb) with vb the grid step in Doppler units (S1 = S):
// Line6fA_kernel voigt.h:1235-1262, in FP64.
// erf(a) - erf(b) for a > b without cancellation in the wings: as
// erfc(b) - erfc(a) when both are positive, erfc(-a) - erfc(-b) when both
// are negative (the same value; the reference subtracts FP32 erff).
__device__ __forceinline__ double erf_diff(double a, double b) {
  if (b >= 0.0) return erfc(b) - erfc(a);
  if (a <= 0.0) return erfc(-a) - erfc(-b);
  return erf(a) - erf(b);
}

__device__ __forceinline__ double profile_a_d(int profile, double x, double y2, double S1,
                                              double vb) {
  if (profile == 3) return S1 * exp(-(x * x));
  if (profile == 4) return S1 * (1.0 / vb) * 0.5 * erf_diff(x + 0.5 * vb, x - 0.5 * vb);
  return S1 / (x * x + y2);  // profile 1 region A, profile 2
}

// Sub-Lorentzian factor chi(|x - nu|) x / nu for a grid point x of a line
// at nu (sLChi voigt.h:47-72 and its use in Line6fAX/BX/CX, voigt.h:1345-
// 1790), in FP64: 1 outside (sl_lo, sl_hi); chi piecewise exponential with
// breakpoints sigma1 < sigma2 < sigma3 and the state's slopes B1, B2, B3.
__device__ __forceinline__ double sublorentz_d(const GridDev &g, const StateDev &st, double x,
                                               double nu) {
  if (!(x > g.sl_lo && x < g.sl_hi)) return 1.0;
  const double d = fabs(x - nu);
  const double s1 = g.sl_sigma[0], s2 = g.sl_sigma[1], s3 = g.sl_sigma[2];
  double chi;
  if (d < s1) chi = 1.0;
  else if (d < s2) chi = exp(-st.sl_B[0] * (d - s1));
  else if (d < s3) chi = exp(-st.sl_B[0] * (s2 - s1) - st.sl_B[1] * (d - s2));
  else chi = exp(-st.sl_B[0] * (s2 - s1) - st.sl_B[1] * (s3 - s2) - st.sl_B[2] * (d - s3));
  return chi * x / nu;
}

// The profile's value at the line's cut edge, x_c = cut iad (cutMode 0),
// cut y (1) or cut (2): Plinth_kernel (voigt.h:1091-1164) in FP64, the Voigt
// profile by the region of r^2 = x_c^2 + y^2; 0 for the binned Gaussian (the
// reference defines none).
// the cut edge in Doppler units: cut iad (cutMode 0), cut y (1), cut (2)
__device__ __forceinline__ double plinth_xc(const GridDev &g, double iad, double vy) {
  return (g.cutMode == 1) ? g.cut * vy : (g.cutMode == 2 ? g.cut : g.cut * iad);
}

__device__ __forceinline__ double plinth_d(const GridDev &g, double S1, double Sc, double iad,
                                           double vy) {
  const double xc = plinth_xc(g, iad, vy);
  const double y2 = vy * vy;
  if (g.profile == 1) {
    const double r2 = xc * xc + y2;
    if (r2 >= 1.0e6) return S1 / r2;
    if (r2 >= 100.0) return S1 * gh2_d(xc, y2);
    return Sc * voigt916_d(xc, vy, erfcx(vy));
  }
  if (g.profile == 4) return 0.0;
  return profile_a_d(g.profile, xc, y2, S1, 0.0);
}

// ------------------------------------------- region C, recurrence form
// Algorithm 916 in FP32 (the series of voigt.h:217-268, Sigmabf, and the
// region-C formula of voigt.h:1662-1682, with a from def_TOLF).  Unlike the
// reference's FP32 kernel, x arrives with FP32 relative accuracy (formed
// from a double-float split of the FP64 offset, not from (numin - nu)/alphaD
// rounded to float) and erfcx(y) is a per-line FP64 constant.  The series
// are rearranged for FP32 throughput:
//   s1 = sum_m R_m exp(-(a^2 m^2 + x^2)) = exp(-x^2) * Sig1(y),
//        Sig1(y) = sum_m exp(-a^2 m^2) R_m  -- a per-line constant;
//   s3 = sum_{m>=1} R_m exp(-(a m - x)^2),  s2 = sum_{m>=1} R_m exp(-(a m + x)^2),
//        R_m = 1 / (a^2 m^2 + y^2).
// The Gaussians of s3 are generated from the centre m_c = rint(x/a) outwards
// with the exact ratio exp(-(a(m+1)-x)^2) / exp(-(a m - x)^2)
//   = exp(-a^2 (2m+1) + 2 a x), itself advanced by the constant exp(-2 a^2):
// three exps instead of one per term.  HK_C916_K terms each side reach
// |a m - x| >= 4.8, where the Gaussian is below 1e-10 of the centre term,
// so the trip counts are fixed (no data-dependent convergence loop).
constexpr int HK_C916_K = 8;

// rcp.approx.ftz.f32: maximum error 1 ulp (PTX ISA), one XU instruction
__device__ __forceinline__ float rcp_fast(float v) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// per-line constant Sig1(y), FP64 at staging
constexpr int HK_SIG1_M = 12;
__device__ __forceinline__ double c916_e(int m) {
  const double a = (double)HK_A916_F;
  return exp(-(a * a * m * m));
}
// e[m-1] = c916_e(m) (a line-independent table, e.g. in shared memory).
// Each term takes the correctly rounded reciprocal of its denominator
// (__drcp_rn, a few instructions) times e_m instead of an FP64 division;
// the sum is rounded to FP32 for the region-C evaluator.
__device__ __forceinline__ double c916_sig1_tab(double y, const double *__restrict__ e) {
  const double a = (double)HK_A916_F;
  const double y2 = y * y;
  double s = 0.0;
#pragma unroll 4
  for (int m = 1; m <= HK_SIG1_M; ++m) {
    const double am2 = a * a * m * m;
    s = __fma_rn(e[m - 1], __drcp_rn(am2 + y2), s);
  }
  return s;
}
// dSig1/dy = sum_m e_m (-2 y) / (a^2 m^2 + y^2)^2 (the mixed adjoint's region C)
__device__ __forceinline__ double c916_dsig1_tab(double y, const double *__restrict__ e) {
  const double a = (double)HK_A916_F;
  const double y2 = y * y;
  double s = 0.0;
#pragma unroll 4
  for (int m = 1; m <= HK_SIG1_M; ++m) {
    const double r = __drcp_rn(a * a * m * m + y2);
    s = __fma_rn(e[m - 1] * r, r, s);
  }
  return -2.0 * y * s;
}
__device__ __forceinline__ double c916_sig1(double y) {
  double e[HK_SIG1_M];
  for (int m = 1; m <= HK_SIG1_M; ++m) e[m - 1] = c916_e(m);
  return c916_sig1_tab(y, e);
}

// R[m-1] = 1 / (a^2 m^2 + y^2), m = 1..HK_C916_MR, is a per-line table built
// once per (line, tile) in shared memory; the recurrence seeds use ex2.approx
// (their arguments are bounded by ~2a^2, so it keeps ~1e-7 relative
// accuracy).
constexpr int HK_C916_MR = 18;  // x < 6 -> m_c <= 10, plus HK_C916_K

__device__ __forceinline__ float ex2_fast(float v) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// Region C with r = |x + iy| >= 6: the asymptotic (Laplace continued
// fraction's) series of the Faddeeva function,
//   w(z) ~ i / (sqrt(pi) z) * sum_{k>=0} c_k u^k,  u = 1/z^2,
//   c_k = (2k-1)!! / 2^k,
// so K(x, y) = Re w = (y Re S - x Im S) / (sqrt(pi) r^2).  HK_ASY_K = 8 terms
// leave c_8 / r^16 < 3e-9 at r = 6 (the series' smallest term is near
// k = r^2, far beyond).  The expansion omits Re exp(-z^2) =
// exp(y^2 - x^2) cos(2xy) (the Stokes term that gives w(x) = exp(-x^2) on
// the real axis); it is added for y < 1 -- for y >= 1 and r >= 6 it is below
// 1e-13 of K.  Against the FP64 Algorithm 916 the FP32 evaluation keeps
// 3e-7 relative error over 6 <= r < 10.
constexpr float HK_ASY_R2 = 36.0f;
constexpr int HK_ASY_K = 8;

__device__ __forceinline__ float voigt_asy(float x, float y) {
  x = fabsf(x);
  const float x2 = x * x, y2 = y * y;
  const float r2 = fmaf(x, x, y2);
  const float ir2 = rcp_fast(r2);
  const float ir4 = ir2 * ir2;
  const float ur = (x2 - y2) * ir4;
  const float ui = -2.0f * x * y * ir4;
  // c_k, k = 0..8
  const float c[HK_ASY_K + 1] = {1.0f, 0.5f, 0.75f, 1.875f, 6.5625f, 29.53125f,
                                 162.421875f, 1055.7421875f, 7918.06640625f};
  float sr = c[HK_ASY_K], si = 0.0f;
#pragma unroll
  for (int k = HK_ASY_K - 1; k >= 0; --k) {
    const float nr = fmaf(sr, ur, fmaf(-si, ui, c[k]));
    si = fmaf(sr, ui, si * ur);
    sr = nr;
  }
  float v = fmaf(y, sr, -x * si) * (0.56418958354775628f * ir2);  // 1/sqrt(pi)
  if (y < 1.0f) v = fmaf(ex2_fast(1.4426950408889634f * (y2 - x2)), __cosf(2.0f * x * y), v);
  return v;
}

// sin(z)^2 for 0 <= z <= 64: z = n pi + r with |r| <= pi/2 (Cody-Waite
// reduction, pi split into its nearest float and the remainder), then
// sin(r) from its Taylor series to r^13 (remainder < (pi/2)^15/15! = 9e-10).
// Near a zero of sin the reduced r keeps its own relative accuracy.
__device__ __forceinline__ float sin_sq(float z) {
  const float n = rintf(z * 0.318309886183790672f);   // 1/pi
  float r = fmaf(-n, 3.14159274101257324f, z);          // float(pi)
  r = fmaf(-n, -8.74227766e-8f, r);                     // pi - float(pi)
  const float r2 = r * r;
  float p = 1.60590438368216146e-10f;                   // 1/13!
  p = fmaf(p, r2, -2.50521083854417188e-8f);            // -1/11!
  p = fmaf(p, r2, 2.75573192239858907e-6f);             // 1/9!
  p = fmaf(p, r2, -1.98412698412698413e-4f);            // -1/7!
  p = fmaf(p, r2, 8.33333333333333333e-3f);             // 1/5!
  p = fmaf(p, r2, -0.166666666666666667f);              // -1/3!
  const float sr = fmaf(p * r2, r, r);
  return sr * sr;
}

// Algorithm 916 with the per-line table R, valid for |x| < 6.3 (m_c <= 10);
// iy = 1/y.  The s2 series stops at the first term below e^-25 of the
// largest (a m + x >= 5.1), so its length falls from 8 at x = 0 to none at
// x >= 4.5.
__device__ __forceinline__ float voigt916_core(float x, float y, float iy, float ey, float sig1,
                                               const float *__restrict__ R) {
  const float a = HK_A916_F;
  const float a2 = a * a;
  const float L2E = 1.4426950408889634f;  // log2(e)
  const float G = 0.48675662279129028f;   // exp(-2 a^2)
  x = fabsf(x);
  const float ex2 = expf(-x * x);
  if (x == 0.f) return ey;
  if (y == 0.f) return ex2;
  const int mc = min(HK_C916_MR - HK_C916_K, max(1, __float2int_rn(x * (1.0f / a))));
  const float mcf = (float)mc;
  const float d = fmaf(a, mcf, -x);
  const float Tc = ex2_fast(-L2E * d * d);
  const float up0 = ex2_fast(L2E * fmaf(-a2, fmaf(2.0f, mcf, 1.0f), 2.0f * a * x));
  const float dn0 = ex2_fast(L2E * fmaf(a2, fmaf(2.0f, mcf, -1.0f), -2.0f * a * x));
  const float *Rc = R + (mc - 1);
  float s3 = Tc * Rc[0];
  float T = Tc, q = up0;
#pragma unroll
  for (int k = 1; k <= HK_C916_K; ++k) {
    T *= q;
    q *= G;
    s3 = fmaf(T, Rc[k], s3);
  }
  T = Tc;
  q = dn0;
#pragma unroll
  for (int k = 1; k <= HK_C916_K; ++k) {
    T *= q;
    q *= G;
    if (mc - k >= 1) s3 = fmaf(T, Rc[-k], s3);
  }
  float s2 = 0.f;
  const int n2 = min(HK_C916_K, __float2int_ru((5.1f - x) * (1.0f / a)));
  if (n2 > 0) {
    // exp(-(a + x)^2) = exp(-x^2) exp(-a^2 - 2 a x)
    float T2 = ex2 * ex2_fast(-L2E * fmaf(2.0f * a, x, a2));
    float q2 = ex2_fast(L2E * fmaf(-3.0f, a2, -2.0f * a * x));
    for (int k = 0; k < n2; ++k) {
      s2 = fmaf(T2, R[k], s2);
      T2 *= q2;
      q2 *= G;
    }
  }
  const float s1 = ex2 * sig1;
  const float sin2 = sin_sq(x * y);
  const float cos2xy = fmaf(-2.0f, sin2, 1.0f);
  const float t2 = sin2 * ex2 * iy;
  const float t3 = y * fmaf(-cos2xy, s1, 0.5f * (s2 + s3));
  return fmaf(ex2 * ey, cos2xy, HK_C916_F * (t2 + t3));
}

// region C in FP32: the asymptotic series for r >= 6, Algorithm 916 below
__device__ __forceinline__ float voigt916_tab(float x, float y, float iy, float ey, float sig1,
                                              const float *__restrict__ R) {
  x = fabsf(x);
  if (fmaf(x, x, y * y) >= HK_ASY_R2) return voigt_asy(x, y);
  return voigt916_core(x, y, iy, ey, sig1, R);
}

// Region C in FP32 with the partial derivatives in x and y (the mixed
// adjoint), y > 0.  r >= 6: the asymptotic series of w and, by a second
// Horner sum, of dw/dz = -(i/sqrt(pi)) u S'(u), S' = sum (2k+1) c_k u^k,
// u = 1/z^2, so dV/dx = Im(u S')/sqrt(pi), dV/dy = Re(u S')/sqrt(pi) (no
// cancellation, unlike -2 z w + 2i/sqrt(pi)), plus the Stokes term
// exp(-z^2) and its derivative -2 z exp(-z^2) for y < 1.  r < 6: Algorithm
// 916 as voigt916_core with every term differentiated: a Gaussian of s3
// (s2) carries 2 (a m - x) (-2 (a m + x)) in x and each R_m = 1 / (a^2 m^2
// + y^2) carries -2 y R_m in y; s1 = e^(-x^2) Sig1(y) with dsig1 = Sig1'(y).
// Float32 emulation against FP64 wofz: V 1.3e-6 relative, the derivatives
// 2e-6 of |w|.
struct VDerF {
  float v, vx, vy;
};

__device__ __forceinline__ VDerF voigt_c_grad_f(float x, float y, float ey, float sig1, float dsig1) {
  const float isp = 0.56418958354775628f;  // 1/sqrt(pi)
  const float L2E = 1.4426950408889634f;
  const float sx = x < 0.f ? -1.f : 1.f;
  x = fabsf(x);
  VDerF o;
  const float x2 = x * x, Y = y * y;
  if (x2 + Y >= HK_ASY_R2) {
    const float ir2 = rcp_fast(x2 + Y), ir4 = ir2 * ir2;
    const float ur = (x2 - Y) * ir4, ui = -2.0f * x * y * ir4;
    const float c[HK_ASY_K + 1] = {1.0f, 0.5f, 0.75f, 1.875f, 6.5625f, 29.53125f,
                                   162.421875f, 1055.7421875f, 7918.06640625f};
    float sr = c[HK_ASY_K], si = 0.f, pr = (2 * HK_ASY_K + 1) * c[HK_ASY_K], pi = 0.f;
#pragma unroll
    for (int k = HK_ASY_K - 1; k >= 0; --k) {
      const float nr = fmaf(sr, ur, fmaf(-si, ui, c[k]));
      si = fmaf(sr, ui, si * ur);
      sr = nr;
      const float qr = fmaf(pr, ur, fmaf(-pi, ui, (float)(2 * k + 1) * c[k]));
      pi = fmaf(pr, ui, pi * ur);
      pr = qr;
    }
    float v = fmaf(y, sr, -x * si) * (isp * ir2);
    float vx = fmaf(ur, pi, ui * pr) * isp;
    float vy = fmaf(ur, pr, -ui * pi) * isp;
    if (y < 1.0f) {
      const float E = ex2_fast(L2E * (Y - x2));
      float s2, c2;
      sincosf(2.0f * x * y, &s2, &c2);
      v = fmaf(E, c2, v);
      vx = fmaf(-2.0f * E, fmaf(x, c2, y * s2), vx);
      vy = fmaf(2.0f * E, fmaf(y, c2, -x * s2), vy);
    }
    o.v = v;
    o.vx = sx * vx;
    o.vy = vy;
    return o;
  }
  if (x == 0.f) {
    o.v = ey;
    o.vx = 0.f;
    o.vy = fmaf(2.0f * y, ey, -2.0f * isp);
    return o;
  }
  const float a = HK_A916_F, a2 = a * a;
  const float G = 0.48675662279129028f;  // exp(-2 a^2)
  const float ex2 = expf(-x2);
  const int mc = min(HK_C916_MR - HK_C916_K, max(1, __float2int_rn(x * (1.0f / a))));
  const float mcf = (float)mc;
  const float d = fmaf(a, mcf, -x);
  const float Tc = ex2_fast(-L2E * d * d);
  const float up0 = ex2_fast(L2E * fmaf(-a2, fmaf(2.0f, mcf, 1.0f), 2.0f * a * x));
  const float dn0 = ex2_fast(L2E * fmaf(a2, fmaf(2.0f, mcf, -1.0f), -2.0f * a * x));
  // s3, sum (a m - x) R T, sum R^2 T
  float Rm = rcp_fast(fmaf(a2 * mcf, mcf, Y));
  float s3 = Tc * Rm, s3w = d * (Tc * Rm), s3f = Rm * (Tc * Rm);
  float T = Tc, q = up0;
#pragma unroll
  for (int k = 1; k <= HK_C916_K; ++k) {
    T *= q;
    q *= G;
    const float mf = mcf + (float)k;
    Rm = rcp_fast(fmaf(a2 * mf, mf, Y));
    const float tr = T * Rm;
    s3 += tr;
    s3w = fmaf(fmaf(a, mf, -x), tr, s3w);
    s3f = fmaf(Rm, tr, s3f);
  }
  T = Tc;
  q = dn0;
#pragma unroll
  for (int k = 1; k <= HK_C916_K; ++k) {
    T *= q;
    q *= G;
    if (mc - k >= 1) {
      const float mf = mcf - (float)k;
      Rm = rcp_fast(fmaf(a2 * mf, mf, Y));
      const float tr = T * Rm;
      s3 += tr;
      s3w = fmaf(fmaf(a, mf, -x), tr, s3w);
      s3f = fmaf(Rm, tr, s3f);
    }
  }
  float s2 = 0.f, s2w = 0.f, s2f = 0.f;
  const int n2 = min(HK_C916_K, __float2int_ru((5.1f - x) * (1.0f / a)));
  if (n2 > 0) {
    float T2 = ex2 * ex2_fast(-L2E * fmaf(2.0f * a, x, a2));
    float q2 = ex2_fast(L2E * fmaf(-3.0f, a2, -2.0f * a * x));
    for (int k = 0; k < n2; ++k) {
      const float mf = (float)(k + 1);
      Rm = rcp_fast(fmaf(a2 * mf, mf, Y));
      const float tr = T2 * Rm;
      s2 += tr;
      s2w = fmaf(fmaf(a, mf, x), tr, s2w);
      s2f = fmaf(Rm, tr, s2f);
      T2 *= q2;
      q2 *= G;
    }
  }
  const float s1 = ex2 * sig1;
  const float s1x = -2.0f * x * s1, s1y = ex2 * dsig1;
  const float s2x = -2.0f * s2w, s2y = -2.0f * y * s2f;
  const float s3x = 2.0f * s3w, s3y = -2.0f * y * s3f;
  const float sin2 = sin_sq(x * y);
  const float cos2 = fmaf(-2.0f, sin2, 1.0f);
  const float sn2 = sinf(2.0f * x * y);
  const float iy = 1.0f / y;
  const float qq = sin2 * iy;  // sin(xy)^2 / y
  const float t2 = ex2 * qq;
  const float B = fmaf(-cos2, s1, 0.5f * (s2 + s3));
  o.v = fmaf(ex2 * ey, cos2, HK_C916_F * fmaf(y, B, t2));
  const float dcx = -2.0f * y * sn2, dcy = -2.0f * x * sn2;
  const float dt2x = ex2 * fmaf(-2.0f * x, qq, sn2), dt2y = ex2 * fmaf(x, sn2, -qq) * iy;
  const float dBx = fmaf(-dcx, s1, fmaf(-cos2, s1x, 0.5f * (s2x + s3x)));
  const float dBy = fmaf(-dcy, s1, fmaf(-cos2, s1y, 0.5f * (s2y + s3y)));
  const float eyp = fmaf(2.0f * y, ey, -2.0f * isp);
  o.vx = sx * fmaf(ey * ex2, fmaf(-2.0f * x, cos2, dcx), HK_C916_F * fmaf(y, dBx, dt2x));
  o.vy = fmaf(ex2, fmaf(eyp, cos2, ey * dcy), HK_C916_F * (B + fmaf(y, dBy, dt2y)));
  return o;
}

// ------------------------------------------------- derivatives (adjoint)
// Value and partial derivatives in x and y of the line shapes of the three
// regions, for the vector-Jacobian product of the opacity.
struct VDer {
  double v, vx, vy;
};

// Algorithm 916 in FP64 with forward-mode derivatives: the series of
// voigt916_d (same terms, same stopping rule) with each term differentiated.
// With k = 2a/pi, q = sin(xy)^2 / y:
//   V  = e^{-x^2} erfcx(y) cos 2xy + k e^{-x^2} q + k y (-cos 2xy s1 + (s2 + s3)/2)
// and d erfcx/dy = 2y erfcx(y) - 2/sqrt(pi).  V is even in x.
// The Gaussian factors of the terms follow from recurrences instead of one
// exp per term: with E_n = exp(-a^2 n^2) (E_n = E_{n-1} exp(-a^2) exp(-2a^2)^{n-1}),
//   exp(-(a^2 n^2 + x^2)) = e^{-x^2} E_n,   exp(-(an + x)^2) = e^{-x^2} E_n R^n,
//   exp(-(d + an)^2) = e^{-d^2} E_n P^n,    exp(-(d' - an)^2) = e^{-d'^2} E_n M^n,
// R = exp(-2a|x|), d = a(n0 - 1) - |x|, P = exp(-2ad), d' = a n0 - |x|,
// M = exp(2ad'): four exps per call in place of four per term (a few ulp
// apart from the direct exps over the 10-15 terms the tolerance needs).
constexpr double HK_E916_A2 = 0.778805723222652;   // exp(-a^2), a = HK_A916_D
constexpr double HK_E916_2A2 = 0.606538354524358;  // exp(-2 a^2)

__host__ __device__ inline double hk_rcp_d(double v) {
#ifdef __CUDA_ARCH__
  return __drcp_rn(v);
#else
  return 1.0 / v;
#endif
}

__host__ __device__ __noinline__ inline VDer voigt916_dd(double x, double y, double ey) {
  const double a = HK_A916_D;
  const double ax = fabs(x), sx = x < 0.0 ? -1.0 : 1.0;
  const double ex2 = exp(-ax * ax);
  const double isp = 0.56418958354775628695;  // 1/sqrt(pi)
  VDer o;
  if (ax == 0.0) {
    o.v = ey;
    o.vx = 0.0;
    o.vy = 2.0 * y * ey - 2.0 * isp;
    return o;
  }
  // s1, s2, s3 and, per sum, the weighted sums its derivatives need:
  //   s1f = sum f^2 e1,  s2w = sum (an + x) f e2,  s2f = sum f^2 e2,
  //   s3w = sum (a n3 - x) f3 e3,  s3f = sum f3^2 e3
  double s1 = 0.0, s2 = 0.0, s3 = 0.0, s1f = 0.0, s2w = 0.0, s2f = 0.0, s3w = 0.0, s3f = 0.0;
  {
    double o1 = 0.0, o2 = 0.0, o3 = 0.0;
    const double yy = y * y;
    const int n0 = (int)ceil(ax / a);
    const double d = a * (n0 - 1) - ax, d2 = a * n0 - ax;
    const double R = exp(-2.0 * a * ax), P = exp(-2.0 * a * d), M = exp(2.0 * a * d2);
    const double ex2p = exp(-d * d), ex2n = exp(-d2 * d2);
    double E = 1.0, gE = HK_E916_A2, Rn = 1.0, Pn = 1.0, Mn = 1.0;
    bool st1 = false, st2 = false, st3 = false;
    for (int n = 1; n < 100; ++n) {
      const int n3p = n0 + n - 1, n3n = n0 - n;
      E *= gE;
      gE *= HK_E916_2A2;
      Rn *= R;
      Pn *= P;
      Mn *= M;
      const double an = a * n, an3p = a * n3p;
      const double f = hk_rcp_d(an * an + yy);
      const double f3p = hk_rcp_d(an3p * an3p + yy);
      const double e1 = ex2 * E;
      const double fe1 = f * e1, fe2 = fe1 * Rn, fe3 = f3p * (ex2p * E * Pn);
      s1 += fe1;
      s1f += f * fe1;
      s2 += fe2;
      s2w += (an + ax) * fe2;
      s2f += f * fe2;
      s3 += fe3;
      s3w += (d + an) * fe3;
      s3f += f3p * fe3;
      if (n3n >= 1) {
        const double an3n = a * n3n;
        const double f3n = hk_rcp_d(an3n * an3n + yy);
        const double fe = f3n * (ex2n * E * Mn);
        s3 += fe;
        s3w += (d2 - an) * fe;
        s3f += f3n * fe;
      }
      if (fabs(s1 - o1) < HK_TOL) st1 = true;
      if (fabs(s2 - o2) < HK_TOL) st2 = true;
      if (fabs(s3 - o3) < HK_TOL) st3 = true;
      if (st1 && st2 && st3) break;
      o1 = s1;
      o2 = s2;
      o3 = s3;
    }
  }
  const double s1x = -2.0 * ax * s1, s1y = -2.0 * y * s1f;
  const double s2x = -2.0 * s2w, s2y = -2.0 * y * s2f;
  const double s3x = 2.0 * s3w, s3y = -2.0 * y * s3f;
  const double xy = ax * y;
  double c2, sn2;
#ifdef __CUDA_ARCH__
  sincos(2.0 * xy, &sn2, &c2);
#else
  sn2 = sin(2.0 * xy);
  c2 = cos(2.0 * xy);
#endif
  const double sn = sin(xy);
  const double k = 2.0 * a / CUDART_PI;
  double q, qy;
  if (y != 0.0) {
    q = sn * sn / y;
    qy = ax * sn2 / y - q / y;
  } else {
    q = 0.0;
    qy = ax * ax;
  }
  const double br = -c2 * s1 + 0.5 * (s2 + s3);
  o.v = ex2 * ey * c2 + k * ex2 * q + k * y * br;
  const double vx = ey * (-2.0 * ax * ex2 * c2 - 2.0 * y * ex2 * sn2) +
                    k * (-2.0 * ax * ex2 * q + ex2 * sn2) +
                    k * y * (2.0 * y * sn2 * s1 - c2 * s1x + 0.5 * (s2x + s3x));
  o.vy = ex2 * ((2.0 * y * ey - 2.0 * isp) * c2 - 2.0 * ax * ey * sn2) + k * ex2 * qy + k * br +
         k * y * (2.0 * ax * sn2 * s1 - c2 * s1y + 0.5 * (s2y + s3y));
  o.vx = sx * vx;
  if (y == 0.0) o.v = ex2;
  return o;
}

// GH2 rational of region B (gh2_d) and its partials in s = x^2 and Y = y^2:
// t = num / den, num = a1 (u + 1) - (4/pi) s, den = u (a1^2 - (6/pi) s),
// u = s + Y, a1 = u + 1.5.
template <class F>
__device__ __forceinline__ void gh2_grad(F s, F Y, F &t, F &ts, F &tY) {
  const F u = s + Y;
  const F a1 = u + F(1.5);
  const F c4 = F(4.0 / CUDART_PI), c6 = F(6.0 / CUDART_PI);
  const F num = a1 * (u + F(1)) - c4 * s;
  const F q = a1 * a1 - c6 * s;
  const F den = u * q;
  t = num / den;
  const F num_s = (u + F(1)) + a1 - c4, num_Y = (u + F(1)) + a1;
  const F den_s = q + u * (F(2) * a1 - c6), den_Y = q + u * F(2) * a1;
  ts = (num_s - t * den_s) / den;
  tY = (num_Y - t * den_Y) / den;
}

}  // namespace hkb
