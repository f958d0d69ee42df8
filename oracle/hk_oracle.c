/*
 * hk_oracle.c -- FP64 CPU restatement of the HELIOS-K opacity hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and the
 * timed CPU baseline.  The product never links or calls this file.
 *
 * Built with -O2 -ffp-contract=off -fopenmp (see oracle/Makefile) so that
 * every FP64 predicate below is the plain IEEE sequence written here.
 * Where the reference's CUDA code is contracted to an FMA by nvcc
 * (a*b + c in one expression), the restatement calls fma() explicitly.
 */
#include "hk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ grid */

/* voigt.h:751-768 (setX_kernel): x_d[id] = numin + id * dnu, contracted. */
double hko_grid_x(double numin, double dnu, int64_t i) {
  return fma((double)i, dnu, numin);
}

/* heliosk.cu:448-455: Nx = (int)((numax - numin) / dnu + 0.5) */
int hko_grid_nx(double numin, double numax, double dnu) {
  return (int)((numax - numin) / dnu + 0.5);
}

void hko_grid_fill(double numin, double dnu, int64_t nx, double *x) {
  for (int64_t i = 0; i < nx; ++i) x[i] = hko_grid_x(numin, dnu, i);
}

/* Bin boundaries heliosk.cu:436-441, binKey_kernel voigt.h:779-805,
 * binIndex_kernel voigt.h:815-832. */
void hko_bin_keys(double numin, double numax, double dnu, int64_t nx, int nbins,
                  int32_t *key, int32_t *bin_index) {
  double *bb = (double *)malloc((size_t)(nbins + 1) * sizeof(double));
  for (int i = 0; i < nbins; ++i)
    bb[i] = numin + i * (numax - numin) / ((double)nbins);
  bb[nbins] = numax;
  for (int64_t id = 0; id < nx; ++id) {
    double nu = hko_grid_x(numin, dnu, id);
    int32_t k = 0;
    /* first bin with bb[i] <= nu < bb[i+1]; the intervals are disjoint so a
     * binary search finds the same bin the reference's linear scan finds */
    int lo = 0, hi = nbins - 1, found = -1;
    while (lo <= hi) {
      int mid = (lo + hi) / 2;
      if (nu < bb[mid]) hi = mid - 1;
      else if (nu >= bb[mid + 1]) lo = mid + 1;
      else { found = mid; break; }
    }
    if (found >= 0) k = found;
    if (nu >= numax) k = nbins;
    key[id] = k;
  }
  if (bin_index) {
    for (int i = 0; i < nbins + 2; ++i) bin_index[i] = 0;
    for (int64_t id = 0; id + 1 < nx; ++id) {
      int32_t b0 = key[id], b1 = key[id + 1];
      if (b1 > b0) bin_index[b1] = (int32_t)(id + 1);
    }
    bin_index[0] = 0;
    bin_index[nbins] = (int32_t)nx;
    bin_index[nbins + 1] = (int32_t)nx;
  }
  free(bb);
}

/* ------------------------------------------------------- partition Q(T) */

/* host.h:9-73 readPartition: walk the table, first row with T1 >= T,
 * linear interpolation between the previous row and that row.
 * Returns 1 on success, 0 on the reference's error conditions. */
int hko_partition_interp(const double *Tq, const double *q, int nq, double T,
                         double *Q_out) {
  double T0, T1 = -1.0, q0, q1 = 1.0, qv = 1.0;
  for (int j = 0; j < 100000; ++j) {
    T0 = T1;
    q0 = q1;
    if (j >= nq) return 0; /* fscanf returned EOF */
    T1 = Tq[j];
    q1 = q[j];
    if (T0 == T1 && T0 < T && j > 0) return 0;
    if (T1 > T && j == 0) return 0;
    if (T0 < T && T1 >= T) {
      double tt = (T - T0) / (T1 - T0);
      qv = (q1 - q0) * tt + q0;
      if (j == 0) qv = q1;
      *Q_out = qv;
      return 1;
    }
  }
  return 0;
}

/* ------------------------------------------------------------ line prep */

/* host.h:598-649 (readFile) followed by voigt.h:331-363 (S2_kernel). */
void hko_prep_hitran(int64_t n, const double *nu, const double *S_file,
                     const double *EL, const double *A, const double *delta,
                     const double *gair, const double *gself,
                     const double *nexp, const int32_t *iso, int niso,
                     const double *iso_mass, const double *iso_ab,
                     const double *iso_Q, double T, double P, double qalphaL,
                     double gammaF, int units, double meanMass, double Sscale,
                     double *out_nu, double *out_S, double *out_iad,
                     double *out_vy) {
  const double c = HKO_H * HKO_C / HKO_KB;
  (void)niso;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int j = iso[i];
    double mass = iso_mass[j] / HKO_NA;
    double Abundance = iso_ab[j];
    double Sscale1 = Sscale;
    if (units == 0) {
      Abundance *= iso_mass[j] / meanMass;
      Sscale1 *= iso_mass[j] / meanMass;
    }
    double Q = iso_Q[j];
    double vy = (1.0 - qalphaL) * gair[i] + qalphaL * gself[i];
    vy *= gammaF;
    double iad0 = HKO_C * sqrt(mass / (2.0 * HKO_KB * T));
    double S = S_file[i] / Q * Abundance * Sscale1;
    /* S2_kernel */
    double nuv = fma(delta[i], P, nu[i]);
    double iad = iad0 / nuv;
    double el = EL[i];
    S *= exp(-el * c / T + el * c / HKO_T0) * (1.0 - exp(-c * nuv / T)) /
         (1.0 - exp(-c * nuv / HKO_T0)) * iad;
    double aL = vy * ((P / HKO_PO_ATM) * pow(HKO_T0 / T, nexp[i]));
    aL = aL + A[i] / (4.0 * M_PI * HKO_C);
    double vyv = aL * iad;
    if (nuv == 0.0) {
      S = 0.0;
      iad = 0.0;
      vyv = 0.0;
    }
    out_nu[i] = nuv;
    out_S[i] = S;
    out_iad[i] = iad;
    out_vy[i] = vyv;
  }
}

/* voigt.h:484-504 (L_kernelExomol) followed by voigt.h:365-397 (Sf_kernel),
 * with the caller-side scalings of heliosk.cu:1064-1070. */
void hko_prep_exomol(int64_t n, const double *nu, const double *S_file,
                     const double *EL, const double *A, double mass_g_mol,
                     double ab, double Q, double defaultL, double defaultn,
                     double T, double P, double gammaF, int units,
                     double meanMass, double Sscale, double *out_nu,
                     double *out_S, double *out_iad, double *out_vy) {
  double mass = mass_g_mol / HKO_NA;
  double Abundance = ab;
  if (units == 0) {
    Abundance *= mass_g_mol / meanMass;
    Sscale *= mass_g_mol / meanMass;
  }
  const double c1 = HKO_H * HKO_C / (HKO_KB * T);
  const double T1 = HKO_T0 / T;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double nuv = nu[i];
    double iad0 = HKO_C * sqrt(mass / (2.0 * HKO_KB * T));
    double Ad = A[i] / (4.0 * M_PI * HKO_C);
    double vy = defaultL * gammaF;
    double S = S_file[i] * Abundance * Sscale / Q;
    double iad = iad0 / nuv;
    S *= exp(-c1 * EL[i]) * (1.0 - exp(-c1 * nuv)) * iad;
    double aL = vy * ((P / HKO_PO_BAR) * pow(T1, defaultn));
    aL = aL + Ad;
    double vyv = aL * iad;
    if (nuv == 0.0) {
      S = 0.0;
      iad = 0.0;
      vyv = 0.0;
    }
    out_nu[i] = nuv;
    out_S[i] = S;
    out_iad[i] = iad;
    out_vy[i] = vyv;
  }
}

/* -------------------------------------------------------------- windows */

typedef struct {
  double numin, dnu, nu, iad, vy2, w;
} wctx;

static inline double w_d(const wctx *c, int64_t i) {
  return hko_grid_x(c->numin, c->dnu, i) - c->nu;
}
static inline double w_r2(const wctx *c, int64_t i) {
  double x = w_d(c, i) * c->iad;
  return x * x + c->vy2;
}
/* predicate kinds: all monotone false..true over the searched range */
enum { P_LEFT_CUT, P_RIGHT_CUT, P_CENTER, P_LEFT_R, P_RIGHT_R };
static inline int w_pred(const wctx *c, int kind, int64_t i, double R) {
  switch (kind) {
  case P_LEFT_CUT: return w_d(c, i) > -c->w;  /* inside from the left  */
  case P_RIGHT_CUT: return w_d(c, i) >= c->w; /* outside on the right   */
  case P_CENTER: return w_d(c, i) >= 0.0;
  case P_LEFT_R: return w_r2(c, i) < R;       /* i < centre            */
  default: return w_r2(c, i) >= R;            /* i >= centre           */
  }
}

/* First index in [lo, hi) where the monotone predicate is true, hi if none.
 * The result does not depend on the estimate e. */
static int64_t first_true(const wctx *c, int kind, double R, int64_t lo,
                          int64_t hi, int64_t e) {
  if (lo >= hi) return lo;
  if (e < lo) e = lo;
  if (e > hi) e = hi;
  /* bracket [a, b]: every index below a is false (or a == lo), b is true
   * (index hi counts as true); gallop outwards from the estimate e */
  int64_t a, b;
  if (e >= hi || w_pred(c, kind, e, R)) {
    b = e;
    int64_t step = 1;
    while (1) {
      int64_t t = b - step;
      if (t < lo) { a = lo; break; }
      if (!w_pred(c, kind, t, R)) { a = t + 1; break; }
      b = t;
      step *= 2;
    }
  } else {
    a = e + 1;
    int64_t step = 1;
    while (1) {
      int64_t t = a - 1 + step;
      if (t >= hi) { b = hi; break; }
      if (w_pred(c, kind, t, R)) { b = t; break; }
      a = t + 1;
      step *= 2;
    }
  }
  /* binary search in [a, b]: pred false before a, true at b (or b == hi) */
  while (a < b) {
    int64_t m = a + (b - a) / 2;
    if (w_pred(c, kind, m, R)) b = m;
    else a = m + 1;
  }
  return a;
}

static int64_t est_index(double nu_edge, double numin, double dnu, int64_t nx) {
  double e = ceil((nu_edge - numin) / dnu);
  if (!(e > -1.0)) return 0;        /* also catches NaN */
  if (e > (double)nx) return nx;
  return (int64_t)e;
}

/* Per-line index windows.  Restates the region classes of nuLimits_kernel
 * (voigt.h:2205-2341) and the per-pair predicates of Line6fA/B/C
 * (voigt.h:1223, 1481, 1662) as exact FP64 index ranges:
 *   cut window  [i0, i1)     : |x_i - nu| < w
 *   B or C      [b0, b1)     : r2 < 1e6   (inside the cut window)
 *   C           [c0, c1)     : r2 < 100   (inside the cut window)
 * win[6*l + 0..5] = i0, b0, c0, c1, b1, i1.
 * Lines with S == 0 or ialphaD == 0 contribute exactly zero in the
 * reference (S2_kernel zeroes them, voigt.h:355-359) and get empty windows. */
void hko_windows(int64_t n, const double *nu, const double *S,
                 const double *iad, const double *vy, double numin, double dnu,
                 int64_t nx, int cutMode, double cut, int64_t *win) {
  hko_windows_p(n, nu, S, iad, vy, numin, dnu, nx, cutMode, cut, 1, win);
}

/* profiles 2-4 have no regions B and C (nuLimits_kernel voigt.h:2250) */
void hko_windows_p(int64_t n, const double *nu, const double *S,
                   const double *iad, const double *vy, double numin, double dnu,
                   int64_t nx, int cutMode, double cut, int profile, int64_t *win) {
  if (cut == 0.0) cut = 1.0e30; /* heliosk.cu:947 */
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < n; ++l) {
    int64_t *o = win + 6 * l;
    if (S[l] == 0.0 || iad[l] == 0.0 || !(iad[l] > 0.0)) {
      for (int k = 0; k < 6; ++k) o[k] = 0;
      continue;
    }
    wctx c;
    c.numin = numin;
    c.dnu = dnu;
    c.nu = nu[l];
    c.iad = iad[l];
    c.vy2 = vy[l] * vy[l];
    double w;
    if (cutMode == 1) w = cut * vy[l] / iad[l];
    else if (cutMode == 2) w = cut / iad[l];
    else w = cut;
    c.w = w;
    int64_t i0 = first_true(&c, P_LEFT_CUT, 0, 0, nx,
                            est_index(c.nu - w, numin, dnu, nx));
    int64_t i1 = first_true(&c, P_RIGHT_CUT, 0, i0, nx,
                            est_index(c.nu + w, numin, dnu, nx));
    if (i1 <= i0) {
      for (int k = 0; k < 6; ++k) o[k] = i0;
      continue;
    }
    int64_t ic = first_true(&c, P_CENTER, 0, i0, i1,
                            est_index(c.nu, numin, dnu, nx));
    int64_t bc[2][2];
    const double Rs[2] = {1.0e6, 100.0};
    for (int r = 0; r < 2; ++r) {
      double R = Rs[r];
      double h2 = R - c.vy2;
      int64_t lo, hi;
      if (profile == 1 && h2 > 0.0) {
        double h = sqrt(h2) / c.iad;
        lo = first_true(&c, P_LEFT_R, R, i0, ic,
                        est_index(c.nu - h, numin, dnu, nx));
        hi = first_true(&c, P_RIGHT_R, R, ic, i1,
                        est_index(c.nu + h, numin, dnu, nx));
      } else {
        lo = ic;
        hi = ic;
      }
      bc[r][0] = lo;
      bc[r][1] = hi;
    }
    o[0] = i0;
    o[1] = bc[0][0];
    o[2] = bc[1][0];
    o[3] = bc[1][1];
    o[4] = bc[0][1];
    o[5] = i1;
  }
}

/* --------------------------------------------------------------- profile */

/* Scaled complementary error function erfcx(y) = exp(y^2) erfc(y), y >= 0.
 * Own implementation from classical expansions (test oracle only):
 *   y < 0.5      : erfc = 1 - erf, erf from its Maclaurin series
 *                  erf(y) = 2/sqrt(pi) sum (-1)^k y^(2k+1) / (k! (2k+1));
 *   0.5 <= y < 2 : erf(y) = 2/sqrt(pi) exp(-y^2) sum 2^k y^(2k+1)/(2k+1)!!
 *                  (all terms positive), erfcx = exp(y^2) - that sum;
 *   y >= 2       : Laplace continued fraction
 *                  sqrt(pi) erfcx(y) = 1/(y + (1/2)/(y + 1/(y + (3/2)/(y + ...))))
 *                  evaluated bottom-up at fixed depth.
 * Checked against scipy.special.erfcx in tests/test_oracle_profile.py. */
double hko_erfcx(double y) {
  const double isqpi = 0.56418958354775628695; /* 1/sqrt(pi) */
  if (y < 0.0) return 2.0 * exp(y * y) - hko_erfcx(-y);
  if (y < 0.5) {
    double y2 = y * y, term = y, sum = y;
    for (int k = 1; k < 60; ++k) {
      term *= -y2 / (double)k;
      double add = term / (double)(2 * k + 1);
      sum += add;
      if (fabs(add) < 1e-18 * fabs(sum)) break;
    }
    return exp(y2) * (1.0 - 2.0 * isqpi * sum);
  }
  if (y < 2.0) {
    double y2 = y * y, term = y, sum = y;
    for (int k = 1; k < 400; ++k) {
      term *= 2.0 * y2 / (double)(2 * k + 1);
      sum += term;
      if (term < 1e-18 * sum) break;
    }
    return exp(y2) - 2.0 * isqpi * sum;
  }
  double f = y;
  for (int k = 400; k >= 1; --k) f = y + (0.5 * k) / f;
  return isqpi / f;
}

/* Zaghloul & Ali, Algorithm 916, as restated in voigt.h:165-216 (Sigmab)
 * and voigt.h:278-300 (voigt_916), FP64 with def_TOL, a = pi/sqrt(-ln(TOL/2)).
 * ey = erfcx(y) (per-line constant). */
static double voigt916_ey(double x, double y, double ey) {
  static double a = 0.0;
  if (a == 0.0) a = M_PI * sqrt(-1.0 / log(HKO_TOL * 0.5));
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  double ex2 = exp(-x * x);
  double ax = fabs(x);
  if (x != 0.0 && y != 0.0) {
    double sold1 = 0.0, sold2 = 0.0, sold3 = 0.0;
    double yy = y * y;
    int n0 = (int)ceil(ax / a);
    int stop1 = 0, stop2 = 0, stop3 = 0;
    for (int n = 1; n < 100; ++n) {
      int n3p = n0 + n - 1;
      int n3n = n0 - n;
      double an = a * n, an3p = a * n3p, an3n = a * n3n;
      double f = 1.0 / (an * an + yy);
      double f3p = 1.0 / (an3p * an3p + yy);
      double f3n = 1.0 / (an3n * an3n + yy);
      s1 += f * exp(-(an * an + ax * ax));
      s2 += f * exp(-(an + ax) * (an + ax));
      s3 += f3p * exp(-(an3p - ax) * (an3p - ax));
      if (n3n >= 1) s3 += f3n * exp(-(an3n - ax) * (an3n - ax));
      if (fabs(s1 - sold1) < HKO_TOL) stop1 = 1;
      if (fabs(s2 - sold2) < HKO_TOL) stop2 = 1;
      if (fabs(s3 - sold3) < HKO_TOL) stop3 = 1;
      if (stop1 && stop2 && stop3) break;
      sold1 = s1;
      sold2 = s2;
      sold3 = s3;
    }
  }
  double xy = ax * y;
  double a2ipi = 2.0 * a / M_PI;
  double cos2xy = cos(2.0 * xy);
  double sinxy = sin(xy);
  double t1 = ex2 * ey * cos2xy;
  if (x != 0.0 && y != 0.0) {
    t1 += a2ipi * ax * sinxy * ex2 * sinxy / xy;
    t1 += a2ipi * y * (-cos2xy * s1 + 0.5 * (s2 + s3));
  }
  if (x == 0.0) t1 = ey;
  if (y == 0.0) t1 = ex2;
  return t1;
}

double hko_voigt916(double x, double y) {
  return voigt916_ey(x, y, hko_erfcx(y));
}

/* region B, 2nd-order Gauss-Hermite, voigt.h:1481-1490; returns t4 such
 * that the contribution is S1 * t4 with S1 = S * y / pi */
double hko_gh2(double x, double y) {
  double t1 = x * x;
  double r2 = t1 + y * y;
  t1 *= 6.0;
  double t2 = r2 + 1.5;
  double t3 = M_PI * t2;
  return (t3 * (2.0 * t2 + r2) - 2.0 * t1) / (3.0 * r2 * (t3 * t2 - t1));
}

/* --------------------------------------------------------------- opacity */

typedef struct {
  int64_t i0;
  int64_t l;
} lkey;

static int cmp_lkey(const void *a, const void *b) {
  const lkey *x = (const lkey *)a, *y = (const lkey *)b;
  if (x->i0 < y->i0) return -1;
  if (x->i0 > y->i0) return 1;
  return (x->l < y->l) ? -1 : (x->l > y->l);
}

/* Sum of the Voigt contributions of all lines onto the grid:
 *   C: S * V(x, y) / sqrt(pi)         (voigt.h:1662-1682, b = 1/sqrt(pi))
 *   B: S1 * t4,   S1 = S * y / pi     (voigt.h:1481-1490; S3_kernel 454)
 *   A: S1 / r2                        (voigt.h:1223-1227)
 * then K = kmin + sum (InitialK_kernel + AddKStreams_kernel, voigt.h:713-742).
 * OpenMP over grid tiles; each tile owns its points, so no atomics. */
void hko_opacity(int64_t n, const double *nu, const double *S,
                 const double *iad, const double *vy, const int64_t *win,
                 double numin, double dnu, int64_t ib, int64_t ie, double kmin,
                 double *K, int nthreads, int64_t pairs_out[3]) {
  hko_opacity_p(n, nu, S, iad, vy, win, numin, dnu, ib, ie, kmin, 1, NULL, NULL, K, nthreads,
                pairs_out);
}

/* sLChi (voigt.h:47-72) times x / nu inside (lo, hi), as Line6fAX/BX/CX
 * apply it; sl = {sigma1, sigma2, sigma3, B1, B2, B3, lo, hi} */
static double sublorentz(const double *sl, double x, double nu) {
  if (!(x > sl[6] && x < sl[7])) return 1.0;
  const double d = fabs(x - nu);
  double chi;
  if (d < sl[0]) chi = 1.0;
  else if (d < sl[1]) chi = exp(-sl[3] * (d - sl[0]));
  else if (d < sl[2]) chi = exp(-sl[3] * (sl[1] - sl[0]) - sl[4] * (d - sl[1]));
  else chi = exp(-sl[3] * (sl[1] - sl[0]) - sl[4] * (sl[2] - sl[1]) - sl[5] * (d - sl[2]));
  return chi * x / nu;
}

/* profiles 2-4 at x (Doppler units): Line6fA_kernel voigt.h:1235-1262 with
 * S1 of S3_kernel voigt.h:452-463 (S y / pi, S / sqrt(pi), S) */
/* erf(a) - erf(b), a > b, through erfc on the same side of zero (no
 * cancellation in the wings) */
static double erf_diff(double a, double b) {
  if (b >= 0.0) return erfc(b) - erfc(a);
  if (a <= 0.0) return erfc(-a) - erfc(-b);
  return erf(a) - erf(b);
}

static double profile_a(int profile, double x, double S, double y, double vb) {
  if (profile == 3) return S / sqrt(M_PI) * exp(-(x * x));
  if (profile == 4) return S * (1.0 / vb) * 0.5 * erf_diff(x + 0.5 * vb, x - 0.5 * vb);
  return S * y / M_PI / (x * x + y * y);
}

/* Plinth_kernel (voigt.h:1091-1164) in FP64: the profile at the cut edge
 * x_c = cut iad (cutMode 0), cut y (1), cut (2); 0 for profile 4 and for
 * lines without a window. */
void hko_plinth(int64_t n, const double *S, const double *iad, const double *vy,
                const int64_t *win, int cutMode, double cut, int profile, double *out) {
  if (cut == 0.0) cut = 1.0e30;
  for (int64_t l = 0; l < n; ++l) {
    const int64_t *o = win + 6 * l;
    out[l] = 0.0;
    if (!(o[5] > o[0]) || profile == 4) continue;
    const double y = vy[l];
    const double xc = (cutMode == 1) ? cut * y : (cutMode == 2 ? cut : cut * iad[l]);
    if (profile != 1) {
      out[l] = profile_a(profile, xc, S[l], y, 0.0);
      continue;
    }
    const double r2 = xc * xc + y * y;
    const double S1 = S[l] * y / M_PI;
    if (r2 >= 1.0e6) {
      out[l] = S1 / r2;
    } else if (r2 >= 100.0) {
      out[l] = S1 * hko_gh2(xc, y);
    } else {
      out[l] = S[l] / sqrt(M_PI) * hko_voigt916(xc, y);
    }
  }
}

void hko_opacity_p(int64_t n, const double *nu, const double *S,
                   const double *iad, const double *vy, const int64_t *win,
                   double numin, double dnu, int64_t ib, int64_t ie, double kmin,
                   int profile, const double *plinth, const double *sl, double *K,
                   int nthreads, int64_t pairs_out[3]) {
  lkey *ord = (lkey *)malloc((size_t)(n > 0 ? n : 1) * sizeof(lkey));
  double *ey = (double *)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
  int64_t m = 0, wmax = 0;
  for (int64_t l = 0; l < n; ++l) {
    const int64_t *o = win + 6 * l;
    if (o[5] > o[0]) {
      ord[m].i0 = o[0];
      ord[m].l = l;
      ++m;
      if (o[5] - o[0] > wmax) wmax = o[5] - o[0];
    }
  }
  qsort(ord, (size_t)m, sizeof(lkey), cmp_lkey);
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < n; ++l) ey[l] = hko_erfcx(vy[l]);

  const int64_t TILE = 4096;
  int64_t ntile = (ie - ib + TILE - 1) / TILE;
  int64_t pa = 0, pb = 0, pc = 0;
  const double isqpi = 1.0 / sqrt(M_PI);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : pa, pb, pc)
  for (int64_t t = 0; t < ntile; ++t) {
    int64_t t0 = ib + t * TILE, t1 = t0 + TILE;
    if (t1 > ie) t1 = ie;
    double acc[4096];
    for (int64_t i = 0; i < t1 - t0; ++i) acc[i] = 0.0;
    /* candidate lines: i0 in (t0 - wmax, t1) */
    int64_t lo = 0, hi = m;
    int64_t key = t0 - wmax;
    while (lo < hi) {
      int64_t mid = (lo + hi) / 2;
      if (ord[mid].i0 <= key) lo = mid + 1;
      else hi = mid;
    }
    for (int64_t q = lo; q < m && ord[q].i0 < t1; ++q) {
      int64_t l = ord[q].l;
      const int64_t *o = win + 6 * l;
      int64_t a0 = o[0] > t0 ? o[0] : t0;
      int64_t a1 = o[5] < t1 ? o[5] : t1;
      if (a0 >= a1) continue;
      double nul = nu[l], il = iad[l], y = vy[l], Sl = S[l];
      double S1 = Sl * y / M_PI;
      double y2 = y * y;
      for (int64_t i = a0; i < a1; ++i) {
        double d = hko_grid_x(numin, dnu, i) - nul;
        double x = d * il;
        double v;
        if (i >= o[2] && i < o[3]) {
          v = Sl * voigt916_ey(x, y, ey[l]) * isqpi;
          ++pc;
        } else if (i >= o[1] && i < o[4]) {
          double t1x = x * x;
          double r2 = t1x + y2;
          t1x *= 6.0;
          double t2 = r2 + 1.5;
          double t3 = M_PI * t2;
          double t4 =
              (t3 * (2.0 * t2 + r2) - 2.0 * t1x) / (3.0 * r2 * (t3 * t2 - t1x));
          v = S1 * t4;
          ++pb;
        } else if (profile != 1) {
          v = profile_a(profile, x, Sl, y, dnu * il);
          ++pa;
        } else {
          double r2 = x * x + y2;
          v = S1 / r2;
          ++pa;
        }
        if (sl) v *= sublorentz(sl, hko_grid_x(numin, dnu, i), nul);
        acc[i - t0] += v;
        if (plinth) acc[i - t0] -= plinth[l];
      }
    }
    for (int64_t i = t0; i < t1; ++i) K[i - ib] = kmin + acc[i - t0];
  }
  if (pairs_out) {
    pairs_out[0] = pa;
    pairs_out[1] = pb;
    pairs_out[2] = pc;
  }
  free(ord);
  free(ey);
}

/* ------------------------------------------------------- k-distribution */

/* resample.h:14-37 (Vandermonde_kernel), column-major V[id + nxb*i]. */
void hko_vandermonde(int nxb, int nc, double *V) {
  for (int id = 0; id < nxb; ++id) {
    double x = id * 2.0 / ((double)nxb - 1.0) - 1.0;
    V[id] = 1.0;
    if (nc > 1) V[id + (int64_t)nxb] = x;
    double t = x, t0 = 1.0;
    for (int i = 2; i < nc; ++i) {
      double tt = t;
      t = fma(2.0 * x, t, -t0);
      t0 = tt;
      V[id + (int64_t)nxb * i] = t;
    }
  }
}

/* resample.h:73-227 (QR_kernel): scaled Householder QR of the nxb x nc
 * matrix in place; C[i] = sigma (v_ii + sigma), D[i] = -scale sigma. */
void hko_qr(int nxb, int nc, double *V, double *C, double *D) {
  for (int i = 0; i < nc; ++i) {
    double *vi = V + (int64_t)nxb * i;
    double scale = 0.0;
    for (int k = i; k < nxb; ++k) scale = fmax(scale, fabs(vi[k]));
    double ss = 0.0;
    for (int k = i; k < nxb; ++k) {
      double v = vi[k] / scale;
      vi[k] = v;
      ss = fma(v, v, ss);
    }
    double s = sqrt(ss);
    double v0 = vi[i];
    double sigma = (v0 < 0.0) ? -s : s;
    vi[i] += sigma;
    C[i] = sigma * (v0 + sigma);
    D[i] = -scale * sigma;
    for (int j = i + 1; j < nc; ++j) {
      double *vj = V + (int64_t)nxb * j;
      double dot = 0.0;
      for (int k = i; k < nxb; ++k) dot = fma(vi[k], vj[k], dot);
      double t = dot / C[i];
      for (int k = i; k < nxb; ++k) vj[k] = fma(-t, vi[k], vj[k]);
    }
  }
}

static int cmp_double(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x < y) ? -1 : (x > y);
}

/* heliosk.cu:2046-2051: sort_by_key(K, binKey) then
 * stable_sort_by_key(binKey, K) == ascending K inside each bin segment. */
void hko_sort_bins(int64_t nx, const int32_t *bin_index, int nbins, double *K) {
  (void)nx;
  for (int b = 0; b <= nbins; ++b) {
    int64_t s = bin_index[b], e = bin_index[b + 1];
    if (e > s) qsort(K + s, (size_t)(e - s), sizeof(double), cmp_double);
  }
}

/* resample.h:362-388 (findCut_kernel), one pass over the state in index
 * order.  Where the kernel's threads could race on one bin (the id == NL-3
 * rule against a later transition), the later index wins here. */
void hko_find_cut(const double *K, int64_t nx, int nxb, double kmin,
                  int nbins, int32_t *nxmin) {
  for (int b = 0; b < nbins; ++b) nxmin[b] = 0;
  for (int64_t id = 0; id < nx - 1; ++id) {
    int64_t ib = id / nxb;
    if (ib >= nbins) break;
    double k = K[id], k1 = K[id + 1];
    if (k <= kmin && k1 > kmin) nxmin[ib] = (int32_t)(id - ib * nxb + 1);
    if (k <= kmin && id % nxb == nxb - 1) nxmin[ib] = nxb;
    if (k <= kmin && id == nx - 3) nxmin[ib] = nxb;
  }
}

/* rescale_kernel f = +1 (resample.h:405-417) for one bin */
static void rescale_fwd(const double *Kb, double *out, int nxb, int nxmin) {
  for (int j = 0; j < nxb; ++j) {
    double ii = fma(1.0 - nxmin / ((double)(nxb - 1)), (double)j, (double)nxmin);
    if (ii >= nxb - 1) ii = 0.999999 * (nxb - 1);
    int il = (int)(ii / ((double)nxb) * nxb);
    double Kl = Kb[il], Kr = Kb[il + 1];
    out[j] = fma(Kr - Kl, ii - il, Kl);
  }
}

/* rescale_kernel f = -1 (resample.h:418-431) for one bin */
static void rescale_inv(const double *Kb, double *out, int nxb, int nxmin,
                        double kmin) {
  for (int j = 0; j < nxb; ++j) {
    double Ki = kmin;
    if (j >= nxmin) {
      double ii = (j - nxmin) / ((double)(nxb - nxmin - 1)) * (nxb - 1);
      if (ii >= nxb - 1) ii = 0.999999 * (nxb - 1);
      int il = (int)(ii / ((double)nxb) * nxb);
      double Kl = Kb[il], Kr = Kb[il + 1];
      Ki = fma(Kr - Kl, ii - il, Kl);
    }
    out[j] = Ki;
  }
}

/* The post-sort chain of heliosk.cu:2139-2193 for one state:
 * findCut -> rescale(+1) -> copyK2 -> lnK -> leastSquare -> coefficients,
 * then (recon != NULL) expfx -> rescale(-1) -> copyK2.
 * K is the per-bin sorted state (nx values) and is overwritten with ln K.
 * leastSquare_kernel (resample.h:243-353) applies only the first nc-1
 * Householder reflections and its back-substitution reduction keeps only
 * the first 64 partial sums; both are restated. */
void hko_kdist(double *K, int64_t nx, int nxb, int nbins, int nc, double kmin,
               double unitScale, const double *V, const double *C,
               const double *D, int32_t *nxmin, double *coeff, double *recon) {
  hko_find_cut(K, nx, nxb, kmin, nbins, nxmin);
  double *tmp = (double *)malloc((size_t)nxb * sizeof(double));
  for (int b = 0; b < nbins; ++b) {
    double *Kb = K + (int64_t)b * nxb;
    if (nxmin[b] > 0) {
      rescale_fwd(Kb, tmp, nxb, nxmin[b]);
      memcpy(Kb, tmp, (size_t)nxb * sizeof(double));
    }
  }
  for (int64_t i = 0; i < nx; ++i) K[i] = log(K[i] * unitScale);
  int lim = nc < 64 ? nc : 64;
  for (int b = 0; b < nbins; ++b) {
    double *bb = K + (int64_t)b * nxb;
    for (int j = 0; j < nc - 1; ++j) {
      const double *vj = V + (int64_t)nxb * j;
      double dot = 0.0;
      for (int k = j; k < nxb; ++k) dot = fma(vj[k], bb[k], dot);
      double t = dot / C[j];
      for (int k = j; k < nxb; ++k) bb[k] = fma(-t, vj[k], bb[k]);
    }
    bb[nc - 1] /= D[nc - 1];
    for (int i = nc - 2; i >= 0; --i) {
      double s = 0.0;
      for (int j = i + 1; j < lim; ++j) s = fma(V[i + (int64_t)nxb * j], bb[j], s);
      bb[i] = (bb[i] - s) / D[i];
    }
    for (int i = 0; i < nc; ++i) coeff[(int64_t)b * nc + i] = bb[i];
  }
  if (recon) {
    for (int b = 0; b < nbins; ++b) {
      const double *cb = coeff + (int64_t)b * nc;
      double *rb = recon + (int64_t)b * nxb;
      /* expfx_kernel, resample.h:497-524 (x uses /Nxb, not /(Nxb-1)) */
      for (int j = 0; j < nxb; ++j) {
        double x = -1.0 + j * 2.0 / ((double)nxb);
        double d1 = 0.0, d2 = 0.0;
        for (int i = nc - 1; i >= 1; --i) {
          double t = d1;
          d1 = fma(2.0 * x, d1, -d2) + cb[i];
          d2 = t;
        }
        double f = fma(x, d1, -d2) + 0.5 * cb[0] + 0.5 * cb[0];
        rb[j] = exp(f) / unitScale;
      }
      if (nxmin[b] > 0) {
        rescale_inv(rb, tmp, nxb, nxmin[b], kmin);
        memcpy(rb, tmp, (size_t)nxb * sizeof(double));
      }
    }
  }
  free(tmp);
}

/* ---------------------------------------------------- reference gradient */

/* Algorithm 916 (voigt916_ey) with forward-mode derivatives in x and y:
 * every series term differentiated, same stopping rule.  With k = 2a/pi and
 * q = sin(xy)^2 / y:
 *   V = e^{-x^2} erfcx(y) cos 2xy + k e^{-x^2} q + k y (-cos 2xy s1 + (s2+s3)/2),
 *   d erfcx/dy = 2y erfcx(y) - 2/sqrt(pi).  Test oracle for the adjoint. */
static void voigt916_grad(double x, double y, double ey, double *v, double *vx, double *vyo) {
  static double a = 0.0;
  if (a == 0.0) a = M_PI * sqrt(-1.0 / log(HKO_TOL * 0.5));
  const double ax = fabs(x), sx = x < 0.0 ? -1.0 : 1.0;
  const double ex2 = exp(-ax * ax), isp = 1.0 / sqrt(M_PI);
  if (ax == 0.0) {
    *v = ey;
    *vx = 0.0;
    *vyo = 2.0 * y * ey - 2.0 * isp;
    return;
  }
  double s1 = 0, s2 = 0, s3 = 0, s1y = 0, s2x = 0, s2y = 0, s3x = 0, s3y = 0;
  double o1 = 0, o2 = 0, o3 = 0;
  const double yy = y * y;
  const int n0 = (int)ceil(ax / a);
  int st1 = 0, st2 = 0, st3 = 0;
  for (int n = 1; n < 100; ++n) {
    const int n3p = n0 + n - 1, n3n = n0 - n;
    const double an = a * n, ap = a * n3p, am = a * n3n;
    const double f = 1.0 / (an * an + yy), fp = 1.0 / (ap * ap + yy), fm = 1.0 / (am * am + yy);
    const double e1 = exp(-(an * an + ax * ax)), e2 = exp(-(an + ax) * (an + ax));
    const double ep = exp(-(ap - ax) * (ap - ax));
    s1 += f * e1;
    s1y -= 2.0 * y * f * f * e1;
    s2 += f * e2;
    s2x -= 2.0 * (an + ax) * f * e2;
    s2y -= 2.0 * y * f * f * e2;
    s3 += fp * ep;
    s3x += 2.0 * (ap - ax) * fp * ep;
    s3y -= 2.0 * y * fp * fp * ep;
    if (n3n >= 1) {
      const double em = exp(-(am - ax) * (am - ax));
      s3 += fm * em;
      s3x += 2.0 * (am - ax) * fm * em;
      s3y -= 2.0 * y * fm * fm * em;
    }
    if (fabs(s1 - o1) < HKO_TOL) st1 = 1;
    if (fabs(s2 - o2) < HKO_TOL) st2 = 1;
    if (fabs(s3 - o3) < HKO_TOL) st3 = 1;
    if (st1 && st2 && st3) break;
    o1 = s1;
    o2 = s2;
    o3 = s3;
  }
  const double s1x = -2.0 * ax * s1;
  const double xy = ax * y, c2 = cos(2.0 * xy), sn2 = sin(2.0 * xy), sn = sin(xy);
  const double k = 2.0 * a / M_PI;
  double q, qy;
  if (y != 0.0) {
    q = sn * sn / y;
    qy = ax * sn2 / y - q / y;
  } else {
    q = 0.0;
    qy = ax * ax;
  }
  const double br = -c2 * s1 + 0.5 * (s2 + s3);
  *v = (y == 0.0) ? ex2 : ex2 * ey * c2 + k * ex2 * q + k * y * br;
  *vx = sx * (ey * (-2.0 * ax * ex2 * c2 - 2.0 * y * ex2 * sn2) + k * (-2.0 * ax * ex2 * q + ex2 * sn2) +
              k * y * (2.0 * y * sn2 * s1 - c2 * s1x + 0.5 * (s2x + s3x)));
  *vyo = ex2 * ((2.0 * y * ey - 2.0 * isp) * c2 - 2.0 * ax * ey * sn2) + k * ex2 * qy + k * br +
         k * y * (2.0 * ax * sn2 * s1 - c2 * s1y + 0.5 * (s2y + s3y));
}

/* region B's GH2 t4 (hko_gh2, voigt.h:1481-1490) in the algebraically equal
 * form num/den, num = a1 (u+1) - (4/pi) s, den = u (a1^2 - (6/pi) s),
 * u = s + Y, a1 = u + 1.5 (s = x^2, Y = y^2), and its partials in s and Y */
static void gh2_grad(double s, double Y, double *t, double *ts, double *tY) {
  const double u = s + Y, a1 = u + 1.5, c4 = 4.0 / M_PI, c6 = 6.0 / M_PI;
  const double num = a1 * (u + 1.0) - c4 * s, q = a1 * a1 - c6 * s, den = u * q;
  *t = num / den;
  *ts = (((u + 1.0) + a1 - c4) - *t * (q + u * (2.0 * a1 - c6))) / den;
  *tY = (((u + 1.0) + a1) - *t * (q + u * 2.0 * a1)) / den;
}

/* Per-line sums of the vector-Jacobian product of K (test oracle of the
 * adjoint): with c_li the contribution of line l to K_i (hko_opacity's
 * regions), G[l] = sum_i u_i c_li, G[n+l] = sum_i u_i dc/dy,
 * G[2n+l] = sum_i u_i dc/dx x_li, G[3n+l] = sum_i u_i dc/dx, i over the line's
 * window inside [0, nx).  OpenMP over lines. */
/* profiles 3-4 (region A only): the shape c with its S1 and dc/dx, dc/dvb
 * (vb = dnu iad, the grid step in Doppler units): Doppler S/sqrt(pi)
 * e^{-x^2}; binned Gaussian S (erf(x+h) - erf(x-h)) / (2 vb), h = vb/2, whose
 * exponentials are taken from the larger one, e^{-(|x|-h)^2}, so neither the
 * difference nor the sum cancels or overflows. */
static void profile34_grad(int profile, double x, double S, double vb, double *c, double *cx,
                           double *cvb) {
  if (profile == 3) {
    const double v = S / sqrt(M_PI) * exp(-(x * x));
    *c = v;
    *cx = -2.0 * x * v;
    *cvb = 0.0;
    return;
  }
  const double h = 0.5 * vb, ax = fabs(x), sx = x < 0.0 ? -1.0 : 1.0;
  const double D = erf_diff(x + h, x - h);
  const double Eb = exp(-(ax - h) * (ax - h));
  const double dE = sx * Eb * expm1(-4.0 * ax * h); /* e^{-(x+h)^2} - e^{-(x-h)^2} */
  const double sE = Eb * (1.0 + exp(-4.0 * ax * h)); /* e^{-(x+h)^2} + e^{-(x-h)^2} */
  const double k = S / (2.0 * vb);
  *c = k * D;
  *cx = k * (2.0 / sqrt(M_PI)) * dE;
  *cvb = k * (sE / sqrt(M_PI) - D / vb);
}

void hko_vjp_sums(int64_t n, const double *nu, const double *S, const double *iad,
                  const double *vy, const int64_t *win, double numin, double dnu, int64_t nx,
                  const double *u, double *G, int profile, int nthreads) {
  const double isp = 1.0 / sqrt(M_PI);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t l = 0; l < n; ++l) {
    const int64_t *o = win + 6 * l;
    double gS = 0, gy = 0, gx = 0, gn = 0;
    const double y = vy[l], Sl = S[l], ey = hko_erfcx(vy[l]);
    const double Sp = Sl / M_PI;
    const int64_t a0 = o[0] > 0 ? o[0] : 0, a1 = o[5] < nx ? o[5] : nx;
    for (int64_t i = a0; i < a1 && Sl != 0.0; ++i) {
      const double x = (hko_grid_x(numin, dnu, i) - nu[l]) * iad[l];
      double c, cx, cy;
      if (profile >= 3) {
        /* the shape depends on iad through x and vb: G_x takes both */
        double cvb;
        const double vb = dnu * iad[l];
        profile34_grad(profile, x, Sl, vb, &c, &cx, &cvb);
        gS += u[i] * c;
        gx += u[i] * (cx * x + cvb * vb);
        gn += u[i] * cx;
        continue;
      }
      if (i >= o[2] && i < o[3]) {
        double v, vx, vyy;
        voigt916_grad(x, y, ey, &v, &vx, &vyy);
        c = Sl * isp * v;
        cx = Sl * isp * vx;
        cy = Sl * isp * vyy;
      } else {
        double t, ts, tY;
        if (i >= o[1] && i < o[4]) {
          gh2_grad(x * x, y * y, &t, &ts, &tY);
        } else {
          t = 1.0 / (x * x + y * y);
          ts = -t * t;
          tY = ts;
        }
        c = Sp * y * t;
        cx = Sp * y * ts * 2.0 * x;
        cy = Sp * (t + 2.0 * y * y * tY);
      }
      gS += u[i] * c;
      gy += u[i] * cy;
      gx += u[i] * cx * x;
      gn += u[i] * cx;
    }
    G[l] = gS;
    G[n + l] = gy;
    G[2 * n + l] = gx;
    G[3 * n + l] = gn;
  }
}

/* ------------------------------------------------ means, transmission */
/* end weights of resample.h:611-619: index idy gets w[idy], index n-1-idy
 * gets w[2-idy] (the reference's mirrored order, kept as it is) */
static const double hko_wS[3] = {-5.0 / 8.0, 1.0 / 6.0, -1.0 / 24.0};

/* resample.h:635-663 */
void hko_planck(double nu, double T, double *B, double *dBdT) {
  if (nu == 0.0) {
    *B = 0.0;
    *dBdT = 0.0;
    return;
  }
  const double nu3 = nu * nu * nu;
  const double t1 = 2.0 * HKO_H * nu3 * HKO_C * HKO_C;
  const double t2 = HKO_H * nu * HKO_C / (HKO_KB * T);
  const double e = exp(t2);
  const double e1 = e - 1.0;
  *B = t1 / e1;
  *dBdT = t1 * t2 / (T * (e - 2.0 + 1.0 / e));
}

/* resample.h:670-773 with useIndividualX = 0 */
void hko_means(const double *x, const double *K, int64_t nx, double T, double *out) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t k = 0; k < nx; ++k) {
    double B, R;
    hko_planck(x[k], T, &B, &R);
    s[0] += B * K[k];
    if (K[k] != 0.0) s[1] += R / K[k];
    s[2] += B;
    s[3] += R;
  }
  for (int idy = 0; idy < 3 && nx >= 3; ++idy) {
    const int64_t a = idy, b = nx - 1 - idy;
    double Ba, Ra, Bb, Rb;
    hko_planck(x[a], T, &Ba, &Ra);
    hko_planck(x[b], T, &Bb, &Rb);
    s[0] += hko_wS[idy] * (Ba * K[a]);
    s[0] += hko_wS[2 - idy] * (Bb * K[b]);
    if (K[a] != 0.0) s[1] += hko_wS[idy] * (Ra / K[a]);
    if (K[b] != 0.0) s[1] += hko_wS[2 - idy] * (Rb / K[b]);
    s[2] += hko_wS[idy] * Ba;
    s[2] += hko_wS[2 - idy] * Bb;
    s[3] += hko_wS[idy] * Ra;
    s[3] += hko_wS[2 - idy] * Rb;
  }
  for (int q = 0; q < 4; ++q) out[q] = s[q];
}

/* resample.h:541-608 */
void hko_transmission(const double *K, int nxb, int nbins, const int32_t *nxmin,
                      double kmin, int nTr, double dTr, double *Tr) {
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nbins; ++b) {
    const double *Kb = K + (int64_t)b * nxb;
    const int nm = nxmin ? nxmin[b] : 0;
    for (int j = 0; j < nTr; ++j) {
      const double m = exp((j - nTr / 2) * dTr);
      double a = 0.0;
      for (int k = 0; k < nxb; ++k) a += exp(-Kb[k] * m);
      for (int idy = 0; idy < 3 && nxb >= 3; ++idy) {
        a += hko_wS[idy] * exp(-Kb[idy] * m);
        a += hko_wS[2 - idy] * exp(-Kb[nxb - 1 - idy] * m);
      }
      Tr[(int64_t)b * nTr + j] = a / ((double)(nxb - 1)) * (nxb - nm) / ((double)nxb) +
                                 exp(-kmin * m) * nm / ((double)nxb);
    }
  }
}
