// hkb_prep.cuh -- one line scaled to one state: the per-(line, state) record
// the Voigt sum stages (sm_100a device code shared by line_prep_kernel and
// the fused T-P table kernel).
//
// Restates S2_kernel / Sf_kernel (voigt.h:331-397) through prep_line, the
// cutoff and S1 rules of S3_kernel (voigt.h:436-482), and the region classes
// of nuLimits_kernel (voigt.h:2205-2341) as the exact FP64 index windows of
// line_windows (hkb_device.cuh).
#pragma once

#include "hkb_device.cuh"

namespace hkb {

// MODE: PREP_ALL writes the record and updates the per-state maxima;
// PREP_STATS only the maxima (the state pass of a sectioned state);
// PREP_RECORDS only the record (one section's lines, the state already
// finalised).
enum { PREP_ALL = 0, PREP_STATS = 1, PREP_RECORDS = 2 };

// Line l of state st: FP64 scaling (prep_line), the global index windows
// (line_windows over [0, Nx)), and the region-C per-line constants erfcx(y)
// and Sig1(y) for lines that have a region-C window; the record goes to
// out[l] (LinePrepF for the mixed form, LinePrep for the plain FP64 form).
// w_loc accumulates the line's cutoff half-width (cm^-1; cutMode 1/2) and
// s1_loc its largest region-A/B term S1 / max(100, y^2) (the power-of-two
// scale of the mixed form's FP32 sums).  e916[m-1] = c916_e(m).
template <bool MIXED, int MODE>
__device__ __forceinline__ void prep_record(const LinesDev &L, const GridDev &g, const StateDev &st,
                                            int64_t l, const double *__restrict__ e916,
                                            void *__restrict__ out, double &w_loc, double &s1_loc) {
  const LineState ls = prep_line(L, st, l);
  int64_t w[6];
  line_windows(g, st, ls, 0, g.nx, w);
  // S1 per profile (S3_kernel voigt.h:452-463)
  const double Sc = ls.S * (1.0 / 1.7724538509055160273);
  const double S1 = g.profile <= 2 ? ls.S * ls.vy / CUDART_PI : (g.profile == 3 ? Sc : ls.S);
  const bool hasC = w[3] > w[2];
  // largest region-A/B term of the line: S1 / r^2 with r^2 >= max(100, y^2)
  // (Voigt: region C covers r < 10), r^2 >= y^2 for the Lorentz profile;
  // S1 for the Doppler profile, S1 / (2 vb) erf(vb / 2) < S1 / sqrt(pi) for
  // the binned Gaussian
  const double Y = ls.vy * ls.vy;
  const double rmin = g.profile == 2 ? Y : (g.profile >= 3 ? 1.0 : fmax(100.0, Y));
  const double term = rmin > 0.0 ? S1 / rmin : 0.0;
  if (MODE == PREP_STATS) {
  } else if (MIXED) {
    const double ey = hasC ? erfcx(ls.vy) : 1.0;
    const float sig1 = hasC ? (float)c916_sig1_tab(ls.vy, e916) : 0.f;
    LinePrepF r;
    r.nu = ls.nu;
    r.iad = ls.iad;
    r.S1 = S1;
    r.Sc = Sc;
    r.y = (float)ls.vy;
    r.ey = (float)ey;
    r.sig1 = sig1;
    const double A2 = 2.0 * Y + 3.0 - 6.0 / CUDART_PI, B2 = (Y + 1.5) * (Y + 1.5);
    r.A1 = (float)(2.0 * Y + 2.5 - 4.0 / CUDART_PI);
    r.B1 = (float)((Y + 1.5) * (Y + 1.0));
    r.D2 = (float)(A2 + Y);
    r.D1 = (float)(B2 + A2 * Y);
    r.D0 = (float)(B2 * Y);
    int ex = -100000;
    if (term > 0.0) frexp(term, &ex);
    r.ex = ex;
    int flags = 0;
    if (w[5] > w[0] && g.profile <= 2) {
      // the largest |x| inside the cut window (at its first or last point)
      const double xa = fabs((grid_x(g, w[0]) - ls.nu) * ls.iad);
      const double xb = fabs((grid_x(g, w[5] - 1) - ls.nu) * ls.iad);
      const double umax = fmax(xa, xb) * fmax(xa, xb) + Y;
      if (umax >= 1e18) flags |= HK_PF_WIDE;
      // (Lorentz: Y >= 2^-60 also keeps the product of two denominators,
      // >= Y^2, a normal float)
      if (rmin < 0x1p-64 * umax || Y > 0x1p60 || (g.profile == 2 && Y < 0x1p-60)) flags |= HK_PF_RANGE;
    }
    r.ext0 = 0.f;
    r.inu = g.subL ? (float)(1.0 / ls.nu) : 0.f;
    if (g.plinth && w[5] > w[0] && S1 > 0.0) {
      // The mixed form takes profile - plinth as t(x) - t(x_c) without
      // cancellation where a point lies in the region of the cut edge x_c
      // (the Lorentzian and GH2 differences factored by x_c - |x|, the
      // Doppler one as t (1 - exp(-(x_c^2 - x^2))) with x_c - |x| from the
      // FP64 offsets); elsewhere the term is at least 4 plinths, so the plain
      // difference keeps FP32 accuracy.  A Voigt line whose cut edge lies in
      // region C or within a factor 4 of a region boundary (r_c^2 < 400, or
      // 0.999e6 <= r_c^2 < 4e6: a point and the edge in different regions
      // with close values) and a line FP32 cannot hold are summed per point
      // in FP64, from the record's FP64 vy, erfcx(vy) and plinth.
      const double xc = plinth_xc(g, ls.iad, ls.vy);
      rec_put_d(&r.ext0, xc);
      bool pl64 = false;
      if (g.profile <= 2) {
        pl64 = (flags & (HK_PF_RANGE | HK_PF_WIDE)) != 0;
        const double rc2 = xc * xc + Y;
        if (g.profile == 1 && (rc2 < 400.0 || (rc2 >= 0.999e6 && rc2 < 4e6))) pl64 = true;
      }
      if (pl64) {
        flags |= HK_PF_RANGE | HK_PF_PL64;
        rec_put_d(&r.y, ls.vy);
        rec_put_d(&r.sig1, ey);
        rec_put_d(&r.B1, plinth_d(g, S1, Sc, ls.iad, ls.vy));
      }
    }
    r.flags = flags;
    // region C's Algorithm-916 part: |x| < sqrt(36 - y^2), from the FP64
    // offsets (a point within rounding of r = 6 may fall on either side;
    // both evaluators hold there)
    int64_t t0 = w[3], t1 = w[3];
    if (w[3] > w[2] && Y < 36.0) {
      const double xt = sqrt(36.0 - Y);
      const double x0 = (g.numin - ls.nu) * ls.iad, vb = g.dnu * ls.iad;
      const double k0 = floor((-xt - x0) / vb) + 1.0, k1 = floor((xt - x0) / vb) + 1.0;
      t0 = (int64_t)fmin(fmax(k0, (double)w[2]), (double)w[3]);
      t1 = (int64_t)fmin(fmax(k1, (double)t0), (double)w[3]);
    }
    r.t0 = (int)t0;
    r.t1 = (int)t1;
    r.i0 = (int)w[0];
    r.b0 = (int)w[1];
    r.c0 = (int)w[2];
    r.c1 = (int)w[3];
    r.b1 = (int)w[4];
    r.i1 = (int)w[5];
    reinterpret_cast<LinePrepF *>(out)[l] = r;
  } else {
    const double ey = hasC ? erfcx(ls.vy) : 1.0;
    const float sig1 = hasC ? (float)c916_sig1_tab(ls.vy, e916) : 0.f;
    LinePrep r;
    r.nu = ls.nu;
    r.iad = ls.iad;
    r.vy = ls.vy;
    r.S1 = S1;
    r.Sc = Sc;
    r.ey = ey;
    r.sig1 = sig1;
    r.i0 = (int)w[0];
    r.b0 = (int)w[1];
    r.c0 = (int)w[2];
    r.c1 = (int)w[3];
    r.b1 = (int)w[4];
    r.i1 = (int)w[5];
    r.dsig1 = hasC ? (float)c916_dsig1_tab(ls.vy, e916) : 0.f;
    r.plinth = (g.plinth && w[5] > w[0]) ? plinth_d(g, S1, Sc, ls.iad, ls.vy) : 0.0;
    reinterpret_cast<LinePrep *>(out)[l] = r;
  }
  if (w[5] > w[0]) s1_loc = fmax(s1_loc, term);
  if (ls.S != 0.0 && ls.iad > 0.0) {
    if (g.cutMode == 1) w_loc = fmax(w_loc, g.cut * ls.vy / ls.iad);
    else if (g.cutMode == 2) w_loc = fmax(w_loc, g.cut / ls.iad);
  }
}

// The state's cutoff bound and FP32 scale from its two maxima (the words of
// the line maxima as non-negative doubles' bits): wmax (cm^-1) the search
// half-width of a tile's lines, s1exp with 2^(40 - s1exp) above the largest
// region-A/B term.
__device__ __forceinline__ void state_scale(const GridDev &g, unsigned long long wbits_w,
                                            unsigned long long wbits_s, double &wmax, int &s1exp) {
  if (g.cutMode == 0) {
    wmax = g.cut;
  } else {
    const double w = __longlong_as_double((long long)wbits_w);
    wmax = w * (1.0 + 1e-9) + 1e-300;
  }
  const double tmax = __longlong_as_double((long long)wbits_s);
  int e = 0;
  if (tmax > 0.0 && isfinite(tmax)) {
    frexp(tmax, &e);  // tmax in [2^(e-1), 2^e)
    e = 40 - e;
  }
  s1exp = e;
}

}  // namespace hkb
