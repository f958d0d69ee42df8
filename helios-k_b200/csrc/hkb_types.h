// hkb_types.h -- plain-data types shared by the host runtime and kernels.
#pragma once

#include <cstdint>

namespace hkb {

// physical constants, define.h:36-45
constexpr double HK_T0 = 296.0;
constexpr double HK_PO_BAR = 0.986923;
constexpr double HK_PO_ATM = 1.0;
constexpr double HK_KB = 1.3806489e-16;
constexpr double HK_H = 6.62606957e-27;
constexpr double HK_C = 2.99792458e10;
constexpr double HK_NA = 6.0221412927e23;
// Voigt series tolerances, define.h:47-48
constexpr double HK_TOL = 1.43e-17;
constexpr float HK_TOLF = 2.48e-12f;
// Algorithm 916 step a = pi * sqrt(-1 / ln(TOL / 2)) (voigt.h:601, and
// heliosk.cu:1656-1658 for the FP32 constants a and c = 2a/pi)
constexpr double HK_A916_D = 0.4999936567001175;
constexpr float HK_A916_F = 0.5999962687492371f;
constexpr float HK_C916_F = 0.38196948170661926f;

constexpr int HK_DB_HITRAN = 0;
constexpr int HK_DB_EXOMOL = 2;
constexpr int HK_MAX_ISO = 64;  // isotopologues of all species of a mixture

// Sorted line list resident in HBM (SoA, FP64).  A null array means the
// column is uniform and its *_c scalar is used instead.
struct LinesDev {
  int64_t n;
  int database;
  const double *nu0;    // line centre, ascending
  const double *Sfile;  // strength as stored in the line file
  const double *EL;     // lower-state energy
  const double *gam;    // ((1-q) gamma_air + q gamma_self) * gammaF  (host.h:640-641)
  const double *nexp;   // temperature exponent
  const double *delta;  // pressure shift (HITRAN)
  const double *Aterm;  // A / (4 pi c)
  const uint8_t *iso;   // isotopologue index (null: 0)
  double EL_c, gam_c, nexp_c, delta_c, Aterm_c;
  // optional per-line multipliers of the scaled strength and of the Lorentz
  // half-width (null: 1), the differentiable line parameters of the adjoint
  const double *sscale, *gscale;
};

struct GridDev {
  double numin, dnu;
  int64_t nx;
  int cutMode;
  double cut;  // 1e30 when the parameter file says 0 (heliosk.cu:947)
  // line profile (define.h:69): 1 Voigt, 2 Lorentz, 3 Doppler, 4 binned
  // Gaussian cross section; plinth 1: every line's profile value at its cut
  // edge is subtracted inside its cut window (removePlinth)
  int profile = 1;
  int plinth = 0;
  // sub-Lorentzian wings (Perrin & Hartmann 1989 chi, voigt.h:1-72): on when
  // subL = 1, for grid points with sl_lo < x < sl_hi; chi's breakpoints
  // sl_sigma (cm^-1); the per-state slopes are StateDev.sl_B
  int subL = 0;
  int pad_g = 0;
  double sl_sigma[3] = {0.0, 0.0, 0.0};
  double sl_lo = 0.0, sl_hi = 0.0;
};

// One line scaled to one state, as written by line_prep_kernel and read by
// the Voigt sum (96 bytes; FP64 parameters, global index windows).
struct __align__(16) LinePrep {
  double nu;    // centre after the pressure shift
  double iad;   // 1 / alphaD
  double vy;    // gammaL / alphaD
  double S1;    // S * vy / pi (regions A, B; Lorentz), S / sqrt(pi) (Doppler), S (binned Gaussian)
  double Sc;    // S / sqrt(pi)     (region C)
  double ey;    // erfcx(vy)        (lines with a region-C window)
  int i0, b0, c0, c1, b1, i1;  // [i0,b0) A [b0,c0) B [c0,c1) C [c1,b1) B [b1,i1) A
  float sig1;   // region-C series constant Sig1(vy)
  float dsig1;  // dSig1/dy (region C of the mixed adjoint)
  double plinth;  // profile value at the cut edge (removePlinth), else 0
};
static_assert(sizeof(LinePrep) == 96, "LinePrep layout");

// The same line and state for the mixed form (112 bytes): everything that
// depends on the line and the state only, so staging a line into a tile adds
// just the tile's offsets and the strength level.
//   A1 = 2Y + 2.5 - 4/pi, B1 = (Y+1.5)(Y+1)      (GH2 numerator, Y = vy^2)
//   D2 = A2 + Y, D1 = B2 + A2 Y, D0 = B2 Y         (GH2 denominator expanded,
//   A2 = 2Y + 3 - 6/pi, B2 = (Y+1.5)^2)
//   ex: frexp exponent of the line's largest region-A/B term S1 / max(100, Y)
//   flags: HK_PF_WIDE  -- some x^2 + Y in the cut window reaches 1e18;
//          HK_PF_RANGE -- the window's terms span more than 2^64, or Y > 2^60:
//                         FP32 sums cannot hold the line (FP64 instead);
//          HK_PF_PL64  -- plinth removal: the line is summed per point in
//                         FP64 (set with HK_PF_RANGE; see below).
constexpr int HK_PF_WIDE = 2, HK_PF_RANGE = 1, HK_PF_PL64 = 4;
//   [t0, t1): the part of region C with |x| < sqrt(36 - y^2) (Algorithm 916
//   in FP32; the rest of region C takes the asymptotic series)
//   ext0, inu: sub-Lorentzian wings: inu = 1 / nu.  Plinth removal (never
//   together with sub-Lorentzian wings in the mixed form): the two words
//   hold the cut edge x_c (double, Doppler units), and an HK_PF_PL64 line,
//   whose FP32 profile fields are unused, holds vy (double) in {y, ey},
//   erfcx(vy) in {sig1, A1} and its plinth in {B1, D2}.
struct __align__(16) LinePrepF {
  double nu, iad;
  double S1, Sc;
  float y, ey, sig1;
  float A1, B1;
  float D2, D1, D0;
  int ex, flags;
  int i0, b0, c0, c1, b1, i1;
  int t0, t1;
  float ext0, inu;
};
static_assert(sizeof(LinePrepF) == 112, "LinePrepF layout");

// a double kept in two consecutive (8-byte aligned) float words of a record
__host__ __device__ inline double rec_get_d(const float *w) { return *reinterpret_cast<const double *>(w); }
__host__ __device__ inline void rec_put_d(float *w, double v) { *reinterpret_cast<double *>(w) = v; }

// Per-(T, P) constants formed on the host.
struct StateDev {
  double T, P;
  double PoverP0;  // P / 1 atm (HITRAN) or P / 1 bar in atm (ExoMol)
  double powbase;  // T0 / T
  double c1;       // h c / (kB T)   (ExoMol strength)
  double wmax;     // upper bound of the cutoff half-width over lines (cm^-1)
  double shift;    // upper bound of |delta| * P
  double kmin;
  double s1scale;    // 2^e, largest region-A/B term S1/max(100, y^2) * 2^e in [2^39, 2^40)
  double s1unscale;  // 2^-e
  int s1exp, pad0;   // e
  double iad0[HK_MAX_ISO];  // c sqrt(m / (2 kB T))
  double Q[HK_MAX_ISO];     // partition function at T
  double ab[HK_MAX_ISO];    // abundance * (m / meanMass) when units == 0
  double ss[HK_MAX_ISO];    // species scale * (m / meanMass) when units == 0
  double dlnQ[HK_MAX_ISO];  // d ln Q / dT of the interpolated partition function
  double sl_B[3];           // sub-Lorentzian slopes alpha + beta exp(-epsilon T)
};
static_assert(sizeof(StateDev) == 2672, "StateDev layout (the host copies it per state)");

}  // namespace hkb
