/*
 * hk_oracle.h -- FP64 CPU restatement of the HELIOS-K opacity hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA path and the timed CPU baseline.  Nothing in the product (libhkb,
 * the heliosk driver, the hkb Python package) links, loads or calls it.
 *
 * Every function names the reference file:line it restates.  Paths are
 * relative to the HELIOS-K source tree.
 *
 * Numerical conventions (both here and in the CUDA kernels):
 *   - grid point          x_i = fma(i, dnu, numin)           (voigt.h:751-768,
 *                          setX_kernel; nvcc contracts numin + id*dnu to an FMA)
 *   - line-centre offset  dnu_i = x_i - nu                    (FP64)
 *   - cutoff              |dnu_i| < w, w = cut (cutMode 0), cut*gammaL (1),
 *                          cut*alphaD (2)                     (voigt.h:436-452)
 *   - Voigt argument      x = dnu_i * ialphaD, y = vy, r2 = x*x + y*y (FP64,
 *                          no contraction)
 *   - regions             C: r2 < 100, B: 100 <= r2 < 1e6, A: r2 >= 1e6
 *                          (voigt.h:1223, 1481, 1662)
 * The oracle is compiled with -ffp-contract=off so these predicates are the
 * IEEE-rounded sequence the CUDA code reproduces with __dmul_rn/__dadd_rn.
 */
#ifndef HK_ORACLE_H
#define HK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* physical constants, define.h:36-45 */
#define HKO_T0 296.0
#define HKO_PO_BAR 0.986923
#define HKO_PO_ATM 1.0
#define HKO_KB 1.3806489e-16
#define HKO_H 6.62606957e-27
#define HKO_C 2.99792458e10
#define HKO_NA 6.0221412927e23
/* Voigt series tolerance, define.h:47 */
#define HKO_TOL 1.43e-17

/* grid */
double hko_grid_x(double numin, double dnu, int64_t i);
int hko_grid_nx(double numin, double numax, double dnu);
void hko_grid_fill(double numin, double dnu, int64_t nx, double *x);
void hko_bin_keys(double numin, double numax, double dnu, int64_t nx, int nbins,
                  int32_t *key, int32_t *bin_index /* nbins+2 */);

/* partition function, host.h:9-73 */
int hko_partition_interp(const double *Tq, const double *q, int nq, double T,
                         double *Q_out);

/* line scaling to one (T,P) state */
void hko_prep_hitran(int64_t n, const double *nu, const double *S_file,
                     const double *EL, const double *A, const double *delta,
                     const double *gair, const double *gself,
                     const double *nexp, const int32_t *iso, int niso,
                     const double *iso_mass, const double *iso_ab,
                     const double *iso_Q, double T, double P, double qalphaL,
                     double gammaF, int units, double meanMass, double Sscale,
                     double *out_nu, double *out_S, double *out_iad,
                     double *out_vy);

void hko_prep_exomol(int64_t n, const double *nu, const double *S_file,
                     const double *EL, const double *A, double mass_g_mol,
                     double ab, double Q, double defaultL, double defaultn,
                     double T, double P, double gammaF, int units,
                     double meanMass, double Sscale, double *out_nu,
                     double *out_S, double *out_iad, double *out_vy);

/* per-line grid windows: [i0,b0) A  [b0,c0) B  [c0,c1) C  [c1,b1) B  [b1,i1) A */
void hko_windows(int64_t n, const double *nu, const double *S,
                 const double *iad, const double *vy, double numin, double dnu,
                 int64_t nx, int cutMode, double cut, int64_t *win /* n*6 */);

/* profile */
double hko_erfcx(double y);
double hko_voigt916(double x, double y);
double hko_gh2(double x, double y);

/* K[i - ib] = kmin + sum over lines (profile 1, Voigt), ib <= i < ie */
/* profile 1..4 (define.h:69); plinth: per-line values subtracted inside
 * each line's window (removePlinth), or NULL; sl: sub-Lorentzian {sigma1,
 * sigma2, sigma3, B1, B2, B3, x_lo, x_hi} (voigt.h:1-72), or NULL */
void hko_windows_p(int64_t n, const double *nu, const double *S,
                   const double *iad, const double *vy, double numin, double dnu,
                   int64_t nx, int cutMode, double cut, int profile, int64_t *win);
void hko_plinth(int64_t n, const double *S, const double *iad, const double *vy,
                const int64_t *win, int cutMode, double cut, int profile, double *out);
void hko_opacity_p(int64_t n, const double *nu, const double *S,
                   const double *iad, const double *vy, const int64_t *win,
                   double numin, double dnu, int64_t ib, int64_t ie, double kmin,
                   int profile, const double *plinth, const double *sl, double *K,
                   int nthreads, int64_t pairs_out[3]);
void hko_opacity(int64_t n, const double *nu, const double *S,
                 const double *iad, const double *vy, const int64_t *win,
                 double numin, double dnu, int64_t ib, int64_t ie, double kmin,
                 double *K, int nthreads, int64_t pairs_out[3]);

/* per-line sums of the vector-Jacobian product of K (G: 4 x n), test
 * oracle of the adjoint */
void hko_vjp_sums(int64_t n, const double *nu, const double *S, const double *iad,
                  const double *vy, const int64_t *win, double numin, double dnu, int64_t nx,
                  const double *u, double *G, int profile, int nthreads);

/* k-distribution fit, resample.h */
void hko_vandermonde(int nxb, int nc, double *V);
void hko_qr(int nxb, int nc, double *V, double *C, double *D);
void hko_sort_bins(int64_t nx, const int32_t *bin_index, int nbins, double *K);
void hko_find_cut(const double *K, int64_t nx, int nxb, double kmin,
                  int nbins, int32_t *nxmin);
void hko_kdist(double *K, int64_t nx, int nxb, int nbins, int nc, double kmin,
               double unitScale, const double *V, const double *C,
               const double *D, int32_t *nxmin, double *coeff /* nbins*nc */,
               double *recon /* nx or NULL */);

/* Planck / Rosseland mean ingredients, resample.h:635-773 (Mean_kernel,
 * IntegrateMean_kernel, equal spacing) on the grid x (nx points, state
 * temperature T): out[0] = sum B K, out[1] = sum over K != 0 of (dB/dT) / K,
 * out[2] = sum B, out[3] = sum dB/dT, each with the reference's end weights
 * (SimpsonCoefficient resample.h:611-619, applied as resample.h:730-747). */
void hko_planck(double nu, double T, double *B, double *dBdT);
void hko_means(const double *x, const double *K, int64_t nx, double T, double *out);
/* Transmission function, resample.h:541-608 (Integrate_kernel): for every
 * bin of nxb points of K (sorted or reconstructed) and m_j = exp((j - nTr/2)
 * dTr), Tr[b nTr + j] = (sum_k exp(-K_k m_j) + end weights) / (nxb - 1)
 * (nxb - Nxmin_b) / nxb + exp(-kmin m_j) Nxmin_b / nxb; nxmin NULL = 0. */
void hko_transmission(const double *K, int nxb, int nbins, const int32_t *nxmin,
                      double kmin, int nTr, double dTr, double *Tr);

#ifdef __cplusplus
}
#endif
#endif
