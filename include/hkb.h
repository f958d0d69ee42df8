/*
 * hkb.h -- C ABI of libhkb, the B200 (sm_100a) opacity engine.
 *
 * The reference (HELIOS-K) is a single executable with no library API; its
 * internal seam for this path is the kernel-launch helpers
 * Line6A_Call/Line6B_Call/Line6C_Call (voigt.h:1820, 1968, 2004) fed by the
 * host readers (host.h, ISO.h) and followed by the post-processing chain of
 * heliosk.cu:2046-2195.  Each entry point below names what it replaces.
 * The heliosk drop-in executable (helios-k_b200/bin/heliosk) is built on
 * these calls and keeps the reference's param.dat / <species>.param inputs
 * and Out_* / Info_* outputs.
 *
 * Conventions
 *  - Every call returns hk_status: 0 = HK_OK, negative = error class; the
 *    message is available from hk_last_error(ctx).  Nothing is printed.
 *  - Pointers are plain host pointers unless a *_on_device flag says the
 *    buffer is device memory of the context's GPU.  Callers own their
 *    buffers; the library owns its device workspace.
 *  - `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *    stream).  Calls with host outputs synchronise that stream before
 *    returning; calls with device outputs are asynchronous on it.
 *  - One context per host thread at a time.
 */
#ifndef HKB_H
#define HKB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hk_ctx hk_ctx;
typedef int hk_status;

enum {
  HK_OK = 0,
  HK_ERR_ARG = -1,         /* invalid argument                          */
  HK_ERR_IO = -2,          /* file missing or unreadable                */
  HK_ERR_FORMAT = -3,      /* malformed parameter / species / line file */
  HK_ERR_RANGE = -4,       /* value outside what the path supports      */
  HK_ERR_CUDA = -5,        /* CUDA runtime error                        */
  HK_ERR_STATE = -6,       /* call order (e.g. no grid set)             */
  HK_ERR_NOMEM = -7,       /* device or host allocation failed          */
  HK_ERR_UNSUPPORTED = -8, /* option outside this build's scope        */
  HK_ERR_TIMEOUT = -9      /* a bounded wait on the GPU ran out         */
};

enum { HK_PRECISION_PLAIN_FP64 = 0, HK_PRECISION_MIXED = 1 };
enum { HK_DATABASE_HITRAN = 0, HK_DATABASE_EXOMOL = 2 };

/* ------------------------------------------------------------ context */

/* Bind a GPU and create the workspace.
 * Replaces cudaSetDevice(param.dev) (heliosk.cu:392) and the K/x/bin
 * allocations of heliosk.cu:712-725. */
hk_ctx *hk_create(int device, hk_status *status);
void hk_destroy(hk_ctx *ctx);
/* Message of the last failed call on this context ("" if none). */
const char *hk_last_error(const hk_ctx *ctx);
const char *hk_version(void);

/* ------------------------------------------------------------ species */

/* Isotopologue table of one species: molar masses (g/mol) and abundances.
 * Replaces Init (ISO.h:16-219) for callers that do not read a .param file.
 * defaultL / defaultn are the ExoMol width defaults (ISO.h:192-206). */
hk_status hk_set_species(hk_ctx *ctx, int database, int niso,
                         const double *mass_g_mol, const double *abundance,
                         double defaultL, double defaultn);

/* Partition-function table (T, Q) of isotopologue `iso`, interpolated per
 * state exactly as readPartition (host.h:9-73). */
hk_status hk_set_partition(hk_ctx *ctx, int iso, int n, const double *T,
                           const double *Q);

/* param.dat keys qalphaL, gammaF, Units (host.h:75-300) and the species
 * abundance scale of a mixture entry (heliosk.cu:787-789).  Defaults:
 * qalphaL = 0.5 (define.h:66), gammaF = 1, units = 0, Sscale = 1. */
hk_status hk_set_options(hk_ctx *ctx, double qalphaL, double gammaF, int units,
                         double Sscale);

/* -------------------------------------------------------------- lines */

/* HITRAN/HITEMP line list as host SoA (copied to HBM, sorted by nu).
 * Fields as in the 68-byte record (host.h:607-615): nu, S, E'', A, delta,
 * gamma_air, gamma_self, n; iso = isotopologue index per line (NULL: 0).
 * Replaces readFile (host.h:598-649) + Copy_Line (host.h:958-967). */
hk_status hk_load_lines_hitran(hk_ctx *ctx, int64_t n, const double *nu,
                               const double *S, const double *EL,
                               const double *A, const double *delta,
                               const double *gair, const double *gself,
                               const double *nexp, const int32_t *iso);

/* ExoMol line list (nu, S, E'', A), widths from hk_set_species defaults.
 * Replaces readFileExomol (host.h:656-668) + L_kernelExomol
 * (voigt.h:484-504). */
hk_status hk_load_lines_exomol(hk_ctx *ctx, int64_t n, const double *nu,
                               const double *S, const double *EL,
                               const double *A);

/* Read <path><species>.param, its partition files and every binary line
 * file whose range can reach [numin - cut, numax + cut] (heliosk.cu:943-956),
 * then load them.  Replaces Init + readPartition + the file loop of
 * heliosk.cu:943-1043.  cut == 0 means no cutoff. */
hk_status hk_load_species_file(hk_ctx *ctx, const char *path,
                               const char *species, double numin, double numax,
                               int cutMode, double cut);

/* Species mixture (param.dat SpeciesFile: "<species> <abundance>" per line),
 * replacing the per-species loop of heliosk.cu:660-700, 784-800: every
 * species' selected line files are loaded into one line list (its
 * isotopologues after the previous species'), each species' strengths scaled
 * by its abundance (1 when nspecies == 1, as the reference), the mean molar
 * mass taken over the mixture; one hk_opacity then sums all species.  All
 * species must share the record format (HITRAN or ExoMol); at most 64
 * isotopologues in all. */
hk_status hk_load_mixture(hk_ctx *ctx, const char *path, int nspecies, const char *const *species,
                          const double *abundance, double numin, double numax, int cutMode,
                          double cut);

/* Collision-induced absorption in place of lines (param.dat ciaSystem;
 * InitCia ISO.h:222-277, readCiaFile host.h:670-785): reads
 * <path><system>_2011.cia (HITRAN CIA format) for the systems H2-H2,
 * H2-H2_eq, H2-H2_norm, H2-He, H2-He_eq, H2-He_norm, H2-CH4_eq, H2-CH4_norm,
 * H2-H; hk_opacity then interpolates it onto the grid for each state (the
 * reference's T and P rules, K in cm^2/g plus kmin).  mass1 (optional) gets
 * the collider mass the reference's units = 1 scaling uses.  Loading lines
 * or species ends CIA mode. */
hk_status hk_load_cia(hk_ctx *ctx, const char *path, const char *system, double *mass1);

int64_t hk_num_lines(const hk_ctx *ctx);

/* --------------------------------------------------------------- grid */

/* Wavenumber grid x_i = numin + i dnu, Nx = (int)((numax-numin)/dnu + 0.5)
 * points in nbins equal bins; cutoff mode/width; K floor kmin.
 * Replaces heliosk.cu:417-476 and InitialK/setX/binKey/binIndex
 * (voigt.h:713-832).  Nx must divide evenly into nbins (heliosk.cu:456). */
hk_status hk_set_grid(hk_ctx *ctx, double numin, double numax, double dnu,
                      int nbins, int cutMode, double cut, double kmin);
int64_t hk_grid_points(const hk_ctx *ctx);

/* ------------------------------------------------------------ compute */

/* Opacity K(nu) of every state (T[s], P[s]) onto the grid:
 * K_out[s * Nx + i], FP64.  precision selects the FP64 plain form or the
 * mixed FP32/FP64 form.  States run in batches sized to the workspace
 * budget (per-line records of all states of a batch); each batch is one
 * persistent Voigt launch.
 * Replaces the per-part / per-pressure loop of heliosk.cu:1051-1776:
 * S2_kernel, the nu sort, S3_kernel, nuLimits/iiLimits, Line6A/B/C_Call and
 * AddKStreams_kernel. */
hk_status hk_opacity(hk_ctx *ctx, int nstates, const double *T, const double *P,
                     int precision, double *K_out, int K_on_device,
                     void *stream);

/* Per-bin sort and Chebyshev k-distribution fit of K (nstates x Nx):
 * coeff_out[(s * nbins + b) * nC + j], nxmin_out[s * nbins + b] (the
 * reference's Nxmin; ystart = min(Nxmin / (Nxb - 1), 1)), optional
 * per-bin sorted K and optional reconstruction (expfx + inverse rescale).
 * Any output pointer may be NULL.  Replaces heliosk.cu:2046-2193
 * (thrust sorts, Vandermonde/QR/findCut/rescale/copyK2/lnK/leastSquare/
 * expfx kernels of resample.h:14-524). */
hk_status hk_kdist(hk_ctx *ctx, int nstates, const double *K, int K_on_device,
                   int nC, double unitScale, double *coeff_out,
                   int32_t *nxmin_out, double *sortedK_out, double *recon_out,
                   int outputs_on_device, void *stream);

/* The same per-bin sort and Chebyshev fit as hk_kdist, for callers that
 * cannot allocate device memory: host programs that give every byte of the
 * GPU to their own memory pool or run under a fixed budget, or that must not
 * make calls which may synchronise the device or fail for lack of memory in
 * the middle of a run.  No counterpart in the reference (its fit allocates
 * with cudaMalloc, heliosk.cu:2090-2106).
 *  - No context, no allocation: it runs on the CURRENT device; K (nstates x
 *    nx), coeff (nstates x nbins x nC), nxmin (nstates x nbins) and the
 *    optional sortedK (nstates x nx) are device pointers owned by the caller.
 *  - Its only scratch is a fixed 2 MiB array in the library (2^18 doubles,
 *    held on every GPU that loads the library until exit): requires
 *    (nx / nbins) * nC + 2 nC <= 262144, and a bin small enough for the
 *    shared-memory sort; larger sizes return HK_ERR_RANGE with a message.
 *  - The first call on a device looks up that array's device address; make
 *    that first call before any stream capture.
 *  - All calls share the array: calls that overlap on the GPU (different
 *    streams, or different host threads) race.  Serialise them.
 *  - Asynchronous on `stream`; on failure a message is written to errbuf.
 *    A CUDA error already pending from an earlier launch of the caller's is
 *    reported as such (HK_ERR_CUDA, left pending) before anything runs. */
hk_status hk_kdist_noalloc(const double *K, int nstates, int64_t nx, int nbins, int nC,
                           double kmin, double unitScale, double *coeff, int32_t *nxmin,
                           double *sortedK, void *stream, char *errbuf, int errbuf_len);

/* Device workspace budgets (bytes): per-(state, line) records of one batch
 * (default 24 GiB) and split-tile partial sums (default 4 GiB).  States whose
 * records exceed the first run in grid sections (bit-identical K). */
hk_status hk_set_workspace(hk_ctx *ctx, double prep_bytes, double part_bytes);

/* Line profile (param.dat `profile`, define.h:69): 1 Voigt (default),
 * 2 Lorentz, 3 Doppler, 4 binned Gaussian cross section (Hill et al. 2012),
 * as Line6fA_kernel (voigt.h:1235-1262) evaluates them over the whole cut
 * window; remove_plinth 1 (param.dat `removePlinth`) subtracts each line's
 * profile value at its cut edge (Plinth_kernel voigt.h:1091-1164) from every
 * point of its window.  All four profiles have a mixed (FP32) form -- the
 * Doppler and binned-Gaussian terms in FP32 where they are normal floats,
 * in FP64 beyond -- and an adjoint.  Plinth removal has a mixed form too (profile -
 * plinth formed without cancellation: factored differences in FP32, and FP64
 * per point for a Voigt line whose cut edge lies in region C or near a
 * region boundary), except with sub-Lorentzian wings (FP64 form); the
 * adjoint refuses it. */
hk_status hk_set_profile(hk_ctx *ctx, int profile, int remove_plinth);

/* Sub-Lorentzian line wings (param.dat subLorentzianfile; Perrin & Hartmann
 * 1989 chi factors, voigt.h:1-72, host.h:489-515): p = {sigma1, sigma2,
 * sigma3, alpha1, beta1, epsilon1, alpha2, beta2, epsilon2, alpha3, beta3,
 * epsilon3, x_lo, x_hi}; every term at a grid point lo < x < hi is multiplied
 * by chi(|x - nu|) x / nu, chi = 1 below sigma1 and exp(-B1 (d - sigma1)
 * ...) beyond, B_k = alpha_k + beta_k exp(-epsilon_k T).  NULL turns it off.
 * The mixed form applies it to the Voigt and Lorentz profiles without
 * plinth removal (the Doppler and binned-Gaussian profiles with it, and
 * either profile with plinth removal too, run the FP64 form); the adjoint
 * refuses it. */
hk_status hk_set_sublorentzian(hk_ctx *ctx, const double *p);

/* --------------------------------------- mean opacities, transmission */

/* Planck and Rosseland mean ingredients of nstates opacities K (nstates x
 * Nx, the states' temperatures T[s]), replacing Mean_kernel +
 * IntegrateMean_kernel (resample.h:635-773; driver heliosk.cu:1953-2020):
 * sums[4 s + q] = sum over the grid of B K (q = 0), of (dB/dT) / K where
 * K != 0 (1), of B (2), of dB/dT (3), each with the reference's end weights.
 * Planck mean = sums[0] / sums[2]; Rosseland mean = sums[3] / sums[1];
 * sums[2] dnu and sums[3] dnu approximate sigma T^4 / pi and 4 sigma T^3 / pi.
 * K is in the library's internal units (hk_opacity's output). */
hk_status hk_means(hk_ctx *ctx, int nstates, const double *T, const double *K, int K_on_device,
                   double *sums, int sums_on_device, void *stream);

/* Transmission function per bin, replacing Integrate_kernel (resample.h:
 * 541-608; driver heliosk.cu:2377-2430): K is nstates x Nx of per-bin values
 * (hk_kdist's sorted K, or its reconstruction when the fit ran), nxmin the
 * fit's Nxmin (nstates x nbins; NULL = 0, as without resampling), kmin the
 * grid's.  Tr[(s nbins + b) nTr + j] for m_j = exp((j - nTr/2) dTr):
 *   (sum_k exp(-K_k m_j) + end weights) / (Nxb - 1) (Nxb - Nxmin) / Nxb
 *   + exp(-kmin m_j) Nxmin / Nxb.
 * K and nxmin are both on the device or both on the host. */
hk_status hk_transmission(hk_ctx *ctx, int nstates, const double *K, const int32_t *nxmin,
                          int inputs_on_device, int nTr, double dTr, double *Tr,
                          int Tr_on_device, void *stream);

/* ------------------------------------------------------ tile shapes */

/* The mixed Voigt kernel runs in one of hk_num_tile_shapes() tile shapes:
 * lines per staged chunk x grid points per tile, run by a number of warps
 * per CTA (shape 0, the default: 128 x 2048, 8 warps).  The shape changes only the order of the FP64 additions (results
 * differ in the last bits, within the same error bound); the plain FP64 form
 * always uses shape 0.  Replaces the reference's kernel self-tuning
 * (doTuning, heliosk.cu:1363-1705; tile widths nkA..nkC, heliosk.cu:968-982). */
int hk_num_tile_shapes(void);
hk_status hk_tile_shape_info(int shape, int *lines_per_chunk, int *points_per_tile, int *warps);

/* mode 0: the fixed shape (hk_set_tile_shape, default 0).
 * mode 1: tune when the probes cost at most a tenth of the call's sweep
 *         (tables and large batches; single states keep the fixed shape).
 * mode 2: tune on the first mixed call after lines, grid or options change.
 * Tuning times each shape on up to 4 probe states of the call over a
 * section of the grid and keeps the fastest until lines, grid or options
 * change.  hk_table_build tunes before recording its graph. */
hk_status hk_set_tuning(hk_ctx *ctx, int mode);
hk_status hk_set_tile_shape(hk_ctx *ctx, int shape);
/* last_shape: the shape of the last mixed call; tuned_shape: the tuner's
 * choice (-1 if not tuned); probe_ms[hk_num_tile_shapes()] (optional): the
 * probe time per shape (-1 if not tuned). */
hk_status hk_tuning_result(hk_ctx *ctx, int *last_shape, int *tuned_shape, double *probe_ms);

/* ----------------------------------------------------------- adjoint */

/* Optional per-line multipliers, in load order (host arrays of
 * hk_num_lines values, each finite and > 0; NULL restores 1): the scaled
 * strength of line l is multiplied by s_scale[l] and its Lorentz half-width
 * gammaL (collisional + natural) by g_scale[l].  They make log S and
 * gammaL per-line parameters of the forward, for gradient-based fitting.
 * Loading a new line list clears them.  No counterpart in the reference. */
hk_status hk_set_line_scales(hk_ctx *ctx, const double *s_scale, const double *g_scale);

/* The same multipliers from DEVICE arrays (load order, hk_num_lines values
 * each, on this context's GPU; NULL restores 1), reordered and checked on
 * the GPU in stream order on `stream` (a cudaStream_t, NULL the legacy
 * stream); the call returns once they are in place, having copied only the
 * check's 8-byte result to the host.  For callers whose parameters live on
 * the GPU (an optimiser's tensors): hk_set_line_scales would take them
 * through host memory twice.  Pointers that are not device memory of this
 * context's GPU are refused (HK_ERR_ARG) before any launch.  A value that is
 * not finite and > 0 fails with HK_ERR_ARG naming its load index, and then
 * both multipliers are restored to 1.  Work on other streams that still
 * reads the previous multipliers must be complete.  No counterpart in the
 * reference. */
hk_status hk_set_line_scales_device(hk_ctx *ctx, const double *s_scale, const double *g_scale,
                                    void *stream);

/* Vector-Jacobian product of the opacity of one state: with the seed
 * u[i] = dLoss/dK_i (Nx values, e.g. w_i / K_i for Loss = sum_i w_i log K_i),
 * returns dLoss/dT (K), dLoss/dP (atm for HITRAN, bar for ExoMol), and per
 * line (load order) dLoss/dlog S_l and dLoss/dgammaL_l (cm).  The forward is
 * recomputed per grid tile (nothing of it is stored); regions A and B are
 * differentiated in the working precision (FP32 in the mixed form, x from
 * the FP64 offset), region C through the FP64 Algorithm-916 series, and the
 * per-line sums are FP64 (accumulated with atomics: the last bits may vary
 * between runs).  Any of dT, dP, dlogS, dgammaL may be NULL.  Synchronous.
 * The four line profiles (Doppler and binned Gaussian in FP64 in either
 * precision) without plinth removal or sub-Lorentzian wings;
 * HK_ERR_UNSUPPORTED with either option.
 * No counterpart in the reference (it computes no derivatives). */
hk_status hk_opacity_vjp(hk_ctx *ctx, double T, double P, int precision, const double *u,
                         int u_on_device, double *dT, double *dP, double *dlogS,
                         double *dgammaL, int outputs_on_device, void *stream);

/* The same vector-Jacobian product with the per-line width gradient taken
 * per log gammaL (dLoss/dlog gammaL = gammaL dLoss/dgammaL, gammaL of this
 * state with its line scale): the natural parameters of a fit of per-line
 * multipliers exp(log g).  With outputs_on_device the per-line results stay
 * on the GPU (no host round trip).  No counterpart in the reference. */
hk_status hk_opacity_vjp_log(hk_ctx *ctx, double T, double P, int precision, const double *u,
                             int u_on_device, double *dT, double *dP, double *dlogS,
                             double *dlogGammaL, int outputs_on_device, void *stream);

/* ------------------------------------------------------------ tables */

/* A whole T-P table as one CUDA graph, recorded once by hk_table_build and
 * replayed by hk_table_run with one graph launch.  Table mode 0 (default):
 * per batch of states whose line records fit the workspace, a line-prep and
 * a persistent Voigt launch, then one k-distribution launch for all states.
 * Table mode 1 (hk_set_table_mode, tables of 4 states or more): two kernels,
 * one persistent launch that scales the lines to every state (records in a
 * ring of per-state slots) and sums every state's Voigt profiles as tickets
 * of one counter (the line prep of state s beside the sums of state s - 1, a
 * slot reused once its previous state's sums are done), then one
 * k-distribution launch.  Both modes give the same bits.  K (nstates x Nx), coeff (nstates x nbins x nC) and nxmin
 * (nstates x nbins) are DEVICE buffers owned by the caller that must stay
 * valid while the table exists; hk_table_build allocates all workspace and
 * synchronises the device; hk_table_run is asynchronous on `stream`.  The
 * results equal those of hk_opacity + hk_kdist on the same states.  A new
 * hk_table_build, hk_table_free or hk_destroy drops the graph; other calls
 * on the same context between runs reuse its workspace, so rebuild after
 * them.  The kernel's waits for other tickets are bounded: hk_table_status
 * synchronises `stream` and returns HK_ERR_TIMEOUT if one of the last run's
 * ran out (its results are then incomplete), else HK_OK.
 * Replaces the reference's one-state-per-run loop (heliosk.cu:1051-2193 run
 * once per pressure of the PFile). */
hk_status hk_table_build(hk_ctx *ctx, int nstates, const double *T, const double *P,
                         int precision, double *K, int nC, double unitScale,
                         double *coeff, int32_t *nxmin);
/* 0: per-batch launches (default); 1: one persistent launch for the sums. */
hk_status hk_set_table_mode(hk_ctx *ctx, int fused);
hk_status hk_table_run(hk_ctx *ctx, void *stream);
hk_status hk_table_status(hk_ctx *ctx, void *stream);
hk_status hk_table_free(hk_ctx *ctx);
/* kernels recorded in the table graph */
int64_t hk_table_kernels(const hk_ctx *ctx);

/* ------------------------------------------------------- diagnostics */

/* kernels launched by the last hk_opacity and the hk_kdist calls after it */
int64_t hk_last_launches(const hk_ctx *ctx);

/* (line, grid point) pairs of one state inside the cutoff windows, by
 * region: pairs3 = {A, B, C} (the algorithmic work of the Voigt sum, from the
 * same windows the sum uses). */
hk_status hk_count_pairs(hk_ctx *ctx, double T, double P, int64_t *pairs3);


/* Per-line state (nu, S, 1/alphaD, gammaL/alphaD) and the six window
 * indices i0, b0, c0, c1, b1, i1 of every loaded line (in load order is NOT
 * kept: lines are in the library's nu-sorted order, see hk_line_order) for
 * one state, computed by the same device code the sum uses.  Any output may
 * be NULL. */
hk_status hk_state_lines(hk_ctx *ctx, double T, double P, double *nu,
                         double *S, double *iad, double *vy, int64_t *win6);

/* Permutation applied at load: sorted position k holds input line order[k]. */
hk_status hk_line_order(hk_ctx *ctx, int64_t *order);

/* Voigt function V(x, y) (region-C formula, Algorithm 916) evaluated by the
 * device code of the given precision. */
hk_status hk_profile_eval(hk_ctx *ctx, int64_t n, const double *x,
                          const double *y, int precision, double *out);

/* Device time of the last hk_opacity / hk_kdist kernels (CUDA events on
 * the launching stream), in milliseconds; and the grid tile size.  After
 * hk_opacity_vjp, voigt_ms is the time of its adjoint kernels. */
hk_status hk_last_timing(const hk_ctx *ctx, double *voigt_ms, double *kdist_ms);
int hk_tile_points(void);

/* FP32 FMA throughput of this GPU at the current clocks (TFLOP/s), from a
 * short all-SM FMA probe; the roofline denominator of the Voigt sum. */
hk_status hk_fp32_peak(hk_ctx *ctx, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* HKB_H */
