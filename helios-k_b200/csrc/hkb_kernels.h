// hkb_kernels.h -- host-side launchers of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "hkb_types.h"

namespace hkb {

// dynamic shared memory budget of one kdist CTA (sm_100: 227 KB per block,
// minus the kernel's static shared arrays)
constexpr int KD_SMEM_LIMIT = 224 * 1024;

// Tile shapes of the mixed Voigt kernel: lines per staged chunk x grid points
// per tile (warps per CTA); shape 0 is the default and the plain FP64 form's
// only shape.
int voigt_num_shapes();
int voigt_tile_points(int shape);
int voigt_chunk_lines(int shape);
int voigt_tile_warps(int shape);
cudaError_t measure_fp32_peak(double *tflops, cudaStream_t stream);

// Vector-Jacobian product of one state's opacity (hkb_adjoint.cu): G_d holds
// 4 x nlines FP64 sums, dTP_d the two scalars; dlogS_d / dgam_d (load order
// through order_d, may be null) the per-line results, dgam_d per gammaL or,
// with log_gamma, per log gammaL.
cudaError_t launch_opacity_vjp(bool mixed, const LinesDev &L, const GridDev &g,
                               const StateDev *state_d, const StateDev &state_h,
                               const LinePrep *prep_d, const double *u_d, unsigned *ticket_d,
                               double *G_d, const int64_t *order_d, double *dlogS_d,
                               double *dgam_d, int log_gamma, double *dTP_d, cudaStream_t stream);

// per-(line, state) records: LinePrepF (mixed) or LinePrep (plain FP64)
cudaError_t launch_line_prep(bool mixed, const LinesDev &L, const GridDev &g, StateDev *states_d,
                             int nstates, void *prep_d, unsigned long long *wbits_d,
                             cudaStream_t stream);
// Sectioned states (a state's records larger than the workspace): the state
// pass (cutoff bound, FP32 scale) over all lines, then one section's records
// at a time; sections find their lines with launch_lower_bound on nu0.
cudaError_t launch_state_stats(const LinesDev &L, const GridDev &g, StateDev *states_d,
                               int nstates, unsigned long long *wbits_d, cudaStream_t stream);
cudaError_t launch_line_records(bool mixed, const LinesDev &L, const GridDev &g,
                                const StateDev *state_d, void *prep_d, cudaStream_t stream);
cudaError_t launch_lower_bound(const double *a_d, int64_t n, const double *q_d, int m,
                               int64_t *out_d, cudaStream_t stream);
// lines [l0, l0 + n) of L as a list of their own
inline LinesDev lines_sub(const LinesDev &L, int64_t l0, int64_t n) {
  LinesDev s = L;
  s.n = n;
  auto off = [l0](const double *p) { return p ? p + l0 : p; };
  s.nu0 = off(L.nu0);
  s.Sfile = off(L.Sfile);
  s.EL = off(L.EL);
  s.gam = off(L.gam);
  s.nexp = off(L.nexp);
  s.delta = off(L.delta);
  s.Aterm = off(L.Aterm);
  s.sscale = off(L.sscale);
  s.gscale = off(L.gscale);
  s.iso = L.iso ? L.iso + l0 : nullptr;
  return s;
}

// Line ingestion (hkb_ingest.cu): binary records or caller columns to the
// library's columns on the device, in load order.
struct IngestSpec {
  int hitran;           // 68-byte HITRAN records (else 32-byte ExoMol)
  int niso;
  char cid[HK_MAX_ISO][4];
  double qalphaL, gammaF, defaultL, defaultn;
  double four_pi_c;     // 4 pi c as the host forms it
  int iso_base;         // the species' first isotopologue index (mixtures)
};
struct LineCols {
  double *nu, *S, *EL, *gam, *nexp, *delta, *Aterm;
  uint8_t *iso;
};
cudaError_t launch_unpack_records(const unsigned char *raw_d, int64_t n, int64_t first,
                                  const IngestSpec &sp, const LineCols &cols,
                                  unsigned long long *bad_d, cudaStream_t stream);
cudaError_t launch_finish_columns(int64_t n, const IngestSpec &sp, const double *gair_d,
                                  const double *gself_d, const double *A_d, const int32_t *iso32_d,
                                  const LineCols &cols, cudaStream_t stream);
cudaError_t column_minmax(int64_t n, const double *v_d, double *scratch_d, double *lo, double *hi,
                          cudaStream_t stream);
cudaError_t launch_gather_u8(int64_t n, const int64_t *order_d, const uint8_t *src_d, uint8_t *dst_d,
                             cudaStream_t stream);

// Collision-induced absorption (hkb_cia.cu): one table set on the device
struct CiaSetDev {
  double T;
  int64_t off;    // first row in the packed nu / cia arrays
  int n;          // rows
  int pad;
  int64_t istop;  // last grid index the set's scan reaches
};
cudaError_t launch_cia(const GridDev &g, const CiaSetDev *sets_d, int nsets, const double *nu_d,
                       const double *cia_d, double T, double P, double mass1, double kmin, int beyond,
                       double *K_d, cudaStream_t stream);

// Mean opacities and transmission function (hkb_means.cu)
size_t means_scratch_doubles(int nstates, int64_t nx);
cudaError_t launch_means(const double *K_d, int64_t k_stride, const GridDev &g, const double *T_d,
                         int nstates, double *scratch_d, double *out_d, cudaStream_t stream);
cudaError_t launch_transmission(const double *K_d, int64_t k_stride, int nstates, int nxb,
                                int nbins, const int *nxmin_d, double kmin, int nTr, double dTr,
                                double *Tr_d, cudaStream_t stream);

cudaError_t launch_count_pairs(const LinesDev &L, const GridDev &g, const StateDev *state_d,
                               unsigned long long *out_d, cudaStream_t stream);
inline size_t line_prep_bytes(bool mixed) { return mixed ? sizeof(LinePrepF) : sizeof(LinePrep); }

// Work plan of one Voigt launch: (state, tile) tickets, each tile's line
// range split into nsplit parts when there are too few tiles to fill the GPU
// (parts are combined in part order through partial_doubles of scratch and
// one counter per tile).
struct VoigtPlan {
  int shape = 0;  // tile shape (mixed form)
  int G = 0;      // grid points per tile of that shape
  int tile0 = 0;  // first tile of the launch (a section of one state's grid)
  int tiles_per_state = 0;
  int64_t tiles = 0;
  int ctas = 0;
  int nsplit = 1;
  size_t partial_doubles = 0;
  size_t counters = 0;
};
VoigtPlan plan_voigt_sum(bool mixed, int shape, int64_t nx, int nstates, int grid_ctas);
// tiles [tile0, tile0 + ntiles) of each state's grid
VoigtPlan plan_voigt_section(bool mixed, int shape, int64_t nx, int tile0, int ntiles, int grid_ctas);
// line-range parts per tile for a grid of nx points in tiles of the shape
int voigt_nsplit(int64_t nx, int shape);
cudaError_t launch_voigt_sum(bool mixed, const VoigtPlan &plan, const void *prep_d,
                             const double *nu0_d, int64_t nlines, const GridDev &g,
                             const StateDev *states_d, unsigned *ticket_d, double *partial_d,
                             unsigned *tile_cnt_d, double *K_d, int64_t k_stride,
                             cudaStream_t stream);

// A whole T-P table as one persistent launch (hkb_voigt.cu): line prep into
// a ring of per-state record slots and the Voigt sums of every state, as
// tickets of one counter (the prep tickets of state s interleaved with the
// sum tickets of state s - 1; a slot is reused once its previous state's
// sums are done).
struct TableFin {  // per state, written by the kernel's last prep ticket of the state
  double wmax;
  int s1exp, pad;
};
static_assert(sizeof(TableFin) == 16, "TableFin layout");
struct TablePlan {
  int shape = 0, G = 0;
  int S = 0, R = 3, slots = 1;  // states, ring slots of the schedule, slots allocated
  int lpt = 0, npb = 0;         // lines per prep ticket, prep tickets per state
  int tps = 0, nsplit = 1;
  long long nsum = 0, total = 0;
  int ctas = 0;
  size_t ring_bytes = 0, partial_doubles = 0, counters = 0;
};
// device buffers of a table launch: the record ring, split-tile partial rows
// and counters (slots x tiles), and the sync block of table_sync_bytes(S)
struct TableBufs {
  void *ring = nullptr;
  double *partial = nullptr;
  unsigned *tile_cnt = nullptr;
  void *sync = nullptr;
};
inline size_t table_sync_bytes(int nstates) {
  // ticket (8) + pad (8), wbits 16 S, fin 16 S, prep/sum counts and ready flags 12 S, error word
  return 16 + 16 * (size_t)nstates + sizeof(TableFin) * (size_t)nstates + 12 * (size_t)nstates + 16;
}
TablePlan plan_table(bool mixed, int shape, int64_t nlines, int64_t nx, int nstates);
cudaError_t launch_voigt_table(bool mixed, const TablePlan &plan, const LinesDev &L, const GridDev &g,
                               const StateDev *states_d, const TableBufs &bufs, double *K_d,
                               int64_t k_stride, cudaStream_t stream);
// the launch's error word in its sync block (0: every wait ended; 1: a wait
// for another ticket ran out and the results are incomplete)
int *table_error_word(void *sync_d, int nstates);

cudaError_t launch_prep_dump(const LinesDev &L, const GridDev &g,
                             const StateDev &st, double *out4_d,
                             long long *win6_d, cudaStream_t stream);

cudaError_t launch_profile_eval(int64_t n, const double *x_d, const double *y_d,
                                int mixed, double *out_d, cudaStream_t stream);

size_t kdist_smem_bytes(int nxb);
size_t kdist_scratch_doubles(int nxb, int nbins, int nstates);

cudaError_t launch_qr(int nxb, int nc, double *V_d, double *C_d, double *D_d,
                      cudaStream_t stream);

cudaError_t launch_kdist(const double *K_d, int64_t k_stride, int nstates,
                         int nxb, int nbins, int nc, double kmin,
                         double unitScale, const double *V_d, const double *C_d,
                         const double *D_d, double *coeff_d, int *nxmin_d,
                         double *sorted_d, double *recon_d, double *scratch_d,
                         cudaStream_t stream);

cudaError_t launch_gather_lines(int64_t n, const int64_t *order_d,
                                const double *src_d, double *dst_d,
                                cudaStream_t stream);
// per-line multipliers (device, load order) into the sorted order; *bad_d:
// the smallest load index of a value that is not finite and > 0, else n
cudaError_t launch_gather_scales(int64_t n, const int64_t *order_d, const double *src_d,
                                 double *dst_d, unsigned long long *bad_d, cudaStream_t stream);

cudaError_t sort_lines_by_nu(int64_t n, double *nu_d, int64_t *order_d,
                             cudaStream_t stream);

}  // namespace hkb
