// hkb_api.cu -- the C ABI of libhkb (declared in include/hkb.h).
//
// Host runtime: context, resident line list, grid, per-state constants and
// the launch sequence.  All arithmetic on lines and grid points runs on the
// GPU; the host only forms per-state scalars (partition-function
// interpolation, Doppler factors) exactly as the reference's host code does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hkb.h"
#include "hkb_formats.h"
#include "hkb_kernels.h"
#include "hkb_types.h"

using namespace hkb;

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, b ? b : 16);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct hk_ctx {
  int device = 0;
  std::string err;
  // species
  int database = HK_DB_HITRAN;
  std::vector<double> iso_mass, iso_ab;
  double defaultL = 0.0, defaultn = 0.0;
  std::vector<std::vector<double>> qT, qQ;
  std::vector<double> iso_ss;  // per-isotopologue species scale (mixtures), empty = 1
  double sl_abe[9] = {};       // sub-Lorentzian alpha, beta, epsilon of B1, B2, B3
  double qalphaL = 0.5, gammaF = 1.0, Sscale = 1.0;
  int units = 0;
  // lines (device, nu-sorted)
  int64_t nlines = 0;
  DevBuf nu0, Sfile, EL, gam, nexp, delta, Aterm, iso, order;
  LinesDev L{};
  double max_abs_delta = 0.0;
  // grid
  bool grid_set = false;
  GridDev g{};
  double numax = 0.0;
  int nbins = 0, nxb = 0;
  double kmin = 0.0;
  // workspace
  DevBuf states, ticket, wbits, Kwork, outwork, scratch, prep;
  DevBuf vpart, vcnt;  // split-tile partial sums and per-tile counters
  DevBuf sscale, gscale, adjwork;  // per-line scales (adjoint parameters), VJP workspace
  size_t prep_budget = (size_t)24 << 30;  // bytes of per-(state, line) records per batch
  size_t part_budget = (size_t)4 << 30;   // bytes of split-tile partial sums per batch
  double voigt_ms_acc = 0.0;
  DevBuf qrV, qrC, qrD;
  int qr_nxb = -1, qr_nc = -1;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool have_voigt_t = false, have_kdist_t = false;
  int64_t launches = 0;  // kernels launched since the last hk_opacity began
  bool voigt_ms_acc_only = false;  // sectioned call: voigt_ms_acc is the whole time
  // tile shape of the mixed Voigt kernel: fixed (tuning 0) or chosen by
  // timed probes (tuning 1 when the probes cost at most a tenth of the
  // call's sweep, tuning 2 always) once per loaded lines, grid and options
  int tuning = 0;
  int shape_fixed = 0;
  bool tuned = false;
  int tuned_shape = 0;
  int last_shape = 0;
  std::vector<double> tune_ms;  // probe time per shape at the last tuning
  DevBuf tunework;              // probe states and their max-term words
  DevBuf meanwork;              // means / transmission inputs, partial sums and outputs
  // collision-induced absorption in place of lines (hk_load_cia)
  bool cia = false;
  std::vector<CiaSet> cia_sets;
  double cia_mass1 = 1.0;
  DevBuf cia_nu, cia_val, cia_tab;
  // T-P table recorded as one CUDA graph (hk_table_build / hk_table_run)
  cudaGraph_t table_graph = nullptr;
  cudaGraphExec_t table_exec = nullptr;
  int64_t table_kernels = 0;
  int table_states = 0;
  int table_fused = 0;  // hk_set_table_mode: 1 = one persistent launch for the table's sums
  DevBuf tsync;  // the table kernel's counters, flags and per-state scales
};

static hk_status fail(hk_ctx *c, hk_status s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return s;
}

#define CUDA_TRY(ctx, expr)                                                   \
  do {                                                                        \
    cudaError_t e_ = (expr);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return fail(ctx, (e_ == cudaErrorMemoryAllocation) ? HK_ERR_NOMEM       \
                                                         : HK_ERR_CUDA,       \
                  "%s: %s", #expr, cudaGetErrorString(e_));                   \
  } while (0)

static void ok(hk_ctx *c) { c->err.clear(); }

extern "C" {

const char *hk_version(void) { return "hkb 0.1 (sm_100a)"; }

hk_ctx *hk_create(int device, hk_status *status) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    if (status) *status = HK_ERR_CUDA;
    return nullptr;
  }
  if (device < 0 || device >= n) {
    if (status) *status = HK_ERR_ARG;
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    if (status) *status = HK_ERR_CUDA;
    return nullptr;
  }
  hk_ctx *c = new hk_ctx();
  c->device = device;
  for (auto &e : c->ev) cudaEventCreate(&e);
  if (c->ticket.ensure(sizeof(unsigned)) != cudaSuccess) {
    delete c;
    if (status) *status = HK_ERR_NOMEM;
    return nullptr;
  }
  if (status) *status = HK_OK;
  return c;
}

static void table_release(hk_ctx *c) {
  if (c->table_exec) cudaGraphExecDestroy(c->table_exec);
  if (c->table_graph) cudaGraphDestroy(c->table_graph);
  c->table_exec = nullptr;
  c->table_graph = nullptr;
  c->table_kernels = 0;
}

void hk_destroy(hk_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  table_release(c);
  for (DevBuf *b : {&c->nu0, &c->Sfile, &c->EL, &c->gam, &c->nexp, &c->delta,
                    &c->Aterm, &c->iso, &c->order, &c->states, &c->ticket,
                    &c->prep, &c->wbits, &c->Kwork, &c->outwork, &c->scratch,
                    &c->qrV, &c->qrC, &c->qrD, &c->vpart, &c->vcnt, &c->sscale, &c->gscale, &c->adjwork,
                    &c->tunework, &c->meanwork, &c->cia_nu, &c->cia_val, &c->cia_tab})
    b->release();
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  delete c;
}

const char *hk_last_error(const hk_ctx *c) { return c ? c->err.c_str() : "null context"; }

int hk_tile_points(void) { return voigt_tile_points(0); }

// ------------------------------------------------------------- species
hk_status hk_set_species(hk_ctx *c, int database, int niso, const double *mass,
                         const double *ab, double defaultL, double defaultn) {
  if (!c) return HK_ERR_ARG;
  if (database != HK_DATABASE_HITRAN && database != HK_DATABASE_EXOMOL)
    return fail(c, HK_ERR_UNSUPPORTED, "database %d: only 0 (HITRAN) and 2 (ExoMol) are on this path", database);
  if (niso < 1 || niso > HK_MAX_ISO || !mass || !ab)
    return fail(c, HK_ERR_ARG, "niso must be 1..%d with mass and abundance arrays", HK_MAX_ISO);
  for (int i = 0; i < niso; ++i)
    if (!(mass[i] > 0.0)) return fail(c, HK_ERR_ARG, "isotopologue %d: mass must be > 0", i);
  c->database = database;
  c->iso_mass.assign(mass, mass + niso);
  c->iso_ab.assign(ab, ab + niso);
  c->defaultL = defaultL;
  c->defaultn = defaultn;
  c->qT.assign(niso, {});
  c->qQ.assign(niso, {});
  c->iso_ss.clear();
  c->cia = false;
  ok(c);
  return HK_OK;
}

hk_status hk_set_partition(hk_ctx *c, int iso, int n, const double *T, const double *Q) {
  if (!c) return HK_ERR_ARG;
  if (iso < 0 || iso >= (int)c->qT.size()) return fail(c, HK_ERR_STATE, "hk_set_species must come first (iso %d)", iso);
  if (n < 1 || !T || !Q) return fail(c, HK_ERR_ARG, "empty partition table");
  c->qT[iso].assign(T, T + n);
  c->qQ[iso].assign(Q, Q + n);
  ok(c);
  return HK_OK;
}

hk_status hk_set_options(hk_ctx *c, double qalphaL, double gammaF, int units, double Sscale) {
  if (!c) return HK_ERR_ARG;
  if (units != 0 && units != 1) return fail(c, HK_ERR_ARG, "units must be 0 or 1");
  c->qalphaL = qalphaL;
  c->gammaF = gammaF;
  c->units = units;
  c->Sscale = Sscale;
  c->tuned = false;
  ok(c);
  return HK_OK;
}

// --------------------------------------------------------------- lines
// ------------------------------------------------------------ ingestion
// Lines arrive as unsorted device columns in load order (from caller arrays
// or from binary records unpacked on the GPU, hkb_ingest.cu); load_device
// sorts them by centre once, gathers each column into sorted order, and keeps
// a column whose values are all equal as a scalar (synthetic HITRAN: A = delta
// = 0; ExoMol: gamma, n from the species defaults).
struct IngestBuf {
  DevBuf cols;  // 7 n doubles + n bytes, plus minmax scratch
  LineCols lc{};
  double *scratch = nullptr;
  cudaError_t alloc(int64_t n) {
    const size_t nd = (size_t)std::max<int64_t>(n, 1);
    cudaError_t e = cols.ensure(7 * nd * sizeof(double) + nd + 2 * 592 * sizeof(double) + 64);
    if (e != cudaSuccess) return e;
    double *p = cols.as<double>();
    lc.nu = p;
    lc.S = p + nd;
    lc.EL = p + 2 * nd;
    lc.gam = p + 3 * nd;
    lc.nexp = p + 4 * nd;
    lc.delta = p + 5 * nd;
    lc.Aterm = p + 6 * nd;
    scratch = p + 7 * nd;
    lc.iso = reinterpret_cast<uint8_t *>(scratch + 2 * 592);
    return cudaSuccess;
  }
};

static IngestSpec ingest_spec(const hk_ctx *c, bool hitran) {
  IngestSpec sp{};
  sp.hitran = hitran ? 1 : 0;
  sp.niso = (int)c->iso_mass.size();
  sp.qalphaL = c->qalphaL;
  sp.gammaF = c->gammaF;
  sp.defaultL = c->defaultL;
  sp.defaultn = c->defaultn;
  sp.four_pi_c = 4.0 * M_PI * HK_C;  // voigt.h:349 divides A by this product
  return sp;
}

static hk_status load_device(hk_ctx *c, int64_t n, IngestBuf &ib, int niso) {
  cudaSetDevice(c->device);
  c->tuned = false;
  c->nlines = 0;
  c->L = LinesDev{};
  c->L.database = c->database;
  if (n == 0) {
    ok(c);
    return HK_OK;
  }
  CUDA_TRY(c, c->nu0.ensure(n * sizeof(double)));
  CUDA_TRY(c, c->order.ensure(n * sizeof(int64_t)));
  CUDA_TRY(c, cudaMemcpy(c->nu0.p, ib.lc.nu, n * sizeof(double), cudaMemcpyDeviceToDevice));
  CUDA_TRY(c, sort_lines_by_nu(n, c->nu0.as<double>(), c->order.as<int64_t>(), 0));
  CUDA_TRY(c, cudaDeviceSynchronize());
  struct Col { DevBuf *buf; double *src; const double **dst; double *cval; bool uni; };
  double dummy = 0.0;
  const double *sfile = nullptr;
  Col cols[6] = {{&c->Sfile, ib.lc.S, &sfile, &dummy, false},
                 {&c->EL, ib.lc.EL, &c->L.EL, &c->L.EL_c, true},
                 {&c->gam, ib.lc.gam, &c->L.gam, &c->L.gam_c, true},
                 {&c->nexp, ib.lc.nexp, &c->L.nexp, &c->L.nexp_c, true},
                 {&c->delta, ib.lc.delta, &c->L.delta, &c->L.delta_c, true},
                 {&c->Aterm, ib.lc.Aterm, &c->L.Aterm, &c->L.Aterm_c, true}};
  for (Col &q : cols) {
    double lo = 0.0, hi = 0.0;
    CUDA_TRY(c, column_minmax(n, q.src, ib.scratch, &lo, &hi, 0));
    *q.cval = lo;
    if (q.buf == &c->delta) c->max_abs_delta = std::max(std::fabs(lo), std::fabs(hi));
    if (q.uni && lo == hi) {
      q.buf->release();
      *q.dst = nullptr;
      continue;
    }
    CUDA_TRY(c, q.buf->ensure(n * sizeof(double)));
    CUDA_TRY(c, launch_gather_lines(n, c->order.as<int64_t>(), q.src, q.buf->as<double>(), 0));
    *q.dst = q.buf->as<double>();
  }
  c->L.Sfile = sfile;
  if (niso <= 1) {
    c->iso.release();
    c->L.iso = nullptr;
  } else {
    CUDA_TRY(c, c->iso.ensure(n));
    CUDA_TRY(c, launch_gather_u8(n, c->order.as<int64_t>(), ib.lc.iso, c->iso.as<uint8_t>(), 0));
    c->L.iso = c->iso.as<uint8_t>();
  }
  CUDA_TRY(c, cudaDeviceSynchronize());
  c->L.nu0 = c->nu0.as<double>();
  c->L.n = n;
  c->nlines = n;
  ok(c);
  return HK_OK;
}

hk_status hk_load_lines_hitran(hk_ctx *c, int64_t n, const double *nu, const double *S,
                               const double *EL, const double *A, const double *delta,
                               const double *gair, const double *gself, const double *nexp,
                               const int32_t *iso) {
  if (!c) return HK_ERR_ARG;
  if (c->iso_mass.empty()) return fail(c, HK_ERR_STATE, "hk_set_species must come before loading lines");
  if (c->database != HK_DB_HITRAN) return fail(c, HK_ERR_STATE, "species database is not HITRAN");
  if (n < 0 || (n > 0 && (!nu || !S || !EL || !A || !delta || !gair || !gself || !nexp)))
    return fail(c, HK_ERR_ARG, "null line array");
  const int niso = (int)c->iso_mass.size();
  if (iso)
    for (int64_t i = 0; i < n; ++i)
      if (iso[i] < 0 || iso[i] >= niso)
        return fail(c, HK_ERR_FORMAT, "line %lld: isotopologue index %d not in the species table", (long long)i, iso[i]);
  cudaSetDevice(c->device);
  IngestBuf ib;
  DevBuf tmp;  // gamma_air, gamma_self, A and the isotopologue indices as given
  const size_t nd = (size_t)std::max<int64_t>(n, 1);
  CUDA_TRY(c, ib.alloc(n));
  CUDA_TRY(c, tmp.ensure(3 * nd * sizeof(double) + nd * sizeof(int32_t)));
  double *ga = tmp.as<double>(), *gs = ga + nd, *Ad = ga + 2 * nd;
  int32_t *iso32 = reinterpret_cast<int32_t *>(ga + 3 * nd);
  const size_t B = (size_t)n * sizeof(double);
  if (n) {
    CUDA_TRY(c, cudaMemcpy(ib.lc.nu, nu, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ib.lc.S, S, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ib.lc.EL, EL, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ib.lc.nexp, nexp, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ib.lc.delta, delta, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ga, gair, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(gs, gself, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(Ad, A, B, cudaMemcpyHostToDevice));
    if (iso) CUDA_TRY(c, cudaMemcpy(iso32, iso, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice));
    CUDA_TRY(c, launch_finish_columns(n, ingest_spec(c, true), ga, gs, Ad, iso ? iso32 : nullptr,
                                      ib.lc, 0));
  }
  tmp.release();
  return load_device(c, n, ib, niso);
}

hk_status hk_load_lines_exomol(hk_ctx *c, int64_t n, const double *nu, const double *S,
                               const double *EL, const double *A) {
  if (!c) return HK_ERR_ARG;
  if (c->iso_mass.empty()) return fail(c, HK_ERR_STATE, "hk_set_species must come before loading lines");
  if (c->database != HK_DB_EXOMOL) return fail(c, HK_ERR_STATE, "species database is not ExoMol");
  if (n < 0 || (n > 0 && (!nu || !S || !EL || !A))) return fail(c, HK_ERR_ARG, "null line array");
  cudaSetDevice(c->device);
  IngestBuf ib;
  DevBuf tmp;  // A as given
  CUDA_TRY(c, ib.alloc(n));
  CUDA_TRY(c, tmp.ensure((size_t)std::max<int64_t>(n, 1) * sizeof(double)));
  const size_t B = (size_t)n * sizeof(double);
  if (n) {
    CUDA_TRY(c, cudaMemcpy(ib.lc.nu, nu, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ib.lc.S, S, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(ib.lc.EL, EL, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaMemcpy(tmp.p, A, B, cudaMemcpyHostToDevice));
    CUDA_TRY(c, launch_finish_columns(n, ingest_spec(c, false), nullptr, nullptr, tmp.as<double>(),
                                      nullptr, ib.lc, 0));
  }
  tmp.release();
  return load_device(c, n, ib, 1);
}

int64_t hk_num_lines(const hk_ctx *c) { return c ? c->nlines : 0; }

hk_status hk_line_order(hk_ctx *c, int64_t *order) {
  if (!c || !order) return HK_ERR_ARG;
  if (c->nlines == 0) return HK_OK;
  cudaSetDevice(c->device);
  CUDA_TRY(c, cudaMemcpy(order, c->order.p, c->nlines * sizeof(int64_t), cudaMemcpyDeviceToHost));
  ok(c);
  return HK_OK;
}

// ---------------------------------------------------------------- grid
hk_status hk_set_grid(hk_ctx *c, double numin, double numax, double dnu, int nbins,
                      int cutMode, double cut, double kmin) {
  if (!c) return HK_ERR_ARG;
  if (!(dnu > 0.0) || !(numax > numin)) return fail(c, HK_ERR_ARG, "need numax > numin and dnu > 0");
  if (nbins < 1) return fail(c, HK_ERR_ARG, "nbins must be >= 1");
  if (cutMode < 0 || cutMode > 2) return fail(c, HK_ERR_ARG, "cutMode must be 0, 1 or 2");
  if (cut < 0.0) return fail(c, HK_ERR_ARG, "cut must be >= 0");
  // heliosk.cu:448-461
  const double nxd = (numax - numin) / dnu + 0.5;
  if (nxd >= 2147483647.0) return fail(c, HK_ERR_RANGE, "Nx too large, integer overflow. %g", nxd);
  const int nx = (int)nxd;
  if (nx % nbins != 0)
    return fail(c, HK_ERR_RANGE, "range cannot be divided evenly in bins. %d %d %g", nx, nbins, nx / (double)nbins);
  c->g.numin = numin;
  c->g.dnu = dnu;
  c->g.nx = nx;
  c->g.cutMode = cutMode;
  c->g.cut = (cut == 0.0) ? 1.0e30 : cut;  // heliosk.cu:947
  c->numax = numax;
  c->nbins = nbins;
  c->nxb = nx / nbins;
  c->kmin = kmin;
  c->grid_set = true;
  c->tuned = false;
  ok(c);
  return HK_OK;
}

int64_t hk_grid_points(const hk_ctx *c) { return (c && c->grid_set) ? c->g.nx : 0; }

// --------------------------------------------------------------- states
static hk_status build_states(hk_ctx *c, int nstates, const double *T, const double *P,
                              std::vector<StateDev> &out) {
  const int niso = (int)c->iso_mass.size();
  // species scale of each isotopologue: Sscale, times the species' abundance
  // in a mixture; mean molar mass over all of them (heliosk.cu:672-686)
  auto sscale = [&](int i) { return c->iso_ss.empty() ? c->Sscale : c->Sscale * c->iso_ss[i]; };
  double meanMass = 0.0;
  for (int i = 0; i < niso; ++i) meanMass += c->iso_ab[i] * c->iso_mass[i] * sscale(i);
  out.assign(nstates, StateDev{});
  for (int s = 0; s < nstates; ++s) {
    StateDev &st = out[s];
    const double Ts = T[s], Ps = P[s];
    if (!(Ts > 0.0)) return fail(c, HK_ERR_ARG, "state %d: T must be > 0", s);
    if (!(Ps >= 0.0)) return fail(c, HK_ERR_ARG, "state %d: P must be >= 0", s);
    st.T = Ts;
    st.P = Ps;
    st.PoverP0 = (c->database == HK_DB_HITRAN) ? Ps / HK_PO_ATM : Ps / HK_PO_BAR;
    st.powbase = HK_T0 / Ts;
    st.c1 = HK_H * HK_C / (HK_KB * Ts);
    st.wmax = c->g.cut;
    st.shift = c->max_abs_delta * Ps;
    st.kmin = c->kmin;
    // subLorentzianB (voigt.h:12-35): B_k = alpha_k + beta_k exp(-epsilon_k T)
    for (int k = 0; k < 3; ++k)
      st.sl_B[k] = c->sl_abe[3 * k] + c->sl_abe[3 * k + 1] * std::exp(-c->sl_abe[3 * k + 2] * Ts);
    for (int j = 0; j < niso; ++j) {
      double Q;
      if (c->qT[j].empty()) return fail(c, HK_ERR_STATE, "no partition table for isotopologue %d", j);
      if (!partition_interp(c->qT[j].data(), c->qQ[j].data(), (int)c->qT[j].size(), Ts, &Q))
        return fail(c, HK_ERR_RANGE, "partition function not valid for given temperature. T: %g (isotopologue %d)", Ts, j);
      const double mass = c->iso_mass[j] / HK_NA;
      st.iad0[j] = HK_C * std::sqrt(mass / (2.0 * HK_KB * Ts));
      st.Q[j] = Q;
      double dl = 0.0;
      partition_dlnq(c->qT[j].data(), c->qQ[j].data(), (int)c->qT[j].size(), Ts, &dl);
      st.dlnQ[j] = dl;
      double Abundance = c->iso_ab[j];
      double Ss = sscale(j);
      if (c->units == 0) {
        Abundance *= c->iso_mass[j] / meanMass;
        Ss *= c->iso_mass[j] / meanMass;
      }
      st.ab[j] = Abundance;
      st.ss[j] = Ss;
    }
  }
  return HK_OK;
}

static hk_status check_ready(hk_ctx *c) {
  if (!c->grid_set) return fail(c, HK_ERR_STATE, "hk_set_grid must come first");
  if (c->iso_mass.empty() && !c->cia) return fail(c, HK_ERR_STATE, "hk_set_species must come first");
  return HK_OK;
}

// States whose per-line records exceed the workspace (e.g. 5e8 ExoMol lines
// at 112 B): a state pass over all lines fixes every state's cutoff bound and
// FP32 scale, then each state's grid is cut into tile sections whose lines --
// a contiguous range of the nu-sorted list -- fit the workspace, and each
// section is prepared and summed on its own.  A tile sees the same lines in
// the same order as in the batched path, so K is bit-identical to it.
static hk_status opacity_sectioned(hk_ctx *c, int nstates, bool mixed, int shape, double *Kd,
                                   cudaStream_t s) {
  const int64_t nx = c->g.nx, n = c->nlines;
  const int G = voigt_tile_points(shape);
  const int tps = (int)((nx + G - 1) / G);
  const size_t rec = line_prep_bytes(mixed);
  const int64_t cap = (int64_t)(c->prep_budget / rec);
  if (cap < 1) return fail(c, HK_ERR_NOMEM, "workspace budget below one line record");
  CUDA_TRY(c, c->prep.ensure((size_t)std::min<int64_t>(cap, n) * rec));
  StateDev *sd = c->states.as<StateDev>();
  CUDA_TRY(c, launch_state_stats(c->L, c->g, sd, nstates, c->wbits.as<unsigned long long>(), s));
  c->launches += 2;
  std::vector<StateDev> hs(nstates);
  CUDA_TRY(c, cudaMemcpyAsync(hs.data(), sd, nstates * sizeof(StateDev), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  CUDA_TRY(c, c->adjwork.ensure(4 * sizeof(double)));
  double *q_d = c->adjwork.as<double>();
  int64_t *lb_d = reinterpret_cast<int64_t *>(q_d + 2);
  auto line_range = [&](int st, int t0, int t1, int64_t &L0, int64_t &L1) -> cudaError_t {
    const double W = hs[st].wmax + hs[st].shift + 2.0 * c->g.dnu;
    const double xlo = std::fma((double)t0 * G, c->g.dnu, c->g.numin) - W;
    const double xhi = std::fma((double)(std::min<int64_t>((int64_t)t1 * G, nx) - 1), c->g.dnu, c->g.numin) + W;
    const double pad = 1e-12 * (std::fabs(xlo) + std::fabs(xhi)) + 1e-300;
    const double q[2] = {xlo - pad, xhi + pad};
    int64_t lb[2];
    cudaError_t e = cudaMemcpyAsync(q_d, q, sizeof q, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_lower_bound(c->L.nu0, n, q_d, 2, lb_d, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(lb, lb_d, sizeof lb, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    L0 = lb[0];
    L1 = lb[1];
    return e;
  };
  for (int st = 0; st < nstates; ++st) {
    struct Sec { int t0, t1; int64_t L0, L1; };
    std::vector<Sec> secs;
    std::vector<std::pair<int, int>> todo{{0, tps}};
    while (!todo.empty()) {
      const std::pair<int, int> tt = todo.back();
      todo.pop_back();
      int64_t L0 = 0, L1 = 0;
      CUDA_TRY(c, line_range(st, tt.first, tt.second, L0, L1));
      if (L1 - L0 <= cap) {
        secs.push_back({tt.first, tt.second, L0, L1});
      } else if (tt.second - tt.first == 1) {
        return fail(c, HK_ERR_NOMEM, "one grid tile reaches %lld lines, above the workspace of %lld records",
                    (long long)(L1 - L0), (long long)cap);
      } else {
        const int mid = (tt.first + tt.second) / 2;
        todo.push_back({mid, tt.second});
        todo.push_back({tt.first, mid});
      }
    }
    for (const Sec &q : secs) {
      const LinesDev Ls = lines_sub(c->L, q.L0, q.L1 - q.L0);
      const VoigtPlan plan = plan_voigt_section(mixed, shape, nx, q.t0, q.t1 - q.t0, 0);
      if (plan.nsplit > 1) {
        CUDA_TRY(c, c->vpart.ensure(plan.partial_doubles * sizeof(double)));
        CUDA_TRY(c, c->vcnt.ensure(plan.counters * sizeof(unsigned)));
      }
      CUDA_TRY(c, launch_line_records(mixed, Ls, c->g, sd + st, c->prep.p, s));
      CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
      CUDA_TRY(c, launch_voigt_sum(mixed, plan, c->prep.p, Ls.nu0, Ls.n, c->g, sd + st,
                                   c->ticket.as<unsigned>(), c->vpart.as<double>(),
                                   c->vcnt.as<unsigned>(), Kd + (size_t)st * nx, nx, s));
      CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
      c->launches += 2;
      float ms = 0.f;
      CUDA_TRY(c, cudaEventSynchronize(c->ev[1]));
      CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
      c->voigt_ms_acc += ms;
    }
  }
  c->have_voigt_t = false;  // all Voigt time is in voigt_ms_acc
  c->voigt_ms_acc_only = true;
  return HK_OK;
}

// ------------------------------------------------------------ autotuner
// The mixed kernel's tile shape (lines per staged chunk x grid points per
// tile; voigt_num_shapes() of them) changes only the order of the FP64
// additions, so every shape meets the same accuracy; the fastest depends on
// the line density, the window widths and the grid.  Like the reference's
// self-tuning of its kernels' tile widths (heliosk.cu:1363-1705, timed trial
// launches), the tuner times each shape on probes of the workload: up to 4 of
// the call's states spread over it, each prepared on its own, on a section of
// the grid in the middle (a quarter of it at least, and two waves of
// tickets), after one warm-up tile per shape.  The choice holds until lines,
// grid or options change.  Its probe outputs land in K rows the call then
// overwrites.
// Whether a call of the given precision runs the mixed form.  It holds the
// Voigt regions and the Lorentz profile (with sub-Lorentzian wings or plinth
// removal), the Doppler profile (with plinth removal too) and the binned
// Gaussian (region A; FP32 where their terms are normal floats, FP64 tails).
// Sub-Lorentzian wings run the FP64 form with plinth removal (chi t - plinth
// is no difference of one function, so no cancellation-free form exists)
// and with the Gaussian profiles.
static bool mixed_form(const hk_ctx *c, int precision) {
  return precision == HK_PRECISION_MIXED && !(c->g.subL && (c->g.plinth || c->g.profile >= 3));
}

static int shape_for(const hk_ctx *c, bool mixed) {
  // the kernels of the Gaussian profiles, plinth removal and sub-Lorentzian
  // wings have the default shape only
  if (!mixed || c->g.profile >= 3 || c->g.plinth || c->g.subL) return 0;
  return (c->tuning != 0 && c->tuned) ? c->tuned_shape : c->shape_fixed;
}

static hk_status tune_shape(hk_ctx *c, int nstates, const std::vector<StateDev> &hs, double *Kd,
                            cudaStream_t s) {
  const int64_t nx = c->g.nx, n = c->nlines;
  const int nsh = voigt_num_shapes();
  const size_t per_state = (size_t)std::max<int64_t>(n, 1) * line_prep_bytes(true);
  int np = std::max(1, std::min({4, nstates / 12, (int)std::min<size_t>(4, c->prep_budget / per_state)}));
  const int G0 = voigt_tile_points(0);  // the widest tile; every shape's tile divides it
  const int tps0 = (int)((nx + G0 - 1) / G0);
  const VoigtPlan p0 = plan_voigt_sum(true, 0, nx, 1, 0);
  const int sec = std::min(tps0, std::max((tps0 + 3) / 4, (2 * p0.ctas + p0.nsplit - 1) / p0.nsplit));
  const int first = (tps0 - sec) / 2;
  const int64_t x0 = (int64_t)first * G0, x1 = std::min<int64_t>((int64_t)(first + sec) * G0, nx);
  if (c->tuning == 1) {
    // probe sweeps in state-equivalents against the call's sweep
    const double cost = (double)nsh * np * (double)(x1 - x0) / (double)nx;
    if (cost > 0.1 * nstates) return HK_OK;
  }
  std::vector<StateDev> ps(np);
  for (int k = 0; k < np; ++k) ps[k] = hs[np == 1 ? 0 : (int)((int64_t)k * (nstates - 1) / (np - 1))];
  CUDA_TRY(c, c->tunework.ensure(np * (sizeof(StateDev) + 2 * sizeof(unsigned long long))));
  StateDev *tsd = c->tunework.as<StateDev>();
  unsigned long long *twb = reinterpret_cast<unsigned long long *>(tsd + np);
  CUDA_TRY(c, cudaMemcpyAsync(tsd, ps.data(), np * sizeof(StateDev), cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, c->prep.ensure((size_t)np * per_state));
  CUDA_TRY(c, launch_line_prep(true, c->L, c->g, tsd, np, c->prep.p, twb, s));
  c->launches += 2;
  c->tune_ms.assign(nsh, -1.0);
  int best = 0;
  for (int v = 0; v < nsh; ++v) {
    const int G = voigt_tile_points(v);
    const int t0 = (int)(x0 / G), nt = (int)((x1 - x0 + G - 1) / G);
    const VoigtPlan pw = plan_voigt_section(true, v, nx, t0, 1, 0);
    const VoigtPlan pl = plan_voigt_section(true, v, nx, t0, nt, pw.ctas);
    if (pl.nsplit > 1) {
      CUDA_TRY(c, c->vpart.ensure(pl.partial_doubles * sizeof(double)));
      CUDA_TRY(c, c->vcnt.ensure(pl.counters * sizeof(unsigned)));
    }
    CUDA_TRY(c, launch_voigt_sum(true, pw, c->prep.p, c->L.nu0, n, c->g, tsd, c->ticket.as<unsigned>(),
                                 c->vpart.as<double>(), c->vcnt.as<unsigned>(), Kd, nx, s));
    double ms_v = 0.0;
    for (int k = 0; k < np; ++k) {
      const char *pk = static_cast<const char *>(c->prep.p) + (size_t)k * per_state;
      CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
      CUDA_TRY(c, launch_voigt_sum(true, pl, pk, c->L.nu0, n, c->g, tsd + k, c->ticket.as<unsigned>(),
                                   c->vpart.as<double>(), c->vcnt.as<unsigned>(), Kd + (size_t)k * nx,
                                   nx, s));
      CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
      CUDA_TRY(c, cudaEventSynchronize(c->ev[1]));
      float ms = 0.f;
      CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
      ms_v += ms;
    }
    c->launches += 1 + np;
    c->tune_ms[v] = ms_v;
    c->voigt_ms_acc += ms_v;  // probe sweeps count as line-sum time
    if (v == 0 || ms_v < c->tune_ms[best]) best = v;  // ties keep the lower shape
  }
  c->tuned_shape = best;
  c->tuned = true;
  return HK_OK;
}

// ------------------------------------------------------------------ CIA
// hk_opacity of a CIA context: per state the sets the reference reads for
// its T (up to the first with T <= T_set; above all of them K = kmin), each
// with the last grid index its scan reaches.
static hk_status opacity_cia(hk_ctx *c, int nstates, const double *T, const double *P, double *K_out,
                             int K_on_device, cudaStream_t s) {
  const int64_t nx = c->g.nx;
  double *Kd = K_out;
  if (!K_on_device) {
    CUDA_TRY(c, c->Kwork.ensure((size_t)nstates * nx * sizeof(double)));
    Kd = c->Kwork.as<double>();
  }
  const int ns = (int)c->cia_sets.size();
  std::vector<CiaSetDev> tab((size_t)nstates * ns);
  std::vector<int> used(nstates), beyond(nstates);
  for (int q = 0; q < nstates; ++q) {
    if (!(T[q] > 0.0) || !(P[q] >= 0.0)) return fail(c, HK_ERR_ARG, "state %d: need T > 0 and P >= 0", q);
    int k = 0;
    int64_t off = 0;
    for (; k < ns; ++k) {
      const CiaSet &cs = c->cia_sets[k];
      const int n = (int)cs.nu.size();
      int64_t istop = nx - 1;
      if (n == 2) {
        istop = 0;
      } else {
        // first grid point at or past nu[n-2] (x_i = numin + i dnu, one FMA)
        int64_t lo = 0, hi = nx;
        while (lo < hi) {
          const int64_t m = lo + (hi - lo) / 2;
          if (std::fma((double)m, c->g.dnu, c->g.numin) >= cs.nu[n - 2]) hi = m;
          else lo = m + 1;
        }
        if (lo < nx) istop = lo;
      }
      tab[(size_t)q * ns + k] = CiaSetDev{cs.T, off, n, 0, istop};
      off += n;
      if (T[q] <= cs.T) break;
    }
    used[q] = std::min(k + 1, ns);
    beyond[q] = (k == ns);  // T above every set: host.h:773-775
  }
  CUDA_TRY(c, c->cia_tab.ensure(std::max<size_t>(tab.size(), 1) * sizeof(CiaSetDev)));
  CUDA_TRY(c, cudaMemcpyAsync(c->cia_tab.p, tab.data(), tab.size() * sizeof(CiaSetDev), cudaMemcpyHostToDevice, s));
  for (int q = 0; q < nstates; ++q)
    CUDA_TRY(c, launch_cia(c->g, c->cia_tab.as<CiaSetDev>() + (size_t)q * ns, used[q], c->cia_nu.as<double>(),
                           c->cia_val.as<double>(), T[q], P[q], c->cia_mass1, c->kmin, beyond[q],
                           Kd + (size_t)q * nx, s));
  c->launches = nstates;
  c->have_voigt_t = false;
  c->voigt_ms_acc = 0.0;
  if (!K_on_device) {
    CUDA_TRY(c, cudaMemcpyAsync(K_out, Kd, (size_t)nstates * nx * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(c, cudaStreamSynchronize(s));  // the set table is pageable host memory
  ok(c);
  return HK_OK;
}

hk_status hk_opacity(hk_ctx *c, int nstates, const double *T, const double *P, int precision,
                     double *K_out, int K_on_device, void *stream) {
  if (!c) return HK_ERR_ARG;
  hk_status st;
  if ((st = check_ready(c)) != HK_OK) return st;
  if (nstates < 1 || !T || !P || !K_out) return fail(c, HK_ERR_ARG, "need nstates >= 1, T, P and K_out");
  if (precision != HK_PRECISION_PLAIN_FP64 && precision != HK_PRECISION_MIXED)
    return fail(c, HK_ERR_ARG, "precision must be 0 (plain FP64) or 1 (mixed)");
  if (nstates > 65535) return fail(c, HK_ERR_RANGE, "at most 65535 states per call");
  cudaSetDevice(c->device);
  cudaStream_t s = (cudaStream_t)stream;
  if (c->cia) return opacity_cia(c, nstates, T, P, K_out, K_on_device, s);
  std::vector<StateDev> hs;
  if ((st = build_states(c, nstates, T, P, hs)) != HK_OK) return st;
  CUDA_TRY(c, c->states.ensure(nstates * sizeof(StateDev)));
  CUDA_TRY(c, c->wbits.ensure(2 * nstates * sizeof(unsigned long long)));
  CUDA_TRY(c, cudaMemcpyAsync(c->states.p, hs.data(), nstates * sizeof(StateDev), cudaMemcpyHostToDevice, s));
  const int64_t nx = c->g.nx;
  double *Kd = K_out;
  if (!K_on_device) {
    CUDA_TRY(c, c->Kwork.ensure((size_t)nstates * nx * sizeof(double)));
    Kd = c->Kwork.as<double>();
  }
  // States run in batches whose per-(state, line) records fit the prep
  // budget; each batch is one prep launch and one persistent Voigt launch.
  const bool mixed = mixed_form(c, precision);
  const size_t per_state = (size_t)std::max<int64_t>(c->nlines, 1) * line_prep_bytes(mixed);
  c->voigt_ms_acc = 0.0;
  c->have_voigt_t = false;
  c->voigt_ms_acc_only = false;
  c->launches = 0;
  if (mixed && c->g.profile <= 2 && !c->g.plinth && !c->g.subL && c->tuning != 0 && !c->tuned && per_state <= c->prep_budget && c->nlines > 0)
    if ((st = tune_shape(c, nstates, hs, Kd, s)) != HK_OK) return st;
  const int shape = shape_for(c, mixed);
  c->last_shape = shape;
  int batch = (int)std::max<size_t>(1, c->prep_budget / per_state);
  const int nsplit = voigt_nsplit(nx, shape);
  if (nsplit > 1) {
    // split tiles keep one partial row per part: bound that scratch too
    const int G = voigt_tile_points(shape);
    const size_t part_per_state = (size_t)((nx + G - 1) / G) * nsplit * G * sizeof(double);
    batch = std::min(batch, (int)std::max<size_t>(1, c->part_budget / part_per_state));
  }
  batch = std::min(batch, nstates);
  if (per_state > c->prep_budget) {
    if ((st = opacity_sectioned(c, nstates, mixed, shape, Kd, s)) != HK_OK) return st;
    batch = nstates;  // nothing left for the batched loop
  } else {
    CUDA_TRY(c, c->prep.ensure((size_t)batch * per_state));
  }
  StateDev *sd = c->states.as<StateDev>();
  unsigned long long *wb = c->wbits.as<unsigned long long>();
  for (int b0 = 0; per_state <= c->prep_budget && b0 < nstates; b0 += batch) {
    const int nb = std::min(batch, nstates - b0);
    const VoigtPlan plan = plan_voigt_sum(mixed, shape, nx, nb, 0);
    c->launches += 3;  // line prep, state finalize, Voigt sum
    if (plan.nsplit > 1) {
      CUDA_TRY(c, c->vpart.ensure(plan.partial_doubles * sizeof(double)));
      CUDA_TRY(c, c->vcnt.ensure(plan.counters * sizeof(unsigned)));
    }
    CUDA_TRY(c, launch_line_prep(mixed, c->L, c->g, sd + b0, nb, c->prep.p, wb + 2 * b0, s));
    CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
    CUDA_TRY(c, launch_voigt_sum(mixed, plan, c->prep.p, c->L.nu0, c->nlines, c->g,
                                 sd + b0, c->ticket.as<unsigned>(), c->vpart.as<double>(),
                                 c->vcnt.as<unsigned>(), Kd + (size_t)b0 * nx, nx, s));
    CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
    c->have_voigt_t = true;
    if (b0 + nb < nstates) {
      // accumulate the Voigt time of earlier batches (the last one is read
      // lazily by hk_last_timing)
      float ms = 0.f;
      CUDA_TRY(c, cudaEventSynchronize(c->ev[1]));
      CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
      c->voigt_ms_acc += ms;
    }
  }
  if (!K_on_device) {
    CUDA_TRY(c, cudaMemcpyAsync(K_out, Kd, (size_t)nstates * nx * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
  }
  ok(c);
  return HK_OK;
}

// -------------------------------------------------------------- kdist
static hk_status ensure_qr(hk_ctx *c, int nc, cudaStream_t s) {
  if (c->qr_nxb == c->nxb && c->qr_nc == nc) return HK_OK;
  CUDA_TRY(c, c->qrV.ensure((size_t)c->nxb * nc * sizeof(double)));
  CUDA_TRY(c, c->qrC.ensure(nc * sizeof(double)));
  CUDA_TRY(c, c->qrD.ensure(nc * sizeof(double)));
  CUDA_TRY(c, launch_qr(c->nxb, nc, c->qrV.as<double>(), c->qrC.as<double>(), c->qrD.as<double>(), s));
  c->qr_nxb = c->nxb;
  c->qr_nc = nc;
  return HK_OK;
}

hk_status hk_kdist(hk_ctx *c, int nstates, const double *K, int K_on_device, int nC,
                   double unitScale, double *coeff_out, int32_t *nxmin_out,
                   double *sortedK_out, double *recon_out, int outputs_on_device, void *stream) {
  if (!c) return HK_ERR_ARG;
  if (!c->grid_set) return fail(c, HK_ERR_STATE, "hk_set_grid must come first");
  if (nstates < 1 || !K) return fail(c, HK_ERR_ARG, "need nstates >= 1 and K");
  if (nstates > 65535) return fail(c, HK_ERR_RANGE, "at most 65535 states per call");
  const bool fit = coeff_out || nxmin_out || recon_out;
  if (fit) {
    if (nC < 1 || nC > 100) return fail(c, HK_ERR_RANGE, "nC must be 1..100 (def_NmaxSample)");
    if (c->nxb < 4 || nC > c->nxb) return fail(c, HK_ERR_RANGE, "need Nxb >= 4 and nC <= Nxb for the fit");
  }
  cudaSetDevice(c->device);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nx = c->g.nx;
  const size_t nK = (size_t)nstates * nx;
  const double *Kd = K;
  if (!K_on_device) {
    CUDA_TRY(c, c->Kwork.ensure(nK * sizeof(double)));
    CUDA_TRY(c, cudaMemcpyAsync(c->Kwork.p, K, nK * sizeof(double), cudaMemcpyHostToDevice, s));
    Kd = c->Kwork.as<double>();
  }
  hk_status st;
  if (fit && (st = ensure_qr(c, nC, s)) != HK_OK) return st;
  // device outputs: caller's or the workspace
  const size_t ncoef = (size_t)nstates * c->nbins * (fit ? nC : 0);
  const size_t nnx = (size_t)nstates * c->nbins;
  double *coef_d = nullptr, *sorted_d = nullptr, *recon_d = nullptr;
  int *nxmin_d = nullptr;
  if (outputs_on_device) {
    coef_d = coeff_out;
    nxmin_d = nxmin_out;
    sorted_d = sortedK_out;
    recon_d = recon_out;
  } else {
    size_t bytes = ncoef * 8 + nnx * 4 + 64 + (sortedK_out ? nK * 8 : 0) + (recon_out ? nK * 8 : 0);
    CUDA_TRY(c, c->outwork.ensure(bytes));
    char *base = (char *)c->outwork.p;
    size_t off = 0;
    if (fit) { coef_d = (double *)(base + off); off += ncoef * 8; }
    if (sortedK_out) { sorted_d = (double *)(base + off); off += nK * 8; }
    if (recon_out) { recon_d = (double *)(base + off); off += nK * 8; }
    if (fit) { nxmin_d = (int *)(base + off); off += nnx * 4; }
  }
  // the fit chain needs Nxmin even if the caller does not ask for it
  DevBuf nxtmp;
  if (fit && !nxmin_d) {
    CUDA_TRY(c, nxtmp.ensure(nnx * sizeof(int)));
    nxmin_d = nxtmp.as<int>();
  }
  double *scr = nullptr;
  const size_t nscr = kdist_scratch_doubles(c->nxb, c->nbins, nstates);
  if (nscr) {
    CUDA_TRY(c, c->scratch.ensure(nscr * sizeof(double)));
    scr = c->scratch.as<double>();
  }
  CUDA_TRY(c, cudaEventRecord(c->ev[2], s));
  c->launches += 1;
  CUDA_TRY(c, launch_kdist(Kd, nx, nstates, c->nxb, c->nbins, fit ? nC : 0, c->kmin, unitScale,
                           c->qrV.as<double>(), c->qrC.as<double>(), c->qrD.as<double>(),
                           fit ? coef_d : nullptr, nxmin_d, sorted_d, recon_d, scr, s));
  CUDA_TRY(c, cudaEventRecord(c->ev[3], s));
  c->have_kdist_t = true;
  if (!outputs_on_device) {
    if (coeff_out) CUDA_TRY(c, cudaMemcpyAsync(coeff_out, coef_d, ncoef * 8, cudaMemcpyDeviceToHost, s));
    if (nxmin_out) CUDA_TRY(c, cudaMemcpyAsync(nxmin_out, nxmin_d, nnx * 4, cudaMemcpyDeviceToHost, s));
    if (sortedK_out) CUDA_TRY(c, cudaMemcpyAsync(sortedK_out, sorted_d, nK * 8, cudaMemcpyDeviceToHost, s));
    if (recon_out) CUDA_TRY(c, cudaMemcpyAsync(recon_out, recon_d, nK * 8, cudaMemcpyDeviceToHost, s));
  }
  if (!outputs_on_device || nxtmp.p) CUDA_TRY(c, cudaStreamSynchronize(s));
  nxtmp.release();
  ok(c);
  return HK_OK;
}

// --------------------------------------------------------- diagnostics
hk_status hk_state_lines(hk_ctx *c, double T, double P, double *nu, double *S, double *iad,
                         double *vy, int64_t *win6) {
  if (!c) return HK_ERR_ARG;
  hk_status st;
  if ((st = check_ready(c)) != HK_OK) return st;
  cudaSetDevice(c->device);
  std::vector<StateDev> hs;
  if ((st = build_states(c, 1, &T, &P, hs)) != HK_OK) return st;
  const int64_t n = c->nlines;
  if (n == 0) return HK_OK;
  DevBuf o4, w6;
  CUDA_TRY(c, o4.ensure(n * 4 * sizeof(double)));
  CUDA_TRY(c, w6.ensure(n * 6 * sizeof(long long)));
  CUDA_TRY(c, launch_prep_dump(c->L, c->g, hs[0], o4.as<double>(), w6.as<long long>(), 0));
  CUDA_TRY(c, cudaDeviceSynchronize());
  std::vector<double> h4(n * 4);
  CUDA_TRY(c, cudaMemcpy(h4.data(), o4.p, n * 4 * sizeof(double), cudaMemcpyDeviceToHost));
  if (win6) CUDA_TRY(c, cudaMemcpy(win6, w6.p, n * 6 * sizeof(long long), cudaMemcpyDeviceToHost));
  for (int64_t l = 0; l < n; ++l) {
    if (nu) nu[l] = h4[4 * l + 0];
    if (S) S[l] = h4[4 * l + 1];
    if (iad) iad[l] = h4[4 * l + 2];
    if (vy) vy[l] = h4[4 * l + 3];
  }
  o4.release();
  w6.release();
  ok(c);
  return HK_OK;
}

hk_status hk_profile_eval(hk_ctx *c, int64_t n, const double *x, const double *y, int precision,
                          double *out) {
  if (!c || n < 0 || (n > 0 && (!x || !y || !out))) return HK_ERR_ARG;
  if (n == 0) return HK_OK;
  cudaSetDevice(c->device);
  DevBuf b;
  CUDA_TRY(c, b.ensure(n * 3 * sizeof(double)));
  double *xd = b.as<double>(), *yd = xd + n, *od = yd + n;
  CUDA_TRY(c, cudaMemcpy(xd, x, n * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(yd, y, n * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(c, launch_profile_eval(n, xd, yd, precision == HK_PRECISION_MIXED, od, 0));
  CUDA_TRY(c, cudaMemcpy(out, od, n * 8, cudaMemcpyDeviceToHost));
  b.release();
  ok(c);
  return HK_OK;
}

// --------------------------------------------------------------- adjoint
hk_status hk_set_workspace(hk_ctx *c, double prep_bytes, double part_bytes) {
  if (!c) return HK_ERR_ARG;
  if (!(prep_bytes >= 1.0) || !(part_bytes >= 1.0))
    return fail(c, HK_ERR_ARG, "workspace budgets must be >= 1 byte");
  c->prep_budget = (size_t)prep_bytes;
  c->part_budget = (size_t)part_bytes;
  table_release(c);
  ok(c);
  return HK_OK;
}

hk_status hk_set_profile(hk_ctx *c, int profile, int remove_plinth) {
  if (!c) return HK_ERR_ARG;
  if (profile < 1 || profile > 4)
    return fail(c, HK_ERR_ARG, "profile must be 1 (Voigt), 2 (Lorentz), 3 (Doppler) or 4 (binned Gaussian)");
  if (remove_plinth != 0 && remove_plinth != 1) return fail(c, HK_ERR_ARG, "remove_plinth must be 0 or 1");
  if (remove_plinth && profile == 4)  // heliosk.cu:410-413
    return fail(c, HK_ERR_UNSUPPORTED, "Error, remove plinth is not supported for profile 4");
  c->g.profile = profile;
  c->g.plinth = remove_plinth;
  c->tuned = false;
  table_release(c);
  ok(c);
  return HK_OK;
}

hk_status hk_set_sublorentzian(hk_ctx *c, const double *p) {
  if (!c) return HK_ERR_ARG;
  if (!p) {
    c->g.subL = 0;
  } else {
    for (int k = 0; k < 14; ++k)
      if (!std::isfinite(p[k])) return fail(c, HK_ERR_ARG, "sub-Lorentzian parameter %d is not finite", k);
    if (!(p[0] <= p[1] && p[1] <= p[2])) return fail(c, HK_ERR_ARG, "need sigma1 <= sigma2 <= sigma3");
    c->g.subL = 1;
    for (int k = 0; k < 3; ++k) c->g.sl_sigma[k] = p[k];
    for (int k = 0; k < 9; ++k) c->sl_abe[k] = p[3 + k];
    c->g.sl_lo = p[12];
    c->g.sl_hi = p[13];
  }
  c->tuned = false;
  table_release(c);
  ok(c);
  return HK_OK;
}

int hk_num_tile_shapes(void) { return voigt_num_shapes(); }

hk_status hk_tile_shape_info(int shape, int *lines_per_chunk, int *points_per_tile, int *warps) {
  if (shape < 0 || shape >= voigt_num_shapes()) return HK_ERR_ARG;
  if (lines_per_chunk) *lines_per_chunk = voigt_chunk_lines(shape);
  if (points_per_tile) *points_per_tile = voigt_tile_points(shape);
  if (warps) *warps = voigt_tile_warps(shape);
  return HK_OK;
}

hk_status hk_set_tuning(hk_ctx *c, int mode) {
  if (!c) return HK_ERR_ARG;
  if (mode < 0 || mode > 2) return fail(c, HK_ERR_ARG, "tuning mode must be 0, 1 or 2");
  c->tuning = mode;
  ok(c);
  return HK_OK;
}

hk_status hk_set_tile_shape(hk_ctx *c, int shape) {
  if (!c) return HK_ERR_ARG;
  if (shape < 0 || shape >= voigt_num_shapes())
    return fail(c, HK_ERR_ARG, "tile shape must be 0..%d", voigt_num_shapes() - 1);
  c->shape_fixed = shape;
  ok(c);
  return HK_OK;
}

hk_status hk_tuning_result(hk_ctx *c, int *last_shape, int *tuned_shape, double *probe_ms) {
  if (!c) return HK_ERR_ARG;
  if (last_shape) *last_shape = c->last_shape;
  if (tuned_shape) *tuned_shape = c->tuned ? c->tuned_shape : -1;
  if (probe_ms)
    for (int v = 0; v < voigt_num_shapes(); ++v)
      probe_ms[v] = (c->tuned && v < (int)c->tune_ms.size()) ? c->tune_ms[v] : -1.0;
  ok(c);
  return HK_OK;
}

hk_status hk_set_line_scales(hk_ctx *c, const double *s_scale, const double *g_scale) {
  if (!c) return HK_ERR_ARG;
  if (c->nlines == 0 && (s_scale || g_scale)) return fail(c, HK_ERR_STATE, "no lines loaded");
  cudaSetDevice(c->device);
  const int64_t n = c->nlines;
  // host arrays are in load order; the device keeps the nu-sorted order
  std::vector<int64_t> ord(n);
  if (n) CUDA_TRY(c, cudaMemcpy(ord.data(), c->order.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
  std::vector<double> tmp(n);
  const double *src[2] = {s_scale, g_scale};
  DevBuf *dst[2] = {&c->sscale, &c->gscale};
  const double **field[2] = {&c->L.sscale, &c->L.gscale};
  for (int q = 0; q < 2; ++q) {
    if (!src[q]) {
      dst[q]->release();
      *field[q] = nullptr;
      continue;
    }
    for (int64_t k = 0; k < n; ++k) {
      const double v = src[q][ord[k]];
      if (!(v > 0.0) || !std::isfinite(v)) return fail(c, HK_ERR_ARG, "line scale %lld must be finite and > 0", (long long)ord[k]);
      tmp[k] = v;
    }
    CUDA_TRY(c, dst[q]->ensure(n * sizeof(double)));
    CUDA_TRY(c, cudaMemcpy(dst[q]->p, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    *field[q] = dst[q]->as<double>();
  }
  ok(c);
  return HK_OK;
}

// true when p is device (or managed) memory of this context's GPU
static bool on_ctx_device(const hk_ctx *c, const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == c->device;
}

hk_status hk_set_line_scales_device(hk_ctx *c, const double *s_scale, const double *g_scale,
                                    void *stream) {
  if (!c) return HK_ERR_ARG;
  if (c->nlines == 0 && (s_scale || g_scale)) return fail(c, HK_ERR_STATE, "no lines loaded");
  cudaSetDevice(c->device);
  const double *src[2] = {s_scale, g_scale};
  for (int q = 0; q < 2; ++q)
    if (src[q] && !on_ctx_device(c, src[q]))
      return fail(c, HK_ERR_ARG, "%s is not device memory of GPU %d", q ? "g_scale" : "s_scale", c->device);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = c->nlines;
  DevBuf *dst[2] = {&c->sscale, &c->gscale};
  const double **field[2] = {&c->L.sscale, &c->L.gscale};
  for (int q = 0; q < 2; ++q) {
    if (!src[q]) {
      dst[q]->release();
      *field[q] = nullptr;
      continue;
    }
    // the values, then the word of the first invalid load index
    CUDA_TRY(c, dst[q]->ensure(n * sizeof(double) + sizeof(unsigned long long)));
    unsigned long long *bad = reinterpret_cast<unsigned long long *>(dst[q]->as<double>() + n);
    CUDA_TRY(c, launch_gather_scales(n, c->order.as<int64_t>(), src[q], dst[q]->as<double>(), bad, s));
    unsigned long long first_bad = 0;
    CUDA_TRY(c, cudaMemcpyAsync(&first_bad, bad, sizeof first_bad, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
    if (first_bad < (unsigned long long)n) {
      // the buffer now holds the invalid values: no multiplier stays in force
      for (int r = 0; r < 2; ++r) {
        dst[r]->release();
        *field[r] = nullptr;
      }
      return fail(c, HK_ERR_ARG, "line scale %lld must be finite and > 0", (long long)first_bad);
    }
    *field[q] = dst[q]->as<double>();
  }
  ok(c);
  return HK_OK;
}

static hk_status opacity_vjp(hk_ctx *c, double T, double P, int precision, const double *u,
                             int u_on_device, double *dT, double *dP, double *dlogS, double *dgammaL,
                             int log_gamma, int outputs_on_device, void *stream) {
  if (!c) return HK_ERR_ARG;
  hk_status st;
  if ((st = check_ready(c)) != HK_OK) return st;
  if (!u) return fail(c, HK_ERR_ARG, "need the seed u (Nx values)");
  if (precision != HK_PRECISION_PLAIN_FP64 && precision != HK_PRECISION_MIXED)
    return fail(c, HK_ERR_ARG, "precision must be 0 (plain FP64) or 1 (mixed)");
  if (c->g.plinth || c->g.subL)
    return fail(c, HK_ERR_UNSUPPORTED,
                "the adjoint is for the line profiles without plinth removal or sub-Lorentzian wings");
  cudaSetDevice(c->device);
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<StateDev> hs;
  if ((st = build_states(c, 1, &T, &P, hs)) != HK_OK) return st;
  const int64_t n = c->nlines, nx = c->g.nx;
  CUDA_TRY(c, c->states.ensure(sizeof(StateDev)));
  CUDA_TRY(c, c->wbits.ensure(2 * sizeof(unsigned long long)));
  CUDA_TRY(c, cudaMemcpyAsync(c->states.p, hs.data(), sizeof(StateDev), cudaMemcpyHostToDevice, s));
  if ((size_t)n * sizeof(LinePrep) > c->prep_budget)
    return fail(c, HK_ERR_RANGE, "the adjoint needs all %lld line records (%zu B) in the workspace (%zu B)",
                (long long)n, (size_t)n * sizeof(LinePrep), c->prep_budget);
  CUDA_TRY(c, c->prep.ensure((size_t)std::max<int64_t>(n, 1) * sizeof(LinePrep)));
  // the plain per-line records (FP64 windows and constants) of this state
  CUDA_TRY(c, launch_line_prep(false, c->L, c->g, c->states.as<StateDev>(), 1, c->prep.p,
                               c->wbits.as<unsigned long long>(), s));
  // the device copy of the state (wmax finalised) drives both passes
  CUDA_TRY(c, cudaMemcpyAsync(hs.data(), c->states.p, sizeof(StateDev), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  const double *ud = u;
  size_t need = 4 * (size_t)std::max<int64_t>(n, 1) + 2;
  if (!u_on_device) need += (size_t)nx;
  if (!outputs_on_device) need += 2 * (size_t)n;
  CUDA_TRY(c, c->adjwork.ensure(need * sizeof(double)));
  double *G = c->adjwork.as<double>();
  double *dTP = G + 4 * std::max<int64_t>(n, 1);
  double *next = dTP + 2;
  if (!u_on_device) {
    CUDA_TRY(c, cudaMemcpyAsync(next, u, nx * sizeof(double), cudaMemcpyHostToDevice, s));
    ud = next;
    next += nx;
  }
  double *dlS = dlogS, *dgm = dgammaL;
  if (!outputs_on_device) {
    dlS = dlogS ? next : nullptr;
    dgm = dgammaL ? next + n : nullptr;
  }
  CUDA_TRY(c, cudaEventRecord(c->ev[0], s));
  CUDA_TRY(c, launch_opacity_vjp(precision == HK_PRECISION_MIXED, c->L, c->g, c->states.as<StateDev>(),
                                 hs[0], c->prep.as<LinePrep>(), ud, c->ticket.as<unsigned>(), G,
                                 c->order.as<int64_t>(), dlS, dgm, log_gamma, dTP, s));
  CUDA_TRY(c, cudaEventRecord(c->ev[1], s));
  c->voigt_ms_acc = 0.0;
  c->voigt_ms_acc_only = false;
  c->have_voigt_t = true;
  double tp[2] = {0.0, 0.0};
  CUDA_TRY(c, cudaMemcpyAsync(tp, dTP, sizeof tp, cudaMemcpyDeviceToHost, s));
  if (!outputs_on_device) {
    if (dlogS) CUDA_TRY(c, cudaMemcpyAsync(dlogS, dlS, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dgammaL) CUDA_TRY(c, cudaMemcpyAsync(dgammaL, dgm, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(c, cudaStreamSynchronize(s));
  if (dT) *dT = tp[0];
  if (dP) *dP = tp[1];
  ok(c);
  return HK_OK;
}

hk_status hk_opacity_vjp(hk_ctx *c, double T, double P, int precision, const double *u,
                         int u_on_device, double *dT, double *dP, double *dlogS, double *dgammaL,
                         int outputs_on_device, void *stream) {
  return opacity_vjp(c, T, P, precision, u, u_on_device, dT, dP, dlogS, dgammaL, 0,
                     outputs_on_device, stream);
}

hk_status hk_opacity_vjp_log(hk_ctx *c, double T, double P, int precision, const double *u,
                             int u_on_device, double *dT, double *dP, double *dlogS,
                             double *dlogGammaL, int outputs_on_device, void *stream) {
  return opacity_vjp(c, T, P, precision, u, u_on_device, dT, dP, dlogS, dlogGammaL, 1,
                     outputs_on_device, stream);
}

// ---------------------------------------------------------------- tables
// Two ways to record a table, with the same bits: the per-batch launches
// (line prep, scale, Voigt sum per batch of states whose records fit the
// workspace; the default, the faster one measured on the 1e7-line, 600-state
// table: 28.6 ms per state against 30.1) and, with hk_set_table_mode(ctx, 1),
// one persistent launch for every state's line prep and sums (two kernels in
// the graph).  Tables of fewer states than this always take the per-batch
// launches: the fused launch can only hide a state's line prep behind
// another state's sums (one 1e7-line state: 31.1 ms per-batch, 32.8 fused).
constexpr int HK_TABLE_FUSED_MIN = 4;

hk_status hk_set_table_mode(hk_ctx *c, int fused) {
  if (!c) return HK_ERR_ARG;
  if (fused != 0 && fused != 1) return fail(c, HK_ERR_ARG, "table mode must be 0 (per batch) or 1 (fused)");
  c->table_fused = fused;
  ok(c);
  return HK_OK;
}

static hk_status table_build_batched(hk_ctx *c, int nstates, bool mixed, int shape, double *K, int nC,
                                     double unitScale, double *coeff, int32_t *nxmin) {
  const int64_t nx = c->g.nx;
  const size_t per_state = (size_t)std::max<int64_t>(c->nlines, 1) * line_prep_bytes(mixed);
  if (per_state > c->prep_budget)
    return fail(c, HK_ERR_UNSUPPORTED, "one state's line records (%zu B) exceed the workspace (%zu B): "
                "tables of such lists run through hk_opacity's sectioned path", per_state, c->prep_budget);
  int batch = (int)std::max<size_t>(1, c->prep_budget / per_state);
  const int nsplit = voigt_nsplit(nx, shape);
  if (nsplit > 1) {
    const int G = voigt_tile_points(shape);
    const size_t part_per_state = (size_t)((nx + G - 1) / G) * nsplit * G * sizeof(double);
    batch = std::min(batch, (int)std::max<size_t>(1, c->part_budget / part_per_state));
  }
  batch = std::min(batch, nstates);
  CUDA_TRY(c, c->prep.ensure((size_t)batch * per_state));
  const VoigtPlan plan0 = plan_voigt_sum(mixed, shape, nx, batch, 0);
  if (plan0.nsplit > 1) {
    CUDA_TRY(c, c->vpart.ensure(plan0.partial_doubles * sizeof(double)));
    CUDA_TRY(c, c->vcnt.ensure(plan0.counters * sizeof(unsigned)));
  }
  hk_status st;
  if ((st = ensure_qr(c, nC, 0)) != HK_OK) return st;
  const size_t nscr = kdist_scratch_doubles(c->nxb, c->nbins, nstates);
  if (nscr) CUDA_TRY(c, c->scratch.ensure(nscr * sizeof(double)));
  CUDA_TRY(c, c->tsync.ensure(table_sync_bytes(nstates)));
  CUDA_TRY(c, cudaMemset(c->tsync.p, 0, table_sync_bytes(nstates)));  // no waits: status stays OK
  CUDA_TRY(c, cudaDeviceSynchronize());
  cudaStream_t cs = nullptr;
  CUDA_TRY(c, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  StateDev *sd = c->states.as<StateDev>();
  unsigned long long *wb = c->wbits.as<unsigned long long>();
  int64_t kernels = 0;
  for (int b0 = 0; e == cudaSuccess && b0 < nstates; b0 += batch) {
    const int nb = std::min(batch, nstates - b0);
    const VoigtPlan plan = plan_voigt_sum(mixed, shape, nx, nb, plan0.ctas);
    e = launch_line_prep(mixed, c->L, c->g, sd + b0, nb, c->prep.p, wb + 2 * b0, cs);
    if (e == cudaSuccess)
      e = launch_voigt_sum(mixed, plan, c->prep.p, c->L.nu0, c->nlines, c->g, sd + b0,
                           c->ticket.as<unsigned>(), c->vpart.as<double>(), c->vcnt.as<unsigned>(),
                           K + (size_t)b0 * nx, nx, cs);
    kernels += 3;  // line prep, state scale, Voigt sum
  }
  if (e == cudaSuccess) {
    e = launch_kdist(K, nx, nstates, c->nxb, c->nbins, nC, c->kmin, unitScale, c->qrV.as<double>(),
                     c->qrC.as<double>(), c->qrD.as<double>(), coeff, nxmin, nullptr, nullptr,
                     nscr ? c->scratch.as<double>() : nullptr, cs);
    kernels += 1;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(c, HK_ERR_CUDA, "recording the table graph: %s",
                cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(c, HK_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  }
  c->table_graph = g;
  c->table_exec = x;
  c->table_kernels = kernels;
  c->table_states = nstates;
  ok(c);
  return HK_OK;
}

hk_status hk_table_build(hk_ctx *c, int nstates, const double *T, const double *P,
                         int precision, double *K, int nC, double unitScale, double *coeff,
                         int32_t *nxmin) {
  if (!c) return HK_ERR_ARG;
  hk_status st;
  if ((st = check_ready(c)) != HK_OK) return st;
  if (nstates < 1 || !T || !P || !K || !coeff || !nxmin)
    return fail(c, HK_ERR_ARG, "need nstates >= 1, T, P and device K, coeff, nxmin");
  if (precision != HK_PRECISION_PLAIN_FP64 && precision != HK_PRECISION_MIXED)
    return fail(c, HK_ERR_ARG, "precision must be 0 (plain FP64) or 1 (mixed)");
  if (nstates > 65535) return fail(c, HK_ERR_RANGE, "at most 65535 states per table");
  if (nC < 1 || nC > 100) return fail(c, HK_ERR_RANGE, "nC must be 1..100 (def_NmaxSample)");
  if (c->nxb < 4 || nC > c->nxb) return fail(c, HK_ERR_RANGE, "need Nxb >= 4 and nC <= Nxb for the fit");
  if (c->cia) return fail(c, HK_ERR_UNSUPPORTED, "CIA contexts have no line table: use hk_opacity");
  cudaSetDevice(c->device);
  table_release(c);
  // everything the graph touches is allocated and uploaded first: capture
  // records only asynchronous memsets and kernels
  std::vector<StateDev> hs;
  if ((st = build_states(c, nstates, T, P, hs)) != HK_OK) return st;
  CUDA_TRY(c, c->states.ensure(nstates * sizeof(StateDev)));
  CUDA_TRY(c, c->wbits.ensure(2 * nstates * sizeof(unsigned long long)));
  CUDA_TRY(c, cudaMemcpy(c->states.p, hs.data(), nstates * sizeof(StateDev), cudaMemcpyHostToDevice));
  const int64_t nx = c->g.nx;
  const bool mixed = mixed_form(c, precision);
  c->launches = 0;
  if (mixed && c->g.profile <= 2 && !c->g.plinth && !c->g.subL && c->tuning != 0 && !c->tuned && c->nlines > 0 &&
      (size_t)std::max<int64_t>(c->nlines, 1) * line_prep_bytes(true) <= c->prep_budget) {
    if ((st = tune_shape(c, nstates, hs, K, 0)) != HK_OK) return st;
    CUDA_TRY(c, cudaDeviceSynchronize());
  }
  const int shape = shape_for(c, mixed);
  c->last_shape = shape;
  if (!c->table_fused || nstates < HK_TABLE_FUSED_MIN)
    return table_build_batched(c, nstates, mixed, shape, K, nC, unitScale, coeff, nxmin);
  // one persistent launch for the whole table: line prep into a ring of
  // per-state record slots and every state's Voigt sums (hkb_voigt.cu)
  const TablePlan tp = plan_table(mixed, shape, c->nlines, nx, nstates);
  if (tp.ring_bytes > c->prep_budget)
    return fail(c, HK_ERR_UNSUPPORTED, "%d states' line records (%zu B) exceed the workspace (%zu B): "
                "tables of such lists run through hk_opacity's sectioned path", tp.slots, tp.ring_bytes,
                c->prep_budget);
  CUDA_TRY(c, c->prep.ensure(tp.ring_bytes));
  if (tp.partial_doubles) CUDA_TRY(c, c->vpart.ensure(tp.partial_doubles * sizeof(double)));
  CUDA_TRY(c, c->vcnt.ensure(std::max<size_t>(tp.counters, 1) * sizeof(unsigned)));
  CUDA_TRY(c, c->tsync.ensure(table_sync_bytes(nstates)));
  if ((st = ensure_qr(c, nC, 0)) != HK_OK) return st;
  const size_t nscr = kdist_scratch_doubles(c->nxb, c->nbins, nstates);
  if (nscr) CUDA_TRY(c, c->scratch.ensure(nscr * sizeof(double)));
  CUDA_TRY(c, cudaDeviceSynchronize());

  TableBufs tb;
  tb.ring = c->prep.p;
  tb.partial = tp.partial_doubles ? c->vpart.as<double>() : nullptr;
  tb.tile_cnt = c->vcnt.as<unsigned>();
  tb.sync = c->tsync.p;
  cudaStream_t cs = nullptr;
  CUDA_TRY(c, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess)
    e = launch_voigt_table(mixed, tp, c->L, c->g, c->states.as<StateDev>(), tb, K, nx, cs);
  if (e == cudaSuccess)
    e = launch_kdist(K, nx, nstates, c->nxb, c->nbins, nC, c->kmin, unitScale, c->qrV.as<double>(),
                     c->qrC.as<double>(), c->qrD.as<double>(), coeff, nxmin, nullptr, nullptr,
                     nscr ? c->scratch.as<double>() : nullptr, cs);
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(c, HK_ERR_CUDA, "recording the table graph: %s",
                cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(c, HK_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  }
  c->table_graph = g;
  c->table_exec = x;
  c->table_kernels = 2;  // the table kernel and the k-distribution kernel
  c->table_states = nstates;
  ok(c);
  return HK_OK;
}

hk_status hk_table_status(hk_ctx *c, void *stream) {
  if (!c) return HK_ERR_ARG;
  if (!c->table_exec) return fail(c, HK_ERR_STATE, "hk_table_build must come first");
  cudaSetDevice(c->device);
  CUDA_TRY(c, cudaStreamSynchronize((cudaStream_t)stream));
  int err = 0;
  CUDA_TRY(c, cudaMemcpy(&err, table_error_word(c->tsync.p, c->table_states), sizeof(int),
                         cudaMemcpyDeviceToHost));
  if (err != 0)
    return fail(c, HK_ERR_TIMEOUT, "a wait inside the table kernel ran out: the last run's results "
                "are incomplete");
  ok(c);
  return HK_OK;
}

hk_status hk_table_run(hk_ctx *c, void *stream) {
  if (!c) return HK_ERR_ARG;
  if (!c->table_exec) return fail(c, HK_ERR_STATE, "hk_table_build must come first");
  cudaSetDevice(c->device);
  CUDA_TRY(c, cudaGraphLaunch(c->table_exec, (cudaStream_t)stream));
  ok(c);
  return HK_OK;
}

hk_status hk_table_free(hk_ctx *c) {
  if (!c) return HK_ERR_ARG;
  cudaSetDevice(c->device);
  table_release(c);
  return HK_OK;
}

int64_t hk_table_kernels(const hk_ctx *c) { return c ? c->table_kernels : 0; }

int64_t hk_last_launches(const hk_ctx *c) { return c ? c->launches : 0; }

// ------------------------------------------- mean opacities, transmission
hk_status hk_means(hk_ctx *c, int nstates, const double *T, const double *K, int K_on_device,
                   double *sums, int sums_on_device, void *stream) {
  if (!c) return HK_ERR_ARG;
  if (!c->grid_set) return fail(c, HK_ERR_STATE, "hk_set_grid must come first");
  if (nstates < 1 || !T || !K || !sums) return fail(c, HK_ERR_ARG, "need nstates >= 1, T, K and sums");
  if (nstates > 65535) return fail(c, HK_ERR_RANGE, "at most 65535 states per call");
  for (int s = 0; s < nstates; ++s)
    if (!(T[s] > 0.0) || !std::isfinite(T[s])) return fail(c, HK_ERR_RANGE, "state %d: T must be finite and > 0", s);
  cudaSetDevice(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nx = c->g.nx;
  const size_t nK = (size_t)nstates * nx;
  const double *Kd = K;
  if (!K_on_device) {
    CUDA_TRY(c, c->Kwork.ensure(nK * sizeof(double)));
    CUDA_TRY(c, cudaMemcpyAsync(c->Kwork.p, K, nK * sizeof(double), cudaMemcpyHostToDevice, st));
    Kd = c->Kwork.as<double>();
  }
  const size_t nscr = means_scratch_doubles(nstates, nx);
  CUDA_TRY(c, c->meanwork.ensure((nscr + 5 * (size_t)nstates) * sizeof(double)));
  double *Td = c->meanwork.as<double>(), *outd = Td + nstates, *scr = outd + 4 * (size_t)nstates;
  CUDA_TRY(c, cudaMemcpyAsync(Td, T, nstates * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(c, launch_means(Kd, nx, c->g, Td, nstates, scr, sums_on_device ? sums : outd, st));
  if (!sums_on_device) {
    CUDA_TRY(c, cudaMemcpyAsync(sums, outd, 4 * (size_t)nstates * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
  } else if (!K_on_device) {
    CUDA_TRY(c, cudaStreamSynchronize(st));  // T's pageable copy
  }
  ok(c);
  return HK_OK;
}

hk_status hk_transmission(hk_ctx *c, int nstates, const double *K, const int32_t *nxmin,
                          int inputs_on_device, int nTr, double dTr, double *Tr,
                          int Tr_on_device, void *stream) {
  if (!c) return HK_ERR_ARG;
  if (!c->grid_set) return fail(c, HK_ERR_STATE, "hk_set_grid must come first");
  if (nstates < 1 || !K || !Tr) return fail(c, HK_ERR_ARG, "need nstates >= 1, K and Tr");
  if (nstates > 65535) return fail(c, HK_ERR_RANGE, "at most 65535 states per call");
  if (nTr < 1) return fail(c, HK_ERR_RANGE, "nTr must be >= 1");
  if (!std::isfinite(dTr)) return fail(c, HK_ERR_RANGE, "dTr must be finite");
  if (c->nxb < 3) return fail(c, HK_ERR_RANGE, "the transmission function needs >= 3 points per bin");
  cudaSetDevice(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nx = c->g.nx;
  const size_t nK = (size_t)nstates * nx, nN = (size_t)nstates * c->nbins;
  const size_t nT = nN * (size_t)nTr;
  const double *Kd = K;
  const int *nmd = reinterpret_cast<const int *>(nxmin);
  double *Trd = Tr;
  size_t need = (inputs_on_device ? 0 : nK) + (Tr_on_device ? 0 : nT) +
                ((!inputs_on_device && nxmin) ? (nN + 1) / 2 : 0);
  CUDA_TRY(c, c->meanwork.ensure(std::max<size_t>(need, 1) * sizeof(double)));
  double *w = c->meanwork.as<double>();
  if (!inputs_on_device) {
    CUDA_TRY(c, cudaMemcpyAsync(w, K, nK * sizeof(double), cudaMemcpyHostToDevice, st));
    Kd = w;
    w += nK;
    if (nxmin) {
      CUDA_TRY(c, cudaMemcpyAsync(w, nxmin, nN * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      nmd = reinterpret_cast<const int *>(w);
      w += (nN + 1) / 2;
    }
  }
  if (!Tr_on_device) Trd = w;
  CUDA_TRY(c, launch_transmission(Kd, nx, nstates, c->nxb, c->nbins, nmd, c->kmin, nTr, dTr, Trd, st));
  if (!Tr_on_device) {
    CUDA_TRY(c, cudaMemcpyAsync(Tr, Trd, nT * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
  } else if (!inputs_on_device) {
    CUDA_TRY(c, cudaStreamSynchronize(st));
  }
  ok(c);
  return HK_OK;
}

hk_status hk_count_pairs(hk_ctx *c, double T, double P, int64_t *pairs3) {
  if (!c || !pairs3) return HK_ERR_ARG;
  hk_status st;
  if ((st = check_ready(c)) != HK_OK) return st;
  cudaSetDevice(c->device);
  std::vector<StateDev> hs;
  if ((st = build_states(c, 1, &T, &P, hs)) != HK_OK) return st;
  CUDA_TRY(c, c->states.ensure(sizeof(StateDev)));
  CUDA_TRY(c, c->adjwork.ensure(4 * sizeof(double)));
  CUDA_TRY(c, cudaMemcpy(c->states.p, hs.data(), sizeof(StateDev), cudaMemcpyHostToDevice));
  unsigned long long *d = reinterpret_cast<unsigned long long *>(c->adjwork.p);
  CUDA_TRY(c, launch_count_pairs(c->L, c->g, c->states.as<StateDev>(), d, 0));
  unsigned long long h[3];
  CUDA_TRY(c, cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost));
  for (int k = 0; k < 3; ++k) pairs3[k] = (int64_t)h[k];
  ok(c);
  return HK_OK;
}

hk_status hk_last_timing(const hk_ctx *c, double *voigt_ms, double *kdist_ms) {
  if (!c) return HK_ERR_ARG;
  float ms = 0.f;
  if (voigt_ms) {
    *voigt_ms = -1.0;
    if (c->voigt_ms_acc_only)
      *voigt_ms = c->voigt_ms_acc;
    else if (c->have_voigt_t && cudaEventSynchronize(c->ev[1]) == cudaSuccess &&
             cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]) == cudaSuccess)
      *voigt_ms = c->voigt_ms_acc + ms;
  }
  if (kdist_ms) {
    *kdist_ms = -1.0;
    if (c->have_kdist_t && cudaEventSynchronize(c->ev[3]) == cudaSuccess &&
        cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]) == cudaSuccess)
      *kdist_ms = ms;
  }
  return HK_OK;
}

hk_status hk_fp32_peak(hk_ctx *c, double *tflops) {
  if (!c || !tflops) return HK_ERR_ARG;
  cudaSetDevice(c->device);
  CUDA_TRY(c, measure_fp32_peak(tflops, 0));
  ok(c);
  return HK_OK;
}

// ---------------------------------------------------------- file loader
// The selected binary line files stream to the GPU in chunks of whole
// records: fread fills one of two pinned buffers while the other's copy and
// unpack run (heliosk.cu:1405-1423 overlaps reads and copies the same way for
// ExoMol, 8192 lines at a time), and the records become columns on the device
// (hkb_ingest.cu).  Nothing of a line list passes through pageable host
// memory beyond the kernel's file cache.
static constexpr int64_t kIngestChunk = 1 << 20;  // records per chunk

// One species' selected files into ib's columns from line base0 on; the
// species' isotopologues are spec.iso_base + (0 .. niso-1).
static hk_status stream_species(hk_ctx *c, const SpeciesInfo &sp, int fi0, int fi1,
                                const IngestSpec &spec, IngestBuf &ib, int64_t base0) {
  const bool hitran = sp.database == HK_DB_HITRAN;
  const size_t rec = hitran ? 68 : 32;
  struct Pipe {
    unsigned char *host[2] = {nullptr, nullptr};
    DevBuf dev[2], bad;
    cudaStream_t st = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    FILE *f = nullptr;
    ~Pipe() {
      if (st) cudaStreamSynchronize(st);
      for (int b = 0; b < 2; ++b) {
        if (host[b]) cudaFreeHost(host[b]);
        if (done[b]) cudaEventDestroy(done[b]);
      }
      if (st) cudaStreamDestroy(st);
      if (f) fclose(f);
    }
  } pp;
  const size_t chunk_bytes = (size_t)kIngestChunk * rec;
  CUDA_TRY(c, cudaStreamCreateWithFlags(&pp.st, cudaStreamNonBlocking));
  for (int b = 0; b < 2; ++b) {
    CUDA_TRY(c, cudaHostAlloc((void **)&pp.host[b], chunk_bytes, cudaHostAllocDefault));
    CUDA_TRY(c, pp.dev[b].ensure(chunk_bytes));
    CUDA_TRY(c, cudaEventCreateWithFlags(&pp.done[b], cudaEventDisableTiming));
  }
  CUDA_TRY(c, pp.bad.ensure(sizeof(unsigned long long)));
  const unsigned long long none = ~0ull;
  CUDA_TRY(c, cudaMemcpy(pp.bad.p, &none, sizeof none, cudaMemcpyHostToDevice));
  int64_t base = base0;
  int b = 0;
  bool used[2] = {false, false};
  for (int fi = fi0; fi < fi1; ++fi) {
    const std::string fname = sp.dataFilename[fi] + "bin";
    pp.f = fopen(fname.c_str(), "rb");
    if (!pp.f) return fail(c, HK_ERR_IO, "Error: line list file not found: %s", fname.c_str());
    const int64_t nl = sp.NL[fi];
    for (int64_t r0 = 0; r0 < nl; r0 += kIngestChunk) {
      const int64_t cnt = std::min<int64_t>(kIngestChunk, nl - r0);
      if (used[b]) CUDA_TRY(c, cudaEventSynchronize(pp.done[b]));  // buffer b is free again
      const size_t got = fread(pp.host[b], rec, (size_t)cnt, pp.f);
      if ((int64_t)got != cnt)
        return fail(c, HK_ERR_FORMAT, "Error: line list file %s is truncated (%lld of %lld records)",
                    fname.c_str(), (long long)(r0 + (int64_t)got), (long long)nl);
      CUDA_TRY(c, cudaMemcpyAsync(pp.dev[b].p, pp.host[b], (size_t)cnt * rec,
                                  cudaMemcpyHostToDevice, pp.st));
      LineCols at = ib.lc;
      for (double **q : {&at.nu, &at.S, &at.EL, &at.gam, &at.nexp, &at.delta, &at.Aterm}) *q += base + r0;
      at.iso += base + r0;
      CUDA_TRY(c, launch_unpack_records(pp.dev[b].as<unsigned char>(), cnt, base + r0, spec, at,
                                        pp.bad.as<unsigned long long>(), pp.st));
      CUDA_TRY(c, cudaEventRecord(pp.done[b], pp.st));
      used[b] = true;
      b ^= 1;
    }
    fclose(pp.f);
    pp.f = nullptr;
    base += nl;
  }
  CUDA_TRY(c, cudaStreamSynchronize(pp.st));
  unsigned long long bad = none;
  CUDA_TRY(c, cudaMemcpy(&bad, pp.bad.p, sizeof bad, cudaMemcpyDeviceToHost));
  if (bad != none) {
    // host.h:624-639: a record whose isotopologue id is not in the species table
    int64_t i = (int64_t)bad - base0;
    int fi = fi0;
    while (fi + 1 < fi1 && i >= sp.NL[fi]) i -= sp.NL[fi++];
    char cid[4] = {0, 0, 0, 0};
    FILE *f = fopen((sp.dataFilename[fi] + "bin").c_str(), "rb");
    if (f) {
      if (fseek(f, (long)(i * (int64_t)rec), SEEK_SET) == 0 && fread(cid, 1, 4, f) != 4) cid[0] = 0;
      fclose(f);
    }
    return fail(c, HK_ERR_FORMAT, "Error: partition function not found. %lld |%.3s|%s|", (long long)i,
                cid, sp.iso[0].cid.c_str());
  }
  return HK_OK;
}

static IngestSpec species_spec(const hk_ctx *c, const SpeciesInfo &sp, int iso_base) {
  IngestSpec spec = ingest_spec(c, sp.database == HK_DB_HITRAN);
  spec.defaultL = sp.defaultL;
  spec.defaultn = sp.defaultn;
  spec.iso_base = iso_base;
  for (size_t k = 0; k < sp.iso.size() && k < (size_t)HK_MAX_ISO; ++k)
    strncpy(spec.cid[k], sp.iso[k].cid.c_str(), 4);  // zero-padded, as strncmp(.., 4) reads it
  return spec;
}

static hk_status stream_line_files(hk_ctx *c, const SpeciesInfo &sp, int fi0, int fi1) {
  int64_t n = 0;
  for (int fi = fi0; fi < fi1; ++fi) n += sp.NL[fi];
  cudaSetDevice(c->device);
  IngestBuf ib;
  CUDA_TRY(c, ib.alloc(n));
  hk_status st = stream_species(c, sp, fi0, fi1, species_spec(c, sp, 0), ib, 0);
  if (st != HK_OK) return st;
  return load_device(c, n, ib, (int)sp.iso.size());
}

hk_status hk_load_cia(hk_ctx *c, const char *path, const char *system, double *mass1) {
  if (!c || !system) return HK_ERR_ARG;
  std::string file;
  int nsets = 0;
  double m1 = 1.0;
  if (!cia_system(system, file, &nsets, &m1))
    return fail(c, HK_ERR_ARG, "unknown cia system %s", system);
  std::vector<CiaSet> sets;
  std::string msg;
  const int rc = read_cia_file(std::string(path ? path : "") + file, nsets, sets, msg);
  if (rc != 0) return fail(c, rc, "%s", msg.c_str());
  std::vector<double> nu, val;
  for (const CiaSet &cs : sets) {
    nu.insert(nu.end(), cs.nu.begin(), cs.nu.end());
    val.insert(val.end(), cs.cia.begin(), cs.cia.end());
  }
  cudaSetDevice(c->device);
  CUDA_TRY(c, c->cia_nu.ensure(nu.size() * sizeof(double)));
  CUDA_TRY(c, c->cia_val.ensure(val.size() * sizeof(double)));
  CUDA_TRY(c, cudaMemcpy(c->cia_nu.p, nu.data(), nu.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(c->cia_val.p, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice));
  // a CIA system has no lines (heliosk.cu:842-845)
  c->nlines = 0;
  c->L = LinesDev{};
  c->iso_mass.clear();
  c->cia_sets = std::move(sets);
  c->cia_mass1 = m1;
  c->cia = true;
  table_release(c);
  if (mass1) *mass1 = m1;
  ok(c);
  return HK_OK;
}

hk_status hk_load_species_file(hk_ctx *c, const char *path, const char *species, double numin,
                               double numax, int cutMode, double cut) {
  if (!c || !species) return HK_ERR_ARG;
  SpeciesInfo sp;
  std::string msg;
  int rc = read_species_param(path ? path : "", species, sp, msg);
  if (rc != 0) return fail(c, rc, "%s", msg.c_str());
  std::vector<double> mass, ab;
  for (auto &iso : sp.iso) {
    mass.push_back(iso.mass);
    ab.push_back(iso.ab);
  }
  hk_status st = hk_set_species(c, sp.database, (int)mass.size(), mass.data(), ab.data(),
                                sp.defaultL, sp.defaultn);
  if (st != HK_OK) return st;
  for (size_t j = 0; j < sp.iso.size(); ++j) {
    std::vector<double> T, Q;
    rc = read_q_file(sp.iso[j].qfile, sp.npfcol, T, Q, msg);
    if (rc != 0) return fail(c, rc, "%s", msg.c_str());
    if ((st = hk_set_partition(c, (int)j, (int)T.size(), T.data(), Q.data())) != HK_OK) return st;
  }
  int fi0, fi1;
  line_file_range(sp, numin, numax, cutMode, cut, &fi0, &fi1);
  return stream_line_files(c, sp, fi0, fi1);
}

// Species mixtures (param.dat SpeciesFile, heliosk.cu:660-700 and 784-800):
// the reference runs its whole line pipeline once per species, scaling that
// species' strengths by its abundance, and sums into one K; the mean molar
// mass (units 0 scaling) is the mixture's.  Here every species' lines go
// into one line list -- isotopologue indices offset per species, the
// abundance as the isotopologues' strength scale -- and one opacity call
// sums them all.
hk_status hk_load_mixture(hk_ctx *c, const char *path, int nspecies, const char *const *species,
                          const double *abundance, double numin, double numax, int cutMode,
                          double cut) {
  if (!c) return HK_ERR_ARG;
  if (nspecies < 1 || !species || (nspecies > 1 && !abundance))
    return fail(c, HK_ERR_ARG, "need nspecies >= 1, species names and (for several) abundances");
  std::vector<SpeciesInfo> sps(nspecies);
  std::string msg;
  int niso = 0;
  for (int s = 0; s < nspecies; ++s) {
    if (!species[s]) return fail(c, HK_ERR_ARG, "species %d: null name", s);
    if (nspecies > 1 && !(abundance[s] >= 0.0 && std::isfinite(abundance[s])))
      return fail(c, HK_ERR_ARG, "species %d: abundance must be finite and >= 0", s);
    int rc = read_species_param(path ? path : "", species[s], sps[s], msg);
    if (rc != 0) return fail(c, rc, "%s", msg.c_str());
    if (sps[s].database != sps[0].database)
      return fail(c, HK_ERR_UNSUPPORTED, "species %s: mixtures of HITRAN- and ExoMol-format species are not supported",
                  species[s]);
    niso += (int)sps[s].iso.size();
  }
  if (niso > HK_MAX_ISO) return fail(c, HK_ERR_RANGE, "the mixture has %d isotopologues, at most %d", niso, HK_MAX_ISO);
  std::vector<double> mass, ab, ss;
  for (int s = 0; s < nspecies; ++s)
    for (auto &iso : sps[s].iso) {
      mass.push_back(iso.mass);
      ab.push_back(iso.ab);
      ss.push_back(nspecies > 1 ? abundance[s] : 1.0);  // heliosk.cu:786-789
    }
  hk_status st = hk_set_species(c, sps[0].database, niso, mass.data(), ab.data(), sps[0].defaultL,
                                sps[0].defaultn);
  if (st != HK_OK) return st;
  int j = 0;
  for (int s = 0; s < nspecies; ++s)
    for (auto &iso : sps[s].iso) {
      std::vector<double> T, Q;
      int rc = read_q_file(iso.qfile, sps[s].npfcol, T, Q, msg);
      if (rc != 0) return fail(c, rc, "%s", msg.c_str());
      if ((st = hk_set_partition(c, j++, (int)T.size(), T.data(), Q.data())) != HK_OK) return st;
    }
  c->iso_ss = ss;
  std::vector<int> f0(nspecies), f1(nspecies);
  int64_t n = 0;
  for (int s = 0; s < nspecies; ++s) {
    line_file_range(sps[s], numin, numax, cutMode, cut, &f0[s], &f1[s]);
    for (int fi = f0[s]; fi < f1[s]; ++fi) n += sps[s].NL[fi];
  }
  cudaSetDevice(c->device);
  IngestBuf ib;
  CUDA_TRY(c, ib.alloc(n));
  int64_t base = 0;
  int iso_base = 0;
  for (int s = 0; s < nspecies; ++s) {
    if ((st = stream_species(c, sps[s], f0[s], f1[s], species_spec(c, sps[s], iso_base), ib, base)) != HK_OK)
      return st;
    for (int fi = f0[s]; fi < f1[s]; ++fi) base += sps[s].NL[fi];
    iso_base += (int)sps[s].iso.size();
  }
  return load_device(c, n, ib, niso);
}

}  // extern "C"
