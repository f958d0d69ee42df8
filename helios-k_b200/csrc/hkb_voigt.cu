// hkb_voigt.cu -- the Voigt line sum onto the wavenumber grid (sm_100a).
//
// One persistent kernel walks (state, grid tile) tickets.  A CTA owns a tile
// of G consecutive grid points, so every output point has exactly one
// writer: there are no atomics on K and no partial-row reduction (the
// reference's 32 KS_d rows + AddKStreams_kernel, voigt.h:728-742, are gone).
// For its tile the CTA
//   1. finds the nu-sorted line range whose cutoff windows can reach the tile
//      (warp-parallel lower_bound),
//   2. stages the lines in chunks of CH through shared memory: each thread
//      loads one line's state record (FP64 parameters and global index
//      windows, written by line_prep_kernel), clips the windows to the tile
//      and forms the line-centre offset at the tile start,
//   3. lets each warp sweep its slice (32 lanes x PPL points) against every staged line:
//      lane-interleaved points (coalesced stores), register accumulators.
// Two precisions share the structure:
//   MIXED: FP32 profile (the offset x from a double-float split of the FP64
//          line-centre offset; region formulas in FP32), strength multiply
//          and grid sum as one FP64 FMA per pair.
//   PLAIN: FP64 everywhere (the "plain FP64 form" used as the GPU baseline).
// Reference: Line6fA/B/C kernels voigt.h:1177-1816 and their launchers
// Line6A_Call/Line6B_Call/Line6C_Call voigt.h:1820-2036.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "hkb_device.cuh"
#include "hkb_kernels.h"
#include "hkb_prep.cuh"

namespace hkb {

// Tile shapes: CH lines per staged chunk x G = WARPS warps * 32 lanes * PPL
// grid points per tile.  The autotuner (hk_set_tuning) picks one per
// workload; shape 0 is the default.  MINB is the CTAs per SM the register
// budget is set for (8 warps: 64 registers at 4, 80 at 3, where shared
// memory allows 3 only; 4 warps of 16 points per lane: 102 registers at 5,
// 64 at 8).  Four warps of 16 points keep the 2048-point tile and spread a
// staged line's per-warp costs (coefficient loads, class ballots) over twice
// the points.
template <int CH_, int PPL_, int MINB_, int WARPS_ = 8>
struct TileShape {
  static constexpr int CH = CH_, PPL = PPL_, MINB = MINB_, WARPS = WARPS_;
  static constexpr int THREADS = 32 * WARPS_;
  static constexpr int SLICE = 32 * PPL_;        // points per warp
  static constexpr int G = WARPS_ * SLICE;       // points per tile
  static_assert(G <= 2048, "a staged line's far-block mask holds 32 blocks of 64 points");
  static_assert(CH % 32 == 0 && CH <= THREADS, "one staging thread per line");
  static_assert(PPL % 2 == 0, "points are processed in pairs");
};
using Shape0 = TileShape<128, 8, 4>;  // default
using Shape1 = TileShape<256, 8, 3>;
using Shape2 = TileShape<64, 8, 4>;
using Shape3 = TileShape<128, 4, 4>;
using Shape4 = TileShape<256, 4, 4>;
using Shape5 = TileShape<128, 16, 5, 4>;
using Shape6 = TileShape<64, 16, 8, 4>;
constexpr int HK_NSHAPES = 7;
constexpr int HK_SHAPE_CH[HK_NSHAPES] = {Shape0::CH, Shape1::CH, Shape2::CH, Shape3::CH,
                                         Shape4::CH, Shape5::CH, Shape6::CH};
constexpr int HK_SHAPE_G[HK_NSHAPES] = {Shape0::G, Shape1::G, Shape2::G, Shape3::G,
                                        Shape4::G, Shape5::G, Shape6::G};
constexpr int HK_SHAPE_WARPS[HK_NSHAPES] = {Shape0::WARPS, Shape1::WARPS, Shape2::WARPS, Shape3::WARPS,
                                            Shape4::WARPS, Shape5::WARPS, Shape6::WARPS};

// Staged line record of the mixed form.  Regions A and B are summed in FP32
// (flushed into the FP64 per-point sums at least once per chunk of lines)
// with the line strength folded into the coefficients:
//   A:  S1f / (s + Y),
//   B:  S1f t4 = (s (S1f s + C1) + C0) / (((s + D2) s + D1) s + D0),
// s = x^2, Y = y^2, S1f = S1 * 2^(s1exp + 96 lev) (below), C1 = S1f A1,
// C0 = S1f B1, and the GH2 denominator (s + Y)(s (s + A2) + B2) expanded:
// D2 = A2 + Y, D1 = B2 + A2 Y, D0 = B2 Y, with A1 = 2Y + 2.5 - 4/pi,
// B1 = (Y+1.5)(Y+1), A2 = 2Y + 3 - 6/pi, B2 = (Y+1.5)^2.  Every coefficient
// is positive, so neither form cancels.
// x at tile point k, every region: x = (k - kc) vb + fr, kc the point
// nearest the line centre (|fr| <= vb/2): the subtraction is exact, so x
// carries ~2 roundings relative to itself (|k - kc| vb <= |x| + vb/2 and
// |x| >= vb/2 off kc) whatever vb, also where x crosses zero.
struct __align__(16) RecF {
  float S1f, C1, C0, D2;
  float D1, D0, nkc, vb;   // nkc = -kc
  float fr, y, ey, sig1;   // y, erfcx(y), region-C series constant
  double Sc;               // S/sqrt(pi) (region C, FP64 sum)
  int i0, b0, c0, c1;      // tile-local window boundaries
  int b1, i1, flags;
  unsigned fmask;          // far-field blocks of the tile (bit b: block b)
  int t0, t1;              // region C: the Algorithm-916 part (tile-local)
};
static_assert(sizeof(RecF) == 96, "RecF layout");

// Profiles 3 (Doppler) and 4 (binned Gaussian) have no regions B and C, so
// their records reuse the GH2 slots: the FP64 offset D0 at the tile start
// and the FP64 grid step vb (Doppler units) in C0..D2 and D1..D0, and, for
// the binned Gaussian, the half step vb / 2 in C1.
__device__ __forceinline__ void gauss_put(RecF &r, double D0, double vb, float h) {
  double *d = reinterpret_cast<double *>(&r.C0);
  d[0] = D0;
  d[1] = vb;
  r.C1 = h;
}
__device__ __forceinline__ double gauss_D0(const RecF &r) { return reinterpret_cast<const double *>(&r.C0)[0]; }
__device__ __forceinline__ double gauss_vb(const RecF &r) { return reinterpret_cast<const double *>(&r.C0)[1]; }

// Strength levels: with 2^(40 - s1exp) the state's largest region-A/B term
// S1 / max(100, Y), a line of level lev = (40 - ex - s1exp) / 96 (ex: the
// exponent of its own largest term) gets S1f = S1 * 2^(s1exp + 96 lev), which
// puts its largest term in (2^-56, 2^40] whatever its strength.  A warp sums
// the lines of one level at a time in FP32 and flushes (exactly unscaled)
// into the FP64 sums when the level changes, so FP32 never holds terms of
// lines more than 2^96 apart, and a line's smallest term (at most 2^64 below
// its largest, else HK_PF_RANGE) stays a normal float.  With those bounds
// S1f s^2 < 2^100 and d0 d1 < 2^120 in region B.
// flags: HK_F_WEAK -- level above HK_MAX_LEVEL (2^768 below the strongest
// line) or HK_PF_RANGE: the line is summed in FP64 with S1f = 1;
// HK_F_WIDE -- some x^2 + Y in the window reaches 1e18, so two region-A
// denominators may not be multiplied in FP32 (paired reciprocals are off);
// with plinth removal, HK_F_PLA / HK_F_PLB -- the cut edge x_c lies in
// region A / B, whose points take the factored difference t(x) - t(x_c);
// HK_F_PL64 -- the line is summed per point in FP64 (HK_PF_PL64).
// The level sits in flags bits 8-11.
constexpr int HK_F_WEAK = 1, HK_F_WIDE = 2, HK_F_PLA = 4, HK_F_PLB = 8, HK_F_PL64 = 16;
constexpr int HK_LEVEL_BITS = 96;
constexpr int HK_MAX_LEVEL = 7;

// Options of the mixed form with their own kernel instantiations: none,
// sub-Lorentzian wings (chi factor), plinth removal.
enum { HK_EXT_NONE = 0, HK_EXT_CHI = 1, HK_EXT_PL = 2 };

// Per staged line with plinth removal (shared memory, beside its RecF):
// x = D0 + k vb in FP64 (k the tile-local point), and
//   factored lines: xd = x_c; plf the plinth in the line's FP32 units (the
//     plain difference, where the term is at least 4 plinths); xcf = x_c;
//     ic = 1 / (x_c^2 + Y) (edge in region A) or 1 / D(x_c^2) (region B);
//     q0..q2 the GH2 difference polynomial (region B);
//   FP64 lines: xd = the plinth, vy and ey = erfcx(vy) in FP64.
struct __align__(16) ExtPL {
  double D0, vb, xd, vy, ey;
  float plf, xcf, ic, q0, q1, q2;
};
static_assert(sizeof(ExtPL) == 64, "ExtPL layout");

// Shared memory of one mixed-form CTA: staged records, the per-line
// region-C denominator tables (8 leading pad floats keep R[m-1-k] of the
// first line in bounds for predicated reads), the per-point FP64 sums, and
// the per-line option data (1 / nu for the chi factor, ExtPL).
constexpr int HK_RPAD = 8;
// Far field (the default option set): each warp's FP64 sums of the blocks'
// Taylor coefficients, HK_FN per 64-point block.
constexpr int HK_FB = 64, HK_FN = 9;
template <class SH, int EXT = HK_EXT_NONE>
constexpr size_t smem_mixed() {
  return sizeof(RecF) * SH::CH + sizeof(float) * (HK_RPAD + SH::CH * HK_C916_MR) +
         sizeof(double) * SH::G +
         (EXT == HK_EXT_CHI ? sizeof(float) * SH::CH
          : EXT == HK_EXT_PL ? sizeof(ExtPL) * SH::CH
                             : sizeof(double) * SH::WARPS * HK_FN * (SH::G / HK_FB));
}

struct __align__(16) RecD {
  double nu, iad, y2, y, S1, Sc, ey, pl;  // pl: plinth (removePlinth), else 0
  int i0, b0, c0, c1, b1, i1, p0, p1;
};

// first index in [0, n) with a[idx] >= v (n if none); all 32 lanes call it
__device__ int64_t lower_bound_warp(const double *__restrict__ a, int64_t n,
                                    double v) {
  const int lane = threadIdx.x & 31;
  int64_t lo = 0, hi = n;
  while (hi - lo > 32) {
    const int64_t span = hi - lo;
    const int64_t pos = lo + ((int64_t)(lane + 1) * span) / 33;
    const bool ge = a[pos] >= v;
    const unsigned m = __ballot_sync(0xffffffffu, ge);
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
  const bool lt = (pos < hi) && (a[pos] < v);
  const unsigned m = __ballot_sync(0xffffffffu, lt);
  return lo + __popc(m);
}

__device__ __forceinline__ int clip_local(int w, int64_t g0, int64_t g1) {
  const int64_t v = (int64_t)w < g0 ? g0 : ((int64_t)w > g1 ? g1 : (int64_t)w);
  return (int)(v - g0);
}

__device__ __forceinline__ float2 f2(double v) {
  const float f = (float)v;
  return make_float2(f, f);
}

// Clip one line's global windows to the tile [g0, g1) and fill the staged
// record.  Clipping the oracle's global boundaries equals searching the
// clipped range, because every window predicate is monotone on its range.
// Lines with S = 0 have empty windows and are staged empty.
//
// Mixed form, in two steps: line_key gives the line's sort key within the
// chunk -- its strength level (0..HK_MAX_LEVEL), HK_MAX_LEVEL + 1 for lines
// summed in FP64 (weak), HK_MAX_LEVEL + 2 for lines without points in the
// tile -- and stage_mixed builds the record for that key.
// Record loads: the Voigt launch reads records another kernel wrote (the
// read-only path is fine); the fused table kernel reads records its own CTAs
// wrote into reused ring slots, so its loads go to L2 (.cg), never through
// a stale L1 or the non-coherent path.
template <bool CG>
__device__ __forceinline__ int4 rec_words(const void *p, int word16) {
  const int4 *q = reinterpret_cast<const int4 *>(p) + word16;
  if constexpr (CG) return __ldcg(q);
  else return *q;
}

template <bool CG, class R>
__device__ __forceinline__ R load_record(const R *p) {
  static_assert(sizeof(R) % 16 == 0, "records are read in 16-byte words");
  R r;
  int4 *d = reinterpret_cast<int4 *>(&r);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(R) / 16); ++k) d[k] = rec_words<CG>(p, k);
  return r;
}

constexpr int HK_NKEY = HK_MAX_LEVEL + 3;
constexpr int HK_KEY_WEAK = HK_MAX_LEVEL + 1, HK_KEY_EMPTY = HK_MAX_LEVEL + 2;

template <bool CG>
__device__ __forceinline__ int line_key(const LinePrepF *__restrict__ P, int64_t l,
                                        int64_t g0, int64_t g1, int s1exp) {
  // words 4 and 5 of the record: {ex, flags, i0, b0}, {c0, c1, b1, i1}
  const int4 w4 = rec_words<CG>(P + l, 4), w5 = rec_words<CG>(P + l, 5);
  const int i0 = clip_local(w4.z, g0, g1), i1 = clip_local(w5.w, g0, g1);
  if (i1 <= i0) return HK_KEY_EMPTY;
  // the state's largest term has exponent 40 - s1exp, so 40 - (ex + s1exp) >= 0
  const int lev = (40 - (w4.x + s1exp)) / HK_LEVEL_BITS;
  if ((w4.y & HK_PF_RANGE) || lev > HK_MAX_LEVEL) return HK_KEY_WEAK;
  return lev;
}

// ------------------------------------------------------------ far field
// Over a 64-point block far from a line's centre the line's term is a smooth
// function of the point, so the tile keeps, per block, the sum over such
// lines of their Taylor expansions about the block centre in the grid offset
// j = k - (blo + 31.5), |j| <= 31.5, and evaluates that one polynomial per
// point at the end of the tile (far_terms; the evaluation closes sum_tile).
// A block is far for a line when it lies inside the line's cut window and
// inside one of regions A and B (no region boundary, no region-C point) and
// its centre is at least HK_FAR_DK grid steps from the line centre.  The
// term's singularities in the complex offset plane are the zeros of
// x^2 + y^2, r0 = |x0 + iy| >= |x0| >= 250 vb away (for small y nearly a
// double pole, whose Taylor remainder after N terms is about (N + 1) rho^N),
// and for GH2 those of its other denominator factor, close to +-i
// sqrt(y^2 + 0.55).  With rho = |j vb| / r0 <= 31.5 / 250.5 = 0.126,
// HK_FN = 9 terms leave 10 * 0.126^9 = 8e-8 of the term, below the FP32
// rounding of the sums (9 terms is what the per-warp FP64 coefficient sums
// leave room for at 4 CTAs per SM; 8 terms needed 315.5 steps for the same
// bound, leaving a wider near zone to the direct sweeps).  FP64 (weak) lines and
// lines with x^2 + y^2 >= 1e18 in their window take the direct sweeps
// throughout.
constexpr float HK_FAR_DK = 250.5f;

// bits [a, b) of a 32-bit mask (a, b clamped to [0, 32])
__device__ __forceinline__ unsigned range_bits(int a, int b) {
  a = max(a, 0);
  b = min(b, 32);
  if (b <= a) return 0u;
  const unsigned hi = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
  return hi & ~((1u << a) - 1u);
}

// The far blocks of a staged line (tile-local record r, line centre at the
// tile point kc): blocks inside the cut window, minus those whose centre
// 64 b + 31.5 lies within HK_FAR_DK of kc, those holding region-C points
// and those a region boundary cuts.
__device__ __forceinline__ unsigned far_blocks(const RecF &r, double kc) {
  if (!(fabs(kc) < 2097152.0)) return 0u;  // block centre - kc exact in FP32
  unsigned m = range_bits((r.i0 + HK_FB - 1) / HK_FB, r.i1 / HK_FB);
  const double lo = (kc - (double)HK_FAR_DK - 31.5) / HK_FB, hi = (kc + (double)HK_FAR_DK - 31.5) / HK_FB;
  m &= ~range_bits((int)floor(lo) + 1, (int)ceil(hi));
  if (r.c0 < r.c1) m &= ~range_bits(r.c0 / HK_FB, (r.c1 + HK_FB - 1) / HK_FB);
  if (r.b0 % HK_FB) m &= ~(1u << (r.b0 / HK_FB));
  if (r.b1 % HK_FB) m &= ~(1u << (r.b1 / HK_FB));
  return m;
}

// The plinth data of a staged line (ExtPL) and its class flag.  S1f: the
// line's FP32 scale (1 for a line summed in FP64); D0, vb: its FP64 offset at
// the tile start and grid step.  GH2 in s = x^2 is S1 N(s) / D(s) with
// N = s^2 + A1 s + B1, D = s^3 + D2 s^2 + D1 s + D0; its difference is
//   t(s) - t(c) = S1 (c - s) Q(s) / (D(s) D(c)),  Q = q2 s^2 + q1 s + q0,
// where (with Y = y^2 and p = 1/pi) every term of q0, q1, q2 is positive:
//   q2 = c^2 + c (2Y + 5/2 - 4p) + Y^2 + 5Y/2 + 3/2,
//   q1 = c^2 (2Y + 5/2 - 4p) + c (4Y^2 + 10Y - 18pY + 27/4 + 24p^2 - 27p)
//        + 2Y^3 + (15/2 - 6p) Y^2 + (39/4 - 15p) Y + 9/2 - 9p,
//   q0 = c^2 (Y^2 + 5Y/2 + 3/2) + c (2Y^3 + (15/2 - 6p) Y^2 + (39/4 - 15p) Y
//        + 9/2 - 9p) + Y^4 + (5 - 2p) Y^3 + (39/4 - 3p) Y^2 + 9Y + 27/8,
// so Q and the product hold FP32 accuracy at any distance from the edge.
template <bool G34>
__device__ __forceinline__ void stage_plinth(const LinePrepF &lp, const GridDev &g, double D0,
                                             double vb, double S1f, RecF &r, ExtPL &e) {
  e.D0 = D0;
  e.vb = vb;
  e.vy = e.ey = 0.0;
  e.plf = e.xcf = e.ic = e.q0 = e.q1 = e.q2 = 0.f;
  const double xc = rec_get_d(&lp.ext0);
  e.xd = xc;
  if (lp.flags & HK_PF_PL64) {
    e.xd = rec_get_d(&lp.B1);
    e.vy = rec_get_d(&lp.y);
    e.ey = rec_get_d(&lp.sig1);
    // the FP32 fields of the record hold FP64 words: give the staged line
    // plain values (its sweep reads none of them)
    r.y = (float)e.vy;
    r.ey = r.sig1 = 0.f;
    r.t0 = r.t1 = r.c0;
    r.flags |= HK_F_PL64;
    return;
  }
  if (!(xc > 0.0)) return;  // no plinth (empty window)
  e.xcf = (float)xc;
  if (G34) return;          // Doppler: the factor 1 - exp(-(x_c^2 - x^2)) per point
  const double c = xc * xc;
  const double Y = (double)lp.y * (double)lp.y;
  if (g.profile == 2 || c + Y >= 2e6) {
    const double ic = 1.0 / (c + Y);
    e.ic = (float)ic;
    e.plf = (float)(S1f * ic);
    r.flags |= HK_F_PLA;
  } else {
    const double D2 = lp.D2, D1 = lp.D1, D0c = lp.D0, A1 = lp.A1, B1 = lp.B1;
    const double Dc = ((c + D2) * c + D1) * c + D0c;
    const double Nc = (c + A1) * c + B1;
    const double p = 0.31830988618379067;
    const double Y2 = Y * Y, Y3 = Y2 * Y, Y4 = Y2 * Y2, c2 = c * c;
    const double k1 = 2.0 * Y + 2.5 - 4.0 * p;
    const double k0 = 2.0 * Y3 + (7.5 - 6.0 * p) * Y2 + (9.75 - 15.0 * p) * Y + 4.5 - 9.0 * p;
    e.q2 = (float)(c2 + c * k1 + Y2 + 2.5 * Y + 1.5);
    e.q1 = (float)(c2 * k1 + c * (4.0 * Y2 + (10.0 - 18.0 * p) * Y + 6.75 + 24.0 * p * p - 27.0 * p) + k0);
    e.q0 = (float)(c2 * (Y2 + 2.5 * Y + 1.5) + c * k0 + Y4 + (5.0 - 2.0 * p) * Y3 +
                   (9.75 - 3.0 * p) * Y2 + 9.0 * Y + 3.375);
    e.ic = (float)(1.0 / Dc);
    e.plf = (float)(S1f * Nc / Dc);
    r.flags |= HK_F_PLB;
  }
}

template <bool CG, bool G34, int EXT = HK_EXT_NONE>
__device__ __forceinline__ void stage_mixed(const LinePrepF *__restrict__ P, const GridDev &g,
                                            int64_t l, int64_t g0, int64_t g1, int s1exp,
                                            int key, RecF &r, void *ext = nullptr) {
  const LinePrepF lp = load_record<CG>(P + l);
  const bool nonempty = key != HK_KEY_EMPTY;
  const bool weak = key == HK_KEY_WEAK;
  const int lev = (weak || !nonempty) ? 0 : key;
  const double D0 = __dmul_rn(__dsub_rn(grid_x(g, g0), lp.nu), lp.iad);
  const double vb = __dmul_rn(g.dnu, lp.iad);
  // the tile point nearest the centre (|kc| <= 2^23 keeps k - kc exact)
  const double kc = fmin(fmax(rint(-D0 / vb), -8388608.0), 8388608.0);
  // S1f = S1 * 2^(s1exp + 96 lev): the line's largest term near 2^40
  const double S1f = weak ? 1.0 : ldexp(lp.S1, s1exp + HK_LEVEL_BITS * lev);
  r.S1f = (float)S1f;
  r.C1 = (float)(S1f * (double)lp.A1);
  r.C0 = (float)(S1f * (double)lp.B1);
  r.D2 = lp.D2;
  r.D1 = lp.D1;
  r.D0 = lp.D0;
  r.nkc = (float)(-kc);
  r.vb = (float)vb;
  r.fr = (float)__fma_rn(kc, vb, D0);
  r.Sc = lp.Sc;
  r.y = lp.y;
  r.ey = lp.ey;
  r.sig1 = lp.sig1;
  r.i0 = nonempty ? clip_local(lp.i0, g0, g1) : 0;
  r.b0 = clip_local(lp.b0, g0, g1);
  r.c0 = clip_local(lp.c0, g0, g1);
  r.c1 = clip_local(lp.c1, g0, g1);
  r.b1 = clip_local(lp.b1, g0, g1);
  r.i1 = nonempty ? clip_local(lp.i1, g0, g1) : 0;
  r.t0 = clip_local(lp.t0, g0, g1);
  r.t1 = clip_local(lp.t1, g0, g1);
  r.flags = ((lp.flags & HK_PF_WIDE) ? HK_F_WIDE : 0) | (weak ? HK_F_WEAK : 0) | (lev << 8);
  r.fmask = (!G34 && EXT == HK_EXT_NONE && nonempty && !weak && !(lp.flags & HK_PF_WIDE))
                ? far_blocks(r, kc)
                : 0u;
  if (EXT == HK_EXT_CHI) *static_cast<float *>(ext) = lp.inu;
  if (EXT == HK_EXT_PL) stage_plinth<G34>(lp, g, D0, vb, S1f, r, *static_cast<ExtPL *>(ext));
  if (G34) {
    // Doppler / binned Gaussian: S1f exp(-u^2) with u = |x| (- vb / 2) is a
    // normal float only for u^2 <= (126 + e) ln 2 (S1f < 2^e), so the FP32
    // sums take [t0, t1), where it is one with room to spare (e - 2 for
    // the Doppler term; e - 30 for the binned Gaussian's erfcx factor), and
    // the points beyond, out to where the FP64 term S1 exp(-u^2) (S1 / vb
    // bounds the binned Gaussian's) falls below 2^-1075 and is exactly 0,
    // are summed in FP64: [i0, t0) and [t1, i1).  Weak lines (FP64 sums)
    // keep their whole window.
    const double h = g.profile == 4 ? 0.5 * vb : 0.0;
    if (g.profile == 4 && !weak) {
      // (erf(x + h) - erf(x - h)) / (2 vb) folded into the strength
      r.S1f = (float)(S1f / (2.0 * vb));
    }
    gauss_put(r, D0, vb, (float)h);
    if (!weak && nonempty) {
      int e = 0;
      frexp((double)r.S1f, &e);
      const double u2 = (double)max(0, (g.profile == 4 ? 96 : 124) + e) * 0.69314718055994531;
      const double xd = sqrt(u2) + h + 1e-6;
      const double S1d = g.profile == 3 ? lp.Sc : lp.Sc * 1.7724538509055160273;
      const double lt = log(fmax(S1d * fmax(1.0, 1.0 / vb), 1e-300));
      const double xt = fmax(xd, sqrt(fmax(746.2 + lt, 0.0)) + h + 1e-6);
      // tile points k with |D0 + k vb| <= xd (FP32) and <= xt (FP64)
      const double n = (double)(g1 - g0);
      const double ka = ceil((-xd - D0) / vb), kb = floor((xd - D0) / vb) + 1.0;
      const double ta = ceil((-xt - D0) / vb), tb = floor((xt - D0) / vb) + 1.0;
      const int k0 = (int)fmin(fmax(ka, 0.0), n), k1 = (int)fmin(fmax(kb, 0.0), n);
      const int u0 = (int)fmin(fmax(ta, 0.0), n), u1 = (int)fmin(fmax(tb, 0.0), n);
      r.i0 = max(r.i0, u0);
      r.i1 = max(r.i0, min(r.i1, u1));
      r.t0 = min(max(r.i0, k0), r.i1);
      r.t1 = max(r.t0, min(r.i1, k1));
      r.b0 = r.c0 = r.c1 = r.b1 = r.i0;  // region A only
    }
  }
}

// region C inside the tile: denominators of the Algorithm-916 series
__device__ __forceinline__ void stage_rtab(float y, float *__restrict__ Rtab) {
  const float a2 = HK_A916_F * HK_A916_F;
  const float Yf = y * y;
#pragma unroll 2
  for (int m = 1; m <= HK_C916_MR; ++m) Rtab[m - 1] = rcp_fast(fmaf(a2 * m, (float)m, Yf));
}

template <bool CG>
__device__ __forceinline__ void stage_plain(const LinePrep *__restrict__ P, int64_t l,
                                            int64_t g0, int64_t g1, RecD *recp) {
  const LinePrep lp = load_record<CG>(P + l);
  int li[6] = {clip_local(lp.i0, g0, g1), clip_local(lp.b0, g0, g1),
               clip_local(lp.c0, g0, g1), clip_local(lp.c1, g0, g1),
               clip_local(lp.b1, g0, g1), clip_local(lp.i1, g0, g1)};
  const bool nonempty = li[5] > li[0] && lp.Sc != 0.0;
  RecD r;
  r.nu = lp.nu;
  r.iad = lp.iad;
  r.y = lp.vy;
  r.y2 = lp.vy * lp.vy;
  r.S1 = lp.S1;
  r.Sc = lp.Sc;
  r.ey = lp.ey;
  r.pl = nonempty ? lp.plinth : 0.0;
  r.i0 = nonempty ? li[0] : 0;
  r.b0 = li[1];
  r.c0 = li[2];
  r.c1 = li[3];
  r.b1 = li[4];
  r.i1 = nonempty ? li[5] : 0;
  r.p0 = r.p1 = 0;
  *recp = r;
}

// ------------------------------------------------------------ FP32 sweep
// Each warp classifies the staged lines against its 256-point slice, 32
// lines per instruction (one lane per line).  With [lo, hi) the line's cut
// window inside the slice:
//   HK_CLS_B   [lo, hi) is the whole slice, inside one region-B part;
//   HK_CLS_A   [lo, hi) is the whole slice, inside region A;
//   HK_CLS_BM  [lo, hi) lies in region B or C (window edge in the slice, or
//              region C in it);
//   HK_CLS_AM  [lo, hi) lies in region A (window edge in the slice);
//   HK_CLS_G   [lo, hi) holds an A/B region boundary;
//   HK_CLS_W   an HK_F_WEAK line (FP64 sums);
//   HK_CLS_BF, HK_CLS_AF  as B and A but for far-field blocks of the slice,
//              which they skip;
// non-intersecting lines cost nothing.  B and A run the packed f32x2 loop
// with no tests; BM and AM run it per 64-point block of pairs, skipping
// blocks without points of their region and masking only the blocks a
// boundary cuts; G tests every point.  Region-C points go to sweep_C and
// are summed in FP64 into the per-point shared sums cacc.
enum { HK_CLS_SKIP = 0, HK_CLS_B, HK_CLS_A, HK_CLS_BM, HK_CLS_AM, HK_CLS_G, HK_CLS_W, HK_CLS_BF, HK_CLS_AF };

// bit q: block q of the slice starting at wb is far for the line
template <int SLICE>
__device__ __forceinline__ unsigned far_mask(const RecF &r, int wb) {
  return (r.fmask >> (wb / HK_FB)) & ((1u << (SLICE / HK_FB)) - 1u);
}

// The line's Taylor coefficients about the centre of block blo (grid units),
// scaled like its FP32 sums (S1f), added to fq.  Region B: GH2 = N(s)/D(s)
// with s = s0 + b j + c j^2 (s0 = x0^2, b = 2 x0 vb, c = vb^2); N and D as
// polynomials in j (every term of each coefficient has the same sign), then
// the quotient series q_n = (N_n - sum_i D_i q_(n-i)) / D_0.  Region A:
// S1f / (d0 + d1 j + d2 j^2), q_n = -(d1 q_(n-1) + d2 q_(n-2)) / d0.
__device__ __forceinline__ void far_terms(const RecF &r, int blo, float (&fq)[HK_FN]) {
  const float x0 = fmaf((float)blo + 31.5f + r.nkc, r.vb, r.fr);
  const float vb = r.vb;
  const float b = 2.0f * x0 * vb, c = vb * vb;
  float q[HK_FN];
  if (blo >= r.b0 && blo + HK_FB <= r.b1) {
    const float S1f = r.S1f, C1 = r.C1, C0 = r.C0, E2 = r.D2, E1 = r.D1, E0 = r.D0;
    const float s0 = x0 * x0;
    // s^2 and s^3 as polynomials in j
    const float t0 = s0 * s0, t1 = 2.0f * s0 * b, t2 = fmaf(b, b, 2.0f * s0 * c), t3 = 2.0f * b * c,
                t4 = c * c;
    const float u0 = t0 * s0, u1 = fmaf(t0, b, t1 * s0), u2 = fmaf(t0, c, fmaf(t1, b, t2 * s0)),
                u3 = fmaf(t1, c, fmaf(t2, b, t3 * s0)), u4 = fmaf(t2, c, fmaf(t3, b, t4 * s0)),
                u5 = fmaf(t3, c, t4 * b), u6 = t4 * c;
    const float N0 = fmaf(S1f, t0, fmaf(C1, s0, C0)), N1 = fmaf(S1f, t1, C1 * b),
                N2 = fmaf(S1f, t2, C1 * c), N3 = S1f * t3, N4 = S1f * t4;
    const float D0 = u0 + fmaf(E2, t0, fmaf(E1, s0, E0)), D1 = u1 + fmaf(E2, t1, E1 * b),
                D2 = u2 + fmaf(E2, t2, E1 * c), D3 = fmaf(E2, t3, u3), D4 = fmaf(E2, t4, u4), D5 = u5,
                D6 = u6;
    const float iD = rcp_fast(D0);  // 1 ulp: one factor on every coefficient
    q[0] = N0 * iD;
    q[1] = fmaf(-D1, q[0], N1) * iD;
    q[2] = fmaf(-D1, q[1], fmaf(-D2, q[0], N2)) * iD;
    q[3] = fmaf(-D1, q[2], fmaf(-D2, q[1], fmaf(-D3, q[0], N3))) * iD;
    q[4] = fmaf(-D1, q[3], fmaf(-D2, q[2], fmaf(-D3, q[1], fmaf(-D4, q[0], N4)))) * iD;
    q[5] = -fmaf(D1, q[4], fmaf(D2, q[3], fmaf(D3, q[2], fmaf(D4, q[1], D5 * q[0])))) * iD;
    q[6] = -fmaf(D1, q[5], fmaf(D2, q[4], fmaf(D3, q[3], fmaf(D4, q[2], fmaf(D5, q[1], D6 * q[0]))))) * iD;
    q[7] = -fmaf(D1, q[6], fmaf(D2, q[5], fmaf(D3, q[4], fmaf(D4, q[3], fmaf(D5, q[2], D6 * q[1]))))) * iD;
    q[8] = -fmaf(D1, q[7], fmaf(D2, q[6], fmaf(D3, q[5], fmaf(D4, q[4], fmaf(D5, q[3], D6 * q[2]))))) * iD;
  } else {
    const float d0 = fmaf(x0, x0, r.y * r.y);
    const float iD = rcp_fast(d0);
    q[0] = r.S1f * iD;
    q[1] = -(b * q[0]) * iD;
#pragma unroll
    for (int n = 2; n < HK_FN; ++n) q[n] = -fmaf(b, q[n - 1], c * q[n - 2]) * iD;
  }
#pragma unroll
  for (int n = 0; n < HK_FN; ++n) fq[n] += q[n];
}

// fq (the FP32 sums of level lev) into the warp's FP64 coefficient sums
__device__ __forceinline__ void far_flush(float (&fq)[HK_FN], double *__restrict__ fdw, int lane,
                                          int nblk, int s1exp, int lev) {
  if (lane < nblk) {
    const double u = ldexp(1.0, -(s1exp + HK_LEVEL_BITS * lev));
#pragma unroll
    for (int n = 0; n < HK_FN; ++n) fdw[n * nblk + lane] = fma((double)fq[n], u, fdw[n * nblk + lane]);
  }
#pragma unroll
  for (int n = 0; n < HK_FN; ++n) fq[n] = 0.f;
}

// fm: the slice's far blocks (FAR), which the direct sweeps skip
template <int SLICE, bool FAR = false>
__device__ __forceinline__ int classify(const RecF &r, int wb, unsigned &fm) {
  fm = 0u;
  const int we = wb + SLICE;
  const int lo = max(r.i0, wb), hi = min(r.i1, we);
  if (hi <= lo) return HK_CLS_SKIP;
  if (r.flags & HK_F_WEAK) return HK_CLS_W;
  if (FAR) {
    fm = far_mask<SLICE>(r, wb);
    if (fm == (1u << (SLICE / HK_FB)) - 1u) return HK_CLS_SKIP;
  }
  const bool full = lo == wb && hi == we;
  const bool noC = r.c0 >= r.c1 || r.c1 <= lo || r.c0 >= hi;
  if (r.b0 <= lo && r.b1 >= hi) return (full && noC) ? (fm ? HK_CLS_BF : HK_CLS_B) : HK_CLS_BM;
  if (r.b0 >= r.b1 || r.b1 <= lo || r.b0 >= hi) return full ? (fm ? HK_CLS_AF : HK_CLS_A) : HK_CLS_AM;
  return HK_CLS_G;
}

// Sub-Lorentzian wings in the mixed form (their own kernel instantiation):
// every term of a grid point lo < x < hi times chi(|x - nu|) x / nu (sLChi
// voigt.h:47-72), chi = exp(-B1 clamp(d - s1, 0, s2 - s1) - B2 clamp(d - s2,
// 0, s3 - s2) - B3 max(d - s3, 0)) -- the reference's piecewise exponential
// written as one continuous expression.  (With plinth removal too, chi t -
// plinth is no difference of one function, so the library runs the pair in
// the FP64 form.)
struct ExtF {
  float s1, s2, s3, B1, B2, B3;  // chi breakpoints (cm^-1) and the state's slopes
  int kl0, kl1;                  // tile points with sl_lo < x < sl_hi
  float dnu;
};

__device__ __forceinline__ ExtF ext_consts(const GridDev &g, const StateDev &st, int64_t g0, int64_t g1) {
  ExtF e;
  e.s1 = (float)g.sl_sigma[0];
  e.s2 = (float)g.sl_sigma[1];
  e.s3 = (float)g.sl_sigma[2];
  e.B1 = (float)st.sl_B[0];
  e.B2 = (float)st.sl_B[1];
  e.B3 = (float)st.sl_B[2];
  e.dnu = (float)g.dnu;
  if (g.subL) {
    // first tile points with x > sl_lo and with x >= sl_hi (x = numin + i dnu)
    int64_t a = g0, b = g1;
    while (a < b) {
      const int64_t m = a + (b - a) / 2;
      if (grid_x(g, m) > g.sl_lo) b = m;
      else a = m + 1;
    }
    int64_t c = a, d = g1;
    while (c < d) {
      const int64_t m = c + (d - c) / 2;
      if (grid_x(g, m) >= g.sl_hi) d = m;
      else c = m + 1;
    }
    e.kl0 = (int)(a - g0);
    e.kl1 = (int)(c - g0);
  } else {
    e.kl0 = e.kl1 = 0;
  }
  return e;
}

// chi(|x - nu|) x / nu at a point x (Doppler units) of a line with grid step
// vb (Doppler units) and 1 / nu = inu: |x - nu| = |x| dnu / vb (cm^-1)
__device__ __forceinline__ float chi_factor(const ExtF &e, float x, float vb, float inu) {
  const float xc = x * (e.dnu / vb);  // x - nu, cm^-1
  const float d = fabsf(xc);
  const float t1 = fminf(fmaxf(d - e.s1, 0.f), e.s2 - e.s1);
  const float t2 = fminf(fmaxf(d - e.s2, 0.f), e.s3 - e.s2);
  const float t3 = fmaxf(d - e.s3, 0.f);
  const float arg = fmaf(-e.B1, t1, fmaf(-e.B2, t2, -e.B3 * t3));
  return ex2_fast(1.4426950408889634f * arg) * fmaf(xc, inu, 1.0f);
}

// 1/d0 and 1/d1 from one reciprocal: R = 1/(d0 d1), then (d1 R, d0 R).
// Callers guarantee d0 d1 < 2^128 (region B: d < r^6 < 1e18).
__device__ __forceinline__ float2 rcp_pair(float2 d) {
  const float R = rcp_fast(d.x * d.y);
  return __fmul2_rn(make_float2(d.y, d.x), make_float2(R, R));
}

// the FP32 constants of regions A and B, read as three 16-byte words and
// duplicated into the pair operands of the packed f32x2 instructions
struct CoefB {
  float2 S1f, C1, C0, D2, D1, D0, nkc, vb, fr;
};

__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }

__device__ __forceinline__ CoefB load_coef(const RecF &rr) {
  const float4 *w = reinterpret_cast<const float4 *>(&rr);
  const float4 w0 = w[0], w1 = w[1];
  CoefB c;
  c.S1f = dup(w0.x);
  c.C1 = dup(w0.y);
  c.C0 = dup(w0.z);
  c.D2 = dup(w0.w);
  c.D1 = dup(w1.x);
  c.D0 = dup(w1.y);
  c.nkc = dup(w1.z);
  c.vb = dup(w1.w);
  c.fr = dup(rr.fr);
  return c;
}

__device__ __forceinline__ float2 x_pair(const CoefB &c, float2 kf) {
  return __ffma2_rn(__fadd2_rn(kf, c.nkc), c.vb, c.fr);
}

// S1f t4 at two points as (numerator, 1/denominator); the reciprocals run
// on the MUFU pipe, beside the FMA pipe that bounds this loop
__device__ __forceinline__ void gh2_pair(const CoefB &c, float2 s, float2 &num, float2 &inv) {
  num = __ffma2_rn(s, __ffma2_rn(c.S1f, s, c.C1), c.C0);
  const float2 den = __ffma2_rn(__ffma2_rn(__fadd2_rn(s, c.D2), s, c.D1), s, c.D0);
  inv = make_float2(rcp_fast(den.x), rcp_fast(den.y));
}

// the pair mask of a cut block: point in [lo, hi) and outside [c0, c1)
__device__ __forceinline__ bool in_run(int k, int lo, int hi, int c0, int c1) {
  return k >= lo && k < hi && !(k >= c0 && k < c1);
}

// region B only, whole slice (SKIP: but the far-field blocks in fm)
template <int PPL, bool SKIP = false>
__device__ __forceinline__ void sweep_B(const RecF &rr, const float2 (&kf)[PPL / 2],
                                        float2 (&a32)[PPL / 2], unsigned fm = 0u) {
  const CoefB c = load_coef(rr);
#pragma unroll
  for (int q = 0; q < PPL / 2; ++q) {
    if (SKIP && ((fm >> q) & 1u)) continue;
    const float2 x = x_pair(c, kf[q]);
    float2 num, inv;
    gh2_pair(c, __fmul2_rn(x, x), num, inv);
    a32[q] = __ffma2_rn(num, inv, a32[q]);
  }
}

// region B points of [lo, hi) minus region C, by 64-point blocks
template <int PPL>
__device__ __forceinline__ void sweep_BM(const RecF &rr, int wb, int lane,
                                         const float2 (&kf)[PPL / 2],
                                         float2 (&a32)[PPL / 2], unsigned fm = 0u) {
  const CoefB c = load_coef(rr);
  const int lo = max(rr.i0, wb), hi = min(rr.i1, wb + 32 * PPL);
  const int c0 = rr.c0, c1 = rr.c1;
#pragma unroll
  for (int q = 0; q < PPL / 2; ++q) {
    const int blo = wb + 64 * q, bhi = blo + 64;
    const int l2 = max(lo, blo), h2 = min(hi, bhi);
    if (l2 >= h2 || (c0 <= l2 && c1 >= h2) || ((fm >> q) & 1u)) continue;  // no region-B point, or far
    const float2 x = x_pair(c, kf[q]);
    float2 s = __fmul2_rn(x, x);
    float2 num, inv;
    if (l2 == blo && h2 == bhi && (c1 <= blo || c0 >= bhi)) {
      gh2_pair(c, s, num, inv);
    } else {
      // masked points take s = 1000 (a finite region-B value) and add 0
      const bool m0 = in_run(blo + lane, lo, hi, c0, c1);
      const bool m1 = in_run(blo + lane + 32, lo, hi, c0, c1);
      s.x = m0 ? s.x : 1000.f;
      s.y = m1 ? s.y : 1000.f;
      gh2_pair(c, s, num, inv);
      num.x = m0 ? num.x : 0.f;
      num.y = m1 ? num.y : 0.f;
    }
    a32[q] = __ffma2_rn(num, inv, a32[q]);
  }
}

// region A, whole slice (AM = false) or the points of [lo, hi) (AM = true);
// both skip the far-field blocks in fm
template <bool AM, int PPL>
__device__ __forceinline__ void sweep_A(const RecF &rr, int wb, int lane,
                                        const float2 (&kf)[PPL / 2],
                                        float2 (&a32)[PPL / 2], unsigned fm = 0u) {
  const CoefB c = load_coef(rr);
  const float Yf = rr.y * rr.y;
  const float2 Y = make_float2(Yf, Yf);
  const bool wide = rr.flags & HK_F_WIDE;
  const int lo = max(rr.i0, wb), hi = min(rr.i1, wb + 32 * PPL);
#pragma unroll
  for (int q = 0; q < PPL / 2; ++q) {
    const int blo = wb + 64 * q, bhi = blo + 64;
    bool m0 = true, m1 = true;
    if ((fm >> q) & 1u) continue;
    if (AM) {
      if (max(lo, blo) >= min(hi, bhi)) continue;
      m0 = blo + lane >= lo && blo + lane < hi;
      m1 = blo + lane + 32 >= lo && blo + lane + 32 < hi;
    }
    const float2 x = x_pair(c, kf[q]);
    float2 u = __ffma2_rn(x, x, Y);
    if (AM) {
      // masked points take u = 1e6 (finite, pairable) and add 0
      u.x = m0 ? u.x : 1e6f;
      u.y = m1 ? u.y : 1e6f;
    }
    float2 inv = wide ? make_float2(rcp_fast(u.x), rcp_fast(u.y)) : rcp_pair(u);
    if (AM) {
      inv.x = m0 ? inv.x : 0.f;
      inv.y = m1 ? inv.y : 0.f;
    }
    a32[q] = __ffma2_rn(c.S1f, inv, a32[q]);
  }
}

// Profiles 3 and 4 (Doppler, binned Gaussian), the points of [lo, hi) in
// the slice: S1f exp(-x^2) and S1f (erf(x + h) - erf(x - h)) (S1f carrying
// 1 / (2 vb)), FP32 but for the Gaussian's exponent: x^2 log2(e) = n + f is
// formed in FP64 from the FP64 offset, so 2^-f (MUFU) and the exponent
// 2^(e - n) of S1f 2^-n keep the term's FP32 accuracy at any |x|.  The
// binned Gaussian takes, on the side of x away from zero, erfc(u) - erfc(v)
// = e^-u^2 (erfcx(u) - erfcx(v) e^(u^2 - v^2)), u = |x| - h, v = |x| + h (no
// cancellation in the wings), and erf(x + h) - erf(x - h) near the centre.
__device__ __forceinline__ float gauss_scaled(double u, float mS, int eS) {
  const double q = u * u * 1.4426950408889634;  // u^2 log2(e)
  const double n = rint(q);
  const float f = (float)(q - n);
  const int et = eS - (int)n;
  const float sc = et >= -126 ? __int_as_float((et + 127) << 23) : 0.f;
  return mS * ex2_fast(-f) * sc;
}

// PL: plinth removal (Doppler): t (1 - exp(-(x_c^2 - x^2))) with
// x_c^2 - x^2 = (x_c - x)(x_c + x) from the FP64 offset, no cancellation.
// The FP32 part [t0, t1) adds to the FP32 sums; the FP64 tails [i0, t0)
// and [t1, i1) add the FP64 form's term to cacc.
template <int PPL, bool PL = false>
__device__ __forceinline__ void sweep_G34(const RecF &rr, int profile, int wb, int lane,
                                          const float2 (&kf)[PPL / 2], float2 (&a32)[PPL / 2],
                                          double *__restrict__ cacc, const ExtPL *pe = nullptr) {
  const int we = wb + 32 * PPL;
  const int lo = max(rr.t0, wb), hi = min(rr.t1, we);
  const double D0 = gauss_D0(rr), vb = gauss_vb(rr);
  if (max(rr.i0, wb) < min(rr.t0, we) || max(rr.t1, wb) < min(rr.i1, we)) {
    const double S1 = profile == 3 ? rr.Sc : rr.Sc * 1.7724538509055160273;  // S / sqrt(pi), S
#pragma unroll 1
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      if ((k >= rr.i0 && k < rr.t0) || (k >= rr.t1 && k < rr.i1)) {
        const double x = fma((double)k, vb, D0);
        double v = profile_a_d(profile, x, 0.0, S1, vb);
        if (PL) {
          const double ax = fabs(x);
          v *= -expm1(-(pe->xd - ax) * (pe->xd + ax));
        }
        cacc[k] += v;
      }
    }
  }
  if (lo >= hi) return;
  const bool full = lo == wb && hi == we;
  const float h = rr.C1;
  int eS = 0;
  const float mS = 2.0f * frexpf(rr.S1f, &eS);  // S1f = mS 2^(eS - 1), mS in [1, 2)
  eS -= 1;
#pragma unroll
  for (int p = 0; p < PPL; ++p) {
    const int k = wb + lane + 32 * p;
    if (!full && !(k >= lo && k < hi)) continue;
    const float kk = (p & 1) ? kf[p >> 1].y : kf[p >> 1].x;
    const double x = fabs(fma((double)kk, vb, D0));
    float t;
    if (profile == 3) {
      t = gauss_scaled(x, mS, eS);
    } else if (x > (double)h) {
      const float u = (float)(x - (double)h), v = (float)(x + (double)h);
      const float w = fmaf(-erfcxf(v), ex2_fast(-4.0f * 1.4426950408889634f * (float)x * h), erfcxf(u));
      t = gauss_scaled(x - (double)h, mS, eS) * w;
    } else {
      const float xf = (float)x;
      t = rr.S1f * (erff(xf + h) - erff(xf - h));
    }
    if (PL) t *= -expm1f(-(float)(pe->xd - x) * (pe->xcf + (float)x));
    if (p & 1) a32[p >> 1].y += t;
    else a32[p >> 1].x += t;
  }
}

// Region C points of the slice, summed in FP64 into cacc, lanes packed by
// evaluator so a warp never runs both: [t0, t1) holds |x| < sqrt(36 - y^2)
// (Algorithm 916), the rest of [lo, hi) has r >= 6 (asymptotic series).  The
// split is the line's own (LinePrepF t0, t1, from the FP64 offsets); a point
// within rounding of r = 6 may take either evaluator (both hold there).
// Points leave their owning lane here, so the warp syncs before cacc is
// touched again.
// EXT: HK_EXT_CHI multiplies the chi factor (ex, inu = 1 / nu); HK_EXT_PL
// subtracts the plinth pld (FP64 units), which a point of region C exceeds
// at least fourfold (the line's edge lies in region A or B, r_c^2 >= 400).
template <int SLICE, int EXT = HK_EXT_NONE>
__device__ __forceinline__ void sweep_C(const RecF &r, const float *__restrict__ Rj,
                                        double *__restrict__ cacc, int wb, int lane,
                                        const ExtF *ex = nullptr, float inu = 0.f, double pld = 0.0) {
  const int lo = max(r.c0, wb), hi = min(r.c1, wb + SLICE);
  if (lo >= hi) return;
  const float nkc = r.nkc, vbf = r.vb, fr = r.fr;
  const float y = r.y, ey = r.ey, sig1 = r.sig1;
  const float iy = y > 0.f ? (float)(1.0 / (double)y) : 0.f;
  const double Sc = r.Sc;
  const int t0 = min(max(r.t0, lo), hi), t1 = min(max(r.t1, t0), hi);
  __syncwarp();
  for (int k = t0 + lane; k < t1; k += 32) {
    const float kk = (float)k;
    const float x = fmaf(kk + nkc, vbf, fr);
    float v = voigt916_core(x, y, iy, ey, sig1, Rj);
    if (EXT == HK_EXT_CHI && k >= ex->kl0 && k < ex->kl1) v *= chi_factor(*ex, x, r.vb, inu);
    cacc[k] = fma(Sc, (double)v, cacc[k]) - pld;
  }
  const int n1 = t0 - lo, ns = n1 + (hi - t1);
  for (int i = lane; i < ns; i += 32) {
    const int k = i < n1 ? lo + i : t1 + (i - n1);
    const float kk = (float)k;
    const float x = fmaf(kk + nkc, vbf, fr);
    float v = voigt_asy(x, y);
    if (EXT == HK_EXT_CHI && k >= ex->kl0 && k < ex->kl1) v *= chi_factor(*ex, x, r.vb, inu);
    cacc[k] = fma(Sc, (double)v, cacc[k]) - pld;
  }
  __syncwarp();
}

// A/B boundaries in the slice, and weak lines: per-point window/region
// tests.  WEAK lines (S1f = 1) add S1 t in FP64 to cacc; the others add
// S1f t to the FP32 sums.  EXT == HK_EXT_CHI: every term times the chi
// factor (ex, inu = 1 / nu).  EXT == HK_EXT_PL: the term less the plinth
// (pe): at a point of the edge's region (HK_F_PLA / HK_F_PLB) the factored
// difference, with x_c - |x| from the FP64 offset, elsewhere t - plinth.
template <bool WEAK, bool G34, int PPL, int EXT = HK_EXT_NONE>
__device__ __forceinline__ void sweep_G(const RecF &r, int wb, int lane,
                                        const float2 (&kf)[PPL / 2],
                                        float2 (&a32)[PPL / 2],
                                        double *__restrict__ cacc, int profile,
                                        const ExtF *ex = nullptr, float inu = 0.f,
                                        const ExtPL *pe = nullptr, unsigned fm = 0u) {
  if (WEAK && G34) {
    // Doppler / binned Gaussian lines summed in FP64: the FP64 form's term
    // (with plinth removal: times 1 - exp(-(x_c^2 - x^2)), x_c - |x| exact)
    const double D0 = gauss_D0(r), vb = gauss_vb(r);
    const double S1 = profile == 3 ? r.Sc : r.Sc * 1.7724538509055160273;  // S / sqrt(pi), S
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      if (k >= r.i0 && k < r.i1) {
        const float kk = (p & 1) ? kf[p >> 1].y : kf[p >> 1].x;
        const double x = fma((double)kk, vb, D0);
        double v = profile_a_d(profile, x, 0.0, S1, vb);
        if (EXT == HK_EXT_PL) {
          const double ax = fabs(x);
          v *= -expm1(-(pe->xd - ax) * (pe->xd + ax));
        }
        cacc[k] += v;
      }
    }
    return;
  }
  // the record lives in shared memory like cacc: read it once into registers
  const int i0 = r.i0, i1 = r.i1, b0 = r.b0, b1 = r.b1, c0 = r.c0, c1 = r.c1;
  const float nkc = r.nkc, vb = r.vb, fr = r.fr;
  const float y = r.y;
  const float Yf = y * y;
  const int we = wb + 32 * PPL;
  if (c0 <= max(i0, wb) && c1 >= min(i1, we)) return;  // region C only
  const float S1f = r.S1f, C1 = r.C1, C0 = r.C0;
  const float D2 = r.D2, D1 = r.D1, D0 = r.D0;
  const double S1w = WEAK ? r.Sc * (double)y * 0.56418958354775628 : 0.0;  // S y / pi
  const int plc = EXT == HK_EXT_PL ? (r.flags & (HK_F_PLA | HK_F_PLB)) : 0;
  const float plf = EXT == HK_EXT_PL ? pe->plf : 0.f;
#pragma unroll
  for (int p = 0; p < PPL; ++p) {
    const int k = wb + lane + 32 * p;
    if (k >= i0 && k < i1 && !(k >= c0 && k < c1) && !((fm >> ((32 * p + lane) >> 6)) & 1u)) {
      const float kk = (p & 1) ? kf[p >> 1].y : kf[p >> 1].x;
      const float x = fmaf(kk + nkc, vb, fr);
      const float s = x * x;
      // the term as (factor, reciprocal), added with one FMA like the packed sweeps
      float f, inv;
      const bool inB = k >= b0 && k < b1;
      if (inB) {
        f = fmaf(s, fmaf(S1f, s, C1), C0);
        inv = rcp_fast(fmaf(fmaf(s + D2, s, D1), s, D0));
      } else {
        f = S1f;
        inv = rcp_fast(fmaf(x, x, Yf));
      }
      if (EXT == HK_EXT_PL) {
        float t;
        if (plc == (inB ? HK_F_PLB : HK_F_PLA)) {
          // (x_c - |x|)(x_c + |x|) = x_c^2 - s; times 1 / (x_c^2 + Y) in
          // region A, times Q(s) / D(x_c^2) in region B
          const float dx = (float)(pe->xd - fabs(fma((double)k, pe->vb, pe->D0)));
          float w = dx * (pe->xcf + fabsf(x)) * pe->ic;
          if (inB) w *= fmaf(fmaf(pe->q2, s, pe->q1), s, pe->q0);
          t = (S1f * inv) * w;
        } else {
          t = fmaf(f, inv, -plf);
        }
        if (WEAK) {
          cacc[k] = fma(S1w, (double)t, cacc[k]);
        } else if (p & 1) {
          a32[p >> 1].y += t;
        } else {
          a32[p >> 1].x += t;
        }
      } else if (EXT == HK_EXT_CHI) {
        float t = f * inv;
        if (k >= ex->kl0 && k < ex->kl1) t *= chi_factor(*ex, x, vb, inu);
        if (WEAK) {
          cacc[k] = fma(S1w, (double)t, cacc[k]);
        } else if (p & 1) {
          a32[p >> 1].y += t;
        } else {
          a32[p >> 1].x += t;
        }
      } else if (WEAK) {
        cacc[k] = fma(S1w, (double)(f * inv), cacc[k]);
      } else if (p & 1) {
        a32[p >> 1].y = fmaf(f, inv, a32[p >> 1].y);
      } else {
        a32[p >> 1].x = fmaf(f, inv, a32[p >> 1].x);
      }
    }
  }
}

// Plinth removal, a line summed per point in FP64 (HK_F_PL64: its cut edge
// lies in region C or close to a region boundary, or FP32 cannot hold it):
// the FP64 form's terms (regions C, B, A) less the plinth, from the line's
// FP64 vy, erfcx(vy) and plinth (pe) and x = D0 + k vb.
template <int PPL>
__device__ __forceinline__ void sweep_pl64(const RecF &r, const ExtPL &pe, int wb, int lane,
                                           double *__restrict__ cacc, int profile) {
  const int we = wb + 32 * PPL;
  if (r.i1 <= wb || r.i0 >= we) return;
  const double vy = pe.vy, Y = vy * vy;
  const double S1 = r.Sc * vy * 0.56418958354775628;  // S vy / pi
#pragma unroll 1
  for (int p = 0; p < PPL; ++p) {
    const int k = wb + lane + 32 * p;
    if (k >= r.i0 && k < r.i1) {
      const double x = fma((double)k, pe.vb, pe.D0);
      double v;
      if (k >= r.c0 && k < r.c1) v = r.Sc * voigt916_d(x, vy, pe.ey);
      else if (k >= r.b0 && k < r.b1) v = S1 * gh2_d(x, Y);
      else v = profile_a_d(profile, x, Y, S1, pe.vb);
      cacc[k] += v - pe.xd;
    }
  }
}

// ------------------------------------------------------------ FP64 sweep
template <int PPL>
__device__ __forceinline__ void sweep_plain(const RecD &r, int wb, int lane,
                                            const double (&xg)[PPL],
                                            double (&acc)[PPL], const GridDev &g,
                                            const StateDev &st) {
  const int we = wb + 32 * PPL;
  if (r.i1 <= wb || r.i0 >= we) return;
  if (g.profile != 1 || g.plinth || g.subL) {
    // profiles 2-4 (region A only), sub-Lorentzian wings and plinth removal:
    // Line6fA/B/C(X) add the profile (times chi x/nu), then subtract the
    // line's plinth, at every window point
    const double vb = g.dnu * r.iad;
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      if (k >= r.i0 && k < r.i1) {
        const double x = (xg[p] - r.nu) * r.iad;
        double v;
        if (k >= r.c0 && k < r.c1) v = r.Sc * voigt916_d(x, r.y, r.ey);
        else if (k >= r.b0 && k < r.b1) v = r.S1 * gh2_d(x, r.y2);
        else v = profile_a_d(g.profile, x, r.y2, r.S1, vb);
        if (g.subL) v *= sublorentz_d(g, st, xg[p], r.nu);
        acc[p] += v;
        acc[p] -= r.pl;
      }
    }
    return;
  }
  const bool full = r.i0 <= wb && r.i1 >= we;
  if (full && ((r.b0 <= wb && r.c0 >= we) || (r.c1 <= wb && r.b1 >= we))) {
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const double x = (xg[p] - r.nu) * r.iad;
      acc[p] += r.S1 * gh2_d(x, r.y2);
    }
  } else if (full && (r.b0 >= we || r.b1 <= wb)) {
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const double x = (xg[p] - r.nu) * r.iad;
      acc[p] += r.S1 / (x * x + r.y2);
    }
  } else {
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      if (k >= r.i0 && k < r.i1) {
        const double x = (xg[p] - r.nu) * r.iad;
        double v;
        if (k >= r.c0 && k < r.c1) v = r.Sc * voigt916_d(x, r.y, r.ey);
        else if (k >= r.b0 && k < r.b1) v = r.S1 * gh2_d(x, r.y2);
        else v = r.S1 / (x * x + r.y2);
        acc[p] += v;
      }
    }
  }
}

// add the FP32 sums of level lev into the FP64 sums (exact unscale) and
// clear them
template <int PPL>
__device__ __forceinline__ void flush_sums(float2 (&a32)[PPL / 2], double *__restrict__ cacc,
                                           int wb, int lane, int s1exp, int lev) {
  const double u = ldexp(1.0, -(s1exp + HK_LEVEL_BITS * lev));
#pragma unroll
  for (int p = 0; p < PPL; ++p) {
    const int k = wb + lane + 32 * p;
    const float v = (p & 1) ? a32[p >> 1].y : a32[p >> 1].x;
    cacc[k] = fma((double)v, u, cacc[k]);
  }
#pragma unroll
  for (int q = 0; q < PPL / 2; ++q) a32[q] = make_float2(0.f, 0.f);
}

// ------------------------------------------------------- one tile's sum
// Everything one ticket of the Voigt sum does: the sum of the lines whose
// windows reach the tile [g0, g1) (the part-th of nsplit parts of its line
// range) into the tile's points, written to Ks (one state's K row) or, for a
// split tile, published to pt (this tile's nsplit partial rows of G points)
// and combined in part order by the CTA that completes the count *cnt.
// wmax and s1exp are the state's search half-width and FP32 scale exponent.
template <bool MIXED, class SH, bool CG, bool G34 = false, int EXT = HK_EXT_NONE>
__device__ __forceinline__ void sum_tile(const void *prep_s, const double *__restrict__ nu0,
                                         int64_t nlines, const GridDev &g, const StateDev &st,
                                         double wmax, int s1exp, int64_t g0, int64_t g1, int part,
                                         int nsplit, double *pt, unsigned *cnt, double *Ks,
                                         unsigned char *smem_dyn) {
  using Rec = typename std::conditional<MIXED, RecF, RecD>::type;
  constexpr int CH = SH::CH, PPL = SH::PPL, SLICE = SH::SLICE, G = SH::G;
  // the far field runs in the mixed form without options (Voigt, Lorentz)
  constexpr bool FAR = MIXED && !G34 && EXT == HK_EXT_NONE;
  constexpr int NBLK = G / HK_FB;  // 64-point blocks of the tile (<= 32)
  static_assert(!FAR || (NBLK <= 32 && SLICE % HK_FB == 0), "far-field block layout");
  Rec *rec = reinterpret_cast<Rec *>(smem_dyn);
  float *Rtab = reinterpret_cast<float *>(smem_dyn + sizeof(Rec) * CH) + HK_RPAD;
  double *cacc = reinterpret_cast<double *>(smem_dyn + sizeof(Rec) * CH +
                                            sizeof(float) * (HK_RPAD + CH * HK_C916_MR));
  __shared__ int s_last;
  __shared__ int s_kcnt[CH / 32][HK_NKEY];  // staged lines per (staging warp, key)
  __shared__ long long s_L0, s_L1;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wb = warp * SLICE;
  const LinePrep *P = reinterpret_cast<const LinePrep *>(prep_s);
  const LinePrepF *PF = reinterpret_cast<const LinePrepF *>(prep_s);
  if (warp == 0) {
    const double W = wmax + st.shift + 2.0 * g.dnu;
    const double xlo = grid_x(g, g0) - W;
    const double xhi = grid_x(g, g1 - 1) + W;
    const double pad = 1e-12 * (fabs(xlo) + fabs(xhi)) + 1e-300;
    const int64_t L0 = lower_bound_warp(nu0, nlines, xlo - pad);
    const int64_t L1 = lower_bound_warp(nu0, nlines, xhi + pad);
    if (lane == 0) {
      s_L0 = L0;
      s_L1 = L1;
    }
  }
  __syncthreads();
  const int64_t L0 = s_L0, L1 = s_L1;
  // per staged line: 1 / nu (chi factor) or ExtPL (plinth), after the
  // per-point sums
  float *ext_inu = reinterpret_cast<float *>(cacc + G);
  ExtPL *ext_pl = reinterpret_cast<ExtPL *>(cacc + G);
  // far field: warp w's coefficient sums fd[(w HK_FN + n) NBLK + block]
  double *fd = cacc + G;
  if (FAR)
    for (int t = lane; t < HK_FN * NBLK; t += 32) fd[warp * HK_FN * NBLK + t] = 0.0;
  ExtF exc;
  if (EXT == HK_EXT_CHI) exc = ext_consts(g, st, g0, g1);
  // chi x / nu is 1 at every point of a tile outside (x_lo, x_hi): such a
  // tile takes the regular sweeps
  const bool chi_tile = EXT == HK_EXT_CHI && exc.kl0 < exc.kl1;

  float2 kf[PPL / 2];   // lane-local point indices, paired {p, p+1}
  float2 a32[PPL / 2];  // mixed: FP32 sums of the current chunk (scaled)
  double acc[PPL], xg[PPL];
#pragma unroll
  for (int p = 0; p < PPL; ++p) {
    const int k = wb + lane + 32 * p;
    acc[p] = 0.0;
    if (MIXED) {
      if (p & 1) {
        kf[p >> 1].y = (float)k;
        a32[p >> 1].y = 0.f;
      } else {
        kf[p >> 1].x = (float)k;
        a32[p >> 1].x = 0.f;
      }
      cacc[k] = 0.0;  // owned by this lane only: no barrier needed
    } else {
      xg[p] = grid_x(g, g0 + k);
    }
  }

  // Chunk c holds the lines L0 + c + q*nch (q < CH): every chunk spans
  // the tile's whole line range, so the costly region-C points of its
  // lines fall into all warp slices instead of one or two (consecutive
  // nu-sorted lines would put a chunk's line cores into a single slice
  // and leave the other warps idle at the barrier).
  const int64_t nL = L1 - L0;
  const int64_t nch = (nL + CH - 1) / CH;
  const int64_t c_begin = nch * part / nsplit, c_end = nch * (part + 1) / nsplit;
  int lcur = 0;  // strength level held in a32 (warp-uniform)
  for (int64_t c = c_begin; c < c_end; ++c) {
    const int cnt_c = (int)((nL - c + nch - 1) / nch);
    if (MIXED) {
      // build the records, then place them sorted by key (stable counting
      // sort over the CH / 32 staging warps), so a warp's 32-line
      // groups mostly hold one strength level
      // (the key pass keeps no record: the record is rebuilt after the
      // scan rather than held in registers across the barrier)
      int key = HK_NKEY, rank = 0;
      const int64_t l = L0 + c + (int64_t)tid * nch;
      if (tid < cnt_c) key = line_key<CG>(PF, l, g0, g1, s1exp);
      if (tid < CH) {
        const unsigned lt = (1u << lane) - 1u;
#pragma unroll
        for (int v = 0; v < HK_NKEY; ++v) {
          const unsigned m = __ballot_sync(0xffffffffu, key == v);
          if (key == v) rank = __popc(m & lt);
          if (lane == 0) s_kcnt[warp][v] = __popc(m);
        }
      }
      __syncthreads();
      if (tid < cnt_c) {
        int pos = rank;
        for (int v = 0; v < key; ++v)
#pragma unroll
          for (int w = 0; w < CH / 32; ++w) pos += s_kcnt[w][v];
        for (int w = 0; w < warp; ++w) pos += s_kcnt[w][key];
        RecF r;
        stage_mixed<CG, G34, EXT>(PF, g, l, g0, g1, s1exp, key, r,
                                  EXT == HK_EXT_PL ? (void *)(ext_pl + pos) : (void *)(ext_inu + pos));
        reinterpret_cast<RecF *>(rec)[pos] = r;
        if (r.c1 > r.c0 && r.i1 > r.i0) stage_rtab(r.y, Rtab + pos * HK_C916_MR);
      }
    } else if (tid < cnt_c) {
      stage_plain<CG>(P, L0 + c + (int64_t)tid * nch, g0, g1, reinterpret_cast<RecD *>(rec) + tid);
    }
    __syncthreads();
    if (MIXED) {
      const RecF *rf = reinterpret_cast<const RecF *>(rec);
      for (int g32 = 0; g32 < cnt_c; g32 += 32) {
        const int j = g32 + lane;
        unsigned fm = 0u;  // the line's far blocks in this slice
        const int cls = (j < cnt_c) ? classify<SLICE, FAR>(rf[j], wb, fm) : HK_CLS_SKIP;
        const int lev = (j < cnt_c) ? (rf[j].flags >> 8) : 0;
        const unsigned bB = __ballot_sync(0xffffffffu, cls == HK_CLS_B);
        const unsigned bA = __ballot_sync(0xffffffffu, cls == HK_CLS_A);
        const unsigned bBM = __ballot_sync(0xffffffffu, cls == HK_CLS_BM);
        const unsigned bAM = __ballot_sync(0xffffffffu, cls == HK_CLS_AM);
        const unsigned bG = __ballot_sync(0xffffffffu, cls == HK_CLS_G);
        const unsigned bBF = FAR ? __ballot_sync(0xffffffffu, cls == HK_CLS_BF) : 0u;
        const unsigned bAF = FAR ? __ballot_sync(0xffffffffu, cls == HK_CLS_AF) : 0u;
        unsigned mW = __ballot_sync(0xffffffffu, cls == HK_CLS_W);
        unsigned live = bB | bA | bBM | bAM | bG | bBF | bAF;
        while (live) {
          // the lines of the current level first; switch level (flushing
          // the FP32 sums) only when none of them is left
          unsigned m = __ballot_sync(0xffffffffu, lev == lcur) & live;
          if (m == 0u) {
            flush_sums<PPL>(a32, cacc, wb, lane, s1exp, lcur);
            lcur = __shfl_sync(0xffffffffu, lev, __ffs(live) - 1);
            m = __ballot_sync(0xffffffffu, lev == lcur) & live;
          }
          live &= ~m;
          if (EXT == HK_EXT_CHI && chi_tile) {
            // every class through the generic sweep with the chi factor
            unsigned mX = m;
            while (mX) {
              const int b = __ffs(mX) - 1;
              mX &= mX - 1;
              const float inu = ext_inu[g32 + b];
              sweep_G<false, false, PPL, EXT>(rf[g32 + b], wb, lane, kf, a32, cacc, g.profile, &exc, inu);
              sweep_C<SLICE, EXT>(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane, &exc, inu);
            }
            continue;
          }
          if constexpr (EXT == HK_EXT_PL && !G34) {
            // every class through the generic sweep less the plinth
            const double u = ldexp(1.0, -(s1exp + HK_LEVEL_BITS * lcur));
            unsigned mX = m;
            while (mX) {
              const int b = __ffs(mX) - 1;
              mX &= mX - 1;
              const ExtPL *pe = ext_pl + g32 + b;
              sweep_G<false, false, PPL, EXT>(rf[g32 + b], wb, lane, kf, a32, cacc, g.profile, nullptr, 0.f,
                                              pe);
              sweep_C<SLICE, EXT>(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane, nullptr, 0.f,
                                  (double)pe->plf * u);
            }
            continue;
          }
          constexpr bool PLG = EXT == HK_EXT_PL && G34;  // Doppler with plinth removal
          unsigned mB = m & bB, mA = m & bA, mBM = m & bBM, mAM = m & bAM, mG = m & bG;
          if constexpr (FAR) {
            unsigned mBF = m & bBF, mAF = m & bAF;
            while (mBF) {
              const int b = __ffs(mBF) - 1;
              mBF &= mBF - 1;
              sweep_B<PPL, true>(rf[g32 + b], kf, a32, __shfl_sync(0xffffffffu, fm, b));
            }
            while (mAF) {
              const int b = __ffs(mAF) - 1;
              mAF &= mAF - 1;
              sweep_A<false, PPL>(rf[g32 + b], wb, lane, kf, a32, __shfl_sync(0xffffffffu, fm, b));
            }
          }
          while (mB) {
            const int b = __ffs(mB) - 1;
            mB &= mB - 1;
            sweep_B<PPL>(rf[g32 + b], kf, a32);
          }
          while (mA) {
            const int b = __ffs(mA) - 1;
            mA &= mA - 1;
            if constexpr (G34) sweep_G34<PPL, PLG>(rf[g32 + b], g.profile, wb, lane, kf, a32, cacc, ext_pl + g32 + b);
            else sweep_A<false, PPL>(rf[g32 + b], wb, lane, kf, a32);
          }
          while (mBM) {
            const int b = __ffs(mBM) - 1;
            mBM &= mBM - 1;
            const unsigned fb = FAR ? __shfl_sync(0xffffffffu, fm, b) : 0u;
            sweep_BM<PPL>(rf[g32 + b], wb, lane, kf, a32, fb);
            sweep_C<SLICE>(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane);
          }
          while (mAM) {
            const int b = __ffs(mAM) - 1;
            mAM &= mAM - 1;
            if constexpr (G34) {
              sweep_G34<PPL, PLG>(rf[g32 + b], g.profile, wb, lane, kf, a32, cacc, ext_pl + g32 + b);
            } else {
              const unsigned fb = FAR ? __shfl_sync(0xffffffffu, fm, b) : 0u;
              sweep_A<true, PPL>(rf[g32 + b], wb, lane, kf, a32, fb);
            }
          }
          while (mG) {
            const int b = __ffs(mG) - 1;
            mG &= mG - 1;
            const unsigned fb = FAR ? __shfl_sync(0xffffffffu, fm, b) : 0u;
            sweep_G<false, G34, PPL>(rf[g32 + b], wb, lane, kf, a32, cacc, g.profile, nullptr, 0.f, nullptr, fb);
            sweep_C<SLICE>(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane);
          }
        }
        while (mW) {
          const int b = __ffs(mW) - 1;
          mW &= mW - 1;
          if (EXT == HK_EXT_CHI && chi_tile) {
            const float inu = ext_inu[g32 + b];
            sweep_G<true, false, PPL, EXT>(rf[g32 + b], wb, lane, kf, a32, cacc, g.profile, &exc, inu);
            sweep_C<SLICE, EXT>(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane, &exc, inu);
          } else if constexpr (EXT == HK_EXT_PL) {
            // FP64 sums (S1f = 1): the plinth per S1 scaled by S1, or the
            // whole line per point in FP64
            const ExtPL *pe = ext_pl + g32 + b;
            const RecF &rw = rf[g32 + b];
            if constexpr (G34) {
              sweep_G<true, true, PPL, EXT>(rw, wb, lane, kf, a32, cacc, g.profile, nullptr, 0.f, pe);
            } else if (rw.flags & HK_F_PL64) {
              sweep_pl64<PPL>(rw, *pe, wb, lane, cacc, g.profile);
            } else {
              sweep_G<true, false, PPL, EXT>(rw, wb, lane, kf, a32, cacc, g.profile, nullptr, 0.f, pe);
              sweep_C<SLICE, EXT>(rw, Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane, nullptr, 0.f,
                                  (double)pe->plf * (rw.Sc * (double)rw.y * 0.56418958354775628));
            }
          } else {
            sweep_G<true, G34, PPL>(rf[g32 + b], wb, lane, kf, a32, cacc, g.profile);
            sweep_C<SLICE>(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane);
          }
        }
      }
      // at most one chunk of lines per FP32 sum
      flush_sums<PPL>(a32, cacc, wb, lane, s1exp, lcur);
      if constexpr (FAR) {
        // far field: warp w takes lines w, w + WARPS, ... (strength-level
        // order), lane = block of the tile
        const int blo = lane * HK_FB;
        double *fdw = fd + warp * HK_FN * NBLK;
        float fq[HK_FN];
#pragma unroll
        for (int n = 0; n < HK_FN; ++n) fq[n] = 0.f;
        int flev = -1;
        for (int j = warp; j < cnt_c; j += SH::WARPS) {
          const RecF &r = rf[j];
          const unsigned fmk = r.fmask;
          if (fmk == 0u) continue;
          const bool far = (fmk >> lane) & 1u;
          const int lev = r.flags >> 8;
          if (lev != flev) {
            if (flev >= 0) far_flush(fq, fdw, lane, NBLK, s1exp, flev);
            flev = lev;
          }
          if (far) far_terms(r, blo, fq);
        }
        if (flev >= 0) far_flush(fq, fdw, lane, NBLK, s1exp, flev);
      }
    } else {
      for (int j = 0; j < cnt_c; ++j)
        sweep_plain<PPL>(reinterpret_cast<const RecD &>(rec[j]), wb, lane, xg, acc, g, st);
    }
    __syncthreads();
  }

  if constexpr (FAR) {
    // the blocks' coefficient sums over the warps (fixed order), then one
    // polynomial per point into the FP64 sums
    __syncthreads();
    for (int t = threadIdx.x; t < HK_FN * NBLK; t += SH::THREADS) {
      double v = fd[t];
      for (int w = 1; w < SH::WARPS; ++w) v += fd[w * HK_FN * NBLK + t];
      fd[t] = v;
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      const int bl = k / HK_FB;
      const double jj = (double)(k - bl * HK_FB) - 31.5;
      double v = fd[(HK_FN - 1) * NBLK + bl];
#pragma unroll
      for (int n = HK_FN - 2; n >= 0; --n) v = fma(v, jj, fd[n * NBLK + bl]);
      cacc[k] += v;
    }
  }
  if (nsplit == 1) {
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      const int64_t gi = g0 + k;
      if (MIXED) acc[p] = cacc[k];
      if (gi < g1) Ks[gi] = st.kmin + acc[p];
    }
  } else {
    // Split tile: publish this part's sums; the CTA that completes the
    // tile's count adds the parts in part order (the result does not
    // depend on which CTA ran which part or when).  The last arriver resets
    // the count, so the counter is ready for the next use of its slot.
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      const int k = wb + lane + 32 * p;
      if (MIXED) acc[p] = cacc[k];
      pt[(int64_t)part * G + k] = acc[p];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(cnt, 1u) == (unsigned)(nsplit - 1));
    __syncthreads();
    if (s_last) {
      __threadfence();
#pragma unroll
      for (int p = 0; p < PPL; ++p) {
        const int k = wb + lane + 32 * p;
        double sum = 0.0;
        for (int j = 0; j < nsplit; ++j) sum += __ldcg(pt + (int64_t)j * G + k);
        const int64_t gi = g0 + k;
        if (gi < g1) Ks[gi] = st.kmin + sum;
      }
      if (tid == 0) atomicExch(cnt, 0u);
    }
  }
}

// ------------------------------------------------------- persistent kernel
// mixed form: SH::MINB CTAs per SM (4: 32 warps, 64 registers)
// G34: the Doppler / binned-Gaussian profiles of the mixed form (their own
// instantiation, so the Voigt and Lorentz kernels carry none of their code)
template <bool MIXED, class SH, bool G34 = false, int EXT = HK_EXT_NONE>
__global__ void __launch_bounds__(SH::THREADS, MIXED ? SH::MINB : 2)
voigt_sum_kernel(const void *__restrict__ prep, const double *__restrict__ nu0,
                 int64_t nlines, GridDev g, const StateDev *__restrict__ states,
                 int tile0, int tiles_per_state, int nsplit, int total_tickets,
                 unsigned *__restrict__ ticket, double *__restrict__ partial,
                 unsigned *__restrict__ tile_cnt, double *__restrict__ K, int64_t k_stride) {
  constexpr int G = SH::G;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ int s_ticket;
  const int tid = threadIdx.x;
  const size_t rec_bytes = MIXED ? sizeof(LinePrepF) : sizeof(LinePrep);
  for (;;) {
    if (tid == 0) s_ticket = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int t = s_ticket;
    if (t >= total_tickets) break;
    // ticket -> (tile of a state, part of that tile's line range)
    const int tt = t / nsplit;
    const int part = t - tt * nsplit;
    const int s = tt / tiles_per_state;
    const int tile = tt - s * tiles_per_state;
    const StateDev &st = states[s];
    const void *prep_s = static_cast<const char *>(prep) + (size_t)s * nlines * rec_bytes;
    const int64_t g0 = (int64_t)(tile0 + tile) * G;
    const int64_t g1 = min(g0 + (int64_t)G, g.nx);
    sum_tile<MIXED, SH, false, G34, EXT>(prep_s, nu0, nlines, g, st, st.wmax, st.s1exp, g0, g1, part, nsplit,
                               partial + (int64_t)tt * nsplit * G, tile_cnt + tt,
                               K + (int64_t)s * k_stride, smem_dyn);
  }
}

// ----------------------------------------------------- T-P table kernel
// A whole T-P table in one persistent launch.  Tickets of two kinds come
// from one 64-bit counter:
//   prep (s, b): lines [b LPT, (b + 1) LPT) of state s scaled into ring slot
//                s mod R (prep_record, the records line_prep_kernel writes);
//                the ticket that completes state s's count turns the state's
//                maxima into its search half-width and FP32 scale and marks
//                the state ready;
//   sum (s, i):  tile i / nsplit, part i mod nsplit of state s (sum_tile).
// Phase p (p = 0 .. S) holds the preps of state p and the sums of state
// p - 1, interleaved one for one from the phase's start (the rest of the
// larger kind follows), so the line prep (FP64 and memory) runs beside the
// Voigt sums (FP32) on the same SMs.  A sum ticket waits until its state is
// ready (its preps were handed out in the previous phase, most of a phase
// earlier); a prep ticket of state s >= R waits until every sum ticket of
// state s - R (its slot's previous user, two phases earlier for R = 3) is
// done.  Every ticket waits only for tickets handed out before it, whose
// CTAs are resident and running, so the waits end (no cycle); each is
// bounded anyway and, once one runs out, every later wait gives up at once
// and the error word tells the host.
struct TableSched {
  int S, R;        // states, ring slots (R >= 2)
  int npb, lpt;    // prep tickets per state, lines per prep ticket
  int tps, nsplit; // tiles per state, parts per tile
  long long nsum;  // sum tickets per state (tps * nsplit)
  long long total; // S * (npb + nsum)
};

// ticket -> (kind, state, index) of the phase order above
__host__ __device__ inline void table_ticket(const TableSched &sc, long long t, bool &prep, int &s,
                                             long long &idx) {
  const long long npb = sc.npb, nsum = sc.nsum, per = npb + nsum;
  const long long k = npb < nsum ? npb : nsum;
  if (t < npb) {  // phase 0: the first state's preps
    prep = true;
    s = 0;
    idx = t;
    return;
  }
  const long long u = t - npb;
  const long long q = u / per;
  if (q >= sc.S - 1) {  // phase S: the last state's sums
    prep = false;
    s = sc.S - 1;
    idx = u - (long long)(sc.S - 1) * per;
    return;
  }
  const int p = 1 + (int)q;
  const long long r = u - q * per;
  if (r < 2 * k) {
    prep = (r & 1) != 0;
    idx = r >> 1;
  } else {
    prep = nsum < npb;
    idx = r - k;
  }
  s = prep ? p : p - 1;
}

constexpr int HK_TABLE_WAIT_POLLS = 1 << 22;  // x >= 256 ns: 1-4 s per wait

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// one thread: wait until *p >= v; false if the wait (or an earlier one) ran out
__device__ bool wait_at_least(const unsigned *p, unsigned v, int *err) {
  for (int it = 0; it < HK_TABLE_WAIT_POLLS; ++it) {
    if (ld_acquire(p) >= v) return true;
    if (*(volatile int *)err != 0) return false;
    __nanosleep(256);
  }
  atomicExch(err, 1);
  return false;
}

// The prep ticket's lines, out of line: the FP64 scaling and window searches
// want more registers than the sum loop's budget, and keeping them in their
// own function keeps their spills out of the sum loop.
template <bool MIXED>
__device__ __noinline__ void prep_lines(const LinesDev &L, const GridDev &g, const StateDev &st,
                                        int64_t l, int64_t l1, int step, const double *e916,
                                        void *out, double &w_loc, double &s1_loc) {
  for (; l < l1; l += step) prep_record<MIXED, PREP_ALL>(L, g, st, l, e916, out, w_loc, s1_loc);
}

// (at most 3 CTAs per SM in the mixed form: the prep tickets' FP64 state
// beside the sums' registers spills at 64 registers per thread)
template <bool MIXED, class SH, bool G34 = false, int EXT = HK_EXT_NONE>
__global__ void __launch_bounds__(SH::THREADS, MIXED ? (SH::MINB > 3 ? 3 : SH::MINB) : 2)
voigt_table_kernel(LinesDev L, GridDev g, const StateDev *__restrict__ states, TableSched sc,
                   void *ring, double *partial, unsigned *tile_cnt, unsigned long long *ticket,
                   unsigned long long *wbits, unsigned *prep_cnt, unsigned *sum_cnt,
                   unsigned *ready, TableFin *fin, int *err, double *__restrict__ K,
                   int64_t k_stride) {
  constexpr int G = SH::G, THREADS = SH::THREADS;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ long long s_ticket;
  __shared__ int s_go;
  __shared__ double s_e916[HK_SIG1_M];
  const int tid = threadIdx.x;
  const size_t rec_bytes = MIXED ? sizeof(LinePrepF) : sizeof(LinePrep);
  const int64_t n = L.n;
  if (tid < HK_SIG1_M) s_e916[tid] = c916_e(tid + 1);
  for (;;) {
    if (tid == 0) s_ticket = (long long)atomicAdd(ticket, 1ull);
    __syncthreads();
    const long long t = s_ticket;
    if (t >= sc.total) break;
    bool prep;
    int s;
    long long idx;
    table_ticket(sc, t, prep, s, idx);
    const int slot = s % sc.R;
    if (tid == 0) {
      bool go;
      if (prep) go = s < sc.R || wait_at_least(sum_cnt + (s - sc.R), (unsigned)sc.nsum, err);
      else go = wait_at_least(ready + s, 1u, err);
      s_go = go;
    }
    __syncthreads();
    const bool go = s_go;
    const StateDev &st = states[s];
    void *ring_s = static_cast<char *>(ring) + (size_t)slot * n * rec_bytes;
    if (prep) {
      double w_loc = 0.0, s1_loc = 0.0;
      if (go) {
        const int64_t l0 = idx * sc.lpt, l1 = min(l0 + (int64_t)sc.lpt, n);
        prep_lines<MIXED>(L, g, st, l0 + tid, l1, THREADS, s_e916, ring_s, w_loc, s1_loc);
      }
      for (int o = 16; o > 0; o >>= 1) {
        w_loc = fmax(w_loc, __shfl_xor_sync(0xffffffffu, w_loc, o));
        s1_loc = fmax(s1_loc, __shfl_xor_sync(0xffffffffu, s1_loc, o));
      }
      if ((tid & 31) == 0) {
        if (g.cutMode != 0) atomicMax(&wbits[2 * s], (unsigned long long)__double_as_longlong(w_loc));
        atomicMax(&wbits[2 * s + 1], (unsigned long long)__double_as_longlong(s1_loc));
      }
      __threadfence();
      __syncthreads();
      if (tid == 0 && atomicAdd(prep_cnt + s, 1u) == (unsigned)(sc.npb - 1)) {
        // the last prep ticket of the state: every other one has published
        __threadfence();
        TableFin f;
        state_scale(g, atomicAdd(&wbits[2 * s], 0ull), atomicAdd(&wbits[2 * s + 1], 0ull), f.wmax,
                    f.s1exp);
        f.pad = 0;
        fin[s] = f;
        __threadfence();
        st_release(ready + s, 1u);
      }
    } else {
      if (go) {
        const TableFin f = {__ldcg(&fin[s].wmax), __ldcg(&fin[s].s1exp), 0};
        const int tile = (int)(idx / sc.nsplit), part = (int)(idx - (long long)tile * sc.nsplit);
        const int64_t g0 = (int64_t)tile * G;
        const int64_t g1 = min(g0 + (int64_t)G, g.nx);
        const size_t tslot = (size_t)slot * sc.tps + tile;
        sum_tile<MIXED, SH, true, G34, EXT>(ring_s, L.nu0, n, g, st, f.wmax, f.s1exp, g0, g1, part, sc.nsplit,
                                  partial + tslot * sc.nsplit * G, tile_cnt + tslot,
                                  K + (int64_t)s * k_stride, smem_dyn);
      }
      // every record read of this ticket has completed: count it
      __threadfence();
      __syncthreads();
      if (tid == 0) atomicAdd(sum_cnt + s, 1u);
    }
  }
}

// ------------------------------------------------------ diagnostics kernels
__global__ void profile_eval_kernel(int64_t n, const double *__restrict__ x,
                                    const double *__restrict__ y, int mixed,
                                    double *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double ey = erfcx(y[i]);
  if (mixed) {
    // same table the Voigt kernel stages per line (padded like Rtab)
    float R[HK_RPAD + HK_C916_MR];
    const float Y = (float)(y[i] * y[i]);
    const float a2 = HK_A916_F * HK_A916_F;
    for (int m = 0; m < HK_RPAD; ++m) R[m] = 0.f;
    for (int m = 1; m <= HK_C916_MR; ++m) R[HK_RPAD + m - 1] = rcp_fast(fmaf(a2 * m, (float)m, Y));
    const float yf = (float)y[i];
    const float iy = yf > 0.f ? (float)(1.0 / (double)yf) : 0.f;
    out[i] = (double)voigt916_tab((float)x[i], yf, iy, (float)ey, (float)c916_sig1(y[i]),
                                  R + HK_RPAD);
  } else {
    out[i] = voigt916_d(x[i], y[i], ey);
  }
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread, every SM
// busy.  Gives the FP32 SIMT peak under the clocks of the current run (the
// roofline denominator of the Voigt sum).
__global__ void fma_peak_kernel(int iters, float seed, float *__restrict__ sink) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 1e-7f + k;
  const float m = 0.9999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == 123.456f) sink[blockIdx.x] = s;  // keeps the chains alive
}

cudaError_t measure_fp32_peak(double *tflops, cudaStream_t stream) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = nsm * 8, threads = 256, iters = 1 << 16;
  float *sink = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&sink, blocks * sizeof(float), stream);
  if (e != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fma_peak_kernel<<<blocks, threads, 0, stream>>>(iters / 8, 1.0f, sink);  // warm-up
  cudaEventRecord(a, stream);
  fma_peak_kernel<<<blocks, threads, 0, stream>>>(iters, 1.0f, sink);
  cudaEventRecord(b, stream);
  e = cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFreeAsync(sink, stream);
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  *tflops = (ms > 0.f) ? flops / (ms * 1e-3) / 1e12 : 0.0;
  return e != cudaSuccess ? e : cudaGetLastError();
}

// ------------------------------------------------------------- launchers
int voigt_num_shapes() { return HK_NSHAPES; }
int voigt_tile_points(int shape) { return HK_SHAPE_G[shape < 0 || shape >= HK_NSHAPES ? 0 : shape]; }
int voigt_chunk_lines(int shape) { return HK_SHAPE_CH[shape < 0 || shape >= HK_NSHAPES ? 0 : shape]; }
int voigt_tile_warps(int shape) { return HK_SHAPE_WARPS[shape < 0 || shape >= HK_NSHAPES ? 0 : shape]; }

// The option instantiation of the mixed form for a grid's options (the
// host runs sub-Lorentzian wings with plinth removal, and the Gaussian
// profiles with sub-Lorentzian wings, in the FP64 form).
static int ext_kind(const GridDev &g) {
  if (g.subL) return HK_EXT_CHI;
  if (g.plinth) return HK_EXT_PL;
  return HK_EXT_NONE;
}

// Calls f(kernel, dynamic shared memory) for the kernel of (precision,
// shape); the plain FP64 form has the default shape only.
template <class F>
static cudaError_t with_kernel(bool mixed, int shape, F &&f, bool g34 = false, int ext = HK_EXT_NONE) {
  using KFn = void (*)(const void *, const double *, int64_t, GridDev, const StateDev *, int, int,
                       int, int, unsigned *, double *, unsigned *, double *, int64_t);
  if (!mixed) return f((KFn)voigt_sum_kernel<false, Shape0>, sizeof(RecD) * Shape0::CH, Shape0::THREADS);
  if (g34 && ext == HK_EXT_PL)
    return f((KFn)voigt_sum_kernel<true, Shape0, true, HK_EXT_PL>, smem_mixed<Shape0, HK_EXT_PL>(),
             Shape0::THREADS);
  if (g34) return f((KFn)voigt_sum_kernel<true, Shape0, true>, smem_mixed<Shape0>(), Shape0::THREADS);
  if (ext == HK_EXT_CHI)
    return f((KFn)voigt_sum_kernel<true, Shape0, false, HK_EXT_CHI>, smem_mixed<Shape0, HK_EXT_CHI>(),
             Shape0::THREADS);
  if (ext == HK_EXT_PL)
    return f((KFn)voigt_sum_kernel<true, Shape0, false, HK_EXT_PL>, smem_mixed<Shape0, HK_EXT_PL>(),
             Shape0::THREADS);
  switch (shape) {
#define HK_SHAPE_CASE(n) \
  case n: return f((KFn)voigt_sum_kernel<true, Shape##n>, smem_mixed<Shape##n>(), Shape##n::THREADS);
    HK_SHAPE_CASE(0)
    HK_SHAPE_CASE(1)
    HK_SHAPE_CASE(2)
    HK_SHAPE_CASE(3)
    HK_SHAPE_CASE(4)
    HK_SHAPE_CASE(5)
    HK_SHAPE_CASE(6)
#undef HK_SHAPE_CASE
    default: return cudaErrorInvalidValue;
  }
}

static int voigt_ctas(bool mixed, int shape) {
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  with_kernel(mixed, shape, [&](auto kfn, size_t smem, int threads) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
  });
  return nsm * (per_sm < 1 ? 1 : per_sm);
}

// Tiles are split along their line range when a state has few tiles: one
// tile's sweep lasts ~1/3 of a 1e7-line state, so an unsplit 1465-tile grid
// ends in a last wave that leaves most of the GPU idle for that long.  The
// split depends on the grid and the tile shape only (HK_TICKETS_PER_STATE,
// about 8 tickets per resident CTA of a 148-SM B200 at 4 CTAs/SM), never on
// the batch or the device, so one state's K is bit-identical however it is
// batched.
constexpr int HK_TICKETS_PER_STATE = 4736;
constexpr int HK_MAX_SPLIT = 8;

int voigt_nsplit(int64_t nx, int shape) {
  const int G = voigt_tile_points(shape);
  const int64_t tps = (nx + G - 1) / G;
  if (tps <= 0) return 1;
  return (int)std::min<int64_t>(HK_MAX_SPLIT,
                                std::max<int64_t>(1, (HK_TICKETS_PER_STATE + tps - 1) / tps));
}

VoigtPlan plan_voigt_section(bool mixed, int shape, int64_t nx, int tile0, int ntiles, int grid_ctas) {
  VoigtPlan pl;
  pl.shape = mixed ? shape : 0;
  pl.G = voigt_tile_points(pl.shape);
  pl.tile0 = tile0;
  pl.tiles_per_state = ntiles;
  pl.tiles = ntiles;
  pl.ctas = grid_ctas > 0 ? grid_ctas : voigt_ctas(mixed, pl.shape);
  pl.nsplit = voigt_nsplit(nx, pl.shape);
  pl.partial_doubles = pl.nsplit > 1 ? (size_t)pl.tiles * pl.nsplit * pl.G : 0;
  pl.counters = pl.nsplit > 1 ? (size_t)pl.tiles : 0;
  return pl;
}

VoigtPlan plan_voigt_sum(bool mixed, int shape, int64_t nx, int nstates, int grid_ctas) {
  const int G = voigt_tile_points(mixed ? shape : 0);
  VoigtPlan pl = plan_voigt_section(mixed, shape, nx, 0, (int)((nx + G - 1) / G), grid_ctas);
  pl.tiles = (int64_t)pl.tiles_per_state * nstates;
  pl.partial_doubles = pl.nsplit > 1 ? (size_t)pl.tiles * pl.nsplit * pl.G : 0;
  pl.counters = pl.nsplit > 1 ? (size_t)pl.tiles : 0;
  return pl;
}

cudaError_t launch_voigt_sum(bool mixed, const VoigtPlan &pl, const void *prep_d,
                             const double *nu0_d, int64_t nlines, const GridDev &g,
                             const StateDev *states_d, unsigned *ticket_d, double *partial_d,
                             unsigned *tile_cnt_d, double *K_d, int64_t k_stride,
                             cudaStream_t stream) {
  const int64_t total64 = pl.tiles * pl.nsplit;
  if (total64 > 0x7fffffff) return cudaErrorInvalidValue;
  if (pl.G != voigt_tile_points(pl.shape)) return cudaErrorInvalidValue;
  if (mixed && (g.profile >= 3 || g.plinth || g.subL) && pl.shape != 0)
    return cudaErrorInvalidValue;  // shape 0 only
  const int total = (int)total64;
  cudaError_t e = cudaMemsetAsync(ticket_d, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  if (total <= 0) return cudaSuccess;
  if (pl.nsplit > 1) {
    if (!partial_d || !tile_cnt_d) return cudaErrorInvalidValue;
    e = cudaMemsetAsync(tile_cnt_d, 0, sizeof(unsigned) * pl.counters, stream);
    if (e != cudaSuccess) return e;
  }
  const int ctas = (int)std::min<int64_t>(pl.ctas, total);
  e = with_kernel(mixed, pl.shape, [&](auto kfn, size_t smem, int threads) {
    if (smem > 48 * 1024) {
      const cudaError_t ea = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (ea != cudaSuccess) return ea;
    }
    kfn<<<ctas, threads, smem, stream>>>(prep_d, nu0_d, nlines, g, states_d, pl.tile0,
                                            pl.tiles_per_state, pl.nsplit, total, ticket_d,
                                            partial_d, tile_cnt_d, K_d, k_stride);
    return cudaGetLastError();
  }, mixed && g.profile >= 3, mixed ? ext_kind(g) : HK_EXT_NONE);
  return e;
}

// The fused table kernel of (precision, shape) and its dynamic shared memory.
template <class F>
static cudaError_t with_table_kernel(bool mixed, int shape, F &&f, bool g34 = false, int ext = HK_EXT_NONE) {
  using KFn = void (*)(LinesDev, GridDev, const StateDev *, TableSched, void *, double *, unsigned *,
                       unsigned long long *, unsigned long long *, unsigned *, unsigned *, unsigned *,
                       TableFin *, int *, double *, int64_t);
  if (!mixed) return f((KFn)voigt_table_kernel<false, Shape0>, sizeof(RecD) * Shape0::CH, Shape0::THREADS);
  if (g34 && ext == HK_EXT_PL)
    return f((KFn)voigt_table_kernel<true, Shape0, true, HK_EXT_PL>, smem_mixed<Shape0, HK_EXT_PL>(),
             Shape0::THREADS);
  if (g34) return f((KFn)voigt_table_kernel<true, Shape0, true>, smem_mixed<Shape0>(), Shape0::THREADS);
  if (ext == HK_EXT_CHI)
    return f((KFn)voigt_table_kernel<true, Shape0, false, HK_EXT_CHI>, smem_mixed<Shape0, HK_EXT_CHI>(),
             Shape0::THREADS);
  if (ext == HK_EXT_PL)
    return f((KFn)voigt_table_kernel<true, Shape0, false, HK_EXT_PL>, smem_mixed<Shape0, HK_EXT_PL>(),
             Shape0::THREADS);
  switch (shape) {
#define HK_SHAPE_CASE(n) \
  case n: return f((KFn)voigt_table_kernel<true, Shape##n>, smem_mixed<Shape##n>(), Shape##n::THREADS);
    HK_SHAPE_CASE(0)
    HK_SHAPE_CASE(1)
    HK_SHAPE_CASE(2)
    HK_SHAPE_CASE(3)
    HK_SHAPE_CASE(4)
    HK_SHAPE_CASE(5)
    HK_SHAPE_CASE(6)
#undef HK_SHAPE_CASE
    default: return cudaErrorInvalidValue;
  }
}

TablePlan plan_table(bool mixed, int shape, int64_t nlines, int64_t nx, int nstates) {
  TablePlan tp;
  tp.shape = mixed ? shape : 0;
  tp.G = voigt_tile_points(tp.shape);
  tp.S = nstates;
  // the preps of state s run beside the sums of state s - 1; a third slot
  // gives the sums of state s - 3 a phase of slack before their slot is reused
  tp.R = 3;
  tp.slots = std::min(tp.R, nstates);
  tp.lpt = 4096;
  tp.npb = (int)std::max<int64_t>(1, (nlines + tp.lpt - 1) / tp.lpt);
  tp.tps = (int)((nx + tp.G - 1) / tp.G);
  tp.nsplit = voigt_nsplit(nx, tp.shape);
  tp.nsum = (long long)tp.tps * tp.nsplit;
  tp.total = (long long)nstates * (tp.npb + tp.nsum);
  tp.ring_bytes = (size_t)tp.slots * (size_t)std::max<int64_t>(nlines, 1) * (mixed ? sizeof(LinePrepF) : sizeof(LinePrep));
  tp.partial_doubles = tp.nsplit > 1 ? (size_t)tp.slots * tp.tps * tp.nsplit * tp.G : 0;
  tp.counters = (size_t)tp.slots * tp.tps;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  with_table_kernel(mixed, tp.shape, [&](auto kfn, size_t smem, int threads) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, threads, smem);
  });
  tp.ctas = nsm * (per_sm < 1 ? 1 : per_sm);
  return tp;
}

cudaError_t launch_voigt_table(bool mixed, const TablePlan &tp, const LinesDev &L, const GridDev &g,
                               const StateDev *states_d, const TableBufs &b, double *K_d,
                               int64_t k_stride, cudaStream_t stream) {
  if (tp.S < 1 || tp.R < 2 || tp.slots != std::min(tp.R, tp.S)) return cudaErrorInvalidValue;
  if (tp.G != voigt_tile_points(tp.shape)) return cudaErrorInvalidValue;
  if (mixed && (g.profile >= 3 || g.plinth || g.subL) && tp.shape != 0)
    return cudaErrorInvalidValue;  // shape 0 only
  if (tp.nsplit > 1 && !b.partial) return cudaErrorInvalidValue;
  // the counters, maxima and flags start from zero on every launch (replay)
  cudaError_t e = cudaMemsetAsync(b.sync, 0, table_sync_bytes(tp.S), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.tile_cnt, 0, sizeof(unsigned) * tp.counters, stream);
  if (e != cudaSuccess) return e;
  TableSched sc;
  sc.S = tp.S;
  sc.R = tp.R;
  sc.npb = tp.npb;
  sc.lpt = tp.lpt;
  sc.tps = tp.tps;
  sc.nsplit = tp.nsplit;
  sc.nsum = tp.nsum;
  sc.total = tp.total;
  // the sync block: ticket, wbits[2S], fin[S], prep_cnt[S], sum_cnt[S], ready[S], err
  char *q = static_cast<char *>(b.sync);
  unsigned long long *ticket = reinterpret_cast<unsigned long long *>(q);
  unsigned long long *wbits = ticket + 2;
  TableFin *fin = reinterpret_cast<TableFin *>(wbits + 2 * (size_t)tp.S);
  unsigned *prep_cnt = reinterpret_cast<unsigned *>(fin + tp.S);
  unsigned *sum_cnt = prep_cnt + tp.S;
  unsigned *ready = sum_cnt + tp.S;
  int *err = reinterpret_cast<int *>(ready + tp.S);
  const int ctas = (int)std::min<long long>(tp.ctas, tp.total);
  return with_table_kernel(mixed, tp.shape, [&](auto kfn, size_t smem, int threads) {
    if (smem > 48 * 1024) {
      const cudaError_t ea = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (ea != cudaSuccess) return ea;
    }
    kfn<<<ctas, threads, smem, stream>>>(L, g, states_d, sc, b.ring, b.partial, b.tile_cnt, ticket, wbits,
                                         prep_cnt, sum_cnt, ready, fin, err, K_d, k_stride);
    return cudaGetLastError();
  }, mixed && g.profile >= 3, mixed ? ext_kind(g) : HK_EXT_NONE);
}

int *table_error_word(void *sync_d, int nstates) {
  char *q = static_cast<char *>(sync_d);
  return reinterpret_cast<int *>(q + 16 + 16 * (size_t)nstates + sizeof(TableFin) * (size_t)nstates +
                                 12 * (size_t)nstates);
}

cudaError_t launch_profile_eval(int64_t n, const double *x_d, const double *y_d,
                                int mixed, double *out_d, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const int b = 128;
  profile_eval_kernel<<<(unsigned)((n + b - 1) / b), b, 0, stream>>>(n, x_d, y_d, mixed, out_d);
  return cudaGetLastError();
}

}  // namespace hkb
