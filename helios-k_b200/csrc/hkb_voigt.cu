// hkb_voigt.cu -- the Voigt line sum onto the wavenumber grid (sm_100a).
//
// One persistent kernel walks (state, grid tile) tickets.  A CTA owns a tile
// of HK_G consecutive grid points, so every output point has exactly one
// writer: there are no atomics on K and no partial-row reduction (the
// reference's 32 KS_d rows + AddKStreams_kernel, voigt.h:728-742, are gone).
// For its tile the CTA
//   1. finds the nu-sorted line range whose cutoff windows can reach the tile
//      (warp-parallel lower_bound),
//   2. stages the lines in chunks of HK_CH through shared memory: each thread
//      loads one line's state record (FP64 parameters and global index
//      windows, written by line_prep_kernel), clips the windows to the tile
//      and forms the line-centre offset at the tile start,
//   3. lets each warp sweep its 256-point slice against every staged line:
//      lane-interleaved points (coalesced stores), register accumulators.
// Two precisions share the structure:
//   MIXED: FP32 profile (the offset x from a double-float split of the FP64
//          line-centre offset; region formulas in FP32), strength multiply
//          and grid sum as one FP64 FMA per pair.
//   PLAIN: FP64 everywhere (the "plain FP64 form" used as the GPU baseline).
// Reference: Line6fA/B/C kernels voigt.h:1177-1816 and their launchers
// Line6A_Call/Line6B_Call/Line6C_Call voigt.h:1820-2036.
#include <cuda_runtime.h>

#include <cstdio>
#include <type_traits>

#include "hkb_device.cuh"
#include "hkb_kernels.h"

namespace hkb {

constexpr int HK_WARPS = 8;
constexpr int HK_THREADS = HK_WARPS * 32;
constexpr int HK_PPL = 8;                    // points per lane
constexpr int HK_SLICE = 32 * HK_PPL;        // points per warp
constexpr int HK_G = HK_WARPS * HK_SLICE;    // points per tile (2048)
constexpr int HK_CH = 128;                   // lines per staged chunk
static_assert(HK_G <= 2048, "k * vb_hi must stay exact in FP32 (11 bits)");

// Staged line record of the mixed form.  The FP32 line constants are stored
// twice ({v, v}) so the packed f32x2 sweep (two grid points per
// instruction) reads them as ready-made float2 operands.
struct __align__(16) RecF {
  float2 dh, dl;           // x at the tile start (hi, lo)
  float2 vbh, vbl;         // x step per grid point (hi, lo)
  float2 Y, A1;            // Y = y^2 and the region-B Horner coefficients
  float2 B1, A2;
  float2 B2;
  double S1, Sc;           // S*y/pi (regions A, B), S/sqrt(pi) (region C)
  float y, ey, sig1;       // y, erfcx(y), region-C series constant
  int i0, b0, c0, c1, b1;  // tile-local window boundaries
  int i1;
};
static_assert(sizeof(RecF) == 128, "RecF layout");

// Shared memory of one mixed-form CTA: staged records, the per-line
// region-C denominator tables (8 leading pad floats keep R[m-1-k] of the
// first line in bounds for predicated reads), and a per-point FP64
// accumulator for the region-C contributions.
constexpr int HK_RPAD = 8;
constexpr size_t HK_SMEM_MIXED = sizeof(RecF) * HK_CH +
                                 sizeof(float) * (HK_RPAD + HK_CH * HK_C916_MR) +
                                 sizeof(double) * HK_G;

struct __align__(16) RecD {
  double nu, iad, y2, y, S1, Sc, ey, pad;
  int i0, b0, c0, c1, b1, i1, p0, p1;
};

// Exact widening of a positive normal float to double with integer ops
// (keeps the conversion off the XU pipe that rcp.approx already uses).
__device__ __forceinline__ double widen_pos(float f) {
  const unsigned u = __float_as_uint(f);
  const unsigned lo = u << 29;
  const unsigned hi = (u >> 3) + (896u << 20);
  return __hiloint2double((int)hi, (int)lo);
}

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

// Clip one line's global windows to the tile [g0, g1) and fill the staged
// record.  Clipping the oracle's global boundaries equals searching the
// clipped range, because every window predicate is monotone on its range.
template <bool MIXED>
__device__ __forceinline__ void stage_line(const LinePrep *__restrict__ P,
                                           const GridDev &g, int64_t l,
                                           int64_t g0, int64_t g1, void *recp,
                                           float *__restrict__ Rtab) {
  const LinePrep lp = P[l];
  int li[6] = {clip_local(lp.i0, g0, g1), clip_local(lp.b0, g0, g1),
               clip_local(lp.c0, g0, g1), clip_local(lp.c1, g0, g1),
               clip_local(lp.b1, g0, g1), clip_local(lp.i1, g0, g1)};
  const bool nonempty = li[5] > li[0];
  if (MIXED) {
    RecF r;
    const double D0 = __dmul_rn(__dsub_rn(grid_x(g, g0), lp.nu), lp.iad);
    const double vb = __dmul_rn(g.dnu, lp.iad);
    const float dh = (float)D0;
    const float dl = (float)(D0 - (double)dh);
    const float vbh = __uint_as_float(__float_as_uint((float)vb) & 0xFFFFF800u);  // 13 bits
    const float vbl = (float)(vb - (double)vbh);
    const double Y = lp.vy * lp.vy;
    const float Yf = (float)Y;
    const float A1 = (float)(2.0 * Y + 2.5 - 4.0 / CUDART_PI);
    const float B1 = (float)((Y + 1.5) * (Y + 1.0));
    const float A2 = (float)(2.0 * Y + 3.0 - 6.0 / CUDART_PI);
    const float B2 = (float)((Y + 1.5) * (Y + 1.5));
    r.dh = make_float2(dh, dh);
    r.dl = make_float2(dl, dl);
    r.vbh = make_float2(vbh, vbh);
    r.vbl = make_float2(vbl, vbl);
    r.Y = make_float2(Yf, Yf);
    r.A1 = make_float2(A1, A1);
    r.B1 = make_float2(B1, B1);
    r.A2 = make_float2(A2, A2);
    r.B2 = make_float2(B2, B2);
    r.y = (float)lp.vy;
    r.S1 = lp.S1;
    r.Sc = lp.Sc;
    r.ey = (float)lp.ey;
    r.sig1 = lp.sig1;
    if (li[3] > li[2]) {
      // region C inside this tile: denominators of the Algorithm-916 series
      const float a2 = HK_A916_F * HK_A916_F;
#pragma unroll 2
      for (int m = 1; m <= HK_C916_MR; ++m) Rtab[m - 1] = rcp_fast(fmaf(a2 * m, (float)m, Yf));
    }
    r.i0 = nonempty ? li[0] : 0;
    r.b0 = li[1];
    r.c0 = li[2];
    r.c1 = li[3];
    r.b1 = li[4];
    r.i1 = nonempty ? li[5] : 0;
    *reinterpret_cast<RecF *>(recp) = r;
  } else {
    RecD r;
    r.nu = lp.nu;
    r.iad = lp.iad;
    r.y = lp.vy;
    r.y2 = lp.vy * lp.vy;
    r.S1 = lp.S1;
    r.Sc = lp.Sc;
    r.ey = lp.ey;
    r.pad = 0.0;
    r.i0 = nonempty ? li[0] : 0;
    r.b0 = li[1];
    r.c0 = li[2];
    r.c1 = li[3];
    r.b1 = li[4];
    r.i1 = nonempty ? li[5] : 0;
    r.p0 = r.p1 = 0;
    *reinterpret_cast<RecD *>(recp) = r;
  }
}

// ------------------------------------------------------------ FP32 sweep
// Region B rational in Horner form with per-line coefficients:
//   t4 = (s (s + A1) + B1) / ((s + Y) (s (s + A2) + B2)),  s = x^2,
//   A1 = 2Y + 2.5 - 4/pi, B1 = (Y+1.5)(Y+1), A2 = 2Y + 3 - 6/pi, B2 = (Y+1.5)^2;
// all terms positive, so no cancellation.
__device__ __forceinline__ float gh2_h(float s, const RecF &r) {
  const float num = fmaf(s, s + r.A1.x, r.B1.x);
  const float q = fmaf(s, s + r.A2.x, r.B2.x);
  return num * rcp_fast((s + r.Y.x) * q);
}

// x at two grid points (kf2 = {k, k + 32}) from the double-float split
__device__ __forceinline__ float2 x_pair(float2 kf2, const RecF &r) {
  return __fadd2_rn(__ffma2_rn(kf2, r.vbh, r.dh), __ffma2_rn(kf2, r.vbl, r.dl));
}

// region-B t4 at two grid points, packed f32x2 (same Horner form as gh2_h)
__device__ __forceinline__ float2 gh2_pair(float2 x, const RecF &r) {
  const float2 s = __fmul2_rn(x, x);
  const float2 num = __ffma2_rn(s, __fadd2_rn(s, r.A1), r.B1);
  const float2 q = __ffma2_rn(s, __fadd2_rn(s, r.A2), r.B2);
  const float2 den = __fmul2_rn(__fadd2_rn(s, r.Y), q);
  return __fmul2_rn(num, make_float2(rcp_fast(den.x), rcp_fast(den.y)));
}

// The profile shape (x, region formula) is FP32; the strength multiply and
// the grid sum are one FP64 FMA, so one state's opacity may span the full
// FP64 range (the strongest lines of a list can exceed the typical opacity
// by more than the FP32 exponent range).
//
// Each warp classifies the staged lines against its 256-point slice, 32
// lines per instruction (one lane per line), and sweeps them by class:
//   HK_CLS_B  slice inside the cut window and inside one region-B part,
//   HK_CLS_A  slice inside the cut window and inside one region-A part,
//   HK_CLS_G  anything else that intersects the slice (window edges,
//             region boundaries, region C),
// so the specialised loops carry no per-pair tests and non-intersecting
// lines cost nothing.  Region-C points are evaluated in a rolled loop and
// summed into the per-point shared accumulator cacc (each point has one
// owning lane: deterministic).
enum { HK_CLS_SKIP = 0, HK_CLS_B = 1, HK_CLS_A = 2, HK_CLS_G = 3 };

__device__ __forceinline__ int classify(const RecF &r, int wb) {
  const int we = wb + HK_SLICE;
  if (r.i1 <= wb || r.i0 >= we) return HK_CLS_SKIP;
  const bool full = r.i0 <= wb && r.i1 >= we;
  if (full && ((r.b0 <= wb && r.c0 >= we) || (r.c1 <= wb && r.b1 >= we))) return HK_CLS_B;
  if (full && (r.b0 >= we || r.b1 <= wb)) return HK_CLS_A;
  return HK_CLS_G;
}

// region B only, two points per packed instruction; the record's first 80
// bytes are read as five 16-byte words
__device__ __forceinline__ void sweep_B(const RecF &rr, const float2 (&kf)[HK_PPL / 2],
                                        double (&acc)[HK_PPL]) {
  const float4 *w = reinterpret_cast<const float4 *>(&rr);
  const float4 w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
  const double S1 = rr.S1;
  const float2 dh = make_float2(w0.x, w0.y), dl = make_float2(w0.z, w0.w);
  const float2 vbh = make_float2(w1.x, w1.y), vbl = make_float2(w1.z, w1.w);
  const float2 Y = make_float2(w2.x, w2.y), A1 = make_float2(w2.z, w2.w);
  const float2 B1 = make_float2(w3.x, w3.y), A2 = make_float2(w3.z, w3.w);
  const float2 B2 = rr.B2;
#pragma unroll
  for (int q = 0; q < HK_PPL / 2; ++q) {
    const float2 x = __fadd2_rn(__ffma2_rn(kf[q], vbh, dh), __ffma2_rn(kf[q], vbl, dl));
    const float2 s = __fmul2_rn(x, x);
    const float2 num = __ffma2_rn(s, __fadd2_rn(s, A1), B1);
    const float2 qq = __ffma2_rn(s, __fadd2_rn(s, A2), B2);
    const float2 den = __fmul2_rn(__fadd2_rn(s, Y), qq);
    const float2 t = __fmul2_rn(num, make_float2(rcp_fast(den.x), rcp_fast(den.y)));
    acc[2 * q] = fma(S1, widen_pos(t.x), acc[2 * q]);
    acc[2 * q + 1] = fma(S1, widen_pos(t.y), acc[2 * q + 1]);
  }
}

// region A only
__device__ __forceinline__ void sweep_A(const RecF &rr, const float2 (&kf)[HK_PPL / 2],
                                        double (&acc)[HK_PPL]) {
  const float4 *w = reinterpret_cast<const float4 *>(&rr);
  const float4 w0 = w[0], w1 = w[1];
  const float2 Y = rr.Y;
  const double S1 = rr.S1;
  const float2 dh = make_float2(w0.x, w0.y), dl = make_float2(w0.z, w0.w);
  const float2 vbh = make_float2(w1.x, w1.y), vbl = make_float2(w1.z, w1.w);
#pragma unroll
  for (int q = 0; q < HK_PPL / 2; ++q) {
    const float2 x = __fadd2_rn(__ffma2_rn(kf[q], vbh, dh), __ffma2_rn(kf[q], vbl, dl));
    const float2 u = __ffma2_rn(x, x, Y);  // unbounded: separate reciprocals
    acc[2 * q] = fma(S1, widen_pos(rcp_fast(u.x)), acc[2 * q]);
    acc[2 * q + 1] = fma(S1, widen_pos(rcp_fast(u.y)), acc[2 * q + 1]);
  }
}

// everything else: per-point window/region tests, region C deferred
__device__ __forceinline__ void sweep_G(const RecF &r, const float *__restrict__ Rj,
                                     double *__restrict__ cacc, int wb, int lane,
                                     const float2 (&kf)[HK_PPL / 2], double (&acc)[HK_PPL]) {
  const int we = wb + HK_SLICE;
  {
#pragma unroll
    for (int p = 0; p < HK_PPL; ++p) {
      const int k = wb + lane + 32 * p;
      if (k >= r.i0 && k < r.i1 && !(k >= r.c0 && k < r.c1)) {
        const float kk = (p & 1) ? kf[p >> 1].y : kf[p >> 1].x;
        const float x = fmaf(kk, r.vbh.x, r.dh.x) + fmaf(kk, r.vbl.x, r.dl.x);
        const float s = x * x;
        const float t = (k >= r.b0 && k < r.b1) ? gh2_h(s, r) : rcp_fast(s + r.Y.x);
        acc[p] = fma(r.S1, widen_pos(t), acc[p]);
      }
    }
    const int lo = max(r.c0, wb), hi = min(r.c1, we);
    if (lo < hi) {
      for (int pp = (lo - wb) >> 5; pp <= (hi - 1 - wb) >> 5; ++pp) {
        const int k = wb + lane + 32 * pp;
        if (k >= lo && k < hi) {
          const float kk = (float)k;
          const float x = fmaf(kk, r.vbh.x, r.dh.x) + fmaf(kk, r.vbl.x, r.dl.x);
          cacc[k] = fma(r.Sc, (double)voigt916_tab(x, r.y, r.ey, r.sig1, Rj), cacc[k]);
        }
      }
    }
  }
}

// ------------------------------------------------------------ FP64 sweep
__device__ __forceinline__ void sweep_plain(const RecD &r, int wb, int lane,
                                            const double (&xg)[HK_PPL],
                                            double (&acc)[HK_PPL]) {
  const int we = wb + HK_SLICE;
  if (r.i1 <= wb || r.i0 >= we) return;
  const bool full = r.i0 <= wb && r.i1 >= we;
  if (full && ((r.b0 <= wb && r.c0 >= we) || (r.c1 <= wb && r.b1 >= we))) {
#pragma unroll
    for (int p = 0; p < HK_PPL; ++p) {
      const double x = (xg[p] - r.nu) * r.iad;
      acc[p] += r.S1 * gh2_d(x, r.y2);
    }
  } else if (full && (r.b0 >= we || r.b1 <= wb)) {
#pragma unroll
    for (int p = 0; p < HK_PPL; ++p) {
      const double x = (xg[p] - r.nu) * r.iad;
      acc[p] += r.S1 / (x * x + r.y2);
    }
  } else {
#pragma unroll
    for (int p = 0; p < HK_PPL; ++p) {
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

// ------------------------------------------------------- persistent kernel
// mixed form: 4 CTAs (32 warps) per SM fit in 64 registers without spills
template <bool MIXED>
__global__ void __launch_bounds__(HK_THREADS, MIXED ? 4 : 2)
voigt_sum_kernel(const LinePrep *__restrict__ prep, const double *__restrict__ nu0,
                 int64_t nlines, GridDev g, const StateDev *__restrict__ states,
                 int tiles_per_state, int total_tickets, unsigned *__restrict__ ticket,
                 double *__restrict__ K, int64_t k_stride) {
  using Rec = typename std::conditional<MIXED, RecF, RecD>::type;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  Rec *rec = reinterpret_cast<Rec *>(smem_dyn);
  float *Rtab = reinterpret_cast<float *>(smem_dyn + sizeof(Rec) * HK_CH) + HK_RPAD;
  double *cacc = reinterpret_cast<double *>(smem_dyn + sizeof(Rec) * HK_CH +
                                            sizeof(float) * (HK_RPAD + HK_CH * HK_C916_MR));
  __shared__ int s_ticket;
  __shared__ long long s_L0, s_L1;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wb = warp * HK_SLICE;

  for (;;) {
    if (tid == 0) s_ticket = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int t = s_ticket;
    if (t >= total_tickets) break;
    const int s = t / tiles_per_state;
    const int tile = t - s * tiles_per_state;
    const StateDev &st = states[s];
    const LinePrep *P = prep + (int64_t)s * nlines;
    const int64_t g0 = (int64_t)tile * HK_G;
    const int64_t g1 = min(g0 + (int64_t)HK_G, g.nx);
    if (warp == 0) {
      const double W = st.wmax + st.shift + 2.0 * g.dnu;
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

    float2 kf[HK_PPL / 2];  // lane-local point indices, paired {p, p+1}
    double acc[HK_PPL], xg[HK_PPL];
#pragma unroll
    for (int p = 0; p < HK_PPL; ++p) {
      const int k = wb + lane + 32 * p;
      acc[p] = 0.0;
      if (MIXED) {
        if (p & 1) kf[p >> 1].y = (float)k;
        else kf[p >> 1].x = (float)k;
        cacc[k] = 0.0;  // owned by this lane only: no barrier needed
      } else {
        xg[p] = grid_x(g, g0 + k);
      }
    }

    // Chunk c holds the lines L0 + c + q*nch (q < HK_CH): every chunk spans
    // the tile's whole line range, so the costly region-C points of its
    // lines fall into all warp slices instead of one or two (consecutive
    // nu-sorted lines would put a chunk's line cores into a single slice
    // and leave the other warps idle at the barrier).
    const int64_t nL = L1 - L0;
    const int64_t nch = (nL + HK_CH - 1) / HK_CH;
    for (int64_t c = 0; c < nch; ++c) {
      const int cnt = (int)((nL - c + nch - 1) / nch);
      if (tid < cnt)
        stage_line<MIXED>(P, g, L0 + c + (int64_t)tid * nch, g0, g1, &rec[tid],
                          Rtab + tid * HK_C916_MR);
      __syncthreads();
      if (MIXED) {
        const RecF *rf = reinterpret_cast<const RecF *>(rec);
        for (int g32 = 0; g32 < cnt; g32 += 32) {
          const int j = g32 + lane;
          const int cls = (j < cnt) ? classify(rf[j], wb) : HK_CLS_SKIP;
          unsigned mB = __ballot_sync(0xffffffffu, cls == HK_CLS_B);
          unsigned mA = __ballot_sync(0xffffffffu, cls == HK_CLS_A);
          unsigned mG = __ballot_sync(0xffffffffu, cls == HK_CLS_G);
          while (mB) {
            const int b = __ffs(mB) - 1;
            mB &= mB - 1;
            sweep_B(rf[g32 + b], kf, acc);
          }
          while (mA) {
            const int b = __ffs(mA) - 1;
            mA &= mA - 1;
            sweep_A(rf[g32 + b], kf, acc);
          }
          while (mG) {
            const int b = __ffs(mG) - 1;
            mG &= mG - 1;
            sweep_G(rf[g32 + b], Rtab + (g32 + b) * HK_C916_MR, cacc, wb, lane, kf, acc);
          }
        }
      } else {
        for (int j = 0; j < cnt; ++j)
          sweep_plain(reinterpret_cast<const RecD &>(rec[j]), wb, lane, xg, acc);
      }
      __syncthreads();
    }

    double *Ks = K + (int64_t)s * k_stride;
#pragma unroll
    for (int p = 0; p < HK_PPL; ++p) {
      const int k = wb + lane + 32 * p;
      const int64_t gi = g0 + k;
      if (MIXED) acc[p] += cacc[k];
      if (gi < g1) Ks[gi] = st.kmin + acc[p];
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
    out[i] = (double)voigt916_tab((float)x[i], (float)y[i], (float)ey, (float)c916_sig1(y[i]),
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
int voigt_tile_points() { return HK_G; }

cudaError_t launch_voigt_sum(bool mixed, const LinePrep *prep_d, const double *nu0_d,
                             int64_t nlines, const GridDev &g, const StateDev *states_d,
                             int nstates, unsigned *ticket_d, double *K_d, int64_t k_stride,
                             int grid_ctas, cudaStream_t stream) {
  const int tps = (int)((g.nx + HK_G - 1) / HK_G);
  const int total = tps * nstates;
  cudaError_t e = cudaMemsetAsync(ticket_d, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  if (total <= 0) return cudaSuccess;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = mixed ? HK_SMEM_MIXED : sizeof(RecD) * HK_CH;
  if (mixed) {
    e = cudaFuncSetAttribute(voigt_sum_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, voigt_sum_kernel<true>, HK_THREADS, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, voigt_sum_kernel<false>, HK_THREADS, smem);
  }
  if (per_sm < 1) per_sm = 1;
  int ctas = grid_ctas > 0 ? grid_ctas : nsm * per_sm;
  if (ctas > total) ctas = total;
  if (mixed)
    voigt_sum_kernel<true><<<ctas, HK_THREADS, smem, stream>>>(prep_d, nu0_d, nlines, g, states_d,
                                                               tps, total, ticket_d, K_d, k_stride);
  else
    voigt_sum_kernel<false><<<ctas, HK_THREADS, smem, stream>>>(prep_d, nu0_d, nlines, g, states_d,
                                                                tps, total, ticket_d, K_d, k_stride);
  return cudaGetLastError();
}

cudaError_t launch_profile_eval(int64_t n, const double *x_d, const double *y_d,
                                int mixed, double *out_d, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const int b = 128;
  profile_eval_kernel<<<(unsigned)((n + b - 1) / b), b, 0, stream>>>(n, x_d, y_d, mixed, out_d);
  return cudaGetLastError();
}

}  // namespace hkb
