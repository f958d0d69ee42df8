// hkb_lines.cu -- line-list residency and the per-state line prep (sm_100a).
//
// The reference sorts every 2^20-line part by nu for every pressure
// (heliosk.cu:1147-1171: thrust::sort_by_key + six gather kernels) and
// rescales it with S2_kernel/S3_kernel (voigt.h:331-482).  Here the list is
// sorted once at load (CUB radix sort on the FP64 centres, one gather per
// column) and stays resident in HBM; line_prep_kernel then scales every line
// to every state of a batch in FP64 and computes its exact index windows,
// one thread per (line, state).  The per-state pressure shift is absorbed by
// widening each tile's line search by max|delta| P.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <climits>

#include "hkb_device.cuh"
#include "hkb_kernels.h"

namespace hkb {

__global__ void gather_kernel(int64_t n, const int64_t *__restrict__ order,
                              const double *__restrict__ src,
                              double *__restrict__ dst) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = src[order[k]];
}

__global__ void iota_kernel(int64_t n, int64_t *__restrict__ v) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    v[k] = k;
}

cudaError_t launch_gather_lines(int64_t n, const int64_t *order_d,
                                const double *src_d, double *dst_d,
                                cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  gather_kernel<<<1184, 256, 0, stream>>>(n, order_d, src_d, dst_d);
  return cudaGetLastError();
}

// Sorts nu_d in place (ascending) and returns the permutation in order_d.
cudaError_t sort_lines_by_nu(int64_t n, double *nu_d, int64_t *order_d,
                             cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  double *keys_out = nullptr;
  int64_t *idx_in = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  cudaError_t e = cudaMallocAsync((void **)&keys_out, n * sizeof(double), stream);
  if (e != cudaSuccess) return e;
  e = cudaMallocAsync((void **)&idx_in, n * sizeof(int64_t), stream);
  if (e != cudaSuccess) return e;
  iota_kernel<<<1184, 256, 0, stream>>>(n, idx_in);
  e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, nu_d, keys_out, idx_in,
                                      order_d, n, 0, 64, stream);
  if (e != cudaSuccess) return e;
  e = cudaMallocAsync(&tmp, tmp_bytes, stream);
  if (e != cudaSuccess) return e;
  e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, nu_d, keys_out, idx_in,
                                      order_d, n, 0, 64, stream);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(nu_d, keys_out, n * sizeof(double), cudaMemcpyDeviceToDevice, stream);
  cudaFreeAsync(tmp, stream);
  cudaFreeAsync(idx_in, stream);
  cudaFreeAsync(keys_out, stream);
  return e != cudaSuccess ? e : cudaGetLastError();
}

// One thread per (line, state): FP64 scaling (prep_line), the global index
// windows (line_windows over [0, Nx)), and the region-C per-line constants
// erfcx(y) and Sig1(y) for lines that have a region-C window.  For cutMode
// 1/2 it also bounds the state's largest cutoff half-width (cm^-1), which
// sizes each tile's line search; and it takes the state's largest region-A/B
// term, which sets the power-of-two scale of the mixed form's FP32 sums.
// wbits holds two words per state: {half-width bits, term bits} (both
// non-negative doubles, so their bit patterns order like the values).
// MODE: PREP_ALL writes the records and the per-state maxima; PREP_STATS only
// the maxima (the state pass of a sectioned state); PREP_RECORDS only the
// records (one section's lines, the state already finalised).
enum { PREP_ALL = 0, PREP_STATS = 1, PREP_RECORDS = 2 };

template <bool MIXED, int MODE>
__global__ void __launch_bounds__(256)
line_prep_kernel(LinesDev L, GridDev g, const StateDev *__restrict__ states,
                 void *__restrict__ out, unsigned long long *__restrict__ wbits) {
  const int s = blockIdx.y;
  const StateDev &st = states[s];
  __shared__ double s_e916[HK_SIG1_M];  // the line-independent terms of Sig1
  if (MODE != PREP_STATS && threadIdx.x < HK_SIG1_M) s_e916[threadIdx.x] = c916_e(threadIdx.x + 1);
  __syncthreads();
  double w_loc = 0.0, s1_loc = 0.0;
  for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < L.n;
       l += (int64_t)gridDim.x * blockDim.x) {
    const LineState ls = prep_line(L, st, l);
    int64_t w[6];
    line_windows(g, st, ls, 0, g.nx, w);
    // S1 per profile (S3_kernel voigt.h:452-463); the mixed form runs profiles 1-2
    const double Sc = ls.S * (1.0 / 1.7724538509055160273);
    const double S1 = (MIXED || g.profile <= 2) ? ls.S * ls.vy / CUDART_PI
                                                : (g.profile == 3 ? Sc : ls.S);
    const bool hasC = w[3] > w[2];
    // largest region-A/B term of the line: S1 / r^2 with r^2 >= max(100, y^2)
    // (Voigt: region C covers r < 10), r^2 >= y^2 for the Lorentz profile
    const double Y = ls.vy * ls.vy;
    const double rmin = g.profile == 2 ? Y : fmax(100.0, Y);
    const double term = rmin > 0.0 ? S1 / rmin : 0.0;
    if (MODE == PREP_STATS) {
    } else if (MIXED) {
      const double ey = hasC ? erfcx(ls.vy) : 1.0;
      const float sig1 = hasC ? (float)c916_sig1_tab(ls.vy, s_e916) : 0.f;
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
      if (w[5] > w[0]) {
        // the largest |x| inside the cut window (at its first or last point)
        const double xa = fabs((grid_x(g, w[0]) - ls.nu) * ls.iad);
        const double xb = fabs((grid_x(g, w[5] - 1) - ls.nu) * ls.iad);
        const double umax = fmax(xa, xb) * fmax(xa, xb) + Y;
        if (umax >= 1e18) flags |= HK_PF_WIDE;
        // (Lorentz: Y >= 2^-60 also keeps the product of two denominators,
        // >= Y^2, a normal float)
        if (rmin < 0x1p-64 * umax || Y > 0x1p60 || (g.profile == 2 && Y < 0x1p-60)) flags |= HK_PF_RANGE;
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
      reinterpret_cast<LinePrepF *>(out)[(int64_t)s * L.n + l] = r;
    } else {
      const double ey = hasC ? erfcx(ls.vy) : 1.0;
      const float sig1 = hasC ? (float)c916_sig1_tab(ls.vy, s_e916) : 0.f;
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
      r.pad = 0;
      r.plinth = (g.plinth && w[5] > w[0]) ? plinth_d(g, S1, Sc, ls.iad, ls.vy) : 0.0;
      reinterpret_cast<LinePrep *>(out)[(int64_t)s * L.n + l] = r;
    }
    if (w[5] > w[0]) s1_loc = fmax(s1_loc, term);
    if (ls.S != 0.0 && ls.iad > 0.0) {
      if (g.cutMode == 1) w_loc = fmax(w_loc, g.cut * ls.vy / ls.iad);
      else if (g.cutMode == 2) w_loc = fmax(w_loc, g.cut / ls.iad);
    }
  }
  if constexpr (MODE != PREP_RECORDS) {
    for (int o = 16; o > 0; o >>= 1) {
      w_loc = fmax(w_loc, __shfl_xor_sync(0xffffffffu, w_loc, o));
      s1_loc = fmax(s1_loc, __shfl_xor_sync(0xffffffffu, s1_loc, o));
    }
    if ((threadIdx.x & 31) == 0) {
      if (g.cutMode != 0) atomicMax(&wbits[2 * s], (unsigned long long)__double_as_longlong(w_loc));
      atomicMax(&wbits[2 * s + 1], (unsigned long long)__double_as_longlong(s1_loc));
    }
  }
}

__global__ void state_finalize_kernel(GridDev g, StateDev *__restrict__ states,
                                      int nstates,
                                      const unsigned long long *__restrict__ wbits) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nstates) return;
  if (g.cutMode == 0) {
    states[s].wmax = g.cut;
  } else {
    const double w = __longlong_as_double((long long)wbits[2 * s]);
    states[s].wmax = w * (1.0 + 1e-9) + 1e-300;
  }
  const double tmax = __longlong_as_double((long long)wbits[2 * s + 1]);
  int e = 0;
  if (tmax > 0.0 && isfinite(tmax)) {
    frexp(tmax, &e);  // tmax in [2^(e-1), 2^e)
    e = 40 - e;
  }
  states[s].s1scale = ldexp(1.0, e);
  states[s].s1unscale = ldexp(1.0, -e);
  states[s].s1exp = e;
}

// Exact (line, grid point) pair counts of one state by region, from the same
// windows the sums use: A = (b0 - i0) + (i1 - b1), B = (c0 - b0) + (b1 - c1),
// C = c1 - c0 (the algorithmic work of the Voigt sum).
__global__ void __launch_bounds__(256)
count_pairs_kernel(LinesDev L, GridDev g, const StateDev *__restrict__ st,
                   unsigned long long *__restrict__ out) {
  __shared__ unsigned long long sa[8], sb[8], sc[8];
  unsigned long long a = 0, b = 0, c = 0;
  for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < L.n;
       l += (int64_t)gridDim.x * blockDim.x) {
    const LineState ls = prep_line(L, *st, l);
    int64_t w[6];
    line_windows(g, *st, ls, 0, g.nx, w);
    a += (unsigned long long)((w[1] - w[0]) + (w[5] - w[4]));
    b += (unsigned long long)((w[2] - w[1]) + (w[4] - w[3]));
    c += (unsigned long long)(w[3] - w[2]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    sb[threadIdx.x >> 5] = b;
    sc[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) {
      a += sa[w];
      b += sb[w];
      c += sc[w];
    }
    atomicAdd(&out[0], a);
    atomicAdd(&out[1], b);
    atomicAdd(&out[2], c);
  }
}

cudaError_t launch_count_pairs(const LinesDev &L, const GridDev &g, const StateDev *state_d,
                               unsigned long long *out_d, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(out_d, 0, 3 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess || L.n == 0) return e;
  const int64_t nb = (L.n + 255) / 256;
  count_pairs_kernel<<<(unsigned)(nb < 4736 ? nb : 4736), 256, 0, stream>>>(L, g, state_d, out_d);
  return cudaGetLastError();
}

cudaError_t launch_line_prep(bool mixed, const LinesDev &L, const GridDev &g, StateDev *states_d,
                             int nstates, void *prep_d, unsigned long long *wbits_d,
                             cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(wbits_d, 0, 2 * nstates * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  if (L.n > 0) {
    const int64_t nb = (L.n + 255) / 256;
    const int bx = (int)(nb < 2368 ? nb : 2368);
    dim3 grid(bx, nstates);
    if (mixed)
      line_prep_kernel<true, PREP_ALL><<<grid, 256, 0, stream>>>(L, g, states_d, prep_d, wbits_d);
    else
      line_prep_kernel<false, PREP_ALL><<<grid, 256, 0, stream>>>(L, g, states_d, prep_d, wbits_d);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  state_finalize_kernel<<<(nstates + 127) / 128, 128, 0, stream>>>(g, states_d, nstates, wbits_d);
  return cudaGetLastError();
}

cudaError_t launch_state_stats(const LinesDev &L, const GridDev &g, StateDev *states_d,
                               int nstates, unsigned long long *wbits_d, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(wbits_d, 0, 2 * nstates * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  if (L.n > 0) {
    const int64_t nb = (L.n + 255) / 256;
    dim3 grid((unsigned)(nb < 2368 ? nb : 2368), nstates);
    line_prep_kernel<true, PREP_STATS><<<grid, 256, 0, stream>>>(L, g, states_d, nullptr, wbits_d);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  state_finalize_kernel<<<(nstates + 127) / 128, 128, 0, stream>>>(g, states_d, nstates, wbits_d);
  return cudaGetLastError();
}

cudaError_t launch_line_records(bool mixed, const LinesDev &L, const GridDev &g,
                                const StateDev *state_d, void *prep_d, cudaStream_t stream) {
  if (L.n == 0) return cudaSuccess;
  const int64_t nb = (L.n + 255) / 256;
  dim3 grid((unsigned)(nb < 2368 ? nb : 2368), 1);
  if (mixed)
    line_prep_kernel<true, PREP_RECORDS><<<grid, 256, 0, stream>>>(L, g, state_d, prep_d, nullptr);
  else
    line_prep_kernel<false, PREP_RECORDS><<<grid, 256, 0, stream>>>(L, g, state_d, prep_d, nullptr);
  return cudaGetLastError();
}

// first index of each query value in the ascending array a (lower bound)
__global__ void lower_bound_kernel(const double *__restrict__ a, int64_t n,
                                   const double *__restrict__ q, int m, int64_t *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double v = q[i];
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  out[i] = lo;
}

cudaError_t launch_lower_bound(const double *a_d, int64_t n, const double *q_d, int m,
                               int64_t *out_d, cudaStream_t stream) {
  if (m <= 0) return cudaSuccess;
  lower_bound_kernel<<<(m + 127) / 128, 128, 0, stream>>>(a_d, n, q_d, m, out_d);
  return cudaGetLastError();
}

// Diagnostics: per-line state and global windows with the exact FP64 S.
__global__ void prep_dump_kernel(LinesDev L, GridDev g, StateDev st,
                                 double *__restrict__ out4,
                                 long long *__restrict__ win6) {
  const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L.n) return;
  const LineState ls = prep_line(L, st, l);
  out4[4 * l + 0] = ls.nu;
  out4[4 * l + 1] = ls.S;
  out4[4 * l + 2] = ls.iad;
  out4[4 * l + 3] = ls.vy;
  int64_t w[6];
  line_windows(g, st, ls, 0, g.nx, w);
  for (int k = 0; k < 6; ++k) win6[6 * l + k] = w[k];
}

cudaError_t launch_prep_dump(const LinesDev &L, const GridDev &g,
                             const StateDev &st, double *out4_d,
                             long long *win6_d, cudaStream_t stream) {
  if (L.n == 0) return cudaSuccess;
  const int b = 128;
  const int64_t nb = (L.n + b - 1) / b;
  prep_dump_kernel<<<(unsigned)nb, b, 0, stream>>>(L, g, st, out4_d, win6_d);
  return cudaGetLastError();
}

}  // namespace hkb
