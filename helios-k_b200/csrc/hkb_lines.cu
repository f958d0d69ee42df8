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
#include "hkb_prep.cuh"

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

// Per-line multipliers from load order into the nu-sorted order, dst[k] =
// src[order[k]], each checked to be finite and > 0: *bad ends as the
// smallest load index of a value that is not (n when all are).
__global__ void bad_init_kernel(unsigned long long *bad, int64_t n) { *bad = (unsigned long long)n; }

__global__ void gather_scales_kernel(int64_t n, const int64_t *__restrict__ order,
                                     const double *__restrict__ src, double *__restrict__ dst,
                                     unsigned long long *bad) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = order[k];
    const double v = src[j];
    dst[k] = v;
    if (!(v > 0.0 && v <= 1.7976931348623157e308)) atomicMin(bad, (unsigned long long)j);
  }
}

cudaError_t launch_gather_scales(int64_t n, const int64_t *order_d, const double *src_d,
                                 double *dst_d, unsigned long long *bad_d, cudaStream_t stream) {
  bad_init_kernel<<<1, 1, 0, stream>>>(bad_d, n);
  if (n > 0) gather_scales_kernel<<<1184, 256, 0, stream>>>(n, order_d, src_d, dst_d, bad_d);
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

// One thread per (line, state): the record of prep_record (hkb_prep.cuh) for
// every line of every state of a batch.  For cutMode 1/2 it also bounds the
// state's largest cutoff half-width (cm^-1), which sizes each tile's line
// search; and it takes the state's largest region-A/B term, which sets the
// power-of-two scale of the mixed form's FP32 sums.  wbits holds two words
// per state: {half-width bits, term bits} (both non-negative doubles, so
// their bit patterns order like the values).
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
  void *out_s = MODE == PREP_STATS ? nullptr
                                   : static_cast<char *>(out) + (size_t)s * L.n * (MIXED ? sizeof(LinePrepF) : sizeof(LinePrep));
  for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < L.n;
       l += (int64_t)gridDim.x * blockDim.x)
    prep_record<MIXED, MODE>(L, g, st, l, s_e916, out_s, w_loc, s1_loc);
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
  double wmax;
  int e;
  state_scale(g, wbits[2 * s], wbits[2 * s + 1], wmax, e);
  states[s].wmax = wmax;
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
