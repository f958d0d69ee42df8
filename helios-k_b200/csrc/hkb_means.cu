// hkb_means.cu -- Planck / Rosseland mean opacities and the transmission
// function of the binned opacity (sm_100a), FP64.
//
// Means (resample.h:635-773, Mean_kernel + IntegrateMean_kernel, equal
// spacing): per state, over the grid,
//   S0 = sum B K,  S1 = sum (dB/dT) / K (K != 0),  S2 = sum B,  S3 = sum dB/dT,
// plus the reference's end weights; Planck mean = S0 / S2, Rosseland mean =
// S3 / S1.  B and dB/dT are formed per point inside the reduction (the
// reference writes them to two Nx arrays first), so one pass reads K once:
// means_partial_kernel sums grid chunks, means_final_kernel adds the chunks
// in a fixed order and the end weights (deterministic).
//
// Transmission (resample.h:541-608, Integrate_kernel): per (state, bin) and
// m_j = exp((j - nTr/2) dTr),
//   Tr_j = (sum_k exp(-K_k m_j) + end weights) / (Nxb - 1) (Nxb - Nxmin) / Nxb
//          + exp(-kmin m_j) Nxmin / Nxb.
// One CTA per (state, bin) stages the bin in shared memory once; each warp
// takes values j and sums its exponentials lane-strided with a shuffle tree
// (no block barrier per j, where the reference reduces 512 threads per j).
#include <cuda_runtime.h>

#include <algorithm>

#include "hkb_device.cuh"
#include "hkb_kernels.h"

namespace hkb {

// resample.h:611-619: index idy gets w[idy], index n-1-idy gets w[2-idy]
__constant__ double c_wS[3] = {-5.0 / 8.0, 1.0 / 6.0, -1.0 / 24.0};

// Mean_kernel's Planck function and its T derivative, same operations
__device__ __forceinline__ void planck_bd(double nu, double T, double &B, double &R) {
  if (nu == 0.0) {
    B = 0.0;
    R = 0.0;
    return;
  }
  const double nu3 = __dmul_rn(__dmul_rn(nu, nu), nu);
  const double t1 = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, HK_H), nu3), HK_C), HK_C);
  const double t2 = __ddiv_rn(__dmul_rn(__dmul_rn(HK_H, nu), HK_C), __dmul_rn(HK_KB, T));
  const double e = exp(t2);
  B = __ddiv_rn(t1, __dsub_rn(e, 1.0));
  R = __ddiv_rn(__dmul_rn(t1, t2), __dmul_rn(T, __dadd_rn(__dsub_rn(e, 2.0), __ddiv_rn(1.0, e))));
}

constexpr int MN_THREADS = 256;

__global__ void __launch_bounds__(MN_THREADS)
means_partial_kernel(const double *__restrict__ K, int64_t k_stride, GridDev g,
                     const double *__restrict__ T, int nchunk, double *__restrict__ part) {
  const int s = blockIdx.y, c = blockIdx.x;
  const double Ts = T[s];
  const double *Ks = K + (int64_t)s * k_stride;
  const int64_t per = (g.nx + nchunk - 1) / nchunk;
  const int64_t i0 = (int64_t)c * per, i1 = min(i0 + per, g.nx);
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t i = i0 + threadIdx.x; i < i1; i += MN_THREADS) {
    double B, R;
    planck_bd(grid_x(g, i), Ts, B, R);
    const double k = Ks[i];
    a[0] = __fma_rn(B, k, a[0]);
    if (k != 0.0) a[1] = __dadd_rn(a[1], __ddiv_rn(R, k));
    a[2] = __dadd_rn(a[2], B);
    a[3] = __dadd_rn(a[3], R);
  }
  __shared__ double red[4][MN_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double v = a[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int k = 0; k < MN_THREADS / 32; ++k) v += red[threadIdx.x][k];
    part[((int64_t)s * nchunk + c) * 4 + threadIdx.x] = v;
  }
}

__global__ void means_final_kernel(const double *__restrict__ K, int64_t k_stride, GridDev g,
                                   const double *__restrict__ T, int nchunk,
                                   const double *__restrict__ part, double *__restrict__ out) {
  const int s = blockIdx.x, q = threadIdx.x;
  if (q >= 4) return;
  double v = 0.0;
  for (int c = 0; c < nchunk; ++c) v += part[((int64_t)s * nchunk + c) * 4 + q];
  const double *Ks = K + (int64_t)s * k_stride;
  const int64_t n = g.nx;
  for (int idy = 0; idy < 3 && n >= 3; ++idy) {
    const int64_t ia[2] = {idy, n - 1 - idy};
    const double wt[2] = {c_wS[idy], c_wS[2 - idy]};
    for (int e = 0; e < 2; ++e) {
      double B, R;
      planck_bd(grid_x(g, ia[e]), T[s], B, R);
      const double k = Ks[ia[e]];
      if (q == 0) v = __dadd_rn(v, __dmul_rn(wt[e], __dmul_rn(B, k)));
      if (q == 1 && k != 0.0) v = __dadd_rn(v, __dmul_rn(wt[e], __ddiv_rn(R, k)));
      if (q == 2) v = __dadd_rn(v, __dmul_rn(wt[e], B));
      if (q == 3) v = __dadd_rn(v, __dmul_rn(wt[e], R));
    }
  }
  out[(int64_t)s * 4 + q] = v;
}

size_t means_scratch_doubles(int nstates, int64_t nx) {
  const int nchunk = (int)std::min<int64_t>(592, std::max<int64_t>(1, nx / 4096));
  return (size_t)nstates * nchunk * 4;
}

cudaError_t launch_means(const double *K_d, int64_t k_stride, const GridDev &g, const double *T_d,
                         int nstates, double *scratch_d, double *out_d, cudaStream_t stream) {
  if (nstates <= 0 || g.nx <= 0) return cudaSuccess;
  const int nchunk = (int)std::min<int64_t>(592, std::max<int64_t>(1, g.nx / 4096));
  dim3 grid(nchunk, nstates);
  means_partial_kernel<<<grid, MN_THREADS, 0, stream>>>(K_d, k_stride, g, T_d, nchunk, scratch_d);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  means_final_kernel<<<nstates, 32, 0, stream>>>(K_d, k_stride, g, T_d, nchunk, scratch_d, out_d);
  return cudaGetLastError();
}

// ------------------------------------------------------------ transmission
constexpr int TR_THREADS = 1024;
constexpr int TR_SMEM_MAX = 200 * 1024;  // bins above stay in global memory (L2)

__global__ void __launch_bounds__(TR_THREADS)
transmission_kernel(const double *__restrict__ K, int64_t k_stride, int nxb, int nbins,
                    const int *__restrict__ nxmin, double kmin, int nTr, double dTr, int use_smem,
                    double *__restrict__ Tr) {
  extern __shared__ __align__(16) double kb_s[];
  const int b = blockIdx.x, s = blockIdx.y;
  const double *src = K + (int64_t)s * k_stride + (int64_t)b * nxb;
  const double *kb = src;
  if (use_smem) {
    for (int k = threadIdx.x; k < nxb; k += TR_THREADS) kb_s[k] = src[k];
    __syncthreads();
    kb = kb_s;
  }
  const int nm = nxmin ? nxmin[(int64_t)s * nbins + b] : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *out = Tr + ((int64_t)s * nbins + b) * nTr;
  for (int j = warp; j < nTr; j += TR_THREADS / 32) {
    const double m = exp((double)(j - nTr / 2) * dTr);
    double a = 0.0;
    for (int k = lane; k < nxb; k += 32) a += exp(-kb[k] * m);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) {
      for (int idy = 0; idy < 3 && nxb >= 3; ++idy) {
        a = __dadd_rn(a, __dmul_rn(c_wS[idy], exp(-kb[idy] * m)));
        a = __dadd_rn(a, __dmul_rn(c_wS[2 - idy], exp(-kb[nxb - 1 - idy] * m)));
      }
      const double t0 = __ddiv_rn(__dmul_rn(__ddiv_rn(a, (double)(nxb - 1)), (double)(nxb - nm)),
                                  (double)nxb);
      const double t1 = __ddiv_rn(__dmul_rn(exp(-kmin * m), (double)nm), (double)nxb);
      out[j] = __dadd_rn(t0, t1);
    }
  }
}

cudaError_t launch_transmission(const double *K_d, int64_t k_stride, int nstates, int nxb,
                                int nbins, const int *nxmin_d, double kmin, int nTr, double dTr,
                                double *Tr_d, cudaStream_t stream) {
  if (nstates <= 0 || nbins <= 0 || nTr <= 0) return cudaSuccess;
  const size_t smem = (size_t)nxb * sizeof(double);
  const int use_smem = smem <= (size_t)TR_SMEM_MAX;
  if (use_smem && smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(transmission_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  dim3 grid(nbins, nstates);
  transmission_kernel<<<grid, TR_THREADS, use_smem ? smem : 0, stream>>>(
      K_d, k_stride, nxb, nbins, nxmin_d, kmin, nTr, dTr, use_smem, Tr_d);
  return cudaGetLastError();
}

}  // namespace hkb
