// hkb_kdist.cu -- per-bin sort + Chebyshev k-distribution fit (sm_100a).
//
// One CTA per (state, bin) does the whole post-processing chain of
// heliosk.cu:2046-2193 on the bin's values while they sit in shared memory:
//   sort (total order on the FP64 bit patterns)          heliosk.cu:2046-2051
//   findCut                                              resample.h:362-388
//   rescale(+1), copyK2                                  resample.h:397-461
//   lnK                                                  resample.h:472-481
//   leastSquare (first nc-1 reflections, back-solve)     resample.h:243-353
//   optional expfx + rescale(-1) reconstruction          resample.h:497-524
// The Householder factorisation of the Chebyshev Vandermonde matrix is done
// once per (Nxb, nC) by qr_kernel (resample.h:14-37, 73-227), a single CTA.
// Bins larger than the shared-memory budget run the same code on a global
// scratch slice.
#include <cuda_runtime.h>

#include <cstdint>
#include <cub/block/block_merge_sort.cuh>

#include "hkb_kernels.h"
#include "hkb_types.h"

namespace hkb {

constexpr int KD_THREADS = 1024;
constexpr int KD_MAX_NC = 100;  // def_NmaxSample, define.h:55

__device__ __forceinline__ uint64_t f2key(double v) {
  const uint64_t b = (uint64_t)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key2f(uint64_t k) {
  const uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// block-wide sum; every thread gets the result
__device__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  double t = (lane < nw) ? red[lane] : 0.0;
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;
}

__device__ double block_max(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  double t = (lane < nw) ? red[lane] : 0.0;
  for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
  return t;
}

// block-wide sum with one barrier: red2 holds two 32-entry buffers used in
// turn by consecutive calls (a thread may start the next call's write while
// others still read this call's buffer, never the same buffer)
__device__ __forceinline__ double block_sum1(double v, double *red2, int parity) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  double *red = red2 + 32 * parity;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  double t = (lane < nw) ? red[lane] : 0.0;
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;
}

// Vandermonde_kernel + QR_kernel (resample.h:14-37, 73-227), one CTA.
// V is column-major nxb x nc; on return it holds the Householder vectors
// below/on the diagonal and R above it; C, D as in the reference.
__global__ void __launch_bounds__(KD_THREADS)
qr_kernel(int nxb, int nc, double *__restrict__ V, double *__restrict__ Cv,
          double *__restrict__ D) {
  __shared__ double red[32];
  for (int id = threadIdx.x; id < nxb; id += blockDim.x) {
    const double x = id * 2.0 / ((double)nxb - 1.0) - 1.0;
    V[id] = 1.0;
    if (nc > 1) V[id + (int64_t)nxb] = x;
    double t = x, t0 = 1.0;
    for (int i = 2; i < nc; ++i) {
      const double tt = t;
      t = __fma_rn(2.0 * x, t, -t0);
      t0 = tt;
      V[id + (int64_t)nxb * i] = t;
    }
  }
  __syncthreads();
  for (int i = 0; i < nc; ++i) {
    double *vi = V + (int64_t)nxb * i;
    double m = 0.0;
    for (int k = i + threadIdx.x; k < nxb; k += blockDim.x) m = fmax(m, fabs(vi[k]));
    const double scale = block_max(m, red);
    double ss = 0.0;
    for (int k = i + threadIdx.x; k < nxb; k += blockDim.x) {
      const double v = vi[k] / scale;
      vi[k] = v;
      ss = __fma_rn(v, v, ss);
    }
    ss = block_sum(ss, red);
    __syncthreads();
    if (threadIdx.x == 0) {
      const double s = sqrt(ss);
      const double v0 = vi[i];
      const double sigma = (v0 < 0.0) ? -s : s;
      vi[i] = v0 + sigma;
      Cv[i] = sigma * (v0 + sigma);
      D[i] = -scale * sigma;
    }
    __syncthreads();
    for (int j = i + 1; j < nc; ++j) {
      double *vj = V + (int64_t)nxb * j;
      double dot = 0.0;
      for (int k = i + threadIdx.x; k < nxb; k += blockDim.x) dot = __fma_rn(vi[k], vj[k], dot);
      dot = block_sum(dot, red);
      const double t = dot / Cv[i];
      for (int k = i + threadIdx.x; k < nxb; k += blockDim.x) vj[k] = __fma_rn(-t, vi[k], vj[k]);
      __syncthreads();
    }
  }
}

struct KdistArgs {
  const double *K;       // nstates x nx, unsorted
  int64_t k_stride;
  int nxb, nbins, nc, pow2;
  double kmin, unitScale;
  const double *V, *Cv, *D;
  double *coeff;         // nstates x nbins x nc
  int *nxmin;            // nstates x nbins
  double *sorted;        // optional nstates x nx
  double *recon;         // optional nstates x nx
  double *scratch;       // global work when the bin does not fit in smem
  int use_smem;
};

struct KeyLess {
  __device__ __forceinline__ bool operator()(uint64_t x, uint64_t y) const { return x < y; }
};

// IPT > 0: the bin is sorted in registers, IPT keys per thread, by a block
// merge sort (CUB's BlockMergeSort: per-thread sort, then log2(1024) rounds of
// merge-path merges through shared memory) -- O(n log n) comparisons where
// the bitonic network needs O(n log^2 n); its tile (1024 IPT + 1 keys) uses
// the key array.  IPT = 0: bitonic network, one shared-memory or global pass
// per stage (bins the merge sort does not hold).  The sorted keys are the
// same either way: the total order of the FP64 bit patterns has no ties
// between distinct values.
template <int IPT>
__global__ void __launch_bounds__(KD_THREADS)
kdist_kernel(KdistArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[64];
  __shared__ int s_trans;
  __shared__ double s_c[KD_MAX_NC], s_cv[KD_MAX_NC], s_d[KD_MAX_NC];
  const int b = blockIdx.x, s = blockIdx.y;
  const int nxb = a.nxb, P2 = a.pow2;
  const int tid = threadIdx.x, nt = blockDim.x;
  uint64_t *keys;
  double *work;
  if (a.use_smem) {
    keys = reinterpret_cast<uint64_t *>(smem_raw);
    work = reinterpret_cast<double *>(smem_raw + (size_t)P2 * 8);
  } else {
    const size_t slot = ((size_t)s * a.nbins + b) * (size_t)(P2 + nxb);
    keys = reinterpret_cast<uint64_t *>(a.scratch + slot);
    work = a.scratch + slot + P2;
  }
  const double *src = a.K + (int64_t)s * a.k_stride + (int64_t)b * nxb;
  constexpr uint64_t KEY_END = 0xffffffffffffffffull;  // after every key of a value
  if (IPT > 0) {
    // coalesced into shared memory, then blocked into registers
    for (int i = tid; i < nxb; i += nt) keys[i] = f2key(src[i]);
  } else {
    for (int i = tid; i < P2; i += nt) keys[i] = (i < nxb) ? f2key(src[i]) : KEY_END;
  }
  for (int i = tid; i < a.nc; i += nt) {
    s_cv[i] = a.Cv[i];
    s_d[i] = a.D[i];
  }
  __syncthreads();

  // sort, ascending
  if (IPT > 0) {
    constexpr int NI = IPT > 0 ? IPT : 1;
    using Sorter = cub::BlockMergeSort<uint64_t, KD_THREADS, NI>;
    uint64_t v[NI];
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const int k = tid * NI + i;
      v[i] = k < nxb ? keys[k] : KEY_END;
    }
    __syncthreads();  // the tile storage below overlays keys[]
    Sorter(*reinterpret_cast<typename Sorter::TempStorage *>(keys)).Sort(v, KeyLess(), nxb, KEY_END);
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const int k = tid * NI + i;
      if (k < nxb) work[k] = key2f(v[i]);
    }
  } else {
    for (int size = 2; size <= P2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int i = tid; i < (P2 >> 1); i += nt) {
          const int pos = 2 * i - (i & (stride - 1));
          const int q = pos + stride;
          const uint64_t x = keys[pos], y = keys[q];
          const bool up = (pos & size) == 0;
          if ((x > y) == up) {
            keys[pos] = y;
            keys[q] = x;
          }
        }
        __syncthreads();
      }
    }
    for (int i = tid; i < nxb; i += nt) work[i] = key2f(keys[i]);
  }
  __syncthreads();
  if (a.sorted) {
    double *dst = a.sorted + (int64_t)s * a.k_stride + (int64_t)b * nxb;
    for (int i = tid; i < nxb; i += nt) dst[i] = work[i];
  }
  if (a.coeff == nullptr) return;

  // findCut (resample.h:362-388) on the sorted bin.  Within a bin at most
  // one index j has K[j] <= kmin < K[j+1]; the empty-bin rules follow it.
  if (tid == 0) s_trans = -1;
  __syncthreads();
  const bool last_bin = (b == a.nbins - 1);
  // transitions at local j <= nxb-2; for the bin's last index the reference's
  // "complete empty bin" rule gives the same Nxb (and the state's last index
  // is never visited: id < NL-1)
  for (int j = tid; j < nxb - 1; j += nt)
    if (work[j] <= a.kmin && work[j + 1] > a.kmin) s_trans = j;
  __syncthreads();
  int nxmin = 0;
  {
    const int jt = s_trans;
    if (jt >= 0) nxmin = jt + 1;
    if (!last_bin) {
      if (work[nxb - 1] <= a.kmin) nxmin = nxb;
    } else if (nxb >= 3 && work[nxb - 3] <= a.kmin) {
      // id == NL-3 rule; a transition at the later id NL-2 wins the race
      nxmin = (jt == nxb - 2) ? nxb - 1 : nxb;
    }
  }
  if (tid == 0) a.nxmin[(int64_t)s * a.nbins + b] = nxmin;

  // rescale(+1) into keys[] (reused as doubles), then copy back
  double *tmp = reinterpret_cast<double *>(keys);
  if (nxmin > 0) {
    for (int j = tid; j < nxb; j += nt) {
      double ii = __fma_rn(1.0 - nxmin / ((double)(nxb - 1)), (double)j, (double)nxmin);
      if (ii >= nxb - 1) ii = 0.999999 * (nxb - 1);
      const int il = (int)(ii / ((double)nxb) * nxb);
      const double Kl = work[il], Kr = work[il + 1];
      tmp[j] = __fma_rn(Kr - Kl, ii - il, Kl);
    }
    __syncthreads();
    for (int j = tid; j < nxb; j += nt) work[j] = tmp[j];
    __syncthreads();
  }
  for (int j = tid; j < nxb; j += nt) work[j] = log(work[j] * a.unitScale);
  __syncthreads();

  // leastSquare_kernel: Q^T b with the first nc-1 reflections.  Thread tid
  // owns the bin elements k = tid + n nt (k >= j) in every reflection, so a
  // reflection needs only its block sum's barrier.
  const int nc = a.nc;
  if (IPT > 0) {
    // (nxb <= 1024 IPT) the thread's entries of V's column in registers, the
    // next column copied asynchronously into the free key array while this
    // one is used; a thread copies and reads only its own entries
    constexpr int NI = IPT > 0 ? IPT : 1;
    double vv[NI];
    double *pbuf = reinterpret_cast<double *>(keys);
#pragma unroll
    for (int n = 0; n < NI; ++n) {
      const int k = tid + n * KD_THREADS;
      vv[n] = (k < nxb && nc > 1) ? a.V[k] : 0.0;
    }
    for (int j = 0; j < nc - 1; ++j) {
      const bool more = j + 1 < nc - 1;
      if (more) {
        const double *vnext = a.V + (int64_t)nxb * (j + 1);
#pragma unroll
        for (int n = 0; n < NI; ++n) {
          const int k = tid + n * KD_THREADS;
          if (k < nxb) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(pbuf + k);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(vnext + k));
          }
        }
        asm volatile("cp.async.commit_group;\n" ::);
      }
      double dot = 0.0;
#pragma unroll
      for (int n = 0; n < NI; ++n) {
        const int k = tid + n * KD_THREADS;
        if (k < nxb && k >= j) dot = __fma_rn(vv[n], work[k], dot);
      }
      dot = block_sum1(dot, red, j & 1);
      const double t = dot / s_cv[j];
#pragma unroll
      for (int n = 0; n < NI; ++n) {
        const int k = tid + n * KD_THREADS;
        if (k < nxb && k >= j) work[k] = __fma_rn(-t, vv[n], work[k]);
      }
      if (more) {
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
#pragma unroll
        for (int n = 0; n < NI; ++n) {
          const int k = tid + n * KD_THREADS;
          vv[n] = k < nxb ? pbuf[k] : 0.0;
        }
      }
    }
  } else {
    for (int j = 0; j < nc - 1; ++j) {
      const double *vj = a.V + (int64_t)nxb * j;
      double dot = 0.0;
      for (int k = tid; k < nxb; k += nt)
        if (k >= j) dot = __fma_rn(vj[k], work[k], dot);
      dot = block_sum1(dot, red, j & 1);
      const double t = dot / s_cv[j];
      for (int k = tid; k < nxb; k += nt)
        if (k >= j) work[k] = __fma_rn(-t, vj[k], work[k]);
    }
  }
  // the R factor's rows used by the back-substitution, copied in parallel
  // into the (now free) key array when it fits
  const int lim = nc < 64 ? nc : 64;
  double *Rb = reinterpret_cast<double *>(keys);
  const bool rb = nc * lim <= P2;
  if (rb)
    for (int q = tid; q < nc * lim; q += nt) Rb[q] = a.V[q / lim + (int64_t)nxb * (q % lim)];
  __syncthreads();
  if (tid == 0) {
    // back-substitution; the reference's reduction keeps 64 partial sums
    double *bb = work;
    bb[nc - 1] /= s_d[nc - 1];
    for (int i = nc - 2; i >= 0; --i) {
      double sum = 0.0;
      for (int j = i + 1; j < lim; ++j)
        sum = __fma_rn(rb ? Rb[i * lim + j] : a.V[i + (int64_t)nxb * j], bb[j], sum);
      bb[i] = (bb[i] - sum) / s_d[i];
    }
    double *co = a.coeff + ((int64_t)s * a.nbins + b) * nc;
    for (int i = 0; i < nc; ++i) {
      co[i] = bb[i];
      s_c[i] = bb[i];
    }
  }
  __syncthreads();
  if (a.recon == nullptr) return;

  // expfx_kernel (x = -1 + 2 j / Nxb) then rescale(-1)
  for (int j = tid; j < nxb; j += nt) {
    const double x = -1.0 + j * 2.0 / ((double)nxb);
    double d1 = 0.0, d2 = 0.0;
    for (int i = nc - 1; i >= 1; --i) {
      const double t = d1;
      d1 = __fma_rn(2.0 * x, d1, -d2) + s_c[i];
      d2 = t;
    }
    const double f = __fma_rn(x, d1, -d2) + 0.5 * s_c[0] + 0.5 * s_c[0];
    work[j] = exp(f) / a.unitScale;
  }
  __syncthreads();
  double *dst = a.recon + (int64_t)s * a.k_stride + (int64_t)b * nxb;
  for (int j = tid; j < nxb; j += nt) {
    double Ki = work[j];
    if (nxmin > 0) {
      Ki = a.kmin;
      if (j >= nxmin) {
        double ii = (j - nxmin) / ((double)(nxb - nxmin - 1)) * (nxb - 1);
        if (ii >= nxb - 1) ii = 0.999999 * (nxb - 1);
        const int il = (int)(ii / ((double)nxb) * nxb);
        const double Kl = work[il], Kr = work[il + 1];
        Ki = __fma_rn(Kr - Kl, ii - il, Kl);
      }
    }
    dst[j] = Ki;
  }
}

static int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

size_t kdist_smem_bytes(int nxb) {
  return (size_t)(next_pow2(nxb) + nxb) * 8;
}

size_t kdist_scratch_doubles(int nxb, int nbins, int nstates) {
  const size_t need = kdist_smem_bytes(nxb);
  if (need <= (size_t)KD_SMEM_LIMIT) return 0;
  return (size_t)nstates * nbins * (size_t)(next_pow2(nxb) + nxb);
}

cudaError_t launch_qr(int nxb, int nc, double *V_d, double *C_d, double *D_d,
                      cudaStream_t stream) {
  qr_kernel<<<1, KD_THREADS, 0, stream>>>(nxb, nc, V_d, C_d, D_d);
  return cudaGetLastError();
}

cudaError_t launch_kdist(const double *K_d, int64_t k_stride, int nstates,
                         int nxb, int nbins, int nc, double kmin,
                         double unitScale, const double *V_d, const double *C_d,
                         const double *D_d, double *coeff_d, int *nxmin_d,
                         double *sorted_d, double *recon_d, double *scratch_d,
                         cudaStream_t stream) {
  if (nstates <= 0 || nbins <= 0) return cudaSuccess;
  KdistArgs a;
  a.K = K_d;
  a.k_stride = k_stride;
  a.nxb = nxb;
  a.nbins = nbins;
  a.nc = nc;
  a.pow2 = next_pow2(nxb);
  a.kmin = kmin;
  a.unitScale = unitScale;
  a.V = V_d;
  a.Cv = C_d;
  a.D = D_d;
  a.coeff = coeff_d;
  a.nxmin = nxmin_d;
  a.sorted = sorted_d;
  a.recon = recon_d;
  a.scratch = scratch_d;
  const size_t smem = kdist_smem_bytes(nxb);
  a.use_smem = smem <= (size_t)KD_SMEM_LIMIT;
  size_t dyn = a.use_smem ? smem : 0;
  if (!a.use_smem && scratch_d == nullptr) return cudaErrorInvalidValue;
  // the merge sort when its tile (1024 IPT + 1 keys) fits the key array
  int ipt = 0;
  if (a.use_smem) {
    static const int kIpt[] = {2, 4, 6, 8, 10, 12};
    for (int q : kIpt)
      if (q * KD_THREADS >= nxb && (size_t)(q * KD_THREADS + 1) <= (size_t)a.pow2) {
        ipt = q;
        break;
      }
  }
  auto run = [&](auto kfn) -> cudaError_t {
    if (a.use_smem) {
      cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
      if (e != cudaSuccess) return e;
    }
    dim3 grid(nbins, nstates);
    kfn<<<grid, KD_THREADS, dyn, stream>>>(a);
    return cudaGetLastError();
  };
  switch (ipt) {
    case 2: return run(kdist_kernel<2>);
    case 4: return run(kdist_kernel<4>);
    case 6: return run(kdist_kernel<6>);
    case 8: return run(kdist_kernel<8>);
    case 10: return run(kdist_kernel<10>);
    case 12: return run(kdist_kernel<12>);
    default: return run(kdist_kernel<0>);
  }
}

}  // namespace hkb
