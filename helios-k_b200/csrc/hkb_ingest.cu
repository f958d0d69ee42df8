// hkb_ingest.cu -- line-list ingestion on the GPU (sm_100a).
//
// The reference reads each line file record by record into host SoA arrays
// (readFile host.h:598-649; readFileExomol host.h:656-668 with 8192-line
// pinned buffers and async copies, heliosk.cu:1405-1423).  Here the binary
// records travel to the GPU as they are -- read in chunks into two pinned
// buffers, each chunk's copy overlapping the read of the next -- and one
// kernel unpacks them into the library's columns:
//   HITRAN 68-byte records  char cid[4]; double nu, S, E'', A, delta,
//                           gamma_air, gamma_self, n   (hitran.cpp:406-414)
//   ExoMol 32-byte records  double nu, S, E'', A       (prepareExomol.cpp:222-225)
// with the combined width gam = ((1-q) gamma_air + q gamma_self) gammaF
// (host.h:640-641; ExoMol: the species default, voigt.h:497) and the
// natural-width term A / (4 pi c) (voigt.h:349, 496), in explicitly rounded
// FP64 so the values equal the host formulas'.
#include <cuda_runtime.h>

#include <cstring>

#include "hkb_device.cuh"
#include "hkb_kernels.h"

namespace hkb {

// strncmp(rec, cid, 4) == 0 for a 4-byte record field and a species cid
__device__ __forceinline__ bool cid_match(const unsigned char *rec, const char (&cid)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const unsigned char a = rec[k], b = (unsigned char)cid[k];
    if (a != b) return false;
    if (a == 0) return true;
  }
  return true;
}

__device__ __forceinline__ double ld_f64(const unsigned char *p) {
  double v;
  memcpy(&v, p, 8);
  return v;
}

__global__ void unpack_records_kernel(const unsigned char *__restrict__ raw, int64_t n,
                                      int64_t first, IngestSpec sp, LineCols cols,
                                      unsigned long long *__restrict__ bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double nu, S, el, A, de = 0.0, ga = 0.0, gs = 0.0, ne = sp.defaultn;
    int j = 0;
    if (sp.hitran) {
      const unsigned char *r = raw + (size_t)i * 68;
      j = -1;
      for (int k = 0; k < sp.niso; ++k)
        if (cid_match(r, sp.cid[k])) j = k;  // the last match, as the host loop
      nu = ld_f64(r + 4);
      S = ld_f64(r + 12);
      el = ld_f64(r + 20);
      A = ld_f64(r + 28);
      de = ld_f64(r + 36);
      ga = ld_f64(r + 44);
      gs = ld_f64(r + 52);
      ne = ld_f64(r + 60);
      if (j < 0) {
        atomicMin(bad, (unsigned long long)(first + i));
        j = 0;
      }
    } else {
      const unsigned char *r = raw + (size_t)i * 32;
      nu = ld_f64(r);
      S = ld_f64(r + 8);
      el = ld_f64(r + 16);
      A = ld_f64(r + 24);
    }
    double gam;
    if (sp.hitran) {
      // ((1 - q) gamma_air + q gamma_self) gammaF, each operation rounded
      gam = __dmul_rn(__dadd_rn(__dmul_rn(__dsub_rn(1.0, sp.qalphaL), ga), __dmul_rn(sp.qalphaL, gs)),
                      sp.gammaF);
    } else {
      gam = __dmul_rn(sp.defaultL, sp.gammaF);
    }
    cols.nu[i] = nu;
    cols.S[i] = S;
    cols.EL[i] = el;
    cols.gam[i] = gam;
    cols.nexp[i] = ne;
    cols.delta[i] = de;
    cols.Aterm[i] = __ddiv_rn(A, sp.four_pi_c);
    cols.iso[i] = (uint8_t)(sp.iso_base + j);
  }
}

// gam and A-term from caller-provided columns already on the device
__global__ void finish_columns_kernel(int64_t n, IngestSpec sp, const double *__restrict__ gair,
                                      const double *__restrict__ gself, const double *__restrict__ A,
                                      const int32_t *__restrict__ iso32, LineCols cols) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (sp.hitran)
      cols.gam[i] = __dmul_rn(__dadd_rn(__dmul_rn(__dsub_rn(1.0, sp.qalphaL), gair[i]),
                                        __dmul_rn(sp.qalphaL, gself[i])), sp.gammaF);
    else
      cols.gam[i] = __dmul_rn(sp.defaultL, sp.gammaF);
    cols.Aterm[i] = __ddiv_rn(A[i], sp.four_pi_c);
    cols.iso[i] = iso32 ? (uint8_t)iso32[i] : (uint8_t)0;
    if (!sp.hitran) {
      cols.nexp[i] = sp.defaultn;
      cols.delta[i] = 0.0;
    }
  }
}

// per-block min and max of a column (the host reduces the blocks)
__global__ void minmax_kernel(int64_t n, const double *__restrict__ v, double *__restrict__ out) {
  __shared__ double smin[256], smax[256];
  double lo = CUDART_INF, hi = -CUDART_INF;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double x = v[i];
    lo = (x < lo || x != x) && lo == lo ? x : lo;  // a NaN sticks
    hi = (x > hi || x != x) && hi == hi ? x : hi;
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double a = smin[threadIdx.x + s], b = smax[threadIdx.x + s];
      if ((a < smin[threadIdx.x] || a != a) && smin[threadIdx.x] == smin[threadIdx.x]) smin[threadIdx.x] = a;
      if ((b > smax[threadIdx.x] || b != b) && smax[threadIdx.x] == smax[threadIdx.x]) smax[threadIdx.x] = b;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = smin[0];
    out[2 * blockIdx.x + 1] = smax[0];
  }
}

__global__ void gather_u8_kernel(int64_t n, const int64_t *__restrict__ order,
                                 const uint8_t *__restrict__ src, uint8_t *__restrict__ dst) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    dst[k] = src[order[k]];
}

cudaError_t launch_unpack_records(const unsigned char *raw_d, int64_t n, int64_t first,
                                  const IngestSpec &sp, const LineCols &cols,
                                  unsigned long long *bad_d, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  unpack_records_kernel<<<2368, 256, 0, stream>>>(raw_d, n, first, sp, cols, bad_d);
  return cudaGetLastError();
}

cudaError_t launch_finish_columns(int64_t n, const IngestSpec &sp, const double *gair_d,
                                  const double *gself_d, const double *A_d, const int32_t *iso32_d,
                                  const LineCols &cols, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  finish_columns_kernel<<<2368, 256, 0, stream>>>(n, sp, gair_d, gself_d, A_d, iso32_d, cols);
  return cudaGetLastError();
}

cudaError_t column_minmax(int64_t n, const double *v_d, double *scratch_d, double *lo, double *hi,
                          cudaStream_t stream) {
  const int blocks = 592;
  double h[2 * blocks];
  *lo = 0.0;
  *hi = 0.0;
  if (n == 0) return cudaSuccess;
  minmax_kernel<<<blocks, 256, 0, stream>>>(n, v_d, scratch_d);
  cudaError_t e = cudaMemcpyAsync(h, scratch_d, sizeof h, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return e;
  double a = h[0], b = h[1];
  for (int k = 1; k < blocks; ++k) {
    const double u = h[2 * k], w = h[2 * k + 1];
    if ((u < a || u != u) && a == a) a = u;
    if ((w > b || w != w) && b == b) b = w;
  }
  *lo = a;
  *hi = b;
  return cudaSuccess;
}

cudaError_t launch_gather_u8(int64_t n, const int64_t *order_d, const uint8_t *src_d, uint8_t *dst_d,
                             cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  gather_u8_kernel<<<1184, 256, 0, stream>>>(n, order_d, src_d, dst_d);
  return cudaGetLastError();
}

}  // namespace hkb
