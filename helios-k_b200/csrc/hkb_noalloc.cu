// hkb_noalloc.cu -- per-bin sort + Chebyshev fit without any device
// allocation, for callers that cannot allocate.
//
// hk_kdist (hkb_api.cu) keeps the Householder factors of the Chebyshev
// Vandermonde matrix in workspace the library allocates with cudaMalloc.
// Some host programs cannot let a library do that: an atmosphere or
// retrieval code that hands every byte of device memory to its own pool or
// runs under a fixed memory budget, or one that must not make calls that
// may synchronise the device or fail for lack of memory in the middle of a
// run.  hk_kdist_noalloc serves them: the caller passes device inputs and
// outputs, and the only scratch (the factors) lives in the fixed file-scope
// array below.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "hkb.h"
#include "hkb_kernels.h"

namespace hkb {

// Fixed scratch: V (Nxb x nC, column-major), then C (nC) and D (nC).
// 2^18 doubles = 2 MiB, held on every GPU that loads the library until the
// process exits.
constexpr long long HK_NOALLOC_DOUBLES = 1LL << 18;
static __device__ __align__(256) double g_kdist_scratch[HK_NOALLOC_DOUBLES];

// Device address of g_kdist_scratch per device.  The symbol name in host
// code is only a host-side stand-in, so the address is looked up once per
// device with that device current.
constexpr int HK_NOALLOC_MAX_DEVICES = 64;
static double *g_scratch_addr[HK_NOALLOC_MAX_DEVICES];
static std::mutex g_scratch_mu;

static hk_status scratch_for_current_device(double **out, char *errbuf, int errlen) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= HK_NOALLOC_MAX_DEVICES) {
    if (errbuf && errlen > 0)
      snprintf(errbuf, errlen, "no usable current CUDA device (%s)", cudaGetErrorString(e));
    return HK_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_kdist_scratch);
    if (e != cudaSuccess || !p) {
      if (errbuf && errlen > 0)
        snprintf(errbuf, errlen, "cudaGetSymbolAddress of the fixed scratch failed: %s",
                 cudaGetErrorString(e));
      return HK_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return HK_OK;
}

}  // namespace hkb

using namespace hkb;

extern "C" hk_status hk_kdist_noalloc(const double *K, int nstates, int64_t nx, int nbins,
                                      int nC, double kmin, double unitScale, double *coeff,
                                      int32_t *nxmin, double *sortedK, void *stream,
                                      char *errbuf, int errbuf_len) {
  auto bad = [&](hk_status s, const char *msg) {
    if (errbuf && errbuf_len > 0) snprintf(errbuf, errbuf_len, "%s", msg);
    return s;
  };
  if (errbuf && errbuf_len > 0) errbuf[0] = '\0';
  // an error left by one of the caller's earlier launches is reported as
  // such (and left pending), not mistaken for a failure of this call
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    if (errbuf && errbuf_len > 0)
      snprintf(errbuf, errbuf_len, "a CUDA error was already pending before this call: %s",
               cudaGetErrorString(pending));
    return HK_ERR_CUDA;
  }
  if (!K || !coeff || !nxmin) return bad(HK_ERR_ARG, "K, coeff and nxmin must be device pointers");
  if (nstates < 1 || nstates > 65535) return bad(HK_ERR_RANGE, "nstates must be 1..65535");
  if (nbins < 1 || nx < 1 || nx % nbins != 0)
    return bad(HK_ERR_RANGE, "nx must be a positive multiple of nbins");
  const long long nxb = nx / nbins;
  if (nxb < 4) return bad(HK_ERR_RANGE, "points per bin must be >= 4");
  if (nxb > (1LL << 30)) return bad(HK_ERR_RANGE, "points per bin must be <= 2^30");
  if (nC < 1 || nC > 100 || nC > nxb) return bad(HK_ERR_RANGE, "nC must be 1..100 and <= points per bin");
  if (nxb * nC + 2LL * nC > HK_NOALLOC_DOUBLES) {
    char m[200];
    snprintf(m, sizeof m,
             "points per bin x nC = %lld x %d exceeds the fixed scratch of %lld doubles "
             "(Nxb * nC + 2 nC must be <= %lld)",
             nxb, nC, HK_NOALLOC_DOUBLES, HK_NOALLOC_DOUBLES);
    return bad(HK_ERR_RANGE, m);
  }
  if (kdist_smem_bytes((int)nxb) > (size_t)KD_SMEM_LIMIT)
    return bad(HK_ERR_RANGE, "bin too large for the shared-memory sort (use hk_kdist)");
  double *base = nullptr;
  const hk_status st = scratch_for_current_device(&base, errbuf, errbuf_len);
  if (st != HK_OK) return st;
  double *V = base;
  double *Cv = base + nxb * nC;
  double *D = Cv + nC;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = launch_qr((int)nxb, nC, V, Cv, D, s);
  if (e == cudaSuccess)
    e = launch_kdist(K, nx, nstates, (int)nxb, nbins, nC, kmin, unitScale, V, Cv, D, coeff,
                     nxmin, sortedK, nullptr, nullptr, s);
  if (e != cudaSuccess) {
    if (errbuf && errbuf_len > 0) snprintf(errbuf, errbuf_len, "CUDA: %s", cudaGetErrorString(e));
    return HK_ERR_CUDA;
  }
  return HK_OK;
}
