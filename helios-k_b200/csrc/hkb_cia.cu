// hkb_cia.cu -- collision-induced absorption on the grid (sm_100a), FP64.
//
// readCiaFile (host.h:670-785) interpolates a HITRAN-format CIA table on the
// host, set by set in file order: linearly in nu inside [nu_j, nu_j+1), the
// sets with T_set <= T overwriting, the first set above T blended linearly
// in T with what the sets before left, and stops after that set; then
// K = cia * rho * NA / mass1 + kmin, rho = P 273.15 / T amagat, or kmin
// everywhere when T lies above every set read.  Here the sets sit on the
// device and one thread per grid point applies the same steps with the same
// rounded operations.  A set's scan in the reference ends right after the
// first grid point that reaches its last interval [nu_N-2, nu_N-1) (the
// "nu1 == numax" exit, host.h:749; with two points, after the first grid
// point): istop is that point's index, computed by the host.
#include <cuda_runtime.h>

#include "hkb_device.cuh"
#include "hkb_kernels.h"

namespace hkb {

constexpr double HK_AMAGAT = 2.6867774e19;  // define.h:43

__global__ void cia_kernel(GridDev g, const CiaSetDev *__restrict__ sets, int nsets,
                           const double *__restrict__ nu, const double *__restrict__ cia, double T,
                           double P, double mass1, double kmin, int beyond, double *__restrict__ K) {
  const double rho1 = __dmul_rn(__ddiv_rn(__dmul_rn(P, 273.15), T), HK_AMAGAT);
  const double na_m = __ddiv_rn(HK_NA, mass1);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.nx;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (beyond) {
      K[i] = kmin;
      continue;
    }
    const double x = grid_x(g, i);
    double k = 0.0;
    for (int s = 0; s < nsets; ++s) {
      const CiaSetDev cs = sets[s];
      if (i > cs.istop) continue;
      const double Tc0 = s > 0 ? sets[s - 1].T : 0.0, Tc1 = cs.T;
      const double *nv = nu + cs.off, *cv = cia + cs.off;
      // last index with nu <= x (-1 if none), the scan's bracket capped at n-2
      int lo = 0, hi = cs.n;
      while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (nv[m] <= x) lo = m + 1;
        else hi = m;
      }
      const int j = min(max(lo - 1, 0), cs.n - 2);
      const double nu0 = nv[j], nu1 = nv[j + 1];
      if (nu0 <= x && x < nu1) {
        const double c0 = cv[j], c1 = cv[j + 1];
        const double v = __dadd_rn(c0, __ddiv_rn(__dmul_rn(__dsub_rn(c1, c0), __dsub_rn(x, nu0)),
                                                 __dsub_rn(nu1, nu0)));
        if (Tc1 <= T) k = v;
        if (T < Tc1 && Tc0 > 0.0)
          k = __dadd_rn(k, __ddiv_rn(__dmul_rn(__dsub_rn(v, k), __dsub_rn(T, Tc0)), __dsub_rn(Tc1, Tc0)));
      }
    }
    K[i] = __dadd_rn(__dmul_rn(__dmul_rn(k, rho1), na_m), kmin);
  }
}

cudaError_t launch_cia(const GridDev &g, const CiaSetDev *sets_d, int nsets, const double *nu_d,
                       const double *cia_d, double T, double P, double mass1, double kmin, int beyond,
                       double *K_d, cudaStream_t stream) {
  if (g.nx <= 0) return cudaSuccess;
  const int64_t nb = (g.nx + 255) / 256;
  cia_kernel<<<(unsigned)(nb < 2368 ? nb : 2368), 256, 0, stream>>>(g, sets_d, nsets, nu_d, cia_d, T, P,
                                                                      mass1, kmin, beyond, K_d);
  return cudaGetLastError();
}

}  // namespace hkb
