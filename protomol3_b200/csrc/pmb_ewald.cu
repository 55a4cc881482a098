// Exact Ewald reciprocal sum, the check path for the PME reciprocal term:
// NonbondedFullEwaldSystemForce::reciprocalTerm (force/nonbonded/NonbondedFullEwaldSystemForce.h:
// 873-1083) over the k-vectors of its initialize (:590-660).
//
// Per k-vector the structure factor S(k) = sum_i q_i sin(k.r_i), C(k) = sum_i q_i cos(k.r_i)
// (one block per k, a fixed-order tree sum, so the result is the same on every run); per atom the
// force k a_k q_i (sin(k.r_i) C(k) - cos(k.r_i) S(k)), a_k = 8 pi / V exp(-k^2 / 4 alpha^2) / k^2.
// The reference builds the sines and cosines of the k.r_i by recurrences over the integer
// indices; here each comes from sincos directly (the two agree to rounding).  Energy and virial
// are summed on the host from S and C in the reference's k order.
#include <cuda_runtime.h>

#include "pmb_internal.h"

namespace pmb {

namespace {

constexpr int EW_THREADS = 256;

__global__ void __launch_bounds__(EW_THREADS) k_ewald_structure(const double *pos, const double *charge, int atom0,
                                                                 int n, const double3 *kv, int nk, double *S,
                                                                 double *Cc) {
  const int k = blockIdx.x;
  if (k >= nk) return;
  const double3 kk = kv[k];
  double s = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < n; i += EW_THREADS) {
    const double *r = pos + 3 * (long long)(atom0 + i);
    const double q = charge[atom0 + i];
    double sn, cs;
    sincos(kk.x * r[0] + kk.y * r[1] + kk.z * r[2], &sn, &cs);
    s += q * sn;
    c += q * cs;
  }
  __shared__ double rs[EW_THREADS], rc[EW_THREADS];
  rs[threadIdx.x] = s;
  rc[threadIdx.x] = c;
  __syncthreads();
  for (int w = EW_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      rs[threadIdx.x] += rs[threadIdx.x + w];
      rc[threadIdx.x] += rc[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    S[k] = rs[0];
    Cc[k] = rc[0];
  }
}

__global__ void __launch_bounds__(EW_THREADS) k_ewald_forces(const double *pos, const double *charge, int atom0,
                                                              int n, const double3 *kv, const double *a, const double *S,
                                                              const double *Cc, int nk, double *fout) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *r = pos + 3 * (long long)(atom0 + i);
  const double q = charge[atom0 + i];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int k = 0; k < nk; k++) {
    const double3 kk = kv[k];
    double sn, cs;
    sincos(kk.x * r[0] + kk.y * r[1] + kk.z * r[2], &sn, &cs);
    const double g = a[k] * (q * sn * Cc[k] - q * cs * S[k]);
    fx += kk.x * g;
    fy += kk.y * g;
    fz += kk.z * g;
  }
  double *f = fout + 3 * (long long)(atom0 + i);
  f[0] = fx;
  f[1] = fy;
  f[2] = fz;
}

}  // namespace

int ewald_recip_launch(const double *pos, const double *charge, int atom0, int n, const double3 *kv,
                       const double *a, int nk, double *S, double *Cc, double *fout, cudaStream_t st) {
  if (n <= 0 || nk <= 0) return 0;
  k_ewald_structure<<<nk, EW_THREADS, 0, st>>>(pos, charge, atom0, n, kv, nk, S, Cc);
  k_ewald_forces<<<(n + EW_THREADS - 1) / EW_THREADS, EW_THREADS, 0, st>>>(pos, charge, atom0, n, kv, a, S, Cc, nk,
                                                                           fout);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace pmb
