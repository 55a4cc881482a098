// Bonded terms, accumulator conversion and the device integrators.
//
// Bonds: BondSystemForce::calcBond (force/bonded/BondSystemForce.h:94-117).
// Angles: AngleSystemForce::calcAngle (force/bonded/AngleSystemForce.h:87-172).
// Leapfrog: LeapfrogIntegrator::doKickdoDrift / doHalfKickdoDrift / run
//   (integrator/leapfrog/LeapfrogIntegrator.cpp:33-104) with h = dt * INV_TIMEFACTOR.
// Langevin: LangevinLeapfrogIntegrator::doHalfKick (integrator/base/LangevinLeapfrogIntegrator.cpp:44-71);
//   the reference's serial Park-Miller generator cannot be reproduced on a GPU, so the Gaussian
//   noise comes from a counter-based generator keyed by (seed, atom, step, component): every
//   trajectory is reproducible bit for bit and independent of how systems are batched.
#include "pmb_internal.h"

namespace pmb {

namespace {

__global__ void k_bonds(const SystemDev s, BondedDev b) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = k < b.nbonds;
  int box = -1;
  double en = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};
  if (valid) {
    int a1 = b.bonds[2 * k], a2 = b.bonds[2 * k + 1];
    box = s.atom_box[a1];
    double r12[3];
    min_diff(s.box[box], s.pos + 3 * a2, s.pos + 3 * a1, r12);  // atom1 - atom2
    double r = sqrt(r12[0] * r12[0] + r12[1] * r12[1] + r12[2] * r12[2]);
    double dpotdr = 2.0 * b.bond_k[k] * (r - b.bond_r0[k]);
    double f1[3] = {r12[0] * (-dpotdr / r), r12[1] * (-dpotdr / r), r12[2] * (-dpotdr / r)};
    for (int c = 0; c < 3; c++) {
      long long v = f2fix(f1[c], FORCE_SCALE);
      red_add(s.facc + 3 * (long long)a1 + c, v);
      red_add(s.facc + 3 * (long long)a2 + c, -v);
    }
    en = b.bond_k[k] * (r - b.bond_r0[k]) * (r - b.bond_r0[k]);
    vir[0] = f1[0] * r12[0]; vir[1] = f1[0] * r12[1]; vir[2] = f1[0] * r12[2];
    vir[3] = f1[1] * r12[1]; vir[4] = f1[1] * r12[2]; vir[5] = f1[2] * r12[2];
  }
  box_accumulate(s.eacc, box, valid, E_BOND, en, b.virial ? vir : nullptr);
}

__global__ void k_angles(const SystemDev s, BondedDev b) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = k < b.nangles;
  int box = -1;
  double en = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};
  if (valid) {
    int a1 = b.angles[3 * k], a2 = b.angles[3 * k + 1], a3 = b.angles[3 * k + 2];
    box = s.atom_box[a1];
    const BoxDev &bx = s.box[box];
    double r12[3], r32[3], r13[3];
    min_diff(bx, s.pos + 3 * a2, s.pos + 3 * a1, r12);
    min_diff(bx, s.pos + 3 * a2, s.pos + 3 * a3, r32);
    min_diff(bx, s.pos + 3 * a3, s.pos + 3 * a1, r13);
    double d12 = sqrt(r12[0] * r12[0] + r12[1] * r12[1] + r12[2] * r12[2]);
    double d32 = sqrt(r32[0] * r32[0] + r32[1] * r32[1] + r32[2] * r32[2]);
    double d13 = sqrt(r13[0] * r13[0] + r13[1] * r13[1] + r13[2] * r13[2]);
    double cr[3] = {r12[1] * r32[2] - r12[2] * r32[1], r12[2] * r32[0] - r12[0] * r32[2],
                    r12[0] * r32[1] - r12[1] * r32[0]};
    double theta = atan2(sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]),
                         r12[0] * r32[0] + r12[1] * r32[1] + r12[2] * r32[2]);
    double sn = sin(theta), cs = cos(theta);
    double kth = b.angle_k[k], th0 = b.angle_theta0[k], ubk = b.ub_k[k], ubr = b.ub_r0[k];
    double dpot = 2.0 * kth * (theta - th0);
    double f1[3], f3[3];
    for (int c = 0; c < 3; c++) {
      double dr12 = r12[c] / d12, dr32 = r32[c] / d32, dr13 = r13[c] / d13;
      double dt1 = (dr12 * cs - dr32) / (sn * d12);
      double dt3 = (dr32 * cs - dr12) / (sn * d32);
      double ub1 = dr13 * (2.0 * ubk * (d13 - ubr));
      f1[c] = -dt1 * dpot - ub1;
      f3[c] = -dt3 * dpot + ub1;
      red_add(s.facc + 3 * (long long)a1 + c, f2fix(f1[c], FORCE_SCALE));
      red_add(s.facc + 3 * (long long)a3 + c, f2fix(f3[c], FORCE_SCALE));
      red_add(s.facc + 3 * (long long)a2 + c, f2fix(-f1[c] - f3[c], FORCE_SCALE));
    }
    en = kth * (theta - th0) * (theta - th0) + ubk * (d13 - ubr) * (d13 - ubr);
    // AngleSystemForce.h:151-170: virial = f1 (x) r12 + f3 (x) r32
    vir[0] = f1[0] * r12[0] + f3[0] * r32[0]; vir[1] = f1[0] * r12[1] + f3[0] * r32[1];
    vir[2] = f1[0] * r12[2] + f3[0] * r32[2]; vir[3] = f1[1] * r12[1] + f3[1] * r32[1];
    vir[4] = f1[1] * r12[2] + f3[1] * r32[2]; vir[5] = f1[2] * r12[2] + f3[2] * r32[2];
  }
  box_accumulate(s.eacc, box, valid, E_ANGLE, en, b.virial ? vir : nullptr);
}

__global__ void k_forces_to_double(const SystemDev s, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * s.natoms) return;
  out[i] = (double)s.facc[i] * (1.0 / FORCE_SCALE);
}

__global__ void k_energies_to_double(const SystemDev s, const double *cst, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.nbox * ACC_PER_BOX) return;
  out[i] = (double)s.eacc[i] * (1.0 / ENERGY_SCALE) + (cst ? cst[i] : 0.0);
}

__global__ void k_zero(long long *a, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = 0;
}

// Counter-based generator: a 4x32 Philox-style bijective mixing round function (Salmon et al.,
// SC'11, "Parallel random numbers: as easy as 1, 2, 3"), 10 rounds, keyed by the seed.
__device__ __forceinline__ uint4 philox10(uint4 c, uint2 k) {
  const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

__device__ __forceinline__ double u01(unsigned a, unsigned b) {
  unsigned long long v = ((unsigned long long)a << 21) ^ (unsigned long long)b;
  v &= (1ull << 53) - 1;
  return ((double)v + 0.5) * (1.0 / 9007199254740992.0);
}

// Box-Muller: three standard normals for (atom, step).
__device__ __forceinline__ void gauss3(unsigned long long seed, int atom, long long step, double g[3]) {
  uint2 key = make_uint2((unsigned)seed, (unsigned)(seed >> 32));
  uint4 c0 = philox10(make_uint4((unsigned)atom, (unsigned)step, (unsigned)(step >> 32), 0u), key);
  uint4 c1 = philox10(make_uint4((unsigned)atom, (unsigned)step, (unsigned)(step >> 32), 1u), key);
  double u1 = u01(c0.x, c0.y), u2 = u01(c0.z, c0.w), u3 = u01(c1.x, c1.y), u4 = u01(c1.z, c1.w);
  double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
  double s1, cc1, s2, cc2;
  sincospi(2.0 * u2, &s1, &cc1);
  sincospi(2.0 * u4, &s2, &cc2);
  g[0] = r1 * cc1;
  g[1] = r1 * s1;
  g[2] = r2 * cc2;
}

// Leapfrog kick (coefficient 1 or 1/2) + drift; the force accumulator is consumed and cleared.
__global__ void k_kick_drift(const SystemDev s, IntegratorDev in, double kick) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < s.nbox * ACC_PER_BOX) s.eacc[i] = 0;
  if (i >= s.natoms) return;
  const double h = in.h, m = in.mass[i];
  long long *fa = s.facc + 3 * (long long)i;
  double *v = in.vel + 3 * (long long)i, *x = in.pos + 3 * (long long)i;
  if (in.kind == 0) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double f = (double)fa[c] * (1.0 / FORCE_SCALE);
      fa[c] = 0;
      // (F * h * 0.5) / m for the half kick, (F * h) / m for the full kick, as the reference
      v[c] += kick == 1.0 ? f * h / m : f * h * 0.5 / m;
      x[c] += v[c] * h;
    }
  } else {
    // Langevin (StandardIntegrator::run, StandardIntegrator.cpp:27-37): per step a noisy half
    // kick, drift, forces, noisy half kick.  The half kick closing step s-1 (noise stream 2s-1)
    // is applied here together with the opening half kick of step s (stream 2s); run() ends
    // with k_half_kick closing the last step.
    const long long step = *in.step;
    const double g = in.gamma;
    const double fdt = (1.0 - exp(-0.5 * g * h)) / g, vdt = exp(-0.5 * g * h);
    const double ndt = sqrt((1.0 - exp(-g * h)) / (2.0 * g));
    const double sq = sqrt(2.0 * in.kT * g / m);
    double ra[3], rb[3];
    gauss3(in.seed, i, 2 * step, ra);
    if (kick == 1.0) gauss3(in.seed, i, 2 * step - 1, rb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double f = (double)fa[c] * (1.0 / FORCE_SCALE);
      fa[c] = 0;
      if (kick == 1.0) v[c] = v[c] * vdt + f * fdt / m + rb[c] * sq * ndt;
      v[c] = v[c] * vdt + f * fdt / m + ra[c] * sq * ndt;
      x[c] += v[c] * h;
    }
  }
}

__global__ void k_half_kick(const SystemDev s, IntegratorDev in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.natoms) return;
  const double h = in.h, m = in.mass[i];
  const long long *fa = s.facc + 3 * (long long)i;
  double *v = in.vel + 3 * (long long)i;
  if (in.kind == 0) {
    for (int c = 0; c < 3; c++) v[c] += ((double)fa[c] * (1.0 / FORCE_SCALE)) * h * 0.5 / m;
  } else {
    const long long step = *in.step;
    const double g = in.gamma;
    const double fdt = (1.0 - exp(-0.5 * g * h)) / g, vdt = exp(-0.5 * g * h);
    const double ndt = sqrt((1.0 - exp(-g * h)) / (2.0 * g));
    const double sq = sqrt(2.0 * in.kT * g / m);
    double rp[3];
    gauss3(in.seed, i, 2 * step - 1, rp);  // closes the last completed step
    for (int c = 0; c < 3; c++)
      v[c] = v[c] * vdt + ((double)fa[c] * (1.0 / FORCE_SCALE)) * fdt / m + rp[c] * sq * ndt;
  }
}

__global__ void k_step_inc(long long *step) { *step += 1; }

__global__ void k_kinetic(const SystemDev s, IntegratorDev in, double *out) {
  // one block per box, fixed-order reduction
  int b = blockIdx.x;
  const BoxDev &bx = s.box[b];
  double acc = 0.0;
  for (int i = bx.atom0 + threadIdx.x; i < bx.atom0 + bx.natoms; i += blockDim.x) {
    const double *v = in.vel + 3 * (long long)i;
    acc += 0.5 * in.mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  __shared__ double red[32];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double r = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    r = warp_sum(r);
    if (threadIdx.x == 0) out[b] = r;
  }
}

// FP32 FMA issue-rate probe: 8 independent dependency chains per thread keep the FMA pipes
// full; the result is written out so nothing is eliminated.
__global__ void k_fma_probe(float *out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = threadIdx.x * 1e-3f + c;
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = fmaf(x[c], a, b);
  float r = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) r += x[c];
  if (r == 1234.5f) out[0] = r;
}

}  // namespace

int fp32_peak_probe(double *tflops) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
  double best = 0.0;
  for (int r = 0; r < 4; r++) {
    cudaEventRecord(e0);
    k_fma_probe<<<blocks, threads>>>(out, iters, 0.999f, 1e-4f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double fl = 2.0 * 8.0 * iters * (double)threads * blocks;
    if (r > 0 && ms > 0) best = fl / (ms * 1e-3) / 1e12 > best ? fl / (ms * 1e-3) / 1e12 : best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *tflops = best;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int bonded_launch(const SystemDev &s, const BondedDev &b, cudaStream_t st) {
  const int T = 256;
  if (b.nbonds > 0) k_bonds<<<(b.nbonds + T - 1) / T, T, 0, st>>>(s, b);
  if (b.nangles > 0) k_angles<<<(b.nangles + T - 1) / T, T, 0, st>>>(s, b);
  return 0;
}

int forces_to_double(const SystemDev &s, double *out, cudaStream_t st) {
  const int T = 256, n = 3 * s.natoms;
  if (n > 0) k_forces_to_double<<<(n + T - 1) / T, T, 0, st>>>(s, out);
  return 0;
}

int energies_to_double(const SystemDev &s, const double *cst, double *out, cudaStream_t st) {
  const int T = 128, n = s.nbox * ACC_PER_BOX;
  k_energies_to_double<<<(n + T - 1) / T, T, 0, st>>>(s, cst, out);
  return 0;
}

int zero_accumulators(const SystemDev &s, cudaStream_t st) {
  const int T = 256;
  long long n = 3LL * s.natoms;
  if (n > 0) k_zero<<<(unsigned)((n + T - 1) / T), T, 0, st>>>(s.facc, n);
  long long ne = (long long)s.nbox * ACC_PER_BOX;
  k_zero<<<(unsigned)((ne + T - 1) / T), T, 0, st>>>(s.eacc, ne);
  return 0;
}

int integrate_kick_drift(const SystemDev &s, const IntegratorDev &in, double kick, cudaStream_t st) {
  const int T = 256;
  int n = s.natoms > s.nbox * ACC_PER_BOX ? s.natoms : s.nbox * ACC_PER_BOX;
  k_kick_drift<<<(n + T - 1) / T, T, 0, st>>>(s, in, kick);
  if (in.kind == 1) k_step_inc<<<1, 1, 0, st>>>(in.step);
  return 0;
}

int integrate_half_kick(const SystemDev &s, const IntegratorDev &in, cudaStream_t st) {
  const int T = 256;
  k_half_kick<<<(s.natoms + T - 1) / T, T, 0, st>>>(s, in);
  return 0;
}

int kinetic_energy(const SystemDev &s, const IntegratorDev &in, double *out, cudaStream_t st) {
  k_kinetic<<<s.nbox, 256, 0, st>>>(s, in, out);
  return 0;
}

}  // namespace pmb
