// Bonded terms, accumulator conversion and the device integrators.
//
// Bonds: BondSystemForce::calcBond (force/bonded/BondSystemForce.h:94-117).
// Angles: AngleSystemForce::calcAngle (force/bonded/AngleSystemForce.h:87-172).
// Leapfrog: LeapfrogIntegrator::doKickdoDrift / doHalfKickdoDrift / run
//   (integrator/leapfrog/LeapfrogIntegrator.cpp:33-104) with h = dt * INV_TIMEFACTOR.
// Langevin: LangevinLeapfrogIntegrator::doHalfKick (integrator/base/LangevinLeapfrogIntegrator.cpp:44-71);
//   the reference's serial Park-Miller generator cannot be reproduced on a GPU, so the Gaussian
//   noise comes from a counter-based generator keyed by (the box's seed, the atom's index within
//   its box, the box's step, component): every trajectory is reproducible bit for bit and
//   independent of how boxes are batched.
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

__global__ void k_forces_to_double(const SystemDev s, double *out, const double *base) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * s.natoms) return;
  const double f = (double)s.facc[i] * (1.0 / FORCE_SCALE);
  out[i] = base ? base[i] + f : f;
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

// One noisy half kick of LangevinLeapfrogIntegrator::doHalfKick (LangevinLeapfrogIntegrator.cpp:
// 66-68): v vdt + (F fdt) / m + (r sq) ndt, every operation rounded on its own (no contraction),
// so that the kick closing a step gives the same bits wherever a run is split into calls.
__device__ __forceinline__ double langevin_half_kick(double v, double f, double r, double vdt, double fdt,
                                                     double m, double sq, double ndt) {
  return __dadd_rn(__dadd_rn(__dmul_rn(v, vdt), __ddiv_rn(__dmul_rn(f, fdt), m)), __dmul_rn(__dmul_rn(r, sq), ndt));
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
      x[c] = __dadd_rn(x[c], __dmul_rn(v[c], h));  // rounded like the reference's x += v * h
    }
  } else {
    // Langevin (StandardIntegrator::run, StandardIntegrator.cpp:27-37): per step a noisy half
    // kick, drift, forces, noisy half kick.  The half kick closing step s-1 (noise stream 2s-1)
    // is applied here together with the opening half kick of step s (stream 2s); run() ends
    // with k_half_kick closing the last step.
    const int b = s.atom_box[i], ia = i - s.box[b].atom0;
    const long long step = *in.step + in.box_step0[b];
    const double g = in.gamma;
    const double fdt = (1.0 - exp(-0.5 * g * h)) / g, vdt = exp(-0.5 * g * h);
    const double ndt = sqrt((1.0 - exp(-g * h)) / (2.0 * g));
    const double sq = sqrt(2.0 * in.kT * g / m);
    double ra[3], rb[3];
    gauss3(in.box_seed[b], ia, 2 * step, ra);
    if (kick == 1.0) gauss3(in.box_seed[b], ia, 2 * step - 1, rb);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double f = (double)fa[c] * (1.0 / FORCE_SCALE);
      fa[c] = 0;
      if (kick == 1.0) v[c] = langevin_half_kick(v[c], f, rb[c], vdt, fdt, m, sq, ndt);
      v[c] = langevin_half_kick(v[c], f, ra[c], vdt, fdt, m, sq, ndt);
      x[c] = __dadd_rn(x[c], __dmul_rn(v[c], h));
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
    const int b = s.atom_box[i], ia = i - s.box[b].atom0;
    const long long step = *in.step + in.box_step0[b];
    const double g = in.gamma;
    const double fdt = (1.0 - exp(-0.5 * g * h)) / g, vdt = exp(-0.5 * g * h);
    const double ndt = sqrt((1.0 - exp(-g * h)) / (2.0 * g));
    const double sq = sqrt(2.0 * in.kT * g / m);
    double rp[3];
    gauss3(in.box_seed[b], ia, 2 * step - 1, rp);  // closes the last completed step
    for (int c = 0; c < 3; c++)
      v[c] = langevin_half_kick(v[c], (double)fa[c] * (1.0 / FORCE_SCALE), rp[c], vdt, fdt, m, sq, ndt);
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

// ------------------------------------------------------------------ SHAKE / RATTLE
// ModifierShake::doExecute (modifier/ModifierShake.cpp:17-75), ModifierRattle::doExecute
// (modifier/ModifierRattle.cpp:17-64) and their error estimates (ModifierMetaShake.cpp:12-33,
// ModifierMetaRattle.cpp:12-31).  The reference sweeps its whole constraint list in order and
// repeats while the mean error over all constraints exceeds epsilon (at most max_iter + 1
// sweeps).  Constraints of different groups share no atom, so a sweep of the list is a sweep of
// every group in list order, and the number of sweeps is the same for all groups.  One thread
// per group, two passes: the scan sweeps its group without writing the state back and adds the
// group's error before each sweep to that sweep's sum (integer atomics, so the sums and the
// count do not depend on the order of the additions); the apply reads the count off the sums and
// takes the state after exactly that many sweeps, from the states the scan kept for the counts
// next to the last application's, or by replaying the sweeps with the same arithmetic, then
// writes positions, velocities and (SHAKE) the reference vectors for the next application.  The
// scan stops two sweeps past the last count; when that is not enough a second scan and apply
// continue from there up to the cap.
// Every operation is rounded as the reference's C++ rounds it (no fused multiply-adds).  With the
// virial on, RATTLE adds its constraint virial (ModifierRattle.cpp:58); SHAKE's term
// (ModifierShake.cpp:65-68) is left out, since the energies are cleared by the force evaluation
// that follows every SHAKE application (integrator/STSIntegrator.cpp:44) and it is never seen.
template <int MA, int MC>
struct ConGroup {
  int nc;
  double x[MA][3], v[MA][3], rm[MA];
  int2 ij[MC];
  double len[MC], ie[MC], rab[MC][3];  // ie = 1 / (2 l^2), for the SHAKE error estimate
};

// register-resident access to a small array by a run-time index
template <int MA>
__device__ __forceinline__ void pick3(const double (&a)[MA][3], int i, double o[3]) {
  o[0] = a[0][0]; o[1] = a[0][1]; o[2] = a[0][2];
#pragma unroll
  for (int k = 1; k < MA; k++)
    if (i == k) { o[0] = a[k][0]; o[1] = a[k][1]; o[2] = a[k][2]; }
}
template <int MA>
__device__ __forceinline__ double pick1(const double (&a)[MA], int i) {
  double o = a[0];
#pragma unroll
  for (int k = 1; k < MA; k++)
    if (i == k) o = a[k];
  return o;
}
template <int MA>
__device__ __forceinline__ void put3(double (&a)[MA][3], int i, const double o[3]) {
#pragma unroll
  for (int k = 0; k < MA; k++)
    if (i == k) { a[k][0] = o[0]; a[k][1] = o[1]; a[k][2] = o[2]; }
}
__device__ __forceinline__ double dot3_rn(const double *a, const double *b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}

template <int MA, int MC>
__device__ void con_load(const ConstraintDev &c, const IntegratorDev &in, int gi, bool shake,
                         ConGroup<MA, MC> &g) {
  const int c0 = c.group_con[gi], a0 = c.group_atom[gi];
  const int na = c.group_atom[gi + 1] - a0;
  g.nc = c.group_con[gi + 1] - c0;
#pragma unroll
  for (int i = 0; i < MA; i++) {
    if (i < na) {
      const int a = c.atoms[a0 + i];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        g.x[i][q] = in.pos[3 * (long long)a + q];
        g.v[i][q] = in.vel[3 * (long long)a + q];
      }
      g.rm[i] = 1.0 / in.mass[a];
    } else {
#pragma unroll
      for (int q = 0; q < 3; q++) g.x[i][q] = g.v[i][q] = 0.0;
      g.rm[i] = 0.0;
    }
  }
#pragma unroll
  for (int k = 0; k < MC; k++) {
    if (k < g.nc) {
      g.ij[k] = c.con_local[c0 + k];
      g.len[k] = c.len[c0 + k];
      g.ie[k] = 1.0 / (2.0 * g.len[k] * g.len[k]);
#pragma unroll
      for (int q = 0; q < 3; q++) g.rab[k][q] = shake ? c.rab[3 * (long long)(c0 + k) + q] : 0.0;
    } else {
      g.ij[k] = make_int2(0, 0);
      g.len[k] = 1.0;
      g.ie[k] = 0.5;
#pragma unroll
      for (int q = 0; q < 3; q++) g.rab[k][q] = 0.0;
    }
  }
}

// sum over the group's constraints of |d^2 - l^2| / (2 l^2), d = x[a2] - x[a1] (the division as a
// product with 1 / (2 l^2): the estimate only feeds the stopping test, whose sums are rounded to
// 2^-40 anyway)
template <int MA, int MC>
__device__ double shake_group_error(const ConGroup<MA, MC> &g) {
  double e = 0.0;
#pragma unroll
  for (int k = 0; k < MC; k++) {
    if (k < g.nc) {
      double p1[3], p2[3], d[3];
      pick3(g.x, g.ij[k].x, p1);
      pick3(g.x, g.ij[k].y, p2);
#pragma unroll
      for (int q = 0; q < 3; q++) d[q] = __dsub_rn(p2[q], p1[q]);
      const double l2 = __dmul_rn(g.len[k], g.len[k]);
      e += fabs(dot3_rn(d, d) - l2) * g.ie[k];
    }
  }
  return e;
}

// sum over the group's constraints of |(x1 - x2).(v1 - v2)|
template <int MA, int MC>
__device__ double rattle_group_error(const ConGroup<MA, MC> &g) {
  double e = 0.0;
#pragma unroll
  for (int k = 0; k < MC; k++) {
    if (k < g.nc) {
      double p1[3], p2[3], v1[3], v2[3], r[3], w[3];
      pick3(g.x, g.ij[k].x, p1);
      pick3(g.x, g.ij[k].y, p2);
      pick3(g.v, g.ij[k].x, v1);
      pick3(g.v, g.ij[k].y, v2);
#pragma unroll
      for (int q = 0; q < 3; q++) {
        w[q] = __dsub_rn(v1[q], v2[q]);
        r[q] = __dsub_rn(p1[q], p2[q]);
      }
      e = __dadd_rn(e, fabs(dot3_rn(r, w)));
    }
  }
  return e;
}

template <int MA, int MC>
__device__ void shake_sweep(ConGroup<MA, MC> &g, double dt) {
#pragma unroll
  for (int k = 0; k < MC; k++) {
    if (k < g.nc) {
      const int a1 = g.ij[k].x, a2 = g.ij[k].y;
      double p1[3], p2[3], v1[3], v2[3], pab[3];
      pick3(g.x, a1, p1);
      pick3(g.x, a2, p2);
      pick3(g.v, a1, v1);
      pick3(g.v, a2, v2);
#pragma unroll
      for (int q = 0; q < 3; q++) pab[q] = __dsub_rn(p1[q], p2[q]);
      const double pabsq = dot3_rn(pab, pab);
      const double rabsq = __dmul_rn(g.len[k], g.len[k]);
      const double diffsq = __dsub_rn(rabsq, pabsq);
      const double rpab = dot3_rn(g.rab[k], pab);
      const double rM1 = pick1(g.rm, a1), rM2 = pick1(g.rm, a2);
      const double gab = __ddiv_rn(diffsq, __dmul_rn(__dmul_rn(2.0, __dadd_rn(rM1, rM2)), rpab));
#pragma unroll
      for (int q = 0; q < 3; q++) {
        double dp = __dmul_rn(g.rab[k][q], gab);
        p1[q] = __dadd_rn(p1[q], __dmul_rn(dp, rM1));
        p2[q] = __dsub_rn(p2[q], __dmul_rn(dp, rM2));
        dp = __ddiv_rn(dp, dt);
        v1[q] = __dadd_rn(v1[q], __dmul_rn(dp, rM1));
        v2[q] = __dsub_rn(v2[q], __dmul_rn(dp, rM2));
      }
      put3(g.x, a1, p1);
      put3(g.x, a2, p2);
      put3(g.v, a1, v1);
      put3(g.v, a2, v2);
    }
  }
}

// vir6 (not null): adds the sweep's virial terms (2 dp) x rab of ModifierRattle.cpp:58, as
// ScalarStructure::addVirial forms them (xx, xy, xz, yy, yz, zz)
template <int MA, int MC>
__device__ void rattle_sweep(ConGroup<MA, MC> &g, double dt, double *vir6 = nullptr) {
#pragma unroll
  for (int k = 0; k < MC; k++) {
    if (k < g.nc) {
      const int a1 = g.ij[k].x, a2 = g.ij[k].y;
      double p1[3], p2[3], v1[3], v2[3], rab[3], vab[3];
      pick3(g.x, a1, p1);
      pick3(g.x, a2, p2);
      pick3(g.v, a1, v1);
      pick3(g.v, a2, v2);
      const double rM1 = pick1(g.rm, a1), rM2 = pick1(g.rm, a2);
#pragma unroll
      for (int q = 0; q < 3; q++) {
        rab[q] = __dsub_rn(p1[q], p2[q]);
        vab[q] = __dsub_rn(v1[q], v2[q]);
      }
      const double rabsq = dot3_rn(rab, rab);
      const double rvab = dot3_rn(rab, vab);
      const double gab = __ddiv_rn(-rvab, __dmul_rn(__dmul_rn(dt, __dadd_rn(rM1, rM2)), rabsq));
      double f2[3];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const double dp = __dmul_rn(rab[q], gab);
        f2[q] = __dmul_rn(dp, 2.0);
        v1[q] = __dadd_rn(v1[q], __dmul_rn(__dmul_rn(dp, dt), rM1));
        v2[q] = __dsub_rn(v2[q], __dmul_rn(__dmul_rn(dp, dt), rM2));
      }
      put3(g.v, a1, v1);
      put3(g.v, a2, v2);
      if (vir6) {
        vir6[0] = __dadd_rn(vir6[0], __dmul_rn(f2[0], rab[0]));
        vir6[1] = __dadd_rn(vir6[1], __dmul_rn(f2[0], rab[1]));
        vir6[2] = __dadd_rn(vir6[2], __dmul_rn(f2[0], rab[2]));
        vir6[3] = __dadd_rn(vir6[3], __dmul_rn(f2[1], rab[1]));
        vir6[4] = __dadd_rn(vir6[4], __dmul_rn(f2[1], rab[2]));
        vir6[5] = __dadd_rn(vir6[5], __dmul_rn(f2[2], rab[2]));
      }
    }
  }
}

constexpr int CON_THREADS = 128;

// SHAKE reference vectors from the current positions (ModifierMetaRattleShake::doInitialize
// takes the positions at initialisation as the last ones)
template <int MA, int MC>
__global__ void k_constraint_init(ConstraintDev c, IntegratorDev in) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= c.ngroup) return;
  ConGroup<MA, MC> g;
  con_load<MA, MC>(c, in, gi, false, g);
  const int c0 = c.group_con[gi];
#pragma unroll
  for (int k = 0; k < MC; k++) {
    if (k < g.nc) {
      double p1[3], p2[3];
      pick3(g.x, g.ij[k].x, p1);
      pick3(g.x, g.ij[k].y, p2);
#pragma unroll
      for (int q = 0; q < 3; q++) c.rab[3 * (long long)(c0 + k) + q] = __dsub_rn(p1[q], p2[q]);
    }
  }
}

template <int MA, int MC, bool RATTLE>
__device__ __forceinline__ void con_sweep(ConGroup<MA, MC> &g, double dt) {
  if constexpr (RATTLE) rattle_sweep(g, dt);
  else shake_sweep(g, dt);
}

template <int MA, int MC, bool RATTLE>
__device__ __forceinline__ double con_error(const ConGroup<MA, MC> &g) {
  if constexpr (RATTLE) return rattle_group_error(g);
  else return shake_group_error(g);
}

template <int MA, int MC>
__device__ __forceinline__ void con_load_or_zero(const ConstraintDev &c, const IntegratorDev &in, int gi,
                                                 bool valid, bool shake, ConGroup<MA, MC> &g) {
  if (valid) {
    con_load<MA, MC>(c, in, gi, shake, g);
  } else {
    g.nc = 0;
#pragma unroll
    for (int i = 0; i < MA; i++) {
#pragma unroll
      for (int q = 0; q < 3; q++) g.x[i][q] = g.v[i][q] = 0.0;
      g.rm[i] = 0.0;
    }
  }
}

// window slot w, component q (x, y, z, vx, vy, vz), group atom i of group gi
__device__ __forceinline__ long long win_at(const ConstraintDev &c, int w, int q, int i, int gi) {
  return (((long long)w * 6 + q) * c.max_atoms + i) * c.ngroup + gi;
}

// Hand-over words after the two rounds of sums in a modifier's error block
constexpr int CON_FLAG = 2 * (CON_MAX_SWEEPS + 1), CON_K1 = CON_FLAG + 1;

// First round: sweeps up to S = min(max_iter, last count + 2); states at the counts around the
// last one go to the window.  Second round (only when the first found no sweep count that meets
// epsilon below the cap): from the state the first apply wrote, up to the remaining budget.
template <int MA, int MC, bool RATTLE, int ROUND>
__global__ void __launch_bounds__(CON_THREADS) k_con_scan(ConstraintDev c, IntegratorDev in) {
  long long *blk = c.err + (RATTLE ? CON_ERR_BLOCK : 0);
  const int maxit = RATTLE ? c.rattle_max : c.shake_max;
  int S, wlo = 0;
  if constexpr (ROUND == 1) {
    const int prev = c.sweeps[RATTLE ? 1 : 0];
    S = min(maxit, prev + 2);
    wlo = max(0, prev - 1);
  } else {
    if (!blk[CON_FLAG]) return;
    S = maxit - (int)blk[CON_K1];
  }
  long long *E = blk + (ROUND == 1 ? 0 : CON_MAX_SWEEPS + 1);
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = gi < c.ngroup;
  ConGroup<MA, MC> g;
  con_load_or_zero<MA, MC>(c, in, gi, valid, !RATTLE, g);
  const int na = valid ? c.group_atom[gi + 1] - c.group_atom[gi] : 0;
  const int lane = threadIdx.x & 31;
  for (int k = 0; k <= S; k++) {
    if (k > 0) con_sweep<MA, MC, RATTLE>(g, c.dt);
    if (ROUND == 1 && k > 0 && k >= wlo && k < wlo + CON_WINDOW) {
#pragma unroll
      for (int i = 0; i < MA; i++) {
        if (i < na) {
#pragma unroll
          for (int q = 0; q < 3; q++) {
            if constexpr (!RATTLE) c.win[win_at(c, k - wlo, q, i, gi)] = g.x[i][q];
            c.win[win_at(c, k - wlo, 3 + q, i, gi)] = g.v[i][q];
          }
        }
      }
    }
    // error before sweep k + 1 into sum k; the warp's sum goes in one atomic
    long long qv = __double2ll_rn(fmin(con_error<MA, MC, RATTLE>(g), c.clamp) * CON_ERR_SCALE);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qv += __shfl_xor_sync(0xffffffffu, qv, o);
    if (lane == 0 && qv) atomicAdd(reinterpret_cast<unsigned long long *>(E + k), (unsigned long long)qv);
  }
}

// The reference's loop: sweep while the mean error exceeds epsilon, at most max_iter + 1 sweeps.
// The first apply takes the count off the first round's sums; when none of them meets epsilon
// below the cap it applies S sweeps and hands over to the second round.
template <int MA, int MC, bool RATTLE, int ROUND>
__global__ void __launch_bounds__(CON_THREADS) k_con_apply(ConstraintDev c, IntegratorDev in) {
  long long *blk = c.err + (RATTLE ? CON_ERR_BLOCK : 0);
  const int maxit = RATTLE ? c.rattle_max : c.shake_max;
  const double eps = RATTLE ? c.rattle_eps : c.shake_eps;
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = gi < c.ngroup;
  int K, wlo = 0, S;
  bool from_window = false, handover = false;
  if constexpr (ROUND == 1) {
    const int prev = c.sweeps[RATTLE ? 1 : 0];
    S = min(maxit, prev + 2);
    wlo = max(0, prev - 1);
    K = 0;
    while (K <= S && (double)blk[K] / CON_ERR_SCALE / c.ncons > eps) K++;
    int cont = 0;
    if (K > S) {
      if (S == maxit) K = maxit + 1;
      else {
        K = S;
        cont = 1;
      }
    }
    if (gi == 0) {
      blk[CON_FLAG] = cont;
      blk[CON_K1] = K;
    }
    handover = cont != 0;
    from_window = K > 0 && K <= S && K >= wlo && K < wlo + CON_WINDOW;
  } else {
    if (!blk[CON_FLAG]) {
      if (gi == 0) c.sweeps[RATTLE ? 1 : 0] = (int)blk[CON_K1];
      return;
    }
    const int s1 = (int)blk[CON_K1];
    S = maxit - s1;
    const long long *E = blk + CON_MAX_SWEEPS + 1;
    K = 0;
    while (K <= S && (double)E[K] / CON_ERR_SCALE / c.ncons > eps) K++;
    if (gi == 0) c.sweeps[RATTLE ? 1 : 0] = s1 + K;
  }
  if (!valid) return;
  ConGroup<MA, MC> g;
  con_load<MA, MC>(c, in, gi, !RATTLE, g);
  const int a0 = c.group_atom[gi], na = c.group_atom[gi + 1] - a0;
  // the constraint virial needs every sweep's multipliers: replay rather than copy
  const bool vir = RATTLE && c.virial;
  if (vir) from_window = false;
  double v6[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (from_window) {
#pragma unroll
    for (int i = 0; i < MA; i++) {
      if (i < na) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
          if constexpr (!RATTLE) g.x[i][q] = c.win[win_at(c, K - wlo, q, i, gi)];
          g.v[i][q] = c.win[win_at(c, K - wlo, 3 + q, i, gi)];
        }
      }
    }
  } else if (vir) {
    for (int k = 0; k < K; k++) rattle_sweep(g, c.dt, v6);
  } else {
    for (int k = 0; k < K; k++) con_sweep<MA, MC, RATTLE>(g, c.dt);
  }
  if (vir) {
    // the group's terms in fixed point (ENERGY_SCALE) into its box's virial slots, row-major
    long long *acc = c.eacc + (long long)c.atom_box[c.atoms[a0]] * ACC_PER_BOX + E_VIR;
    const int slot[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const long long v = f2fix(v6[k], ENERGY_SCALE);
      if (!v) continue;
      red_add(acc + slot[k][0], v);
      if (slot[k][1] != slot[k][0]) red_add(acc + slot[k][1], v);
    }
  }
#pragma unroll
  for (int i = 0; i < MA; i++) {
    if (i < na) {
      const long long a = c.atoms[a0 + i];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        if constexpr (!RATTLE) in.pos[3 * a + q] = g.x[i][q];
        in.vel[3 * a + q] = g.v[i][q];
      }
    }
  }
  // the next SHAKE's reference vectors; not yet when the second round still sweeps against the
  // current ones
  if (!RATTLE && !handover) {
    const int c0 = c.group_con[gi];
#pragma unroll
    for (int k = 0; k < MC; k++) {
      if (k < g.nc) {
        double p1[3], p2[3];
        pick3(g.x, g.ij[k].x, p1);
        pick3(g.x, g.ij[k].y, p2);
#pragma unroll
        for (int q = 0; q < 3; q++) c.rab[3 * (long long)(c0 + k) + q] = __dsub_rn(p1[q], p2[q]);
      }
    }
  }
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

int forces_to_double(const SystemDev &s, double *out, cudaStream_t st, const double *base) {
  const int T = 256, n = 3 * s.natoms;
  if (n > 0) k_forces_to_double<<<(n + T - 1) / T, T, 0, st>>>(s, out, base);
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

template <int MA, int MC, bool RATTLE>
static void constraints_apply_t(const ConstraintDev &c, const IntegratorDev &in, cudaStream_t st) {
  const int blocks = (c.ngroup + CON_THREADS - 1) / CON_THREADS;
  k_con_scan<MA, MC, RATTLE, 1><<<blocks, CON_THREADS, 0, st>>>(c, in);
  k_con_apply<MA, MC, RATTLE, 1><<<blocks, CON_THREADS, 0, st>>>(c, in);
  k_con_scan<MA, MC, RATTLE, 2><<<blocks, CON_THREADS, 0, st>>>(c, in);
  k_con_apply<MA, MC, RATTLE, 2><<<blocks, CON_THREADS, 0, st>>>(c, in);
}

int constraints_init(const ConstraintDev &c, const IntegratorDev &in, cudaStream_t st) {
  if (c.ngroup <= 0) return 0;
  const int blocks = (c.ngroup + CON_THREADS - 1) / CON_THREADS;
  if (c.max_atoms <= 3 && c.max_cons <= 3)
    k_constraint_init<3, 3><<<blocks, CON_THREADS, 0, st>>>(c, in);
  else
    k_constraint_init<CON_MAX_ATOMS, CON_MAX_CONS><<<blocks, CON_THREADS, 0, st>>>(c, in);
  return 0;
}

// One SHAKE (rattle = 0) or RATTLE (rattle = 1) application: clear the modifier's sums and
// hand-over words, then scan and apply, twice (the second round returns at once unless the first
// stopped short of both epsilon and the cap).
int constraints_apply(const ConstraintDev &c, const IntegratorDev &in, int rattle, cudaStream_t st) {
  if (c.ngroup <= 0) return 0;
  cudaError_t e = cudaMemsetAsync(c.err + (rattle ? CON_ERR_BLOCK : 0), 0, sizeof(long long) * CON_ERR_BLOCK, st);
  if (e != cudaSuccess) return 1;
  const bool water = c.max_atoms <= 3 && c.max_cons <= 3;
  if (rattle) {
    if (water) constraints_apply_t<3, 3, true>(c, in, st);
    else constraints_apply_t<CON_MAX_ATOMS, CON_MAX_CONS, true>(c, in, st);
  } else {
    if (water) constraints_apply_t<3, 3, false>(c, in, st);
    else constraints_apply_t<CON_MAX_ATOMS, CON_MAX_CONS, false>(c, in, st);
  }
  return 0;
}

}  // namespace pmb
