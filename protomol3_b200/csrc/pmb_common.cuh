// Shared device-side definitions of the B200 nonbonded / PME force path.
//
// Layout conventions (all arrays device-resident, one system = a batch of >= 1 periodic boxes):
//   * atoms of all boxes are concatenated in the caller's order ("original order");
//   * a box's atoms are re-ordered into "slots" (Hilbert order of a fine cell grid) grouped in
//     blocks of BLOCK slots; a box owns whole blocks, padding slots carry orig = -1;
//   * forces accumulate in int64 fixed point (FORCE_SCALE) in original order, energies and
//     virials per box in int64 fixed point (ENERGY_SCALE): integer addition is associative, so
//     every sum is bit-reproducible whatever the launch order or atomic interleaving;
//   * the PME charge grid accumulates in int64 fixed point (GRID_SCALE).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pmb {

constexpr double FORCE_SCALE = 1099511627776.0;   // 2^40 per kcal/mol/A
constexpr double ENERGY_SCALE = 4294967296.0;     // 2^32 per kcal/mol
constexpr double GRID_SCALE = 1099511627776.0;    // 2^40 per scaled-charge unit
constexpr float FORCE_SCALE_F = 1099511627776.0f;
constexpr float GRID_SCALE_F = 1099511627776.0f;

// Energy / virial accumulator slots per box (ScalarStructure order for the first four).
enum { E_COUL = 0, E_LJ = 1, E_BOND = 2, E_ANGLE = 3, E_VIR = 4, ACC_PER_BOX = 16 };

enum { SW_CUTOFF = 0, SW_C1 = 1, SW_C2 = 2 };

constexpr int BLOCK = 8;           // atoms per i-cluster (a lane group; the j-chunk is 32 atoms)
constexpr int GROUPS = 32 / BLOCK; // lane groups per warp
static_assert(BLOCK == 8 || BLOCK == 16, "i-cluster of 8 or 16 atoms");
constexpr int JCHUNK = 32;         // j-atoms per tile
#ifndef PAIR_TILE_CHUNK
#define PAIR_TILE_CHUNK 8
#endif
constexpr int TILE_CHUNK = PAIR_TILE_CHUNK;  // consecutive tiles per warp assignment of the pair
                                             // kernel; each box's tiles start at a multiple of it
constexpr int JSAME = 1 << 30;     // j-list flag: the j-atom shares a molecule with the i-cluster
constexpr int MAX_LJ_TYPES = 32;   // LJ table kept in shared memory up to this many types

struct BoxDev {
  double L[3], Lr[3];    // edges and reciprocals
  double H[3], H2[3], D; // minimal-image helpers of PeriodicBoundaryConditions (myH, myH2, myD)
  int atom0, natoms;     // original-order atom range
  int blk0, nblk;        // block range; slots [blk0*32, (blk0+nblk)*32)
  int key0;              // first sort bin of this box
  int nc[3];             // sort grid (cells per edge)
  int multi_image;       // Ewald real space must loop lattice images (edge < 2 cutoff)
  int lat0, nlat;        // lattice vectors for multi-image boxes (first is (0,0,0))
  int pad_;
};

// Switching function constants (switch/C1SwitchingFunction.cpp:12-16, C2SwitchingFunction.cpp:12-18).
struct SwitchDev {
  int kind;
  double rc2, ron2, s1, s2, s3, c15_1, c05_3, c15_3;
};

// Pair-kernel parameters shared by all boxes of a batch.
struct PairParams {
  int do_lj, coul_mode;          // coul_mode: 0 none, 1 plain Coulomb with switch, 2 Ewald real
  SwitchDev lj_sw, coul_sw;
  double cut2;                   // pair rejection radius^2 (max of active cutoffs)
  double lj_cut2, coul_cut2;
  double alpha, a2pi;            // Ewald splitting and 2 alpha / sqrt(pi)
  double coulomb_scaling;        // for MODIFIED exclusions
  int ntypes;
  int virial;
};

__host__ __device__ inline long long f2fix(double v, double scale) {
#ifdef __CUDA_ARCH__
  return __double2ll_rn(v * scale);
#else
  return (long long)llrint(v * scale);
#endif
}

__device__ inline long long f2fix(float v, float scale) { return __float2ll_rn(v * scale); }

__device__ inline void red_add(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

// Deterministic double -> fixed conversion of warp partial sums, added to an accumulator.
__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Adds one energy (slot) and optionally a symmetric virial (xx xy xz yy yz zz) per lane to the
// per-box accumulators.  Every term is rounded to fixed point on its own, so a box's sum does not
// depend on which terms of other boxes share its warps; when every valid lane of the warp belongs
// to the same box the warp adds the integers first (one atomic per warp instead of 32 on the
// same address).
__device__ inline void box_accumulate(long long *eacc, int box, bool valid, int slot, double e,
                                      const double *vir6) {
  const int lane = threadIdx.x & 31;
  const unsigned act = __ballot_sync(0xffffffffu, valid);
  if (!act) return;
  const int b0 = __shfl_sync(0xffffffffu, box, __ffs(act) - 1);
  const bool same = __all_sync(0xffffffffu, !valid || box == b0);
  const int map[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};
  const long long ev = valid ? f2fix(e, ENERGY_SCALE) : 0;
  long long vv[6] = {0, 0, 0, 0, 0, 0};
  if (vir6 && valid)
    for (int c = 0; c < 6; c++) vv[c] = f2fix(vir6[c], ENERGY_SCALE);
  if (same) {
    const long long es = warp_sum_ll(ev);
    long long vs[6];
    if (vir6)
      for (int c = 0; c < 6; c++) vs[c] = warp_sum_ll(vv[c]);
    if (lane == 0) {
      long long *acc = eacc + (long long)b0 * ACC_PER_BOX;
      red_add(acc + slot, es);
      if (vir6)
        for (int c = 0; c < 6; c++) {
          red_add(acc + E_VIR + map[c][0], vs[c]);
          if (map[c][1] != map[c][0]) red_add(acc + E_VIR + map[c][1], vs[c]);
        }
    }
  } else if (valid) {
    long long *acc = eacc + (long long)box * ACC_PER_BOX;
    red_add(acc + slot, ev);
    if (vir6)
      for (int c = 0; c < 6; c++) {
        red_add(acc + E_VIR + map[c][0], vv[c]);
        if (map[c][1] != map[c][0]) red_add(acc + E_VIR + map[c][1], vv[c]);
      }
  }
}

// Switching function value and derivative/r (same branch structure as the reference).
template <typename T>
__device__ __forceinline__ void switch_eval(const SwitchDev &w, T r2, T &val, T &der) {
  if (w.kind == SW_C2) {
    der = T(0);
    if (r2 > T(w.rc2)) val = T(0);
    else if (r2 >= T(w.ron2)) {
      T c2 = T(w.rc2) - r2;
      T c4 = c2 * (T(w.s2) + T(2) * r2);
      val = T(w.s1) * (c2 * c4);
      der = T(w.s3) * (c2 * c2 - c4);
    } else val = T(1);
  } else if (w.kind == SW_C1) {
    if (r2 > T(w.rc2)) { val = T(0); der = T(0); return; }
    T dist = sqrt(r2);
    val = T(1) - dist * (T(w.c15_1) - r2 * T(w.c05_3));
    der = -T(w.c15_1) / dist + dist * T(w.c15_3);
  } else {
    der = T(0);
    val = (r2 > T(w.rc2)) ? T(0) : T(1);
  }
}

// Abramowitz & Stegun 7.1.26 polynomial used by the reference's Ewald real space
// (base/MathUtilities.cpp:39-49).
__device__ __forceinline__ double poly5(double ar) {
  double t = 1.0 / (1.0 + 0.3275911 * ar);
  return t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
}
__device__ __forceinline__ float poly5f(float ar) {
  float t = __frcp_rn(fmaf(0.3275911f, ar, 1.0f));
  return t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f))));
}

// Minimal-image difference c2 - c1 with the reference's branch structure
// (topology/PeriodicBoundaryConditions.h:72-110).
__device__ __forceinline__ double min_diff(const BoxDev &b, const double *c1, const double *c2,
                                           double d[3]) {
  d[0] = c2[0] - c1[0];
  d[1] = c2[1] - c1[1];
  d[2] = c2[2] - c1[2];
  double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  if (r2 > b.D) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (d[k] < -b.H2[k]) d[k] += b.H[k];
      else if (d[k] > b.H2[k]) d[k] -= b.H[k];
    }
    r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 > b.D) {
#pragma unroll
      for (int k = 0; k < 3; k++) d[k] -= b.L[k] * rint(b.Lr[k] * d[k]);
      r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    }
  }
  return r2;
}

}  // namespace pmb
