// Fused nonbonded pair kernel: Lennard-Jones with C1/C2/cutoff switching plus either cutoff
// Coulomb (switched) or the Ewald real-space term, over the (block I, 32 j-atoms) tiles built by
// pmb_nblist.cu.
//
// Replaces, per pair, OneAtomPair::doOneAtomPair / OneAtomPairTwo::doOneAtomPair
// (force/OneAtomPair.h:47-106, force/OneAtomPairTwo.h:30-96) with LennardJonesForce::operator()
// (force/LennardJonesForce.h:28-60), CoulombForce::operator() (force/CoulombForce.h:29-40) and
// the PME real-space body (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:644-700).
//
// Warp-tiled: lane l owns i-atom l of block I; the 32 j-atoms are staged in shared memory and
// visited in 32 rotations, the j-force accumulators travel with the rotation through warp
// shuffles (Newton's third law inside the tile).  Forces leave the kernel as int64 fixed point
// (one atomic per j-atom per tile, one per i-atom per run of tiles of the same block); energies
// and virials are summed per tile in a fixed shuffle order and added in fixed point, so results
// are bit-identical from run to run.
//
// Two arithmetic paths share the structure:
//   * FP64 ("plain"): raw double positions, the reference's minimal-image branches, IEEE
//     division/sqrt/exp and the A&S erfc polynomial exactly as the reference evaluates them;
//   * mixed: positions as 32-bit fractional fixed point per box edge, so the minimal image is the
//     wrap-around of an int32 difference and the pair vector keeps full FP32 precision however
//     large the box; FP32 arithmetic with MUFU rsqrt/exp/rcp.
#include "pmb_internal.h"

namespace pmb {

namespace {

constexpr int PAIR_THREADS = 256;
constexpr int PAIR_WARPS = PAIR_THREADS / 32;
constexpr int CHUNK = 4;  // consecutive tiles per warp assignment

__device__ __forceinline__ int excl_check(const SystemDev &s, int oi, int oj) {
  int a = s.excl_start[oi], e = s.excl_start[oi + 1];
  for (int k = a; k < e; k++)
    if (s.excl_partner[k] == oj) return s.excl_kind[k];
  return 0;
}

template <typename T>
struct Acc {
  T fi[3], fj[3], elj, ec, vir[6];
};

template <bool MIXED>
struct SlotData;
template <>
struct SlotData<true> {
  uint4 p;   // fixed x, y, z, q bits
  int4 m;    // orig, mol, type, box
};
template <>
struct SlotData<false> {
  double4 p; // x, y, z, q
  int4 m;
};

template <typename T, bool LJ, int COUL, bool VIR>
__device__ __forceinline__ void pair_terms(const PairParams &p, const SystemDev &s, int ex,
                                           T r2, T dx, T dy, T dz, T qi, T qj,
                                           const T *ljrow, bool multi, const BoxDev *b,
                                           const double *lat, Acc<T> &a, T fjv[3]) {
  constexpr bool F32 = sizeof(T) == 4;
  T fs = T(0);
  if (ex != 2) {
    T rd2, rinv;
    if constexpr (F32) {
      rinv = rsqrtf(r2);
      rd2 = rinv * rinv;
    } else {
      rd2 = 1.0 / r2;
      rinv = T(0);
    }
    if constexpr (LJ) {
      if (r2 <= T(p.lj_cut2)) {
        T A = ex == 1 ? ljrow[2] : ljrow[0];
        T B = ex == 1 ? ljrow[3] : ljrow[1];
        T r6 = rd2 * rd2 * rd2, r12 = r6 * r6, r6B = B * r6, r12A = A * r12;
        T e = r12A - r6B;
        T f = T(12) * r12A * rd2 - T(6) * r6B * rd2;
        T val, der;
        switch_eval<T>(p.lj_sw, r2, val, der);
        f = f * val - e * der;
        e = e * val;
        a.elj += e;
        fs += f;
      }
    }
    if constexpr (COUL == 1) {
      if (r2 <= T(p.coul_cut2)) {
        T e;
        if constexpr (F32) e = qi * qj * rinv;
        else e = qi * qj * sqrt(rd2);
        if (ex == 1) e *= T(p.coulomb_scaling);
        T f = e * rd2;
        T val, der;
        switch_eval<T>(p.coul_sw, r2, val, der);
        f = f * val - e * der;
        e = e * val;
        a.ec += e;
        fs += f;
      }
    }
    if constexpr (COUL == 2) {
      if (r2 <= T(p.coul_cut2)) {
        T qq = qi * qj;
        if (ex == 1) qq *= T(p.coulomb_scaling);
        T e, f;
        if constexpr (F32) {
          T r = r2 * rinv, ar = T(p.alpha) * r;
          T g = qq * __expf(-ar * ar);
          e = poly5f(ar) * g * rinv;
          f = (e + T(p.a2pi) * g) * rd2;
        } else {
          T r = sqrt(r2), rr = 1.0 / r, ar = p.alpha * r;
          T g = qq * exp(-ar * ar);
          e = poly5(ar) * g * rr;
          f = (e + p.a2pi * g) * rr * rr;
        }
        T val, der;
        switch_eval<T>(p.coul_sw, r2, val, der);
        f = f * val - e * der;
        e = e * val;
        a.ec += e;
        fs += f;
      }
    }
  }
  T fx = dx * fs, fy = dy * fs, fz = dz * fs;
  if constexpr (VIR) {
    a.vir[0] += fx * dx; a.vir[1] += fx * dy; a.vir[2] += fx * dz;
    a.vir[3] += fy * dy; a.vir[4] += fy * dz; a.vir[5] += fz * dz;
  }
  if constexpr (COUL == 2) {
    // Lattice images beyond the minimal one (boxes with an edge below twice the cutoff):
    // NonbondedPMEwaldSystemForce.h:644-650 loops myLattice for every pair; FULL exclusions skip
    // only the first image and MODIFIED scaling applies to the first image only.
    if (multi) {
      for (int k = 1; k < b->nlat; k++) {
        const double *lv = lat + 3 * (b->lat0 + k);
        T rx = dx + T(lv[0]), ry = dy + T(lv[1]), rz = dz + T(lv[2]);
        T rr2 = rx * rx + ry * ry + rz * rz;
        if (rr2 > T(p.coul_cut2)) continue;
        T qq = qi * qj, e, f;
        if constexpr (F32) {
          T ri = rsqrtf(rr2), r = rr2 * ri, ar = T(p.alpha) * r;
          T g = qq * __expf(-ar * ar);
          e = poly5f(ar) * g * ri;
          f = (e + T(p.a2pi) * g) * ri * ri;
        } else {
          T r = sqrt(rr2), ri = 1.0 / r, ar = p.alpha * r;
          T g = qq * exp(-ar * ar);
          e = poly5(ar) * g * ri;
          f = (e + p.a2pi * g) * ri * ri;
        }
        T val, der;
        switch_eval<T>(p.coul_sw, rr2, val, der);
        f = f * val - e * der;
        e = e * val;
        a.ec += e;
        T gx = rx * f, gy = ry * f, gz = rz * f;
        fx += gx; fy += gy; fz += gz;
        if constexpr (VIR) {
          a.vir[0] += gx * rx; a.vir[1] += gx * ry; a.vir[2] += gx * rz;
          a.vir[3] += gy * ry; a.vir[4] += gy * rz; a.vir[5] += gz * rz;
        }
      }
    }
  }
  a.fi[0] -= fx; a.fi[1] -= fy; a.fi[2] -= fz;
  fjv[0] += fx; fjv[1] += fy; fjv[2] += fz;
}

template <bool MIXED, bool LJ, int COUL, bool VIR>
__global__ void __launch_bounds__(PAIR_THREADS) k_pair(SystemDev s, NbListDev nb, PairParams p,
                                                       const double *ljd, const double *lat) {
  using T = typename std::conditional<MIXED, float, double>::type;
  extern __shared__ unsigned char smem_raw[];
  T *lj = reinterpret_cast<T *>(smem_raw);                       // [nt*nt*4]
  const int nt = p.ntypes;
  size_t ljbytes = ((size_t)nt * nt * 4 * sizeof(T) + 15) & ~(size_t)15;
  SlotData<MIXED> *stage = reinterpret_cast<SlotData<MIXED> *>(smem_raw + ljbytes);
  for (int k = threadIdx.x; k < nt * nt * 4; k += blockDim.x) lj[k] = T(ljd[k]);
  __syncthreads();

  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  SlotData<MIXED> *sj = stage + wib * 32;
  const int gwarp = blockIdx.x * PAIR_WARPS + wib, nwarps = gridDim.x * PAIR_WARPS;
  int total = nb.tile_off[nb.nblk_total];
  if (total > nb.tile_cap) total = nb.tile_cap;

  int curI = -1, curBox = -1;
  long long ifix[3] = {0, 0, 0};
  long long efix_lj = 0, efix_c = 0, vfix[6] = {0, 0, 0, 0, 0, 0};
  SlotData<MIXED> si;
  const BoxDev *bx = nullptr;
  T sx = 0, sy = 0, sz = 0;

  auto flush_i = [&]() {
    if (curI >= 0 && si.m.x >= 0) {
      long long *f = s.facc + 3 * (long long)si.m.x;
      if (ifix[0]) red_add(f, ifix[0]);
      if (ifix[1]) red_add(f + 1, ifix[1]);
      if (ifix[2]) red_add(f + 2, ifix[2]);
    }
    ifix[0] = ifix[1] = ifix[2] = 0;
  };
  auto flush_e = [&]() {
    if (curBox >= 0 && lane == 0) {
      long long *e = s.eacc + (long long)curBox * ACC_PER_BOX;
      if (efix_lj) red_add(e + E_LJ, efix_lj);
      if (efix_c) red_add(e + E_COUL, efix_c);
      if constexpr (VIR) {
        // xx xy xz yy yz zz -> 3x3 row-major (symmetric)
        const int map[6][2] = {{0, -1}, {1, 3}, {2, 6}, {4, -1}, {5, 7}, {8, -1}};
        for (int c = 0; c < 6; c++) {
          if (!vfix[c]) continue;
          red_add(e + E_VIR + map[c][0], vfix[c]);
          if (map[c][1] >= 0) red_add(e + E_VIR + map[c][1], vfix[c]);
        }
      }
    }
    efix_lj = efix_c = 0;
    for (int c = 0; c < 6; c++) vfix[c] = 0;
  };

  for (int c0 = gwarp * CHUNK; c0 < total; c0 += nwarps * CHUNK) {
    int cend = min(c0 + CHUNK, total);
    for (int u = c0; u < cend; u++) {
      const int I = nb.tile_blk[u], k = nb.tile_k[u];
      if (I < 0 || I >= nb.nblk_total || k < 0 ||
          (k > 0 && (k - 1) * 32 >= nb.jcap_off[I + 1] - nb.jcap_off[I]))
        continue;  // unreachable with a consistent tile map; keeps every access in bounds
      if (I != curI) {
        flush_i();
        curI = I;
        const int sl = I * BLOCK + lane;
        si.m = nb.slot_meta[sl];
        if constexpr (MIXED) si.p = nb.slot_fx[sl];
        else si.p = nb.slot_pq[sl];
        int bidx = __shfl_sync(0xffffffffu, si.m.w, 0);
        if (bidx != curBox) {
          flush_e();
          curBox = bidx;
          bx = s.box + bidx;
          if constexpr (MIXED) {
            sx = T(bx->L[0] * (1.0 / 4294967296.0));
            sy = T(bx->L[1] * (1.0 / 4294967296.0));
            sz = T(bx->L[2] * (1.0 / 4294967296.0));
          }
        }
      }
      const bool diag = (k == 0);
      const int jsl = diag ? I * BLOCK + lane : nb.jlist[nb.jcap_off[I] + (k - 1) * 32 + lane];
      SlotData<MIXED> mine;
      if (jsl >= 0) {
        mine.m = nb.slot_meta[jsl];
        if constexpr (MIXED) mine.p = nb.slot_fx[jsl];
        else mine.p = nb.slot_pq[jsl];
      } else {
        mine.m = make_int4(-1, -1, 0, curBox);
        if constexpr (MIXED) mine.p = make_uint4(0, 0, 0, 0);
        else mine.p = make_double4(0, 0, 0, 0);
      }
      __syncwarp();
      sj[lane] = mine;
      __syncwarp();

      Acc<T> a;
      a.fi[0] = a.fi[1] = a.fi[2] = T(0);
      a.elj = a.ec = T(0);
      for (int c = 0; c < 6; c++) a.vir[c] = T(0);
      T fj[3] = {T(0), T(0), T(0)};
      const bool ivalid = si.m.x >= 0;
      const int ti = si.m.z;
      T qi;
      if constexpr (MIXED) qi = __uint_as_float(si.p.w);
      else qi = si.p.w;
      const bool multi = bx->multi_image != 0;

#pragma unroll 2
      for (int st = 0; st < 32; st++) {
        const int jj = (lane + st) & 31;
        const SlotData<MIXED> dj = sj[jj];
        bool ok = ivalid && dj.m.x >= 0 && (!diag || jj > lane);
        T dx, dy, dz, r2;
        if constexpr (MIXED) {
          dx = T((int)(dj.p.x - si.p.x)) * sx;
          dy = T((int)(dj.p.y - si.p.y)) * sy;
          dz = T((int)(dj.p.z - si.p.z)) * sz;
          r2 = dx * dx + dy * dy + dz * dz;
        } else {
          double c1[3] = {si.p.x, si.p.y, si.p.z}, c2[3] = {dj.p.x, dj.p.y, dj.p.z}, d[3];
          r2 = min_diff(*bx, c1, c2, d);
          dx = d[0]; dy = d[1]; dz = d[2];
        }
        if (ok && r2 <= T(p.cut2)) {
          int ex = 0;
          if (si.m.y == dj.m.y) ex = excl_check(s, si.m.x, dj.m.x);
          T qj;
          if constexpr (MIXED) qj = __uint_as_float(dj.p.w);
          else qj = dj.p.w;
          pair_terms<T, LJ, COUL, VIR>(p, s, ex, r2, dx, dy, dz, qi, qj,
                                        lj + 4 * (ti * nt + dj.m.z), multi, bx, lat, a, fj);
        }
        // rotate j-force accumulators: lane l takes over the one for j-atom (l + st + 1) & 31
        fj[0] = __shfl_sync(0xffffffffu, fj[0], (lane + 1) & 31);
        fj[1] = __shfl_sync(0xffffffffu, fj[1], (lane + 1) & 31);
        fj[2] = __shfl_sync(0xffffffffu, fj[2], (lane + 1) & 31);
      }
      // after 32 rotations lane l holds the accumulator of j-atom l
      if (diag) {
        a.fi[0] += fj[0]; a.fi[1] += fj[1]; a.fi[2] += fj[2];
      } else if (mine.m.x >= 0) {
        long long *f = s.facc + 3 * (long long)mine.m.x;
        long long v0 = f2fix(fj[0], (T)FORCE_SCALE), v1 = f2fix(fj[1], (T)FORCE_SCALE),
                  v2 = f2fix(fj[2], (T)FORCE_SCALE);
        if (v0) red_add(f, v0);
        if (v1) red_add(f + 1, v1);
        if (v2) red_add(f + 2, v2);
      }
      ifix[0] += f2fix(a.fi[0], (T)FORCE_SCALE);
      ifix[1] += f2fix(a.fi[1], (T)FORCE_SCALE);
      ifix[2] += f2fix(a.fi[2], (T)FORCE_SCALE);
      // energies: fixed-order warp sums per tile, then fixed point
      double el = (double)warp_sum(a.elj), ecc = (double)warp_sum(a.ec);
      efix_lj += f2fix(el, ENERGY_SCALE);
      efix_c += f2fix(ecc, ENERGY_SCALE);
      if constexpr (VIR) {
        for (int c = 0; c < 6; c++) vfix[c] += f2fix((double)warp_sum(a.vir[c]), ENERGY_SCALE);
      }
    }
  }
  flush_i();
  flush_e();
}

template <bool MIXED, bool LJ, int COUL, bool VIR>
int launch_t(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st) {
  auto kern = k_pair<MIXED, LJ, COUL, VIR>;
  using T = typename std::conditional<MIXED, float, double>::type;
  size_t ljbytes = ((size_t)pl.p.ntypes * pl.p.ntypes * 4 * sizeof(T) + 15) & ~(size_t)15;
  size_t smem = ljbytes + PAIR_WARPS * 32 * sizeof(SlotData<MIXED>);
  static int configured = 0, grid = 0;
  static size_t conf_smem = 0;
  if (!configured || conf_smem != smem) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, nsm = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, PAIR_THREADS, smem);
    if (occ < 1) occ = 1;
    grid = nsm * occ;
    configured = 1;
    conf_smem = smem;
  }
  kern<<<grid, PAIR_THREADS, smem, st>>>(s, nb, pl.p, pl.lj, pl.lattice);
  return 0;
}

template <bool MIXED>
int launch_p(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st) {
  const bool v = pl.p.virial != 0;
  if (pl.p.do_lj) {
    switch (pl.p.coul_mode) {
      case 0: return v ? launch_t<MIXED, true, 0, true>(s, nb, pl, st) : launch_t<MIXED, true, 0, false>(s, nb, pl, st);
      case 1: return v ? launch_t<MIXED, true, 1, true>(s, nb, pl, st) : launch_t<MIXED, true, 1, false>(s, nb, pl, st);
      default: return v ? launch_t<MIXED, true, 2, true>(s, nb, pl, st) : launch_t<MIXED, true, 2, false>(s, nb, pl, st);
    }
  }
  switch (pl.p.coul_mode) {
    case 1: return v ? launch_t<MIXED, false, 1, true>(s, nb, pl, st) : launch_t<MIXED, false, 1, false>(s, nb, pl, st);
    case 2: return v ? launch_t<MIXED, false, 2, true>(s, nb, pl, st) : launch_t<MIXED, false, 2, false>(s, nb, pl, st);
    default: return 0;
  }
}

}  // namespace

int pair_launch(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st) {
  if (pl.p.ntypes > MAX_LJ_TYPES) return -1;
  return pl.precision ? launch_p<true>(s, nb, pl, st) : launch_p<false>(s, nb, pl, st);
}

}  // namespace pmb
