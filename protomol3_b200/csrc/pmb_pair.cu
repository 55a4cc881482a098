// Fused nonbonded pair kernel: Lennard-Jones with C1/C2/cutoff switching plus either cutoff
// Coulomb (switched) or the Ewald real-space term, over the (8-atom i-cluster, 32 j-atoms)
// tiles built by pmb_nblist.cu.
//
// Replaces, per pair, OneAtomPair::doOneAtomPair / OneAtomPairTwo::doOneAtomPair
// (force/OneAtomPair.h:47-106, force/OneAtomPairTwo.h:30-96) with LennardJonesForce::operator()
// (force/LennardJonesForce.h:28-60), CoulombForce::operator() (force/CoulombForce.h:29-40) and
// the PME real-space body (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:644-700).
//
// Warp tiling: the BLOCK atoms of cluster I sit once in each of the GROUPS lane groups of the
// warp; the 32 j-atoms of the tile are staged in shared memory, lane group g visits j-atoms
// [g BLOCK, (g + 1) BLOCK) in rotations; the j-force accumulators travel with the rotation
// through shuffles inside the group (Newton's third law inside the tile), the groups' i-forces
// are combined once per tile.  A cluster's j-list opens with its own atoms (pairs j > i of lane
// group 0 in its first tile).  Forces leave as int64 fixed point by slot (one atomic per j-atom
// and per i-atom per tile); energies and virials are summed per lane and added in fixed point,
// so results are bit-identical run to run.
//
// The inner loop is branch-free: every lane evaluates the potentials on a clamped distance and
// the result is masked, because about half of the pairs of a tile lie outside the cutoff and a
// divergent branch would cost more than the masked arithmetic.  The switching functions of the
// common force sets are compile-time template parameters; other combinations use a generic
// instance with run-time switches.
//
// Two arithmetic paths share the structure:
//   * FP64 ("plain"): raw double positions, the reference's minimal image (d - L rint(d/L) gives
//     the same double as its single-wrap branches), IEEE division/sqrt/exp and the A&S erfc
//     polynomial exactly as the reference evaluates them;
//   * mixed: positions as 32-bit fractional fixed point per box edge, so the minimal image is the
//     wrap-around of an int32 difference and the pair vector keeps full FP32 precision however
//     large the box; FP32 arithmetic with MUFU rsqrt/exp2/rcp.
#include <cuda.h>

#include <mutex>
#include <type_traits>

#include "pmb_internal.h"

namespace pmb {

namespace {

// 128-thread blocks, 5 per SM for the mixed kernels (up to 102 registers: no spills, 20 warps per
// SM) measured faster than 256-thread blocks at 3 per SM (80 registers, spills): 167 against 170 us
#ifndef PAIR_BLOCK_THREADS
#define PAIR_BLOCK_THREADS 128
#endif
constexpr int PAIR_THREADS = PAIR_BLOCK_THREADS;
constexpr int PAIR_WARPS = PAIR_THREADS / 32;
constexpr int CHUNK = TILE_CHUNK;  // consecutive tiles per warp assignment

// switch / potential selectors (template parameters)
constexpr int SWR = -1;   // read the switching function kind at run time
constexpr int NONE = -2;  // potential absent

__device__ __forceinline__ int excl_check(const SystemDev &s, int oi, int oj) {
  int a = s.excl_start[oi], e = s.excl_start[oi + 1];
  for (int k = a; k < e; k++)
    if (s.excl_partner[k] == oj) return s.excl_kind[k];
  return 0;
}

// Pair parameters in the arithmetic type of the kernel, converted once on the host (the same
// round-to-nearest conversion the device would do), so the inner loop reads FP32 constants
// directly instead of converting FP64 parameters per pair.
template <typename T>
struct SwitchT {
  int kind;
  T rc2, ron2, s1, s2, s3, c15_1, c05_3, c15_3;
};
template <typename T>
struct ParamsT {
  int do_lj, ntypes;
  int lj_all, coul_all;  // the LJ / Coulomb cutoff covers the pair rejection radius
  SwitchT<T> lj_sw, coul_sw;
  T cut2, lj_cut2, coul_cut2, alpha, a2pi, coulomb_scaling;
  T kexp;  // -alpha^2 log2(e): exp(-alpha^2 r^2) = 2^(kexp r^2)
};

template <typename T>
SwitchT<T> switch_t(const SwitchDev &w) {
  SwitchT<T> o;
  o.kind = w.kind;
  o.rc2 = (T)w.rc2; o.ron2 = (T)w.ron2; o.s1 = (T)w.s1; o.s2 = (T)w.s2; o.s3 = (T)w.s3;
  o.c15_1 = (T)w.c15_1; o.c05_3 = (T)w.c05_3; o.c15_3 = (T)w.c15_3;
  return o;
}
template <typename T>
ParamsT<T> params_t(const PairParams &p) {
  ParamsT<T> o;
  o.do_lj = p.do_lj;
  o.ntypes = p.ntypes;
  o.lj_all = p.lj_cut2 >= p.cut2;
  o.coul_all = p.coul_cut2 >= p.cut2;
  o.lj_sw = switch_t<T>(p.lj_sw);
  o.coul_sw = switch_t<T>(p.coul_sw);
  o.cut2 = (T)p.cut2; o.lj_cut2 = (T)p.lj_cut2; o.coul_cut2 = (T)p.coul_cut2;
  o.alpha = (T)p.alpha; o.a2pi = (T)p.a2pi; o.coulomb_scaling = (T)p.coulomb_scaling;
  o.kexp = (T)(-p.alpha * p.alpha * 1.4426950408889634);
  return o;
}

// Switching function with compile-time kind K (SWR: run time).  value/derivative on r2 < rc2.
template <int K, typename T>
__device__ __forceinline__ void sw_apply(const SwitchT<T> &w, T r2, T &e, T &f) {
  const int kind = K == SWR ? w.kind : K;
  if (kind == SW_C2) {
    T c2 = T(w.rc2) - r2;
    T c4 = c2 * (T(w.s2) + T(2) * r2);
    bool on = r2 >= T(w.ron2);
    T val = on ? T(w.s1) * (c2 * c4) : T(1);
    T der = on ? T(w.s3) * (c2 * c2 - c4) : T(0);
    f = f * val - e * der;
    e = e * val;
  } else if (kind == SW_C1) {
    T dist = sqrt(r2);
    T val = T(1) - dist * (T(w.c15_1) - r2 * T(w.c05_3));
    T der = -T(w.c15_1) / dist + dist * T(w.c15_3);
    f = f * val - e * der;
    e = e * val;
  }
  // SW_CUTOFF: value 1 inside the cutoff, derivative 0
}

template <typename T>
struct Acc {
  T fi[3], elj, ec, vir[6];
};

// MUFU approximations for the FP32 path (hand-written PTX; flush-to-zero is harmless here:
// every operand is far from the denormal range).
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2_ftz(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// One pair: LJ (kind LSW) + Coulomb (mode CM: 0 none, 1 plain, 2 Ewald; switch CSW).
// Returns the scalar force/r; energies accumulate into a.  Masked lanes ('in' false) see zero
// parameters (A = B = q = 0), so every term vanishes without output selects.
template <bool MIXED, int LSW, int CM, int CSW>
__device__ __forceinline__ typename std::conditional<MIXED, float, double>::type pair_force(
    const ParamsT<typename std::conditional<MIXED, float, double>::type> &p, bool in, int ex,
    typename std::conditional<MIXED, float, double>::type r2,
    typename std::conditional<MIXED, float, double>::type qq,
    typename std::conditional<MIXED, float2, double2>::type ab,
    Acc<typename std::conditional<MIXED, float, double>::type> &a) {
  using T = typename std::conditional<MIXED, float, double>::type;
  const T r2s = in ? r2 : T(1);
  T rd2, rinv;
  if constexpr (MIXED) {
    rinv = rsqrt_ftz(r2s);
    rd2 = rinv * rinv;
  } else {
    rd2 = 1.0 / r2s;
    rinv = T(0);
  }
  T fs = T(0);
  if constexpr (LSW != NONE) {
    bool use = LSW != SWR || p.do_lj;
    if (use) {
      const bool inl = in && (p.lj_all || r2s <= p.lj_cut2);
      const T A = inl ? ab.x : T(0), B = inl ? ab.y : T(0);
      T r6 = rd2 * rd2 * rd2, r12 = r6 * r6, r6B = B * r6, r12A = A * r12;
      T e = r12A - r6B;
      T f = T(12) * r12A * rd2 - T(6) * r6B * rd2;
      sw_apply<LSW>(p.lj_sw, r2s, e, f);
      a.elj += e;
      fs += f;
    }
  }
  if constexpr (CM != 0) {
    const bool inc = in && (p.coul_all || r2s <= p.coul_cut2);
    T q = inc ? qq : T(0);
    if (ex == 1) q *= T(p.coulomb_scaling);
    T e, f;
    if constexpr (CM == 1) {
      if constexpr (MIXED) e = q * rinv;
      else e = q * sqrt(rd2);
      f = e * rd2;
    } else if constexpr (MIXED) {
      T r = r2s * rinv, ar = T(p.alpha) * r;
      T g = q * ex2_ftz(ar * ar * -1.4426950408889634f);
      T t = rcp_ftz(fmaf(0.3275911f, ar, 1.0f));
      T poly = t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f))));
      e = poly * g * rinv;
      f = (e + T(p.a2pi) * g) * rd2;
    } else {
      T r = sqrt(r2s), rr = 1.0 / r, ar = p.alpha * r;
      T g = q * exp(-ar * ar);
      e = poly5(ar) * g * rr;
      f = (e + p.a2pi * g) * rr * rr;
    }
    sw_apply<CSW>(p.coul_sw, r2s, e, f);
    a.ec += e;
    fs += f;
  }
  return fs;
}

// Shared-memory image of one j-atom of a tile (scalar path).  Mixed: coordinates relative to the
// first atom of the i-cluster (exact fixed-point difference converted to FP32 and scaled once per
// tile, not per pair: about 1 ulp at 13 A, 1e-6 A); padding atoms sit at -1e6 A (i padding at
// +1e6 A) so the cutoff test masks them.
template <bool MIXED>
struct JStage;
template <>
struct JStage<true> {
  float4 p;  // x, y, z relative, q
  int2 m;    // molecule, type
};
template <>
struct JStage<false> {
  double4 p;  // raw x, y, z, q
  int2 m;
};

// ------------------------------------------------------------------ packed FP32 tiles (mixed)
// Tiles whose j-atoms share no molecule with the i-cluster (no exclusion can apply; the list
// build flags the others) run on the two-wide FP32 instructions of sm_100 (FADD2 / FMUL2 /
// FFMA2): every lane evaluates two pairs per step, its i-atom with j-atoms jl and jl + HALF of its
// lane group, so HALF steps cover the group and each FP32 instruction issues two pairs' work.
// The j-atoms are staged as pairs {j, j + HALF} (x x' y y' | z z' q q' | type type'), each entry
// written twice (li and li + BLOCK), so step st reads entry li + st at a constant offset.
// Masking multiplies the parameters by 0/1 instead of selecting per result, and the C2 switch is
// evaluated at max(r2, ron2): its value there is 1 and its derivative 0 up to rounding, which
// removes the inner-radius branch.  Far pairs stay finite (relative coordinates are bounded by
// the box and the +-1e6 A sentinels), so masked terms are exact zeros.
constexpr int HALF = BLOCK / 2;
constexpr int GSTRIDE = 2 * BLOCK + 8;  // entries per lane group; +8 puts groups on other banks
constexpr int FAST_ENTRIES = GROUPS * GSTRIDE;
#ifndef PAIR2_UNROLL
#define PAIR2_UNROLL 4
#endif
constexpr int PAIR2_STEPS_UNROLLED = PAIR2_UNROLL;
#ifndef PAIR_MINB
#define PAIR_MINB 5  // resident blocks per SM of the mixed kernels
#endif
#ifndef PAIR_MINB_FP64
#define PAIR_MINB_FP64 5  // resident blocks per SM of the FP64 kernels (no virial, one image): 96 registers
#endif

// Operations whose operands are all per-pair values use the two-wide instructions; those with a
// constant operand (kernel parameters, polynomial coefficients) are issued as two scalar
// instructions, which read the constant bank directly instead of materialising a register pair
// per use (PAIR2_CONST_MODE 0: two-wide for those too; 2: everything scalar).
#ifndef PAIR2_CONST_MODE
#define PAIR2_CONST_MODE 0
#endif
__device__ __forceinline__ float2 sp2(float v) { return make_float2(v, v); }
#if PAIR2_CONST_MODE == 2
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
}
#else
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
#endif
#if PAIR2_CONST_MODE == 0
__device__ __forceinline__ float2 mulk(float2 a, float k) { return mul2(a, sp2(k)); }
__device__ __forceinline__ float2 fmak(float2 a, float k, float2 b) { return fma2(a, sp2(k), b); }
__device__ __forceinline__ float2 fmakk(float2 a, float k, float c) { return fma2(a, sp2(k), sp2(c)); }
__device__ __forceinline__ float2 fmaK(float2 a, float2 b, float c) { return fma2(a, b, sp2(c)); }
#else
// a k, a k + b, a k + c, a b + c with scalar constants k, c
__device__ __forceinline__ float2 mulk(float2 a, float k) { return make_float2(a.x * k, a.y * k); }
__device__ __forceinline__ float2 fmak(float2 a, float k, float2 b) {
  return make_float2(fmaf(a.x, k, b.x), fmaf(a.y, k, b.y));
}
__device__ __forceinline__ float2 fmakk(float2 a, float k, float c) {
  return make_float2(fmaf(a.x, k, c), fmaf(a.y, k, c));
}
__device__ __forceinline__ float2 fmaK(float2 a, float2 b, float c) {
  return make_float2(fmaf(a.x, b.x, c), fmaf(a.y, b.y, c));
}
#endif
// 1.0f where a <= b, else 0.0f (one SET instruction)
__device__ __forceinline__ float le_mask(float a, float b) {
  float r;
  asm("set.le.f32.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Asynchronous global -> shared copies (cp.async, L1-allocating) used to prefetch the next tile's
// j-list entries and slot records while the current tile computes.
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int K>
__device__ __forceinline__ void sw_apply2(const SwitchT<float> &w, float2 r2, float2 rinv, float2 &e,
                                          float2 &f) {
  const int kind = K == SWR ? w.kind : K;
  if (kind == SW_C2) {
    const float2 rc = make_float2(fmaxf(r2.x, w.ron2), fmaxf(r2.y, w.ron2));
    const float2 c2 = fmakk(rc, -1.f, w.rc2);
    const float2 nc4 = mul2(c2, fmakk(rc, -2.f, -w.s2));  // -c2 (s2 + 2 r2)
    const float2 val = mul2(mulk(c2, -w.s1), nc4);
    const float2 nder = mulk(fma2(c2, c2, nc4), -w.s3);
    f = fma2(e, nder, mul2(f, val));
    e = mul2(e, val);
  } else if (kind == SW_C1) {
    const float2 dist = mul2(r2, rinv);
    const float2 t = fmakk(r2, -w.c05_3, w.c15_1);
    const float2 val = fmakk(mul2(dist, t), -1.f, 1.f);
    const float2 nder = fmak(dist, -w.c15_3, mulk(rinv, w.c15_1));
    f = fma2(e, nder, mul2(f, val));
    e = mul2(e, val);
  }
}

struct Acc2 {
  float2 fi[3], fj[3], elj, ec, vir[6];
};

// HALF steps of one lane over its lane group's j-pairs; fi collects +f (the i-force is -fi).
// sa: this lane's first entry of the packed staging positions (z, charges at + FAST_ENTRIES);
// sty: its first entry of the packed types.  ALL: the LJ and Coulomb cutoffs both cover the pair
// cutoff (the common case), so the pair mask is the only one (chosen per tile, not per step).
template <int LSW, int CM, int CSW, bool VIR, bool ALL>
__device__ __forceinline__ void tile_pairs2(const ParamsT<float> &p, const float2 *__restrict__ ljab,
                                            int tio, const float4 *sa, const int2 *sty, int nxt,
                                            float xi, float yi, float zi, float qi, Acc2 &a) {
  const float2 nx = sp2(-xi), ny = sp2(-yi), nz = sp2(-zi), qi2 = sp2(qi);
#pragma unroll PAIR2_STEPS_UNROLLED
  for (int st = 0; st < HALF; st++) {
    const float4 u = sa[st], v = sa[FAST_ENTRIES + st];
    const int2 ty = sty[st];
    const float2 dx = add2(make_float2(u.x, u.y), nx), dy = add2(make_float2(u.z, u.w), ny),
                 dz = add2(make_float2(v.x, v.y), nz);
    const float2 r2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
    const float2 m = make_float2(le_mask(r2.x, p.cut2), le_mask(r2.y, p.cut2));
    const float2 rinv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    const float2 rd2 = mul2(rinv, rinv);
    float2 fs = sp2(0.f);
    if constexpr (LSW != NONE) {
      if (LSW != SWR || p.do_lj) {
        float2 ml = m;
        if (!ALL && !p.lj_all) ml = mul2(m, make_float2(le_mask(r2.x, p.lj_cut2), le_mask(r2.y, p.lj_cut2)));
        const float2 pa = ljab[tio + ty.x], pb = ljab[tio + ty.y];
        const float2 A = mul2(make_float2(pa.x, pb.x), ml), B = mul2(make_float2(pa.y, pb.y), ml);
        const float2 r6 = mul2(mul2(rd2, rd2), rd2);
        const float2 r6B = mul2(B, r6), r12A = mul2(A, mul2(r6, r6));
        float2 e = fmak(r6B, -1.f, r12A);
        float2 f = mul2(fmak(r12A, 12.f, mulk(r6B, -6.f)), rd2);
        sw_apply2<LSW>(p.lj_sw, r2, rinv, e, f);
        a.elj = add2(a.elj, e);
        fs = f;
      }
    }
    if constexpr (CM != 0) {
      float2 mc = m;
      if (!ALL && !p.coul_all) mc = mul2(m, make_float2(le_mask(r2.x, p.coul_cut2), le_mask(r2.y, p.coul_cut2)));
      const float2 q = mul2(make_float2(v.z, v.w), mul2(mc, qi2));
      float2 e, f;
      if constexpr (CM == 1) {
        e = mul2(q, rinv);
        f = mul2(e, rd2);
      } else {
        // erfc(a r) by Abramowitz & Stegun 7.1.26 as the reference evaluates it, exp(-a^2 r^2)
        // as 2^(r^2 kexp) with kexp = -a^2 log2(e)
        const float2 ar = mulk(mul2(r2, rinv), p.alpha);
        const float2 xe = mulk(r2, p.kexp);
        const float2 g = mul2(q, make_float2(ex2_ftz(xe.x), ex2_ftz(xe.y)));
        const float2 den = fmakk(ar, 0.3275911f, 1.f);
        const float2 t = make_float2(rcp_ftz(den.x), rcp_ftz(den.y));
        float2 h = fmakk(t, 1.061405429f, -1.453152027f);
        h = fmaK(t, h, 1.421413741f);
        h = fmaK(t, h, -0.284496736f);
        h = fmaK(t, h, 0.254829592f);
        e = mul2(mul2(mul2(t, h), g), rinv);
        f = mul2(fmak(g, p.a2pi, e), rd2);
      }
      sw_apply2<CSW>(p.coul_sw, r2, rinv, e, f);
      a.ec = add2(a.ec, e);
      fs = add2(fs, f);
    }
    const float2 fx = mul2(dx, fs), fy = mul2(dy, fs), fz = mul2(dz, fs);
    if constexpr (VIR) {
      a.vir[0] = fma2(fx, dx, a.vir[0]); a.vir[1] = fma2(fx, dy, a.vir[1]);
      a.vir[2] = fma2(fx, dz, a.vir[2]); a.vir[3] = fma2(fy, dy, a.vir[3]);
      a.vir[4] = fma2(fy, dz, a.vir[4]); a.vir[5] = fma2(fz, dz, a.vir[5]);
    }
    a.fi[0] = add2(a.fi[0], fx); a.fi[1] = add2(a.fi[1], fy); a.fi[2] = add2(a.fi[2], fz);
    a.fj[0] = add2(a.fj[0], fx); a.fj[1] = add2(a.fj[1], fy); a.fj[2] = add2(a.fj[2], fz);
    // rotate both j-force accumulators inside the lane group
#pragma unroll
    for (int c = 0; c < 3; c++)
      a.fj[c] = make_float2(__shfl_sync(0xffffffffu, a.fj[c].x, nxt), __shfl_sync(0xffffffffu, a.fj[c].y, nxt));
  }
}

// Bytes of one warp's j-staging region: the scalar layout (positions, metadata, original index as
// separate unit-stride arrays, bank-conflict free for 32 distinct j-atoms) or, mixed only, the
// packed layout; a tile uses one of them.
template <bool MIXED>
constexpr size_t warp_stage_bytes() {
  using JP = decltype(JStage<MIXED>::p);
  const size_t scalar = 32 * (sizeof(JP) + sizeof(int2) + sizeof(int));
  const size_t packed = MIXED ? FAST_ENTRIES * (2 * sizeof(float4) + sizeof(int2)) : 0;
  return ((scalar > packed ? scalar : packed) + 15) & ~(size_t)15;
}

// Per-warp constants of the current box and i-cluster.
struct WarpCtx {
  double s[3];     // box edge / 2^32: fractional fixed point to A
  float sf[3];     // the same in FP32 (j-atom staging: one conversion and one product per axis)
  float L[3], Lr[3];
  unsigned r0[3];  // fixed-point position of cluster atom 0 (mixed relative coordinates)
  int pad_;
};

// Bytes of one warp's prefetch region: the j-list entries of a chunk of tiles, and two buffers of
// slot records (position, metadata) and raw j-list words for the tile in flight and the next.
template <bool MIXED>
constexpr size_t warp_pref_bytes() {
  return 2 * 32 * (MIXED ? sizeof(uint4) : sizeof(double4)) + 2 * 32 * sizeof(int4) + CHUNK * 32 * sizeof(int) +
         2 * 32 * sizeof(int);
}

template <bool MIXED, int LSW, int CM, int CSW, bool VIR, bool MULTI>
__global__ void __launch_bounds__(PAIR_THREADS, (MIXED && !VIR && !MULTI) ? PAIR_MINB : (!MIXED && !VIR && !MULTI) ? PAIR_MINB_FP64 : 2)
    k_pair(SystemDev s, NbListDev nb, PairParams p,
           ParamsT<typename std::conditional<MIXED, float, double>::type> pt, const double *ljd,
           const double *lat, int blk_lo, int blk_hi, int wslot) {
  using T = typename std::conditional<MIXED, float, double>::type;
  using T2 = typename std::conditional<MIXED, float2, double2>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nt = p.ntypes, ntt = nt * nt;
  T2 *ljab = reinterpret_cast<T2 *>(smem_raw);  // [ntt] {A, B} then [ntt] {A14, B14}
  size_t ljbytes = ((size_t)2 * ntt * sizeof(T2) + 15) & ~(size_t)15;
  for (int k = threadIdx.x; k < ntt; k += blockDim.x) {
    ljab[k] = T2{T(ljd[4 * k]), T(ljd[4 * k + 1])};
    ljab[ntt + k] = T2{T(ljd[4 * k + 2]), T(ljd[4 * k + 3])};
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gb = lane & ~(BLOCK - 1), li = lane & (BLOCK - 1);  // lane group base, i-atom
  using JP = decltype(JStage<MIXED>::p);
  unsigned char *wstage = smem_raw + ljbytes + wib * warp_stage_bytes<MIXED>();
  JP *sjp = reinterpret_cast<JP *>(wstage);
  int2 *sjm = reinterpret_cast<int2 *>(sjp + 32);
  int *sorig = reinterpret_cast<int *>(sjm + 32);
  // packed layout (mixed): this lane's group and i-atom entry
  const int qe = (gb / BLOCK) * GSTRIDE + li;
  float4 *qa = reinterpret_cast<float4 *>(wstage) + qe;
  float4 *qb = qa + FAST_ENTRIES;
  int2 *qt = reinterpret_cast<int2 *>(reinterpret_cast<float4 *>(wstage) + 2 * FAST_ENTRIES) + qe;
  const int gwarp = blockIdx.x * PAIR_WARPS + wib, nwarps = gridDim.x * PAIR_WARPS;
  // this launch's tiles: those of blocks [blk_lo, blk_hi)
  int t_lo = nb.tile_start[blk_lo], t_hi = nb.tile_start[blk_hi];
  if (t_hi > nb.tile_cap) t_hi = nb.tile_cap;
  if (t_lo > t_hi) t_lo = t_hi;

  int curI = -1, curBox = -1;
  // energies (and virials) per lane: summed in the arithmetic type over a chunk of tiles, then
  // added in fixed point to this lane's slots in shared memory; summed over the warp and added to
  // the box accumulators when the box changes
  T el_acc = T(0), ec_acc = T(0), v_acc[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  constexpr int NE = VIR ? 8 : 2;
  long long *wsum = reinterpret_cast<long long *>(
      smem_raw + ljbytes + PAIR_WARPS * (warp_stage_bytes<MIXED>() + sizeof(WarpCtx))) + wib * NE * 32;
#pragma unroll
  for (int c = 0; c < NE; c++) wsum[c * 32 + lane] = 0;
  int4 im = make_int4(-1, -1, 0, 0);   // orig, mol, type, box of this lane's i-atom
  T xi = 0, yi = 0, zi = 0, qi = 0;     // i-atom position (relative for the mixed path)
  const BoxDev *bx = nullptr;
  bool wrap = !MIXED;
  // per-warp constants of the current box and cluster, kept in shared memory rather than in
  // registers (they are read once per tile)
  WarpCtx *ctx = reinterpret_cast<WarpCtx *>(smem_raw + ljbytes + PAIR_WARPS * warp_stage_bytes<MIXED>()) + wib;

  // forces accumulate by slot, one component-major array per axis: the j-atoms of a tile come
  // in runs of consecutive slots, so a lane group's atomics touch two sectors per axis rather than
  // eight scattered atoms (pair_fold moves them to original order afterwards)
  const long long nsl = nb.nslot;
  // i-forces of the current cluster per lane: the scalar path's in fi_acc, the packed path's
  // (+f, the i-force is -fi) in a2p.fi; combined over the lane groups and added by slot when the
  // cluster changes.  The packed path's energies and virial also accumulate in a2p over a chunk.
  T fi_acc[3] = {T(0), T(0), T(0)};
  Acc2 a2p;
#pragma unroll
  for (int c = 0; c < 3; c++) a2p.fi[c] = a2p.fj[c] = sp2(0.f);
  a2p.elj = a2p.ec = sp2(0.f);
#pragma unroll
  for (int c = 0; c < 6; c++) a2p.vir[c] = sp2(0.f);
  auto flush_fi = [&]() {  // warp-uniform
    T f[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      f[c] = fi_acc[c];
      if constexpr (MIXED) f[c] -= a2p.fi[c].x + a2p.fi[c].y;
    }
#pragma unroll
    for (int o = BLOCK; o < 32; o <<= 1)
#pragma unroll
      for (int c = 0; c < 3; c++) f[c] += __shfl_xor_sync(0xffffffffu, f[c], o);
    if (curI >= 0 && gb == 0 && im.x >= 0) {
      long long *fs = nb.fslot + (long long)curI * BLOCK + li;
      const long long v0 = f2fix(f[0], (T)FORCE_SCALE), v1 = f2fix(f[1], (T)FORCE_SCALE),
                      v2 = f2fix(f[2], (T)FORCE_SCALE);
      if (v0) red_add(fs, v0);
      if (v1) red_add(fs + nsl, v1);
      if (v2) red_add(fs + 2 * nsl, v2);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      fi_acc[c] = T(0);
      a2p.fi[c] = sp2(0.f);
    }
  };
  auto spill_e = [&]() {
    if constexpr (MIXED) {
      el_acc += a2p.elj.x + a2p.elj.y;
      ec_acc += a2p.ec.x + a2p.ec.y;
      a2p.elj = a2p.ec = sp2(0.f);
      if constexpr (VIR) {
#pragma unroll
        for (int c = 0; c < 6; c++) {
          v_acc[c] += a2p.vir[c].x + a2p.vir[c].y;
          a2p.vir[c] = sp2(0.f);
        }
      }
    }
    wsum[lane] += f2fix(el_acc, (T)ENERGY_SCALE);
    wsum[32 + lane] += f2fix(ec_acc, (T)ENERGY_SCALE);
    el_acc = ec_acc = T(0);
    if constexpr (VIR) {
#pragma unroll
      for (int c = 0; c < 6; c++) {
        wsum[(2 + c) * 32 + lane] += f2fix(v_acc[c], (T)ENERGY_SCALE);
        v_acc[c] = T(0);
      }
    }
  };
  auto flush_e = [&]() {  // warp-uniform
    spill_e();
    const long long el = warp_sum_ll(wsum[lane]), ec = warp_sum_ll(wsum[32 + lane]);
    long long vs[6] = {0, 0, 0, 0, 0, 0};
    if constexpr (VIR)
      for (int c = 0; c < 6; c++) vs[c] = warp_sum_ll(wsum[(2 + c) * 32 + lane]);
    if (curBox >= 0 && lane == 0) {
      long long *e = s.eacc + (long long)curBox * ACC_PER_BOX;
      if (el) red_add(e + E_LJ, el);
      if (ec) red_add(e + E_COUL, ec);
      if constexpr (VIR) {
        const int map[6][2] = {{0, -1}, {1, 3}, {2, 6}, {4, -1}, {5, 7}, {8, -1}};
        for (int c = 0; c < 6; c++) {
          if (!vs[c]) continue;
          red_add(e + E_VIR + map[c][0], vs[c]);
          if (map[c][1] >= 0) red_add(e + E_VIR + map[c][1], vs[c]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NE; c++) wsum[c * 32 + lane] = 0;
  };
  // stage one slot (or padding) as this lane's j-atom
  // (padding slots of a box's last cluster, orig < 0, become sentinels as well: they carry no
  // charge but an LJ type, and must never meet a real atom)
  // prefetch region: slot records [2][32], metadata [2][32], a chunk's j-list words [CHUNK][32],
  // raw j-list words of the buffered tiles [2][32]
  using RawP = typename std::conditional<MIXED, uint4, double4>::type;
  unsigned char *wpref = smem_raw + ljbytes +
                         PAIR_WARPS * (warp_stage_bytes<MIXED>() + sizeof(WarpCtx) + NE * 32 * sizeof(long long)) +
                         wib * warp_pref_bytes<MIXED>();
  RawP *rawP = reinterpret_cast<RawP *>(wpref);
  int4 *rawM = reinterpret_cast<int4 *>(rawP + 64);
  int *jbuf = reinterpret_cast<int *>(rawM + 64);
  int *rawJ = jbuf + CHUNK * 32;
  int tI = -1, tk = -1, tjb = 0;  // lane t < CHUNK: block, index and j-list offset of chunk tile t
  // issues the copies of tile t's slot records into buffer b (warp-uniform; one commit group)
  auto prefetch = [&](int t, int b) {
    const int It = __shfl_sync(0xffffffffu, tI, t), kt = __shfl_sync(0xffffffffu, tk, t);
    int jr = -1;
    if (It >= 0) jr = jbuf[t * 32 + lane];
    rawJ[b * 32 + lane] = jr;
    const int sl = jr < 0 ? -1 : (jr & ~JSAME);
    if (sl >= 0) {
      if constexpr (MIXED) {
        cp_async16(rawP + b * 32 + lane, nb.slot_fx + sl);
      } else {
        cp_async16(rawP + b * 32 + lane, nb.slot_pq + sl);
        cp_async16(reinterpret_cast<unsigned char *>(rawP + b * 32 + lane) + 16,
                   reinterpret_cast<const unsigned char *>(nb.slot_pq + sl) + 16);
      }
      cp_async16(rawM + b * 32 + lane, nb.slot_meta + sl);
    }
    cp_async_commit();
  };
  // stage this lane's j-atom of buffer b (or padding)
  auto stage_slot = [&](int sl, int b, JStage<MIXED> &js, int &orig) {
    const int4 m = sl >= 0 ? rawM[b * 32 + lane] : make_int4(-1, -1, 0, 0);
    if (m.x >= 0) {
      orig = m.x;
      js.m = make_int2(m.y, m.z);
      if constexpr (MIXED) {
        const uint4 f = rawP[b * 32 + lane];
        js.p = make_float4((float)(int)(f.x - ctx->r0[0]) * ctx->sf[0],
                           (float)(int)(f.y - ctx->r0[1]) * ctx->sf[1],
                           (float)(int)(f.z - ctx->r0[2]) * ctx->sf[2], __uint_as_float(f.w));
      } else {
        js.p = rawP[b * 32 + lane];
      }
    } else {
      orig = -1;
      js.m = make_int2(-1, 0);
      if constexpr (MIXED) js.p = make_float4(-1e6f, -1e6f, -1e6f, 0.f);
      else js.p = make_double4(-1e6, -1e6, -1e6, 0.0);
    }
  };

  // Tiles go to warps in chunks of CHUNK consecutive tiles: chunk gwarp first, then the next
  // unclaimed chunk from the launch's counter (ctl[6 + 2 wslot]), so warps that start late (SMs busy with the PME
  // kernels beside this one) take fewer chunks.  The floating-point partial sums (i-forces,
  // energies, virial) are closed at every chunk end, so the result does not depend on which warp
  // took which chunk.  Per chunk the tile records and their j-list words are fetched once (one
  // round trip each); each tile's slot records are copied one tile ahead into the other buffer,
  // so only the first tile of a chunk waits for them.
  unsigned *wq = nb.ctl + 6 + 2 * wslot;
  const int nchunk = (t_hi - t_lo + CHUNK - 1) / CHUNK;
  for (int ci = gwarp; ci < nchunk;) {
    int tnext = 0;
    if (lane == 0) tnext = nwarps + (int)atomicAdd(wq, 1u);  // claimed now, read at chunk end
    const int c0 = t_lo + ci * CHUNK;
    const int nc = min(CHUNK, t_hi - c0);
    tI = -1;
    tk = -1;
    tjb = 0;
    if (lane < nc) {
      const int I = nb.tile_blk[c0 + lane], k = nb.tile_k[c0 + lane];
      // an inconsistent tile record is skipped (unreachable; keeps every access in bounds)
      if (I >= 0 && I < nb.nblk_total && k >= 0) {
        const int j0 = nb.jcap_off[I], j1 = nb.jcap_off[I + 1];
        if (k * JCHUNK < j1 - j0) {
          tI = I;
          tk = k;
          tjb = j0 + k * JCHUNK;
        }
      }
    }
    for (int t = 0; t < nc; t++) {
      const int It = __shfl_sync(0xffffffffu, tI, t), kt = __shfl_sync(0xffffffffu, tk, t),
                jb = __shfl_sync(0xffffffffu, tjb, t);
      if (It >= 0) cp_async4(jbuf + t * 32 + lane, nb.jlist + jb + lane);
    }
    cp_async_commit();
    cp_async_wait<0>();
    prefetch(0, 0);
    for (int t = 0; t < nc; t++) {
      if (t + 1 < nc) prefetch(t + 1, (t + 1) & 1);
      else cp_async_commit();  // an empty group keeps the wait count below uniform
      cp_async_wait<1>();      // tile t's copies (all but the newest group) have landed
      const int buf = t & 1;
      const int I = __shfl_sync(0xffffffffu, tI, t), k = __shfl_sync(0xffffffffu, tk, t);
      if (I < 0) continue;
      if (I != curI) {
        flush_fi();
        curI = I;
        const int sl = I * BLOCK + li;
        im = nb.slot_meta[sl];
        const int bidx = __shfl_sync(0xffffffffu, im.w, 0);
        if (bidx != curBox) {
          flush_e();
          curBox = bidx;
          bx = s.box + bidx;
          __syncwarp();
          if (lane == 0)
            for (int c = 0; c < 3; c++) {
              ctx->s[c] = bx->L[c] * (1.0 / 4294967296.0);
              ctx->sf[c] = (float)(bx->L[c] * (1.0 / 4294967296.0));
              ctx->L[c] = (float)bx->L[c];
              ctx->Lr[c] = (float)bx->Lr[c];
            }
        }
        if constexpr (MIXED) {
          // coordinates relative to cluster atom 0 are minimal-image differences whenever
          // L/2 > cutoff + cluster extent; otherwise (small boxes) every pair is wrapped again
          const uint4 lo = nb.blk_lo[I], hi = nb.blk_hi[I];
          const double rmax = sqrt(p.cut2) + 1e-3;
          const double sx = bx->L[0] * (1.0 / 4294967296.0), sy = bx->L[1] * (1.0 / 4294967296.0),
                       sz = bx->L[2] * (1.0 / 4294967296.0);
          wrap = bx->multi_image || (double)(hi.x - lo.x) * sx + rmax >= 0.5 * bx->L[0] ||
                 (double)(hi.y - lo.y) * sy + rmax >= 0.5 * bx->L[1] ||
                 (double)(hi.z - lo.z) * sz + rmax >= 0.5 * bx->L[2];
          const uint4 f = nb.slot_fx[sl];
          const unsigned rx0 = __shfl_sync(0xffffffffu, f.x, 0), ry0 = __shfl_sync(0xffffffffu, f.y, 0),
                         rz0 = __shfl_sync(0xffffffffu, f.z, 0);
          __syncwarp();
          if (lane == 0) {
            ctx->r0[0] = rx0;
            ctx->r0[1] = ry0;
            ctx->r0[2] = rz0;
          }
          __syncwarp();
          if (im.x >= 0) {
            xi = (float)((double)(int)(f.x - rx0) * sx);
            yi = (float)((double)(int)(f.y - ry0) * sy);
            zi = (float)((double)(int)(f.z - rz0) * sz);
          } else {
            xi = yi = zi = 1e6f;
          }
          qi = __uint_as_float(f.w);
        } else {
          const double4 q4 = nb.slot_pq[sl];
          if (im.x >= 0) {
            xi = q4.x; yi = q4.y; zi = q4.z;
          } else {
            xi = yi = zi = 1e6;
          }
          qi = q4.w;
        }
      }
      // 32 listed j-atoms, JSAME marking those that share a molecule with the cluster; the first
      // tile opens with the cluster's own atoms (lane group 0, pairs j > i only)
      const bool diag = (k == 0);
      const int jraw = rawJ[buf * 32 + lane];
      const int jsl = jraw < 0 ? -1 : (jraw & ~JSAME);
      const bool same = diag || __any_sync(0xffffffffu, jraw >= 0 && (jraw & JSAME));
      JStage<MIXED> mine;
      int jorig;
      stage_slot(jsl, buf, mine, jorig);
      const int tio = im.z * nt;
      const int nxt = gb | ((li + 1) & (BLOCK - 1));
      T tfj[3];  // this lane's j-atom force of the tile

      bool packed = false;
      if constexpr (MIXED) {
        if (!wrap && !same) {
          packed = true;
          // the pair partner (j + HALF) of this lane's j-atom, then two copies of the entry
          const float4 P = mine.p;
          const float px = __shfl_xor_sync(0xffffffffu, P.x, HALF), py = __shfl_xor_sync(0xffffffffu, P.y, HALF),
                      pz = __shfl_xor_sync(0xffffffffu, P.z, HALF), pq = __shfl_xor_sync(0xffffffffu, P.w, HALF);
          const int ptype = __shfl_xor_sync(0xffffffffu, mine.m.y, HALF);
          const float4 ea = make_float4(P.x, px, P.y, py), eb = make_float4(P.z, pz, P.w, pq);
          const int2 et = make_int2(mine.m.y, ptype);
          __syncwarp();
          qa[0] = ea; qa[BLOCK] = ea;
          qb[0] = eb; qb[BLOCK] = eb;
          qt[0] = et; qt[BLOCK] = et;
          __syncwarp();
#pragma unroll
          for (int c = 0; c < 3; c++) a2p.fj[c] = sp2(0.f);
          if (pt.lj_all && pt.coul_all)
            tile_pairs2<LSW, CM, CSW, VIR, true>(pt, reinterpret_cast<const float2 *>(ljab), tio, qa, qt, nxt, xi,
                                                 yi, zi, qi, a2p);
          else
            tile_pairs2<LSW, CM, CSW, VIR, false>(pt, reinterpret_cast<const float2 *>(ljab), tio, qa, qt, nxt,
                                                  xi, yi, zi, qi, a2p);
          // after HALF rotations: .y holds this lane's j-atom, .x that of the lane HALF away
#pragma unroll
          for (int c = 0; c < 3; c++) tfj[c] = a2p.fj[c].y + __shfl_xor_sync(0xffffffffu, a2p.fj[c].x, HALF);
        }
      }
      if (!packed) {
        __syncwarp();
        sjp[lane] = mine.p;
        sjm[lane] = mine.m;
        sorig[lane] = jorig;
        __syncwarp();

        Acc<T> a;
        a.fi[0] = a.fi[1] = a.fi[2] = T(0);
        a.elj = a.ec = T(0);
        for (int c = 0; c < 6; c++) a.vir[c] = T(0);
        T fj[3] = {T(0), T(0), T(0)};
        const T cut2 = pt.cut2;

        const bool ivalid = im.x >= 0;
        auto body = [&](auto diag_tag, auto wrap_tag) {
          constexpr bool DIAG = decltype(diag_tag)::value;
          constexpr bool WRAP = decltype(wrap_tag)::value;
#pragma unroll 2
          for (int st = 0; st < BLOCK; st++) {
            const int jl = (li + st) & (BLOCK - 1);
            JStage<MIXED> dj;
            dj.p = sjp[gb | jl];
            dj.m = sjm[gb | jl];
            T dx = T(dj.p.x) - xi, dy = T(dj.p.y) - yi, dz = T(dj.p.z) - zi;
            if constexpr (!MIXED) {
              // the reference's minimal image: d - L rint(d / L) equals its single-wrap result
              dx -= bx->L[0] * rint(bx->Lr[0] * dx);
              dy -= bx->L[1] * rint(bx->Lr[1] * dy);
              dz -= bx->L[2] * rint(bx->Lr[2] * dz);
            } else if constexpr (WRAP) {
              dx -= ctx->L[0] * rintf(ctx->Lr[0] * dx);
              dy -= ctx->L[1] * rintf(ctx->Lr[1] * dy);
              dz -= ctx->L[2] * rintf(ctx->Lr[2] * dz);
            }
            const T r2 = dx * dx + dy * dy + dz * dz;
            bool in = r2 <= cut2;
            if constexpr (WRAP) in = in && ivalid && dj.m.x >= 0;  // sentinels do not survive a wrap
            if constexpr (DIAG) in = in && (gb != 0 || jl > li);
            int ex = 0;
            if (in && im.y == dj.m.x) {
              ex = excl_check(s, im.x, sorig[gb | jl]);
              if (ex == 2) in = false;
            }
            T2 ab;
            if constexpr (LSW != NONE) ab = ljab[(ex == 1 ? ntt : 0) + tio + dj.m.y];
            else ab = T2{T(0), T(0)};
            T fs = pair_force<MIXED, LSW, CM, CSW>(pt, in, ex, r2, qi * T(dj.p.w), ab, a);
            T fx = dx * fs, fy = dy * fs, fz = dz * fs;
            if constexpr (VIR) {
              a.vir[0] += fx * dx; a.vir[1] += fx * dy; a.vir[2] += fx * dz;
              a.vir[3] += fy * dy; a.vir[4] += fy * dz; a.vir[5] += fz * dz;
            }
            if constexpr (CM == 2 && MULTI && WRAP) {
              // Lattice images beyond the minimal one (edge below twice the cutoff): the reference
              // loops myLattice for every pair (NonbondedPMEwaldSystemForce.h:644-650); FULL
              // exclusions skip only the first image, MODIFIED scaling applies to it only.
              if (bx->multi_image) {
                bool pv = dj.m.x >= 0 && im.x >= 0;
                if constexpr (DIAG) pv = pv && (gb != 0 || jl > li);
                for (int kk = 1; kk < bx->nlat; kk++) {
                  const double *lv = lat + 3 * (bx->lat0 + kk);
                  T rx = dx + T(lv[0]), ry = dy + T(lv[1]), rz = dz + T(lv[2]);
                  T rr2 = rx * rx + ry * ry + rz * rz;
                  bool inl = pv && rr2 <= pt.coul_cut2;
                  Acc<T> b2;
                  b2.elj = T(0);
                  b2.ec = T(0);
                  T g = pair_force<MIXED, NONE, 2, CSW>(pt, inl, 0, rr2, qi * T(dj.p.w), T2{T(0), T(0)}, b2);
                  a.ec += b2.ec;
                  T gx = rx * g, gy = ry * g, gz = rz * g;
                  fx += gx; fy += gy; fz += gz;
                  if constexpr (VIR) {
                    a.vir[0] += gx * rx; a.vir[1] += gx * ry; a.vir[2] += gx * rz;
                    a.vir[3] += gy * ry; a.vir[4] += gy * rz; a.vir[5] += gz * rz;
                  }
                }
              }
            }
            a.fi[0] -= fx; a.fi[1] -= fy; a.fi[2] -= fz;
            fj[0] += fx; fj[1] += fy; fj[2] += fz;
            // rotate j-force accumulators inside the lane group
            fj[0] = __shfl_sync(0xffffffffu, fj[0], nxt);
            fj[1] = __shfl_sync(0xffffffffu, fj[1], nxt);
            fj[2] = __shfl_sync(0xffffffffu, fj[2], nxt);
          }
        };
        bool unwrapped = false;
        if constexpr (MIXED) {
          if (!wrap) {
            unwrapped = true;
            if (diag) body(std::true_type{}, std::false_type{});
            else body(std::false_type{}, std::false_type{});
          }
        }
        if (!unwrapped) {
          if (diag) body(std::true_type{}, std::true_type{});
          else body(std::false_type{}, std::true_type{});
        }
        // after BLOCK rotations lane l holds the accumulator of j-atom l of the tile
#pragma unroll
        for (int c = 0; c < 3; c++) {
          fi_acc[c] += a.fi[c];
          tfj[c] = fj[c];
        }
        el_acc += a.elj;
        ec_acc += a.ec;
        if constexpr (VIR)
          for (int c = 0; c < 6; c++) v_acc[c] += a.vir[c];
      }

      if (diag && gb == 0) {  // own atom li: its j-side force joins its i-side force
#pragma unroll
        for (int c = 0; c < 3; c++) fi_acc[c] += tfj[c];
      } else if (jorig >= 0) {
        long long *f = nb.fslot + jsl;
        long long v0 = f2fix(tfj[0], (T)FORCE_SCALE), v1 = f2fix(tfj[1], (T)FORCE_SCALE),
                  v2 = f2fix(tfj[2], (T)FORCE_SCALE);
        red_add(f, v0);
        red_add(f + nsl, v1);
        red_add(f + 2 * nsl, v2);
      }
    }
    spill_e();
    flush_fi();
    ci = __shfl_sync(0xffffffffu, tnext, 0);
  }
  flush_fi();
  flush_e();
  // the last warp to finish resets the chunk counter for the next launch (every warp has made
  // its last claim before it counts itself here)
  if (lane == 0 && atomicAdd(wq + 1, 1u) == (unsigned)nwarps - 1u) {
    atomicExch(wq, 0u);
    atomicExch(wq + 1, 0u);
  }
}

template <bool MIXED, int LSW, int CM, int CSW, bool VIR, bool MULTI = false>
int launch_t(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st) {
  if constexpr (CM == 2 && !MULTI) {
    if (pl.multi) return launch_t<MIXED, LSW, CM, CSW, VIR, true>(s, nb, pl, st);
  }
  auto kern = k_pair<MIXED, LSW, CM, CSW, VIR, MULTI>;
  using T2 = typename std::conditional<MIXED, float2, double2>::type;
  const int ntt = pl.p.ntypes * pl.p.ntypes;
  size_t ljbytes = ((size_t)2 * ntt * sizeof(T2) + 15) & ~(size_t)15;
  size_t smem = ljbytes + PAIR_WARPS * (warp_stage_bytes<MIXED>() + sizeof(WarpCtx) +
                                        (VIR ? 8 : 2) * 32 * sizeof(long long) + warp_pref_bytes<MIXED>());
  // per device: the SM count, the resident blocks and the shared-memory limit they were found for
  static int n_sm[PMB_MAX_DEVICES] = {}, occupancy[PMB_MAX_DEVICES] = {};
  static size_t conf_smem[PMB_MAX_DEVICES] = {};
  const int slot = device_slot();
  if (!n_sm[slot] || conf_smem[slot] != smem) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, nsm = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, PAIR_THREADS, smem);
    if (occ < 1) occ = 1;
    n_sm[slot] = nsm;
    occupancy[slot] = occ;
    conf_smem[slot] = smem;
  }
  // persistent: every resident CTA walks its share of the tiles (chunks claimed from a counter,
  // so any grid size gives the same result)
  const int occ = occupancy[slot];
  const int per_sm = pl.ctas_per_sm > 0 && pl.ctas_per_sm < occ ? pl.ctas_per_sm : occ;
  const int grid = n_sm[slot] * per_sm;
  using T = typename std::conditional<MIXED, float, double>::type;
  kern<<<grid, PAIR_THREADS, smem, st>>>(s, nb, pl.p, params_t<T>(pl.p), pl.lj, pl.lattice, pl.blk_lo, pl.blk_hi,
                                         pl.wslot);
  return 0;
}

template <bool MIXED, bool VIR>
int launch_v(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st) {
  const PairParams &p = pl.p;
  const int lk = p.do_lj ? p.lj_sw.kind : NONE, ck = p.coul_sw.kind;
  // specialised force sets: LJ C2 + Ewald real (cutoff), LJ C2 + Coulomb C2, LJ C2 alone,
  // Ewald real alone
  if (lk == SW_C2 && p.coul_mode == 2 && ck == SW_CUTOFF) return launch_t<MIXED, SW_C2, 2, SW_CUTOFF, VIR>(s, nb, pl, st);
  if (lk == SW_C2 && p.coul_mode == 1 && ck == SW_C2) return launch_t<MIXED, SW_C2, 1, SW_C2, VIR>(s, nb, pl, st);
  if (lk == SW_C2 && p.coul_mode == 0) return launch_t<MIXED, SW_C2, 0, SW_CUTOFF, VIR>(s, nb, pl, st);
  if (lk == NONE && p.coul_mode == 2 && ck == SW_CUTOFF) return launch_t<MIXED, NONE, 2, SW_CUTOFF, VIR>(s, nb, pl, st);
  // generic: switching functions (and the LJ term) chosen at run time
  switch (p.coul_mode) {
    case 0: return launch_t<MIXED, SWR, 0, SWR, VIR>(s, nb, pl, st);
    case 1: return launch_t<MIXED, SWR, 1, SWR, VIR>(s, nb, pl, st);
    default: return launch_t<MIXED, SWR, 2, SWR, VIR>(s, nb, pl, st);
  }
}

}  // namespace

// Adds the slot-ordered pair forces to the original-order accumulator and clears them (one thread
// per slot; each atom owns one slot, so the read-modify-write needs no atomics).
__global__ void k_pair_fold(SystemDev s, NbListDev nb) {
  const int sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= nb.nslot) return;
  const int o = nb.slot_orig[sl];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    long long *p = nb.fslot + (long long)c * nb.nslot + sl;
    const long long v = *p;
    if (v) {
      *p = 0;
      if (o >= 0) s.facc[3 * (long long)o + c] += v;
    }
  }
}

int pair_fold(const SystemDev &s, const NbListDev &nb, cudaStream_t st) {
  const int T = 256;
  if (nb.nslot > 0) k_pair_fold<<<(nb.nslot + T - 1) / T, T, 0, st>>>(s, nb);
  return 0;
}

int pair_launch(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st) {
  if (pl.p.ntypes > MAX_LJ_TYPES) return -1;
  if (pl.precision) return pl.p.virial ? launch_v<true, true>(s, nb, pl, st) : launch_v<true, false>(s, nb, pl, st);
  return pl.p.virial ? launch_v<false, true>(s, nb, pl, st) : launch_v<false, false>(s, nb, pl, st);
}

// ======================================================================= allocation-free variant
// All-pairs FP64 variant of the cutoff pair kernel for callers that may not allocate device
// memory: no neighbour list, every pair of a box visited from both sides (each thread sums the
// full force on its own atom in registers and stores it, so forces need no accumulator and no
// atomics); energies and the virial count each pair once (j > i) and are added in fixed point to
// per-box accumulators that live in a static device array instead of the system's buffers.
namespace {

constexpr int AP_THREADS = 128;

// Fixed-point energy / virial accumulators of the allocation-free pass,
// [STATIC_MAX_BOXES][ACC_PER_BOX] int64 = 128 KiB.  Zeroed by every call before use.
static __device__ __align__(256) long long g_static_eacc[STATIC_MAX_BOXES * ACC_PER_BOX];

template <int CM, bool VIR>
__global__ void __launch_bounds__(AP_THREADS)
    k_pair_allpairs(SystemDev s, ParamsT<double> p, const double *ljd, const double *pos, double *fout,
                    long long *eacc) {
  __shared__ double4 sp[AP_THREADS];  // j-atoms of the tile: x, y, z, q
  __shared__ int2 sm[AP_THREADS];     // molecule, type
  const int b = blockIdx.y;
  const BoxDev &bx = s.box[b];
  const int n = bx.natoms;
  if ((int)blockIdx.x * AP_THREADS >= n) return;  // whole block: no atom of this box left
  const int li = blockIdx.x * AP_THREADS + threadIdx.x;
  const bool valid = li < n;
  const int i = bx.atom0 + (valid ? li : 0);
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2], qi = s.charge[i];
  const int mi = s.molecule[i], ti = s.type[i], nt = p.ntypes;
  double fi[3] = {0.0, 0.0, 0.0}, elj = 0.0, ec = 0.0, vir[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int j0 = 0; j0 < n; j0 += AP_THREADS) {
    __syncthreads();
    const int lj = j0 + threadIdx.x;
    if (lj < n) {
      const int j = bx.atom0 + lj;
      sp[threadIdx.x] = make_double4(pos[3 * j], pos[3 * j + 1], pos[3 * j + 2], s.charge[j]);
      sm[threadIdx.x] = make_int2(s.molecule[j], s.type[j]);
    }
    __syncthreads();
    const int nj = min(AP_THREADS, n - j0);
    for (int k = 0; k < nj; k++) {
      const double4 pj = sp[k];
      const int2 mj = sm[k];
      double dx = pj.x - xi, dy = pj.y - yi, dz = pj.z - zi;
      // the reference's minimal image: d - L rint(d / L) equals its single-wrap result
      dx -= bx.L[0] * rint(bx.Lr[0] * dx);
      dy -= bx.L[1] * rint(bx.Lr[1] * dy);
      dz -= bx.L[2] * rint(bx.Lr[2] * dz);
      const double r2 = dx * dx + dy * dy + dz * dz;
      bool in = valid && j0 + k != li && r2 <= p.cut2;
      int ex = 0;
      if (in && mj.x == mi) {
        ex = excl_check(s, i, bx.atom0 + j0 + k);
        if (ex == 2) in = false;
      }
      const double *ab = ljd + 4 * (ti * nt + mj.y) + (ex == 1 ? 2 : 0);
      Acc<double> t;
      t.elj = t.ec = 0.0;
      const double fs = pair_force<false, SWR, CM, SWR>(p, in, ex, r2, qi * pj.w, double2{ab[0], ab[1]}, t);
      const double fx = dx * fs, fy = dy * fs, fz = dz * fs;
      fi[0] -= fx;
      fi[1] -= fy;
      fi[2] -= fz;
      if (j0 + k > li) {
        elj += t.elj;
        ec += t.ec;
        if constexpr (VIR) {
          vir[0] += fx * dx; vir[1] += fx * dy; vir[2] += fx * dz;
          vir[3] += fy * dy; vir[4] += fy * dz; vir[5] += fz * dz;
        }
      }
    }
  }
  if (valid) {
    fout[3 * i] = fi[0];
    fout[3 * i + 1] = fi[1];
    fout[3 * i + 2] = fi[2];
  }
  box_accumulate(eacc, b, valid, E_LJ, elj, nullptr);
  box_accumulate(eacc, b, valid, E_COUL, ec, VIR ? vir : nullptr);
}

}  // namespace

// Identity of the calling thread's current CUDA context (cuCtxGetId, unique over the process's
// life even when a context is destroyed and another gets its handle), through the driver entry
// points the runtime hands out, so the library does not link the driver library itself.  0 when
// it cannot be had.
static unsigned long long current_context_id() {
  using get_current_t = CUresult (*)(CUcontext *);
  using get_id_t = CUresult (*)(CUcontext, unsigned long long *);
  static get_current_t get_current = nullptr;
  static get_id_t get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void *f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<get_current_t>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<get_id_t>(f);
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// The device address of the static scratch in the current context, looked up once per device
// and context: an address belongs to the context it was taken in, so a context made after
// cudaDeviceReset gets its own lookup.
cudaError_t static_eacc_address(long long **out) {
  constexpr int MAX_DEV = 64;
  static std::mutex mu;
  static long long *addr[MAX_DEV] = {};
  static unsigned long long ctx[MAX_DEV] = {};
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEV) return cudaErrorInvalidDevice;
  const unsigned long long id = current_context_id();
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev] || id != ctx[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_eacc);
    if (e != cudaSuccess) return e;
    addr[dev] = static_cast<long long *>(p);
    ctx[dev] = id;
  }
  *out = addr[dev];
  return cudaSuccess;
}

cudaError_t pair_allpairs_launch(const SystemDev &s, const PairParams &p, const double *ljd,
                                 const double *pos, double *fout, long long *eacc,
                                 int max_box_atoms, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(eacc, 0, sizeof(long long) * ACC_PER_BOX * s.nbox, st);
  if (e != cudaSuccess) return e;
  if (max_box_atoms > 0) {
    const ParamsT<double> pd = params_t<double>(p);
    dim3 grid((max_box_atoms + AP_THREADS - 1) / AP_THREADS, s.nbox);
    if (p.coul_mode == 1) {
      if (p.virial) k_pair_allpairs<1, true><<<grid, AP_THREADS, 0, st>>>(s, pd, ljd, pos, fout, eacc);
      else k_pair_allpairs<1, false><<<grid, AP_THREADS, 0, st>>>(s, pd, ljd, pos, fout, eacc);
    } else {
      if (p.virial) k_pair_allpairs<0, true><<<grid, AP_THREADS, 0, st>>>(s, pd, ljd, pos, fout, eacc);
      else k_pair_allpairs<0, false><<<grid, AP_THREADS, 0, st>>>(s, pd, ljd, pos, fout, eacc);
    }
  }
  return cudaGetLastError();
}

}  // namespace pmb
