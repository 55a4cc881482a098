// Particle-mesh Ewald reciprocal term and exclusion corrections.
//
// Reference: mdl/interface/force/nonbonded/Grid.h (anterpolateCharge :107-154, interpolateForce
// :158-189, scalarSum :236-341, initialize :498-586, dftmod :588-600), BSpline.cpp:55-105,
// NonbondedPMEwaldSystemForce.h (reciprocalTerm :812-864, correctionTerm :874-911).
//
// Pipeline per step (every kernel batched over the boxes of a system):
//   k_spread      B-spline weights, 64 int64 fixed-point atomics per atom slot (order 4: four
//                 threads per slot, one x-plane of the stencil each)
//   k_fft_z_fwd   z-lines of the fixed-point grid (cleared as it is read), two real lines packed
//                 per complex FFT, half spectrum written as [kz][x][y]
//   k_fft_y       y-lines of the half spectrum (groups of up to 16 rows of one kz plane)
//   k_fft_x_infl  x-lines (groups of up to 16 columns): forward FFT, influence function multiply
//                 with energy and virial partials added to the box accumulators, inverse FFT
//   k_fft_y       inverse y-lines
//   k_fft_z_inv   inverse z transform back to the real potential grid [x][y][z]
//   k_gather      one thread per atom slot, 64-point stencil, fixed-point force atomics
// The transforms are unnormalised, as the reference's ZFFT/FFTW calls; r2c/c2r replace the
// reference's full complex transform of a real grid (identical result: the spectrum is Hermitian
// and the influence function even in m).
#include <type_traits>

#include "pmb_internal.h"

namespace pmb {

namespace {

constexpr int MAXP = 8;  // largest supported interpolation order

template <typename T>
struct C2;
template <>
struct C2<float> {
  using t = float2;
};
template <>
struct C2<double> {
  using t = double2;
};

__device__ __forceinline__ float2 cmk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 cmk(double a, double b) { return make_double2(a, b); }

template <typename T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T2>
__device__ __forceinline__ T2 cadd(T2 a, T2 b) { return cmk(a.x + b.x, a.y + b.y); }
template <typename T2>
__device__ __forceinline__ T2 csub(T2 a, T2 b) { return cmk(a.x - b.x, a.y - b.y); }
// multiply by (i * sign)
template <typename T2>
__device__ __forceinline__ T2 cis(T2 a, int sign) { return sign > 0 ? cmk(-a.y, a.x) : cmk(a.y, -a.x); }
template <typename T2, typename S>
__device__ __forceinline__ T2 cscale(T2 a, S s) { return cmk(a.x * s, a.y * s); }

// Small DFTs X_k = sum_n x_n exp(sign 2 pi i n k / R).
template <int R, typename T2>
__device__ __forceinline__ void dft_small(T2 *v, int sign) {
  using S = decltype(v[0].x);
  if constexpr (R == 2) {
    T2 a = cadd(v[0], v[1]), b = csub(v[0], v[1]);
    v[0] = a; v[1] = b;
  } else if constexpr (R == 3) {
    const S h = S(0.86602540378443864676);
    T2 t1 = cadd(v[1], v[2]);
    T2 t2 = csub(v[0], cscale(t1, S(0.5)));
    T2 t3 = cis(cscale(csub(v[1], v[2]), h), sign);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  } else if constexpr (R == 4) {
    T2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]), c = cadd(v[1], v[3]);
    T2 d = cis(csub(v[1], v[3]), sign);
    v[0] = cadd(a, c); v[1] = cadd(b, d); v[2] = csub(a, c); v[3] = csub(b, d);
  } else if constexpr (R == 5) {
    const S c1 = S(0.30901699437494742410), c2 = S(-0.80901699437494742410),
            s1 = S(0.95105651629515357212), s2 = S(0.58778525229247312917);
    T2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    T2 a1 = cadd(v[0], cadd(cscale(t1, c1), cscale(t2, c2)));
    T2 a2 = cadd(v[0], cadd(cscale(t1, c2), cscale(t2, c1)));
    T2 b1 = cis(cadd(cscale(t3, s1), cscale(t4, s2)), sign);
    T2 b2 = cis(csub(cscale(t3, s2), cscale(t4, s1)), sign);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1); v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2); v[3] = csub(a2, b2);
  }
}

// dft_small for R = 1 .. 5 (R = 1: nothing to do).
template <int R, typename T2>
__device__ __forceinline__ void dft_small_any(T2 *v, int sign) {
  if constexpr (R > 1) dft_small<R>(v, sign);
}

// floor(a / d) for 0 <= a < 2^21 from r ~ 1/d (a few ulp suffice: (a + 1/2) / d stays at least
// 1/(2d) away from an integer), without an integer division.
__device__ __forceinline__ int divf(int a, float r) { return __float2int_rz(((float)a + 0.5f) * r); }
__device__ __forceinline__ float rcpf(int d) { return __fdividef(1.0f, (float)d); }

// One Stockham stage, out of place (src -> dst): each thread takes whole butterflies (R inputs
// read, twiddled, transformed and written), so only R values are live at a time.
template <int R, typename T2>
__device__ __forceinline__ void fft_stage(const T2 *__restrict__ src, T2 *__restrict__ dst, int n,
                                          int nlines, int lstride, int estride, int Ns,
                                          const T2 *tw, int sign) {
  const int nb = n / R, total = nb * nlines, step = n / (Ns * R);
  const float rnb = rcpf(nb), rnl = rcpf(nlines), rns = rcpf(Ns);
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    // contiguous lines: consecutive threads take consecutive butterflies of one line;
    // strided lines: consecutive threads take the same butterfly of consecutive lines
    int line, j;
    if (estride == 1) {
      line = divf(b, rnb);
      j = b - line * nb;
    } else {
      j = divf(b, rnl);
      line = b - j * nlines;
    }
    const T2 *Ls = src + line * lstride;
    T2 *Ld = dst + line * lstride;
    T2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = Ls[(j + r * nb) * estride];
    const int jq = divf(j, rns), k = j - jq * Ns;
#pragma unroll
    for (int r = 1; r < R; r++) {
      T2 w = tw[r * k * step];
      if (sign > 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_small<R>(v, sign);
    const int out = jq * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) Ld[(out + r * Ns) * estride] = v[r];
  }
  __syncthreads();
}

// Batched 1-D FFTs of length n over shared memory (element e of line l at
// buf[l*lstride + e*estride]); radices[0..nrad) multiply to n.  Stages alternate between buf
// and tmp (same layout); returns the buffer holding the result.
template <typename T2>
__device__ T2 *fft_lines(T2 *buf, T2 *tmp, int n, int nlines, int lstride, int estride,
                         const int *radices, int nrad, const T2 *tw, int sign) {
  int Ns = 1;
  T2 *src = buf, *dst = tmp;
  for (int s = 0; s < nrad; s++) {
    const int R = radices[s];
    if (R == 4) fft_stage<4>(src, dst, n, nlines, lstride, estride, Ns, tw, sign);
    else if (R == 2) fft_stage<2>(src, dst, n, nlines, lstride, estride, Ns, tw, sign);
    else if (R == 3) fft_stage<3>(src, dst, n, nlines, lstride, estride, Ns, tw, sign);
    else fft_stage<5>(src, dst, n, nlines, lstride, estride, Ns, tw, sign);
    Ns *= R;
    T2 *t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// B-spline weights of order P at w (BSpline::set, BSpline.cpp:55-105).
template <typename T>
__device__ __forceinline__ void bspline(int P, T w, T *th, T *dth) {
  if (P == 2) {
    th[1] = w; th[0] = T(1) - w;
    if (dth) { dth[1] = T(1); dth[0] = T(-1); }
    return;
  }
  th[P - 1] = T(0);
  th[1] = w;
  th[0] = T(1) - w;
  #pragma unroll
  for (int k = 2; k < P - 1; k++) {
    T div = T(1) / T(k);
    th[k] = div * w * th[k - 1];
    #pragma unroll
    for (int j = 1; j < k; j++)
      th[k - j] = div * ((w + T(j)) * th[k - j - 1] + (T(k + 1 - j) - w) * th[k - j]);
    th[0] = div * (T(1) - w) * th[0];
  }
  if (dth) {
    dth[0] = -th[0];
    #pragma unroll
    for (int j = 1; j <= P - 1; j++) dth[j] = th[j - 1] - th[j];
  }
  T div = T(1) / (T(P) - T(1));
  th[P - 1] = div * w * th[P - 2];
  #pragma unroll
  for (int j = 1; j < P - 1; j++)
    th[P - 1 - j] = div * ((w + T(j)) * th[P - j - 2] + (T(P - j) - w) * th[P - 1 - j]);
  th[0] = div * (T(1) - w) * th[0];
}

// Grid coordinate of one dimension: base index (already offset by -(P-1)/2 and wrapped to
// [0, n)) and the fractional weight w.
template <bool MIXED>
__device__ __forceinline__ void grid_coord(unsigned fx, double x, double hr, int n, int P, int &base,
                                           typename std::conditional<MIXED, float, double>::type &w) {
  int iu;
  if constexpr (MIXED) {
    unsigned long long prod = (unsigned long long)fx * (unsigned)n;
    iu = (int)(prod >> 32);
    w = (float)(unsigned)(prod & 0xffffffffull) * 2.3283064365386963e-10f;
  } else {
    // Grid.h:110-121: u = x n / L wrapped into [0, n) by repeated +-n, then truncated.
    double u = x * hr;
    for (int it = 0; it < 4 && u < 0.0; it++) u += n;
    for (int it = 0; it < 4 && u >= n; it++) u -= n;
    if (!(u >= 0.0 && u < n)) {
      u -= n * floor(u / n);
      if (!(u >= 0.0 && u < n)) u = 0.0;
    }
    iu = (int)u;
    w = u - iu;
  }
  base = iu - (P - 1) / 2 + n;  // myNXOffset = -(order-1)/2 + n
}

// x mod n for 0 <= x < 3n (a stencil index: base in [n - (p-1)/2, 2n) plus an offset below p,
// with n >= p), without an integer division.
__device__ __forceinline__ int wrap3(int x, int n) {
  x = x >= n ? x - n : x;
  return x >= n ? x - n : x;
}

// PC > 0: interpolation order fixed at compile time (weights stay in registers); PC = 0: run time.
template <bool MIXED, int PC>
__global__ void k_spread(NbListDev nb, PmeDev pm) {
  using T = typename std::conditional<MIXED, float, double>::type;
  int sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= nb.nslot) return;
  int4 m = nb.slot_meta[sl];
  if (m.x < 0) return;
  const PmeBoxPlan &pl = pm.plan[m.w];
  const int P = PC > 0 ? PC : pm.order;
  T th[3][MAXP];
  int base[3];
  T q;
  if constexpr (MIXED) {
    uint4 f = nb.slot_fx[sl];
    unsigned fx[3] = {f.x, f.y, f.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T w;
      grid_coord<true>(fx[d], 0.0, 0.0, pl.n[d], P, base[d], w);
      bspline<T>(P, w, th[d], nullptr);
    }
    q = __uint_as_float(f.w);
  } else {
    double4 pq = nb.slot_pq[sl];
    double x[3] = {pq.x, pq.y, pq.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T w;
      grid_coord<false>(0u, x[d], pl.hr[d], pl.n[d], P, base[d], w);
      bspline<T>(P, w, th[d], nullptr);
    }
    q = pq.w;
  }
  const int nx = pl.n[0], ny = pl.n[1], nz = pl.n[2];
  long long *g = pm.qgrid + pl.grid0;
  #pragma unroll
  for (int i = 0; i < P; i++) {
    T a = q * th[0][i];
    int i1 = wrap3(i + base[0], nx);
    #pragma unroll
    for (int j = 0; j < P; j++) {
      T ab = a * th[1][j];
      int j1 = wrap3(j + base[1], ny);
      long long *row = g + ((long long)i1 * ny + j1) * nz;
      #pragma unroll
      for (int k = 0; k < P; k++) {
        int k1 = wrap3(k + base[2], nz);
        long long v = f2fix(ab * th[2][k], (T)GRID_SCALE);
        if (v) red_add(row + k1, v);
      }
    }
  }
}

// B-spline weights and grid bases of one slot for order 4 (the common case).
template <bool MIXED, bool DERIV>
__device__ __forceinline__ void weights4(const PmeBoxPlan &pl, uint4 f, double4 pq,
                                         typename std::conditional<MIXED, float, double>::type th[3][4],
                                         typename std::conditional<MIXED, float, double>::type dth[3][4],
                                         int base[3], typename std::conditional<MIXED, float, double>::type &q) {
  using T = typename std::conditional<MIXED, float, double>::type;
  if constexpr (MIXED) {
    const unsigned fx[3] = {f.x, f.y, f.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T w;
      grid_coord<true>(fx[d], 0.0, 0.0, pl.n[d], 4, base[d], w);
      bspline<T>(4, w, th[d], DERIV ? dth[d] : nullptr);
    }
    q = __uint_as_float(f.w);
  } else {
    const double x[3] = {pq.x, pq.y, pq.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T w;
      grid_coord<false>(0u, x[d], pl.hr[d], pl.n[d], 4, base[d], w);
      bspline<T>(4, w, th[d], DERIV ? dth[d] : nullptr);
    }
    q = pq.w;
  }
}

// v[p] for a run-time p in [0, 4) without indexing a register array (which would go to local
// memory).
template <typename T>
__device__ __forceinline__ T pick4(const T v[4], int p) {
  return p == 0 ? v[0] : (p == 1 ? v[1] : (p == 2 ? v[2] : v[3]));
}

// Order 4 with four threads per atom slot: thread p adds the 16 points of z-offset p of the
// stencil (the same values, in the same order of products, as the one-thread form), so that at
// every step the slot's four threads add to four consecutive grid words (one or two 32-byte
// sectors) rather than to four x-planes (four sectors).
template <bool MIXED>
__global__ void k_spread4(NbListDev nb, PmeDev pm) {
  using T = typename std::conditional<MIXED, float, double>::type;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int sl = (int)(t >> 2), p = (int)(t & 3);
  if (sl >= nb.nslot) return;
  // the slot's metadata and position are loaded together (one round trip)
  const int4 m = nb.slot_meta[sl];
  uint4 f4 = make_uint4(0, 0, 0, 0);
  double4 p4 = make_double4(0, 0, 0, 0);
  if constexpr (MIXED) f4 = nb.slot_fx[sl];
  else p4 = nb.slot_pq[sl];
  if (m.x < 0) return;
  const PmeBoxPlan &pl = pm.plan[m.w];
  T th[3][4];
  int base[3];
  T q;
  weights4<MIXED, false>(pl, f4, p4, th, th, base, q);
  const int nx = pl.n[0], ny = pl.n[1], nz = pl.n[2];
  long long *g = pm.qgrid + pl.grid0;
  const T c2 = pick4(th[2], p);
  long long *col = g + wrap3(p + base[2], nz);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const T a = q * th[0][i];
    const int i1 = wrap3(i + base[0], nx);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int j1 = wrap3(j + base[1], ny);
      const long long v = f2fix(a * th[1][j] * c2, (T)GRID_SCALE);
      if (v) red_add(col + ((long long)i1 * ny + j1) * nz, v);
    }
  }
}

template <bool MIXED, int PC>
__global__ void k_gather(const SystemDev s, NbListDev nb, PmeDev pm) {
  using T = typename std::conditional<MIXED, float, double>::type;
  int sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= nb.nslot) return;
  // the slot's metadata and position are loaded together (one round trip)
  int4 m = nb.slot_meta[sl];
  uint4 f4 = make_uint4(0, 0, 0, 0);
  double4 pq = make_double4(0, 0, 0, 0);
  if constexpr (MIXED) f4 = nb.slot_fx[sl];
  else pq = nb.slot_pq[sl];
  if (m.x < 0) return;
  const PmeBoxPlan &pl = pm.plan[m.w];
  const int P = PC > 0 ? PC : pm.order;
  T th[3][MAXP], dth[3][MAXP];
  int base[3];
  T q;
  if constexpr (MIXED) {
    unsigned fx[3] = {f4.x, f4.y, f4.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T w;
      grid_coord<true>(fx[d], 0.0, 0.0, pl.n[d], P, base[d], w);
      bspline<T>(P, w, th[d], dth[d]);
    }
    q = __uint_as_float(f4.w);
  } else {
    double x[3] = {pq.x, pq.y, pq.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      T w;
      grid_coord<false>(0u, x[d], pl.hr[d], pl.n[d], P, base[d], w);
      bspline<T>(P, w, th[d], dth[d]);
    }
    q = pq.w;
  }
  const int nx = pl.n[0], ny = pl.n[1], nz = pl.n[2];
  const T *g = reinterpret_cast<const T *>(pm.rgrid) + pl.grid0;
  T fx = 0, fy = 0, fz = 0;
  #pragma unroll
  for (int i = 0; i < P; i++) {
    int i1 = wrap3(i + base[0], nx);
    #pragma unroll
    for (int j = 0; j < P; j++) {
      int j1 = wrap3(j + base[1], ny);
      T xij = dth[0][i] * th[1][j], yij = th[0][i] * dth[1][j], zij = th[0][i] * th[1][j];
      const T *row = g + ((long long)i1 * ny + j1) * nz;
      #pragma unroll
      for (int k = 0; k < P; k++) {
        int k1 = wrap3(k + base[2], nz);
        T term = row[k1];
        fx -= term * xij * th[2][k];
        fy -= term * yij * th[2][k];
        fz -= term * zij * dth[2][k];
      }
    }
  }
  long long *f = s.facc + 3 * (long long)m.x;
  red_add(f, f2fix((double)(fx * T(pl.hr[0]) * q), FORCE_SCALE));
  red_add(f + 1, f2fix((double)(fy * T(pl.hr[1]) * q), FORCE_SCALE));
  red_add(f + 2, f2fix((double)(fz * T(pl.hr[2]) * q), FORCE_SCALE));
}

// Order 4 with four threads per atom slot: thread p reads z-offset p of the stencil, so that at
// every step the slot's four threads read four consecutive grid words; the four partial forces
// are summed over the slot's lanes.  Every lane takes part in the shuffles (slots out of range
// or padding add zeros).
template <bool MIXED>
__global__ void k_gather4(const SystemDev s, NbListDev nb, PmeDev pm) {
  using T = typename std::conditional<MIXED, float, double>::type;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int sl = (int)(t >> 2), p = (int)(t & 3);
  const bool in = sl < nb.nslot;
  const int4 m = in ? nb.slot_meta[sl] : make_int4(-1, -1, 0, 0);
  uint4 f4 = make_uint4(0, 0, 0, 0);
  double4 pq = make_double4(0, 0, 0, 0);
  if (in) {
    if constexpr (MIXED) f4 = nb.slot_fx[sl];
    else pq = nb.slot_pq[sl];
  }
  const bool ok = m.x >= 0;
  T fx = 0, fy = 0, fz = 0, q = 0;
  const PmeBoxPlan *pl = ok ? pm.plan + m.w : nullptr;
  if (ok) {
    T th[3][4], dth[3][4];
    int base[3];
    weights4<MIXED, true>(*pl, f4, pq, th, dth, base, q);
    const int nx = pl->n[0], ny = pl->n[1], nz = pl->n[2];
    const T *col = reinterpret_cast<const T *>(pm.rgrid) + pl->grid0 + wrap3(p + base[2], nz);
    const T tz = pick4(th[2], p), dz = pick4(dth[2], p);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int i1 = wrap3(i + base[0], nx);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int j1 = wrap3(j + base[1], ny);
        const T xij = dth[0][i] * th[1][j], yij = th[0][i] * dth[1][j], zij = th[0][i] * th[1][j];
        const T term = col[((long long)i1 * ny + j1) * nz];
        fx -= term * xij * tz;
        fy -= term * yij * tz;
        fz -= term * zij * dz;
      }
    }
  }
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (ok && p == 0) {
    long long *f = s.facc + 3 * (long long)m.x;
    red_add(f, f2fix((double)(fx * T(pl->hr[0]) * q), FORCE_SCALE));
    red_add(f + 1, f2fix((double)(fy * T(pl->hr[1]) * q), FORCE_SCALE));
    red_add(f + 2, f2fix((double)(fz * T(pl->hr[2]) * q), FORCE_SCALE));
  }
}

constexpr int ZT = 128;         // threads of the z-line kernels
constexpr int ZMAXE = 8 * 256;  // 8 packed line pairs x nz <= 256, per ping-pong buffer

template <typename T>
__global__ void __launch_bounds__(ZT, 8) k_fft_z_fwd(PmeDev pm) {
  using T2 = typename C2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 wk = pm.zwork[blockIdx.x];
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int nx = pl.n[0], ny = pl.n[1], nz = pl.n[2], x = wk.y, y0 = wk.z, cnt = wk.w;
  const int npair = (cnt + 1) / 2;
  T2 *tw = reinterpret_cast<T2 *>(smem_raw);
  T2 *buf = tw + 256, *tmp = buf + pm.zbuf;
  for (int k = threadIdx.x; k < nz; k += ZT) {
    if constexpr (sizeof(T) == 4) tw[k] = pm.twiddlef[pl.tw0[2] + k];
    else tw[k] = pm.twiddle[pl.tw0[2] + k];
  }
  long long *g = pm.qgrid + pl.grid0 + ((long long)x * ny + y0) * nz;
  // the work item's lines are one contiguous run of cnt * nz grid values: read them all (no
  // store in between, so the loads overlap), then clear the charge grid for the next step, each
  // thread the values it read itself
  const int nrun = cnt * nz;
  const float rnz = rcpf(nz), rnp = rcpf(npair);
#pragma unroll 4
  for (int e = threadIdx.x; e < npair * 2 * nz; e += ZT) {
    const long long q = e < nrun ? __ldcs(g + e) : 0ll;
    const int line = divf(e, rnz), z = e - line * nz;
    T *dst = reinterpret_cast<T *>(buf + (line >> 1) * nz + z);
    dst[line & 1] = T((double)q * (1.0 / GRID_SCALE));
  }
  for (int e = threadIdx.x; e < nrun; e += ZT) g[e] = 0;
  __syncthreads();
  const T2 *res = fft_lines(buf, tmp, nz, npair, nz, 1, pm.radix + pl.rad0[2], pl.nrad[2], tw, -1);
  const int nh = nz / 2 + 1;
  T2 *C = reinterpret_cast<T2 *>(pm.cgrid) + pl.cgrid0;
  for (int e = threadIdx.x; e < npair * nh; e += ZT) {
    const int k = divf(e, rnp), pi = e - k * npair;
    T2 zk = res[pi * nz + k], zn = res[pi * nz + (k == 0 ? 0 : nz - k)];
    // X = (Z_k + conj(Z_{n-k})) / 2, Y = -i/2 (Z_k - conj(Z_{n-k}))
    T2 X = cmk(T(0.5) * (zk.x + zn.x), T(0.5) * (zk.y - zn.y));
    T2 Y = cmk(T(0.5) * (zk.y + zn.y), T(-0.5) * (zk.x - zn.x));
    T2 *row = C + ((long long)k * nx + x) * ny + y0 + 2 * pi;
    row[0] = X;
    if (2 * pi + 1 < cnt) row[1] = Y;
  }
}

template <typename T>
__global__ void __launch_bounds__(ZT, 8) k_fft_z_inv(PmeDev pm) {
  using T2 = typename C2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 wk = pm.zwork[blockIdx.x];
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int nx = pl.n[0], ny = pl.n[1], nz = pl.n[2], x = wk.y, y0 = wk.z, cnt = wk.w;
  const int npair = (cnt + 1) / 2, nh = nz / 2 + 1;
  T2 *tw = reinterpret_cast<T2 *>(smem_raw);
  T2 *buf = tw + 256, *tmp = buf + pm.zbuf;
  for (int k = threadIdx.x; k < nz; k += ZT) {
    if constexpr (sizeof(T) == 4) tw[k] = pm.twiddlef[pl.tw0[2] + k];
    else tw[k] = pm.twiddle[pl.tw0[2] + k];
  }
  const T2 *C = reinterpret_cast<const T2 *>(pm.cgrid) + pl.cgrid0;
  const float rnz = rcpf(nz), rnp = rcpf(npair);
  for (int e = threadIdx.x; e < npair * nh; e += ZT) {
    const int k = divf(e, rnp), pi = e - k * npair;
    const T2 *row = C + ((long long)k * nx + x) * ny + y0 + 2 * pi;
    T2 X = row[0];
    T2 Y = (2 * pi + 1 < cnt) ? row[1] : cmk(T(0), T(0));
    if (k == 0 || (2 * k == nz)) {
      X.y = T(0);
      Y.y = T(0);
    }
    buf[pi * nz + k] = cmk(X.x - Y.y, X.y + Y.x);
    if (k > 0 && 2 * k != nz) buf[pi * nz + nz - k] = cmk(X.x + Y.y, Y.x - X.y);
  }
  __syncthreads();
  const T2 *res = fft_lines(buf, tmp, nz, npair, nz, 1, pm.radix + pl.rad0[2], pl.nrad[2], tw, +1);
  T *R = reinterpret_cast<T *>(pm.rgrid) + pl.grid0 + ((long long)x * ny + y0) * nz;
  for (int e = threadIdx.x; e < cnt * nz; e += ZT) {
    const int line = divf(e, rnz), z = e - line * nz;
    T2 v = res[(line >> 1) * nz + z];
    R[(long long)line * nz + z] = (line & 1) ? v.y : v.x;
  }
}

template <int THREADS, typename T>
__device__ __forceinline__ double block_sum(double v, double *red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < THREADS / 32 ? red[threadIdx.x] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

constexpr int LT = 128;          // threads of the y- and x-line kernels
constexpr int LMAXE = 2048;      // complex elements per line-kernel CTA, per ping-pong buffer

// y-lines of the half spectrum: rows C[kz][x][0..ny) of one work item are contiguous.
template <typename T>
__global__ void __launch_bounds__(LT, 8) k_fft_y(PmeDev pm, int sign) {
  using T2 = typename C2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 wk = pm.ywork[blockIdx.x];  // box, kz, x0, rows
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int nx = pl.n[0], ny = pl.n[1], kz = wk.y, x0 = wk.z, rows = wk.w;
  T2 *tw = reinterpret_cast<T2 *>(smem_raw + 32 * sizeof(double));
  T2 *buf = tw + 256, *tmp = buf + pm.lbuf;
  for (int k = threadIdx.x; k < ny; k += LT) {
    if constexpr (sizeof(T) == 4) tw[k] = pm.twiddlef[pl.tw0[1] + k];
    else tw[k] = pm.twiddle[pl.tw0[1] + k];
  }
  T2 *C = reinterpret_cast<T2 *>(pm.cgrid) + pl.cgrid0 + ((long long)kz * nx + x0) * ny;
  const int ne = rows * ny;
  for (int e = threadIdx.x; e < ne; e += LT) buf[e] = C[e];
  __syncthreads();
  const T2 *res = fft_lines(buf, tmp, ny, rows, ny, 1, pm.radix + pl.rad0[1], pl.nrad[1], tw, sign);
  for (int e = threadIdx.x; e < ne; e += LT) C[e] = res[e];
}

// x-lines (columns y0..y0+cols of one kz plane): forward FFT, influence function with energy and
// virial (Grid.h:236-341, half spectrum kz <= nz/2 with the doubling of interior kz), inverse FFT.
template <typename T>
__global__ void __launch_bounds__(LT, 8) k_fft_x_infl(const SystemDev s, PmeDev pm) {
  using T2 = typename C2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 wk = pm.xwork[blockIdx.x];  // box, kz, y0, cols
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int nx = pl.n[0], ny = pl.n[1], nz = pl.n[2], kz = wk.y, y0 = wk.z, cols = wk.w;
  double *red = reinterpret_cast<double *>(smem_raw);  // 32 doubles
  T2 *tw = reinterpret_cast<T2 *>(smem_raw + 32 * sizeof(double));
  T2 *buf = tw + 256, *tmp = buf + pm.lbuf;  // buf[x * cols + c]
  for (int k = threadIdx.x; k < nx; k += LT) {
    if constexpr (sizeof(T) == 4) tw[k] = pm.twiddlef[pl.tw0[0] + k];
    else tw[k] = pm.twiddle[pl.tw0[0] + k];
  }
  T2 *C = reinterpret_cast<T2 *>(pm.cgrid) + pl.cgrid0 + (long long)kz * nx * ny + y0;
  const int ne = nx * cols;
  const float rcols = rcpf(cols);
  for (int e = threadIdx.x; e < ne; e += LT) {
    const int x = divf(e, rcols), c = e - x * cols;
    buf[e] = C[(long long)x * ny + c];
  }
  __syncthreads();
  T2 *spec = fft_lines(buf, tmp, nx, cols, 1, cols, pm.radix + pl.rad0[0], pl.nrad[0], tw, -1);
  T2 *other = spec == buf ? tmp : buf;
  // influence function of this plane's columns (precomputed per plan, 0 at m = 0)
  const T *th = reinterpret_cast<const T *>(pm.theta) + pl.cgrid0 + (long long)kz * nx * ny + y0;
  const double mk = kz * pl.mr[2];
  const double wz = (kz > 0 && ((2 * kz != nz) || (nz & 1))) ? 2.0 : 1.0;
  double en = 0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  for (int e = threadIdx.x; e < ne; e += LT) {
    const int i = divf(e, rcols), cc = e - i * cols;
    const T theta = th[(long long)i * ny + cc];
    T2 c = spec[e];
    double qq = (double)c.x * (double)c.x + (double)c.y * (double)c.y;
    double ee = wz * qq * (double)theta;
    en += ee;
    if (pm.virial && theta != T(0)) {
      const int j = y0 + cc;
      int i0 = i <= nx / 2 ? i : i - nx, j0 = j <= ny / 2 ? j : j - ny;
      double mi = i0 * pl.mr[0], mj = j0 * pl.mr[1];
      double m2 = mi * mi + mj * mj + mk * mk;
      double v = 2.0 * (1.0 / m2 + pl.fac);
      vxx += ee * (1.0 - v * mi * mi); vxy -= ee * (v * mi * mj); vxz -= ee * (v * mi * mk);
      vyy += ee * (1.0 - v * mj * mj); vyz -= ee * (v * mj * mk); vzz += ee * (1.0 - v * mk * mk);
    }
    spec[e] = cmk(c.x * theta, c.y * theta);
  }
  // the CTA's energy (x 0.5, Grid.h:319-337) and virial partials go to the box accumulators in
  // fixed point (a fixed reduction order per CTA, integer sums across CTAs)
  double part[7] = {en, vxx, vxy, vxz, vyy, vyz, vzz};
  const int np = pm.virial ? 7 : 1;
  long long *eb = s.eacc + (long long)wk.x * ACC_PER_BOX;
  const int slot[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};  // xx xy xz yy yz zz
  for (int c = 0; c < np; c++) {
    const double r = block_sum<LT, T>(part[c], red);
    if (threadIdx.x == 0) {
      const long long v = f2fix(r * 0.5, ENERGY_SCALE);
      if (c == 0) {
        red_add(eb + E_COUL, v);
      } else {
        red_add(eb + E_VIR + slot[c - 1][0], v);
        if (slot[c - 1][1] != slot[c - 1][0]) red_add(eb + E_VIR + slot[c - 1][1], v);
      }
    }
  }
  __syncthreads();
  const T2 *res = fft_lines(spec, other, nx, cols, 1, cols, pm.radix + pl.rad0[0], pl.nrad[0], tw, +1);
  for (int e = threadIdx.x; e < ne; e += LT) {
    const int x = divf(e, rcols), c = e - x * cols;
    C[(long long)x * ny + c] = res[e];
  }
}

// ------------------------------------------------------------ warp-shuffle transforms (n = 32 R)
// One line of n = 32 R points per warp, no shared-memory stages and no block barrier: lane l
// holds points l, l + 32, ..., l + 32 (R - 1) in registers.  Forward: an R-point DFT over the
// registers, the factors W_n^(l k1), then a 32-point decimation-in-frequency transform across
// the lanes (five xor-shuffle butterfly stages); register k1 of lane l then holds X[k1 + R b(l)],
// b = 5-bit reversal.  Inverse: consumes exactly that layout, decimation-in-time across the
// lanes, the conjugate factors, the R-point DFT over the registers, and leaves point
// l + 32 r in register r.  The factors come from the plan's table W_n^k = exp(-2 pi i k / n).
__device__ __forceinline__ int brev5(int l) { return (int)(__brev((unsigned)l) >> 27); }

template <typename T2>
__device__ __forceinline__ T2 shfl_xor2(T2 v, int d) {
  return cmk(__shfl_xor_sync(0xffffffffu, v.x, d), __shfl_xor_sync(0xffffffffu, v.y, d));
}
template <typename T2>
__device__ __forceinline__ T2 cmulc(T2 a, T2 w) {  // a * conj(w)
  return cmk(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

// Per-lane factors: st[s] = w_(2d)^(l mod d) for d = 16 >> s (w_m = exp(-2 pi i / m)), and
// rk[k1] = W_n^(l k1).
template <int R, typename T2>
struct WarpTw {
  T2 st[5], rk[R];
};
template <int R, typename T2, typename TW>
__device__ __forceinline__ WarpTw<R, T2> warp_twiddles(const TW *tw) {
  const int lane = threadIdx.x & 31;
  WarpTw<R, T2> w;
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int d = 16 >> s, j = lane & (d - 1);
    const TW t = tw[j * (16 / d) * R];
    w.st[s] = cmk(t.x, t.y);
  }
#pragma unroll
  for (int k = 0; k < R; k++) {
    const TW t = tw[lane * k];
    w.rk[k] = cmk(t.x, t.y);
  }
  return w;
}

template <int R, typename T2>
__device__ __forceinline__ void warp_fft_fwd(T2 v[R], const WarpTw<R, T2> &w) {
  const int lane = threadIdx.x & 31;
  dft_small_any<R>(v, -1);
#pragma unroll
  for (int k = 1; k < R; k++) v[k] = cmul(v[k], w.rk[k]);
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int d = 16 >> s;
    const bool up = (lane & d) != 0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const T2 p = shfl_xor2(v[k], d);
      v[k] = up ? cmul(csub(p, v[k]), w.st[s]) : cadd(v[k], p);
    }
  }
}

template <int R, typename T2>
__device__ __forceinline__ void warp_fft_inv(T2 v[R], const WarpTw<R, T2> &w) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 4; s >= 0; s--) {
    const int d = 16 >> s;
    const bool up = (lane & d) != 0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const T2 t = up ? cmulc(v[k], w.st[s]) : v[k];
      const T2 p = shfl_xor2(t, d);
      v[k] = up ? csub(p, t) : cadd(v[k], p);
    }
  }
#pragma unroll
  for (int k = 1; k < R; k++) v[k] = cmulc(v[k], w.rk[k]);
  dft_small_any<R>(v, +1);
}

constexpr int WT = 128;  // threads of the warp-transform y kernel (one row per warp)
constexpr int WX = PME_WX_THREADS;  // threads of the warp-transform x kernel (one column per warp)

// y-lines with n_y = 32 R: row C[kz][x][0..ny) per warp, up to WT / 32 rows per work item.
// The forward result is put back into natural order through a per-warp shared-memory line; the
// inverse reads its input in the forward's lane order through it.
template <typename T, int R>
__global__ void __launch_bounds__(WT) k_fft_y_warp(PmeDev pm, int sign) {
  using T2 = typename C2<T>::t;
  __shared__ T2 sline[WT / 32][32 * R];
  const int4 wk = pm.ywork[blockIdx.x];  // box, kz, x0, rows
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int nx = pl.n[0], w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= wk.w) return;  // warp-uniform; no block barrier below
  constexpr int ny = 32 * R;
  T2 *row = reinterpret_cast<T2 *>(pm.cgrid) + pl.cgrid0 + ((long long)wk.y * nx + wk.z + w) * ny;
  WarpTw<R, T2> tw;
  if constexpr (sizeof(T) == 4) tw = warp_twiddles<R, T2>(pm.twiddlef + pl.tw0[1]);
  else tw = warp_twiddles<R, T2>(pm.twiddle + pl.tw0[1]);
  T2 *sl = sline[w];
  T2 v[R];
  const int b = brev5(lane);
  if (sign < 0) {
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = row[r * 32 + lane];
    warp_fft_fwd<R>(v, tw);
#pragma unroll
    for (int k = 0; k < R; k++) sl[k + R * b] = v[k];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; r++) row[r * 32 + lane] = sl[r * 32 + lane];
  } else {
#pragma unroll
    for (int r = 0; r < R; r++) sl[r * 32 + lane] = row[r * 32 + lane];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = sl[k + R * b];
    warp_fft_inv<R>(v, tw);
#pragma unroll
    for (int r = 0; r < R; r++) row[r * 32 + lane] = v[r];
  }
}

// x-lines with n_x = 32 R (columns y0..y0+cols of one kz plane, one per warp): forward
// transform, influence function with energy and virial (as k_fft_x_infl), inverse transform.
// The block is staged through shared memory (coalesced rows in and out); between the two
// transforms each point stays in its lane's registers.
template <typename T, int R>
__global__ void __launch_bounds__(WX, 3) k_fft_x_warp(const SystemDev s, PmeDev pm) {
  using T2 = typename C2<T>::t;
  constexpr int nx = 32 * R, NW = WX / 32, SP = nx + 1;  // padded column stride
  __shared__ T2 sb[NW * SP];
  __shared__ T sth[NW * SP];  // the block's influence function, staged like the spectrum
  __shared__ double red[32];
  const int4 wk = pm.xwork[blockIdx.x];  // box, kz, y0, cols
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int ny = pl.n[1], nz = pl.n[2], kz = wk.y, y0 = wk.z, cols = wk.w;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T2 *C = reinterpret_cast<T2 *>(pm.cgrid) + pl.cgrid0 + (long long)kz * nx * ny + y0;
  const T *thg = reinterpret_cast<const T *>(pm.theta) + pl.cgrid0 + (long long)kz * nx * ny + y0;
  const float rcols = rcpf(cols);
  for (int e = threadIdx.x; e < nx * cols; e += WX) {
    const int x = divf(e, rcols), c = e - x * cols;
    sb[c * SP + x] = C[(long long)x * ny + c];
    sth[c * SP + x] = thg[(long long)x * ny + c];
  }
  __syncthreads();
  double en = 0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
  T2 v[R];
  if (w < cols) {
    WarpTw<R, T2> tw;
    if constexpr (sizeof(T) == 4) tw = warp_twiddles<R, T2>(pm.twiddlef + pl.tw0[0]);
    else tw = warp_twiddles<R, T2>(pm.twiddle + pl.tw0[0]);
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = sb[w * SP + r * 32 + lane];
    warp_fft_fwd<R>(v, tw);
    const T *th = sth + w * SP;
    const double mk = kz * pl.mr[2];
    const double wz = (kz > 0 && ((2 * kz != nz) || (nz & 1))) ? 2.0 : 1.0;
    const int j = y0 + w, j0 = j <= ny / 2 ? j : j - ny;
    const double mj = j0 * pl.mr[1];
    const int b = brev5(lane);
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int i = k + R * b;
      const T theta = th[i];
      const T2 c = v[k];
      const double qq = (double)c.x * (double)c.x + (double)c.y * (double)c.y;
      const double ee = wz * qq * (double)theta;
      en += ee;
      if (pm.virial && theta != T(0)) {
        const int i0 = i <= nx / 2 ? i : i - nx;
        const double mi = i0 * pl.mr[0];
        const double m2 = mi * mi + mj * mj + mk * mk;
        const double vv = 2.0 * (1.0 / m2 + pl.fac);
        vxx += ee * (1.0 - vv * mi * mi); vxy -= ee * (vv * mi * mj); vxz -= ee * (vv * mi * mk);
        vyy += ee * (1.0 - vv * mj * mj); vyz -= ee * (vv * mj * mk); vzz += ee * (1.0 - vv * mk * mk);
      }
      v[k] = cmk(c.x * theta, c.y * theta);
    }
    warp_fft_inv<R>(v, tw);
#pragma unroll
    for (int r = 0; r < R; r++) sb[w * SP + r * 32 + lane] = v[r];
  }
  // the CTA's energy (x 0.5, Grid.h:319-337) and virial partials in fixed point, as k_fft_x_infl
  const double part[7] = {en, vxx, vxy, vxz, vyy, vyz, vzz};
  const int np = pm.virial ? 7 : 1;
  long long *eb = s.eacc + (long long)wk.x * ACC_PER_BOX;
  const int slot[6][2] = {{0, 0}, {1, 3}, {2, 6}, {4, 4}, {5, 7}, {8, 8}};  // xx xy xz yy yz zz
  for (int c = 0; c < np; c++) {
    const double r = block_sum<WX, T>(part[c], red);
    if (threadIdx.x == 0) {
      const long long q = f2fix(r * 0.5, ENERGY_SCALE);
      if (c == 0) {
        red_add(eb + E_COUL, q);
      } else {
        red_add(eb + E_VIR + slot[c - 1][0], q);
        if (slot[c - 1][1] != slot[c - 1][0]) red_add(eb + E_VIR + slot[c - 1][1], q);
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nx * cols; e += WX) {
    const int x = divf(e, rcols), c = e - x * cols;
    C[(long long)x * ny + c] = sb[c * SP + x];
  }
}

constexpr int WZ = 128;  // threads of the warp z kernel: up to 8 lines (4 pairs) per work item

// z-lines with n_z = 32 R, c2r (as k_fft_z_inv): the z_inv work item's lines (x, y0 .. y0 + cnt)
// as cnt / 2 packed pairs, one per warp, rebuilt from the half spectrum (read in rows of cnt
// consecutive y through shared memory), written to the real potential grid [x][y][z].  (The r2c
// forward pass keeps the shared-memory kernel: its warp form was no faster.)
template <typename T, int R>
__global__ void __launch_bounds__(WZ) k_fft_z_inv_warp(PmeDev pm) {
  using T2 = typename C2<T>::t;
  constexpr int nz = 32 * R, nh = nz / 2 + 1, NP = WZ / 32;
  __shared__ T2 zl[NP][nz];
  __shared__ T2 in[nh * 2 * NP];  // [k][line]
  const int4 wk = pm.zwork[blockIdx.x];
  const PmeBoxPlan &pl = pm.plan[wk.x];
  const int nx = pl.n[0], ny = pl.n[1], x = wk.y, y0 = wk.z, cnt = wk.w;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T2 *C = reinterpret_cast<const T2 *>(pm.cgrid) + pl.cgrid0;
  for (int e = threadIdx.x; e < nh * cnt; e += WZ) {
    const int k = e / cnt, c = e - k * cnt;
    in[k * 2 * NP + c] = C[((long long)k * nx + x) * ny + y0 + c];
  }
  __syncthreads();
  if (2 * w >= cnt) return;  // warp-uniform; no block barrier below
  const bool two = 2 * w + 1 < cnt;
  for (int k = lane; k < nh; k += 32) {
    T2 X = in[k * 2 * NP + 2 * w];
    T2 Y = two ? in[k * 2 * NP + 2 * w + 1] : cmk(T(0), T(0));
    if (k == 0 || 2 * k == nz) {
      X.y = T(0);
      Y.y = T(0);
    }
    // Z_k = X_k + i Y_k and Z_{n-k} = conj(X_k) + i conj(Y_k)
    zl[w][k] = cmk(X.x - Y.y, X.y + Y.x);
    if (k > 0 && 2 * k != nz) zl[w][nz - k] = cmk(X.x + Y.y, Y.x - X.y);
  }
  __syncwarp();
  WarpTw<R, T2> tw;
  if constexpr (sizeof(T) == 4) tw = warp_twiddles<R, T2>(pm.twiddlef + pl.tw0[2]);
  else tw = warp_twiddles<R, T2>(pm.twiddle + pl.tw0[2]);
  const int b = brev5(lane);
  T2 v[R];
#pragma unroll
  for (int k = 0; k < R; k++) v[k] = zl[w][k + R * b];
  warp_fft_inv<R>(v, tw);
  T *Rg = reinterpret_cast<T *>(pm.rgrid) + pl.grid0 + ((long long)x * ny + y0 + 2 * w) * nz;
#pragma unroll
  for (int r = 0; r < R; r++) {
    Rg[r * 32 + lane] = v[r].x;
    if (two) Rg[nz + r * 32 + lane] = v[r].y;
  }
}

// Exclusion correction in FP64 with the exact erf (NonbondedPMEwaldSystemForce.h:874-911).
__global__ void k_correction(const SystemDev s, const int *pairs, const int *kind, int n,
                             double alpha, double a2pi, double csf, int virial) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = k < n;
  double en = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};
  int box = -1;
  if (valid) {
    int a1 = pairs[2 * k], a2 = pairs[2 * k + 1];
    box = s.atom_box[a1];
    const BoxDev &b = s.box[box];
    double rij[3];
    double r2 = min_diff(b, s.pos + 3 * a1, s.pos + 3 * a2, rij);
    double qq = s.charge[a1] * s.charge[a2];
    if (kind[k] == 1) qq *= 1 - csf;
    double r = sqrt(r2), rr = 1 / r, e = erf(alpha * r) * rr;
    en = -qq * e;
    double fs = qq * (a2pi * exp(-alpha * alpha * r2) - e) * rr * rr;
    double fij[3] = {rij[0] * fs, rij[1] * fs, rij[2] * fs};
    long long *f1 = s.facc + 3 * (long long)a1, *f2 = s.facc + 3 * (long long)a2;
    for (int c = 0; c < 3; c++) {
      long long v = f2fix(fij[c], FORCE_SCALE);
      red_add(f1 + c, -v);
      red_add(f2 + c, v);
    }
    vir[0] = fij[0] * rij[0]; vir[1] = fij[0] * rij[1]; vir[2] = fij[0] * rij[2];
    vir[3] = fij[1] * rij[1]; vir[4] = fij[1] * rij[2]; vir[5] = fij[2] * rij[2];
  }
  box_accumulate(s.eacc, box, valid, E_COUL, en, virial ? vir : nullptr);
}

template <typename T>
int recip_t(const SystemDev &s, const NbListDev &nb, const PmeDev &pm, cudaStream_t st,
            StageMark mark, void *mctx) {
  using T2 = typename C2<T>::t;
  const int TB = 256;
  constexpr bool MIXED = sizeof(T) == 4;
  const long long n4 = 4ll * nb.nslot;
  if (pm.order == 4) k_spread4<MIXED><<<(unsigned)((n4 + TB - 1) / TB), TB, 0, st>>>(nb, pm);
  else k_spread<MIXED, 0><<<(nb.nslot + TB - 1) / TB, TB, 0, st>>>(nb, pm);
  if (mark) mark(mctx, "pme_spread");
  // shared memory sized to the largest work item of the plan (caps ZMAXE / LMAXE)
  const size_t zsmem = sizeof(T2) * (256 + 2 * (size_t)pm.zbuf);
  static bool zconf[PMB_MAX_DEVICES] = {}, lconf[PMB_MAX_DEVICES] = {};  // per device
  const int dev = device_slot();
  if (!zconf[dev]) {
    const int zcap = (int)(sizeof(T2) * (256 + 2 * (size_t)ZMAXE));
    cudaFuncSetAttribute(k_fft_z_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, zcap);
    cudaFuncSetAttribute(k_fft_z_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, zcap);
    zconf[dev] = true;
  }
  k_fft_z_fwd<T><<<pm.nzwork, ZT, zsmem, st>>>(pm);
  const size_t lsmem = 32 * sizeof(double) + sizeof(T2) * (256 + 2 * (size_t)pm.lbuf);
  if (!lconf[dev]) {
    const int lcap = (int)(32 * sizeof(double) + sizeof(T2) * (256 + 2 * (size_t)LMAXE));
    cudaFuncSetAttribute(k_fft_y<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lcap);
    cudaFuncSetAttribute(k_fft_x_infl<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lcap);
    lconf[dev] = true;
  }
  auto fft_y = [&](int sign) {
    switch (pm.wy) {
      case 1: k_fft_y_warp<T, 1><<<pm.nywork, WT, 0, st>>>(pm, sign); break;
      case 2: k_fft_y_warp<T, 2><<<pm.nywork, WT, 0, st>>>(pm, sign); break;
      case 3: k_fft_y_warp<T, 3><<<pm.nywork, WT, 0, st>>>(pm, sign); break;
      case 4: k_fft_y_warp<T, 4><<<pm.nywork, WT, 0, st>>>(pm, sign); break;
      case 5: k_fft_y_warp<T, 5><<<pm.nywork, WT, 0, st>>>(pm, sign); break;
      default: k_fft_y<T><<<pm.nywork, LT, lsmem, st>>>(pm, sign);
    }
  };
  fft_y(-1);
  switch (pm.wx) {
    case 1: k_fft_x_warp<T, 1><<<pm.nxwork, WX, 0, st>>>(s, pm); break;
    case 2: k_fft_x_warp<T, 2><<<pm.nxwork, WX, 0, st>>>(s, pm); break;
    case 3: k_fft_x_warp<T, 3><<<pm.nxwork, WX, 0, st>>>(s, pm); break;
    case 4: k_fft_x_warp<T, 4><<<pm.nxwork, WX, 0, st>>>(s, pm); break;
    case 5: k_fft_x_warp<T, 5><<<pm.nxwork, WX, 0, st>>>(s, pm); break;
    default: k_fft_x_infl<T><<<pm.nxwork, LT, lsmem, st>>>(s, pm);
  }
  fft_y(+1);
  switch (pm.wz) {
    case 1: k_fft_z_inv_warp<T, 1><<<pm.nzwork, WZ, 0, st>>>(pm); break;
    case 2: k_fft_z_inv_warp<T, 2><<<pm.nzwork, WZ, 0, st>>>(pm); break;
    case 3: k_fft_z_inv_warp<T, 3><<<pm.nzwork, WZ, 0, st>>>(pm); break;
    case 4: k_fft_z_inv_warp<T, 4><<<pm.nzwork, WZ, 0, st>>>(pm); break;
    case 5: k_fft_z_inv_warp<T, 5><<<pm.nzwork, WZ, 0, st>>>(pm); break;
    default: k_fft_z_inv<T><<<pm.nzwork, ZT, zsmem, st>>>(pm);
  }
  if (mark) mark(mctx, "pme_fft");
  if (pm.order == 4) k_gather4<MIXED><<<(unsigned)((4ll * nb.nslot + TB - 1) / TB), TB, 0, st>>>(s, nb, pm);
  else k_gather<MIXED, 0><<<(nb.nslot + TB - 1) / TB, TB, 0, st>>>(s, nb, pm);
  if (mark) mark(mctx, "pme_gather");
  return 0;
}

}  // namespace

int pme_line_capacity() { return LMAXE; }

int pme_recip_launch(const SystemDev &s, const NbListDev &nb, const PmeDev &pm, cudaStream_t st,
                     StageMark mark, void *mctx) {
  return pm.precision ? recip_t<float>(s, nb, pm, st, mark, mctx)
                      : recip_t<double>(s, nb, pm, st, mark, mctx);
}

int pme_correction_launch(const SystemDev &s, const PmeDev &pm, const int *excl_pairs,
                          const int *excl_kind, int nexcl, double coulomb_scaling, cudaStream_t st) {
  if (nexcl <= 0) return 0;
  const int TB = 256;
  k_correction<<<(nexcl + TB - 1) / TB, TB, 0, st>>>(s, excl_pairs, excl_kind, nexcl, pm.alpha,
                                                     pm.a2pi, coulomb_scaling, pm.virial);
  return 0;
}

}  // namespace pmb
