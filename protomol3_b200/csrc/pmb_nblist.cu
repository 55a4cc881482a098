// Device cell-list / neighbour build: the B200 replacement of Topology::updateCellLists
// (topology/Topology.h:44-81) and CellListEnumerator<PBC, CubicCellManager>
// (topology/CellListEnumeratorPeriodicBoundaries.h:25-134).
//
// Instead of linked cell lists walked pair-of-cells by pair-of-cells, atoms are binned on a fine
// Hilbert-ordered grid with a deterministic counting sort, packed into 8-atom blocks of slots,
// and each block I gets a compacted list of atoms of blocks J > I that lie within the list
// cutoff of I's bounding box.  The pair kernel then sees (I, 32 j-atoms) tiles; the pair set it
// evaluates is exactly the reference's: every unordered pair once, minimal image, r^2 <= rc^2.
#include "pmb_internal.h"

namespace pmb {

namespace {

constexpr int SCAN_CHUNK = 4096;  // elements per CTA (1024 threads x 4)

// Index of cell (x, y, z) along a 3-D Hilbert curve over a 2^bits grid (J. Skilling, "Programming
// the Hilbert curve", AIP Conf. Proc. 707, 381 (2004): axes -> transposed index, then bit
// interleave).  Consecutive cells are face neighbours, so a run of slots never jumps across the
// box the way a Morton order does at its octant boundaries.
__device__ __forceinline__ unsigned hilbert3(unsigned x, unsigned y, unsigned z, int bits) {
  if (bits <= 0) return 0u;
  unsigned X[3] = {x, y, z};
  const unsigned M = 1u << (bits - 1);
  for (unsigned Q = M; Q > 1; Q >>= 1) {
    const unsigned P = Q - 1;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        unsigned t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  unsigned t = 0;
  for (unsigned Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  unsigned h = 0;
  for (int b = bits - 1; b >= 0; b--)
#pragma unroll
    for (int i = 0; i < 3; i++) h = (h << 1) | ((X[i] >> b) & 1u);
  return h;
}

__device__ __forceinline__ unsigned frac_fixed(double x, double Lr) {
  double u = x * Lr;
  u -= floor(u);
  double s = u * 4294967296.0;
  if (!(s >= 0.0)) s = 0.0;                 // also catches NaN
  if (s >= 4294967295.0) s = 4294967295.0;
  return (unsigned)s;
}

// ---------------------------------------------------------------- scans
__device__ int block_exclusive_scan(int v, int *total) {
  __shared__ int warp_tot[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int nw = blockDim.x >> 5;
    int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  int off = w > 0 ? warp_tot[w - 1] : 0;
  if (total) *total = warp_tot[(blockDim.x >> 5) - 1];
  __syncthreads();
  return off + x - v;
}

__global__ void k_scan_reduce(const int *in, int n, int *chunk, const unsigned *go) {
  if (go && !go[1]) return;
  long long base = (long long)blockIdx.x * SCAN_CHUNK + threadIdx.x * 4;
  int s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (base + k < n) s += in[base + k];
  int tot;
  block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) chunk[blockIdx.x] = tot;
}

__global__ void k_scan_chunks(int *chunk, int nchunk, const unsigned *go) {
  if (go && !go[1]) return;
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b = 0; b < nchunk; b += blockDim.x) {
    int i = b + threadIdx.x;
    int v = i < nchunk ? chunk[i] : 0;
    int tot;
    int ex = block_exclusive_scan(v, &tot);
    if (i < nchunk) chunk[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) chunk[nchunk] = carry;
}

__global__ void k_scan_apply(const int *in, int n, const int *chunk, int *out, const unsigned *go) {
  if (go && !go[1]) return;
  long long base = (long long)blockIdx.x * SCAN_CHUNK + threadIdx.x * 4;
  int v[4], s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  int ex = block_exclusive_scan(s, nullptr) + chunk[blockIdx.x];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = chunk[gridDim.x];
}

// ---------------------------------------------------------------- binning and sort
// Rebuild decision, box by box: max |x - x_ref|^2 over each box's atoms (box_d2), then the last
// block sets box_rb[b] for every box that moved more than half the skin and ctl[1] when any did
// (no host round trip); ctl = {-, any box rebuilds, finished blocks, forced rebuild of all}.
// It reads every position of every evaluation, so it also raises status[2] for a non-finite
// one (the host reports PMB_ERR_NUMERIC; every later kernel maps such a position to an in-range
// cell and grid index, so nothing reads out of bounds meanwhile), and, for a system whose boxes
// stand in for vacuum (ctl[10]), status[3] once the atoms of a box spread over half an edge
// (the minimal image would no longer be the plain difference).
__device__ __forceinline__ int ford(float f) {  // order-preserving int image of a float
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float fuord(int o) { return __int_as_float(o >= 0 ? o : o ^ 0x7fffffff); }

__global__ void k_disp_check(SystemDev s, NbListDev nb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f;
  int box = -1;
  const bool vacuum = nb.ctl[10] != 0u;
  if (i < s.natoms) {
    box = s.atom_box[i];
    const double x = s.pos[3 * i], y = s.pos[3 * i + 1], z = s.pos[3 * i + 2];
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicExch(&nb.status[2], 1);
    if (vacuum) {
      int *e = nb.vext + 6 * s.atom_box[i];
      const double p[3] = {x, y, z};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int o = ford((float)p[d]);
        atomicMin(e + d, o);
        atomicMax(e + 3 + d, o);
      }
      __threadfence();
    }
    double dx = x - nb.xref[3 * i], dy = y - nb.xref[3 * i + 1], dz = z - nb.xref[3 * i + 2];
    double r2 = dx * dx + dy * dy + dz * dz;
    d2 = r2 < 3.0e38 ? (float)r2 : 3.0e38f;
    if (!(d2 >= 0.f)) d2 = 3.0e38f;  // NaN positions force a rebuild
  }
  // per-box maxima (float bits of non-negative values order as unsigned): a warp whose atoms
  // belong to one box takes its maximum first, and the block adds one atomic per run of such
  // warps of the same box
  __shared__ int wbox[32];
  __shared__ float wmax[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned act = __ballot_sync(0xffffffffu, box >= 0);
  int wb = -1;  // the warp's box when all its atoms share one, else -1 (atomics already added)
  float m = 0.f;
  if (act) {
    const int b0 = __shfl_sync(0xffffffffu, box, __ffs(act) - 1);
    if (__all_sync(0xffffffffu, box < 0 || box == b0)) {
      m = d2;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      wb = b0;
    } else if (box >= 0) {
      atomicMax(&nb.box_d2[box], __float_as_uint(d2));
    }
  }
  if (lane == 0) {
    wbox[w] = wb;
    wmax[w] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (int)(blockDim.x >> 5);
    for (int k = 0; k < nw;) {
      const int b = wbox[k];
      float mm = wmax[k];
      int k2 = k + 1;
      for (; k2 < nw && wbox[k2] == b; k2++) mm = fmaxf(mm, wmax[k2]);
      if (b >= 0) atomicMax(&nb.box_d2[b], __float_as_uint(mm));
      k = k2;
    }
  }
  __threadfence();
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) last = atomicAdd(&nb.ctl[2], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const bool forced = nb.ctl[3] != 0u;
  int any = 0;
  for (int b = threadIdx.x; b < s.nbox; b += blockDim.x) {
    const float mx = __uint_as_float(atomicExch(&nb.box_d2[b], 0u));  // read and reset
    const unsigned rb = (forced || mx > nb.half_skin2) ? 1u : 0u;
    nb.box_rb[b] = rb;
    any |= (int)rb;
    if (vacuum)
      for (int d = 0; d < 3; d++) {
        // read and reset for the next evaluation
        const float lo = fuord(atomicExch(nb.vext + 6 * b + d, 0x7fffffff));
        const float hi = fuord(atomicExch(nb.vext + 6 * b + 3 + d, (int)0x80000000));
        if (!((double)hi - (double)lo < 0.5 * s.box[b].L[d])) atomicExch(&nb.status[3], 1);
      }
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    nb.ctl[1] = any ? 1u : 0u;
    if (any) ++*reinterpret_cast<unsigned long long *>(nb.ctl + 4);
    nb.ctl[2] = 0u;
    nb.ctl[3] = 0u;
  }
}

__global__ void k_zero_bins(int *bin_count, int n, const unsigned *go) {
  if (!go[1]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= n) bin_count[i] = 0;
}

__global__ void k_bin(SystemDev s, int *key, int *rank, int *bin_count, const unsigned *go, const unsigned *rb) {
  if (!go[1]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.natoms) return;
  const int bi = s.atom_box[i];
  if (!rb[bi]) return;  // the box keeps its slots
  const BoxDev &b = s.box[bi];
  unsigned c[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    unsigned f = frac_fixed(s.pos[3 * i + k], b.Lr[k]);
    c[k] = (unsigned)(((unsigned long long)f * (unsigned)b.nc[k]) >> 32);
  }
  int kk = b.key0 + (int)hilbert3(c[0], c[1], c[2], __ffs(b.nc[0]) - 1);
  key[i] = kk;
  rank[i] = atomicAdd(&bin_count[kk], 1);
}

__global__ void k_scatter(SystemDev s, const int *key, const int *rank, const int *bin_start,
                          int *slot_orig, const unsigned *go, const unsigned *rb) {
  if (!go[1]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.natoms) return;
  const int bi = s.atom_box[i];
  if (!rb[bi]) return;
  const BoxDev &b = s.box[bi];
  int base = b.blk0 * BLOCK - bin_start[b.key0];
  slot_orig[base + bin_start[key[i]] + rank[i]] = i;
}

// Makes the within-bin order deterministic (ascending original index).
__global__ void k_sort_bins(SystemDev s, const int *bin_box, const int *bin_start,
                            const int *bin_count, int nkeys, int *slot_orig, const unsigned *go) {
  if (!go[1]) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nkeys) return;
  int cnt = bin_count[k];
  if (cnt < 2) return;
  const BoxDev &b = s.box[bin_box[k]];
  int *p = slot_orig + b.blk0 * BLOCK - bin_start[b.key0] + bin_start[k];
  for (int a = 1; a < cnt; a++) {
    int v = p[a], j = a - 1;
    while (j >= 0 && p[j] > v) {
      p[j + 1] = p[j];
      j--;
    }
    p[j + 1] = v;
  }
}

__global__ void k_pack(SystemDev s, NbListDev nb, int want_fp64) {
  int sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= nb.nslot) return;
  int o = nb.slot_orig[sl];
  if (o < 0) {
    nb.slot_meta[sl] = make_int4(-1, -1, 0, nb.blk_box[sl / BLOCK]);
    nb.slot_fx[sl] = make_uint4(0, 0, 0, 0);
    if (want_fp64) nb.slot_pq[sl] = make_double4(0, 0, 0, 0);
    return;
  }
  int bi = s.atom_box[o];
  const BoxDev &b = s.box[bi];
  double x = s.pos[3 * o], y = s.pos[3 * o + 1], z = s.pos[3 * o + 2], q = s.charge[o];
  if (nb.ctl[1] && nb.box_rb[bi]) {  // the box's list is rebuilt this step: new reference positions
    nb.xref[3 * o] = x;
    nb.xref[3 * o + 1] = y;
    nb.xref[3 * o + 2] = z;
  }
  nb.slot_meta[sl] = make_int4(o, s.molecule[o], s.type[o], bi);
  nb.slot_fx[sl] = make_uint4(frac_fixed(x, b.Lr[0]), frac_fixed(y, b.Lr[1]),
                              frac_fixed(z, b.Lr[2]), __float_as_uint((float)q));
  if (want_fp64) nb.slot_pq[sl] = make_double4(x, y, z, q);
}

// Bounding box of every BLOCK-slot block in fractional fixed point; a warp covers GROUPS blocks.
__global__ void k_block_bbox(NbListDev nb) {
  if (!nb.ctl[1]) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int blk = t / BLOCK, lane = threadIdx.x & 31;
  bool inr = blk < nb.nblk_total;
  int sl = inr ? t : 0;
  bool valid = inr && nb.slot_orig[sl] >= 0;
  uint4 f = inr ? nb.slot_fx[sl] : make_uint4(0, 0, 0, 0);
  unsigned lo[3] = {valid ? f.x : 0xffffffffu, valid ? f.y : 0xffffffffu, valid ? f.z : 0xffffffffu};
  unsigned hi[3] = {valid ? f.x : 0u, valid ? f.y : 0u, valid ? f.z : 0u};
#pragma unroll
  for (int o = BLOCK / 2; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  unsigned bal = __ballot_sync(0xffffffffu, valid);
  int cnt = __popc(bal & (((1u << BLOCK) - 1u) << (lane & ~(BLOCK - 1))));
  if (inr && (lane & (BLOCK - 1)) == 0 && nb.box_rb[nb.blk_box[blk]]) {
    if (cnt == 0) lo[0] = lo[1] = lo[2] = hi[0] = hi[1] = hi[2] = 0;
    nb.blk_lo[blk] = make_uint4(lo[0], lo[1], lo[2], (unsigned)cnt);
    nb.blk_hi[blk] = make_uint4(hi[0], hi[1], hi[2], 0u);
    nb.blk_c[blk] = make_uint4(lo[0] + (hi[0] - lo[0]) / 2u, lo[1] + (hi[1] - lo[1]) / 2u,
                               lo[2] + (hi[2] - lo[2]) / 2u, (unsigned)cnt);
    nb.blk_h[blk] = make_uint4((hi[0] - lo[0]) / 2u + 1u, (hi[1] - lo[1]) / 2u + 1u, (hi[2] - lo[2]) / 2u + 1u, 0u);
  }
}

// Union extents of each run of 32 consecutive blocks (one warp per superblock).  Blocks of
// different boxes may share a superblock: the union then only enlarges, which never culls a
// true candidate.
__global__ void k_superblock_bbox(NbListDev nb) {
  if (!nb.ctl[1]) return;
  const int S = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (S >= nb.nsblk) return;
  const int J = S * 32 + lane;
  uint4 lo = make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0u), hi = make_uint4(0u, 0u, 0u, 0u);
  if (J < nb.nblk_total) {
    const uint4 l = nb.blk_lo[J];
    if (l.w > 0) {
      lo = l;
      hi = nb.blk_hi[J];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = min(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
    lo.y = min(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
    lo.z = min(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
    lo.w += __shfl_xor_sync(0xffffffffu, lo.w, o);
    hi.x = max(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
    hi.y = max(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
    hi.z = max(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
  }
  if (lane == 0) {
    if (lo.w == 0) lo.x = lo.y = lo.z = hi.x = hi.y = hi.z = 0;
    nb.sblk_lo[S] = lo;
    nb.sblk_hi[S] = hi;
    nb.sblk_c[S] = make_uint4(lo.x + (hi.x - lo.x) / 2u, lo.y + (hi.y - lo.y) / 2u, lo.z + (hi.z - lo.z) / 2u, lo.w);
    nb.sblk_h[S] = make_uint4((hi.x - lo.x) / 2u + 1u, (hi.y - lo.y) / 2u + 1u, (hi.z - lo.z) / 2u + 1u, 0u);
  }
}

// Gap^2 (A^2) between the box (c1, h1 half extents in A) and the box (c2, h2 fixed-point half
// extents) in FP32: the fixed-point difference (minimal image by 32-bit wrap-around) converts
// with an error of < 1e-5 A, far below the 1e-3 A margin of the list radius over the cutoff.
__device__ __forceinline__ float gap2f(const float sL[3], const unsigned c1[3], const float h1[3],
                                       uint4 c2, uint4 h2) {
  const unsigned c[3] = {c2.x, c2.y, c2.z}, h[3] = {h2.x, h2.y, h2.z};
  float g2 = 0.f;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float d = fmaxf((fabsf((float)(int)(c[k] - c1[k])) - (float)h[k]) * sL[k] - h1[k], 0.f);
    g2 = fmaf(d, d, g2);
  }
  return g2;
}

#ifndef BL_BLOCK_THREADS
#define BL_BLOCK_THREADS 256
#endif
#ifndef BL_MINB
#define BL_MINB 4
#endif
constexpr int BL_THREADS = BL_BLOCK_THREADS;
constexpr int BL_CAP = 128;  // candidate blocks buffered per warp before their atoms are tested

// One warp per block I: its own slots, then the candidate blocks J > I of the same box by
// bounding-box gap (superblocks of 32 blocks first), compacted into a shared-memory list, then
// the atoms of GROUPS listed blocks per pass within the list cutoff of I's box, compacted into
// I's j-list (tiles of 32 entries).  The loads of the next pass are issued before the current
// pass is tested.
__global__ void __launch_bounds__(BL_THREADS, BL_MINB) k_build_lists(SystemDev s, NbListDev nb, double rlist2) {
  __shared__ int cand_all[BL_THREADS / 32][BL_CAP];
  if (!nb.ctl[1]) return;
  const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (I >= nb.nblk_total) return;
  int *cl = cand_all[threadIdx.x >> 5];
  const int bi = nb.blk_box[I];
  if (!nb.box_rb[bi]) return;  // the box keeps its list
  const BoxDev &b = s.box[bi];
  const uint4 cIv = nb.blk_c[I], hIv = nb.blk_h[I];
  if (cIv.w == 0) {
    if (lane == 0) nb.jcount[I] = 0;
    return;
  }
  const float sL[3] = {(float)(b.L[0] * (1.0 / 4294967296.0)), (float)(b.L[1] * (1.0 / 4294967296.0)),
                       (float)(b.L[2] * (1.0 / 4294967296.0))};
  const unsigned cI[3] = {cIv.x, cIv.y, cIv.z};
  const float hI[3] = {(float)hIv.x * sL[0], (float)hIv.y * sL[1], (float)hIv.z * sL[2]};
  const int jend = b.blk0 + b.nblk;
  const int cap = nb.jcap_off[I + 1] - nb.jcap_off[I];
  int *out = nb.jlist + nb.jcap_off[I];
  const bool multi = b.multi_image != 0;
  const float rl2 = (float)rlist2;
  const int g = lane / BLOCK, li = lane & (BLOCK - 1);
  // molecules of the cluster's atoms (-2: padding): a listed j-atom of one of them is flagged
  // JSAME, so the pair kernel runs the exclusion test only on tiles holding such an atom; the
  // block's own slots open its list (the pair kernel takes j > i among them)
  // and the block's atom positions (fixed point; padding atoms far away): a candidate atom is
  // listed when it is within the list radius of one of them, the exact Verlet condition per
  // pair (the bounding-box gap alone would list about a third more atoms)
  // (in shared memory, FP32 relative to the block's first atom; padding atoms far away)
  // stored as pairs of atoms {t, t + BLOCK/2}: x x' y y' | z z' (two-wide FP32 tests)
  __shared__ float4 ipos_all[BL_THREADS / 32][BLOCK];
  float4 *ipos = ipos_all[threadIdx.x >> 5];
  int imol[BLOCK];
  unsigned r0[3];
  {
    const int4 m = nb.slot_meta[I * BLOCK + li];
    const uint4 f = nb.slot_fx[I * BLOCK + li];
    if (lane < BLOCK) out[lane] = m.x >= 0 ? ((I * BLOCK + lane) | JSAME) : -1;
    const int mine = m.x >= 0 ? m.y : -2;
#pragma unroll
    for (int t = 0; t < BLOCK; t++) imol[t] = __shfl_sync(0xffffffffu, mine, t);
    r0[0] = __shfl_sync(0xffffffffu, f.x, 0);
    r0[1] = __shfl_sync(0xffffffffu, f.y, 0);
    r0[2] = __shfl_sync(0xffffffffu, f.z, 0);
    float px = 1e6f, py = 1e6f, pz = 1e6f;
    if (m.x >= 0) {
      px = (float)(int)(f.x - r0[0]) * sL[0];
      py = (float)(int)(f.y - r0[1]) * sL[1];
      pz = (float)(int)(f.z - r0[2]) * sL[2];
    }
    const float qx = __shfl_down_sync(0xffffffffu, px, BLOCK / 2), qy = __shfl_down_sync(0xffffffffu, py, BLOCK / 2),
                qz = __shfl_down_sync(0xffffffffu, pz, BLOCK / 2);
    if (lane < BLOCK / 2) {
      ipos[2 * lane] = make_float4(px, qx, py, qy);
      ipos[2 * lane + 1] = make_float4(pz, qz, 0.f, 0.f);
    }
    __syncwarp();
  }
  // offsets from the first atom are minimal images of candidate-atom differences unless the box
  // is under about twice the list radius plus the block's extent: then each difference is
  // wrapped again
  const float rlf = sqrtf(rl2);
  const bool rewrap = rlf + 2.f * hI[0] >= 0.5f * (float)b.L[0] || rlf + 2.f * hI[1] >= 0.5f * (float)b.L[1] ||
                      rlf + 2.f * hI[2] >= 0.5f * (float)b.L[2];
  const float Lf[3] = {(float)b.L[0], (float)b.L[1], (float)b.L[2]},
              Lrf[3] = {(float)b.Lr[0], (float)b.Lr[1], (float)b.Lr[2]};
  auto near_any = [&](uint4 f) {
    const float px = (float)(int)(f.x - r0[0]) * sL[0], py = (float)(int)(f.y - r0[1]) * sL[1],
                pz = (float)(int)(f.z - r0[2]) * sL[2];
    bool near = false;
    if (rewrap) {
#pragma unroll
      for (int t = 0; t < BLOCK / 2; t++) {
        const float4 a = ipos[2 * t], c = ipos[2 * t + 1];
        const float qx[2] = {a.x, a.y}, qy[2] = {a.z, a.w}, qz[2] = {c.x, c.y};
#pragma unroll
        for (int u = 0; u < 2; u++) {
          float dx = px - qx[u], dy = py - qy[u], dz = pz - qz[u];
          dx -= Lf[0] * rintf(dx * Lrf[0]);
          dy -= Lf[1] * rintf(dy * Lrf[1]);
          dz -= Lf[2] * rintf(dz * Lrf[2]);
          near |= fmaf(dz, dz, fmaf(dy, dy, dx * dx)) <= rl2;
        }
      }
      return near;
    }
    const float2 nx2 = make_float2(-px, -px), ny2 = make_float2(-py, -py), nz2 = make_float2(-pz, -pz);
#pragma unroll
    for (int t = 0; t < BLOCK / 2; t++) {
      const float4 a = ipos[2 * t], c = ipos[2 * t + 1];
      const float2 dx = __fadd2_rn(make_float2(a.x, a.y), nx2), dy = __fadd2_rn(make_float2(a.z, a.w), ny2),
                   dz = __fadd2_rn(make_float2(c.x, c.y), nz2);
      const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
      near |= (r2.x <= rl2) | (r2.y <= rl2);
    }
    return near;
  };
  int count = BLOCK, ncand = 0;
  bool overflow = false;

  // atoms of the listed candidate blocks, GROUPS blocks (32 slots) per pass
  auto atoms = [&]() {
    __syncwarp();
    int sl = g < ncand ? cl[g] * BLOCK + li : -1;
    int4 m = make_int4(-1, -1, 0, 0);
    uint4 f = make_uint4(0, 0, 0, 0);
    if (sl >= 0) {
      m = nb.slot_meta[sl];
      f = nb.slot_fx[sl];
    }
    for (int p = 0; p < ncand; p += GROUPS) {
      const int q = p + GROUPS + g;
      const int sl2 = q < ncand ? cl[q] * BLOCK + li : -1;
      int4 m2 = make_int4(-1, -1, 0, 0);
      uint4 f2 = make_uint4(0, 0, 0, 0);
      if (sl2 >= 0) {
        m2 = nb.slot_meta[sl2];
        f2 = nb.slot_fx[sl2];
      }
      const bool take = m.x >= 0 && (multi || (gap2f(sL, cI, hI, f, make_uint4(0, 0, 0, 0)) <= rl2 && near_any(f)));
      const unsigned tm = __ballot_sync(0xffffffffu, take);
      const int n = __popc(tm);
      if (count + n > cap) {
        overflow = true;
        break;
      }
      if (take) {
        bool same = false;
#pragma unroll
        for (int t = 0; t < BLOCK; t++) same |= m.y == imol[t];
        out[count + __popc(tm & ((1u << lane) - 1u))] = same ? (sl | JSAME) : sl;
      }
      count += n;
      sl = sl2;
      m = m2;
      f = f2;
    }
    ncand = 0;
    __syncwarp();
  };

  // superblocks (runs of 32 blocks), 32 per ballot; then the 32 blocks of each candidate one
  const int send = (jend + 31) / 32;
  for (int S0 = (I + 1) / 32; S0 < send && !overflow; S0 += 32) {
    const int S = S0 + lane;
    bool scand = false;
    if (S < send) {
      const uint4 cS = nb.sblk_c[S];
      if (cS.w > 0) scand = multi || gap2f(sL, cI, hI, cS, nb.sblk_h[S]) <= rl2;
    }
    unsigned sm = __ballot_sync(0xffffffffu, scand);
    while (sm && !overflow) {
      const int J = (S0 + __ffs(sm) - 1) * 32 + lane;
      sm &= sm - 1;
      bool cand = false;
      if (J > I && J < jend) {
        const uint4 cJ = nb.blk_c[J];
        if (cJ.w > 0) cand = multi || gap2f(sL, cI, hI, cJ, nb.blk_h[J]) <= rl2;
      }
      const unsigned m = __ballot_sync(0xffffffffu, cand);
      if (ncand + __popc(m) > BL_CAP) atoms();
      if (cand) cl[ncand + __popc(m & ((1u << lane) - 1u))] = J;
      ncand += __popc(m);
    }
  }
  if (!overflow && ncand > 0) atoms();
  const int padded = (count + 31) & ~31;
  if (!overflow)
    for (int k = count + lane; k < padded; k += 32) out[k] = -1;
  if (lane == 0) {
    if (overflow) atomicExch(&nb.status[0], 1);
    nb.jcount[I] = overflow ? 0 : padded / 32;
  }
}

// Padding that starts every box's tiles at a multiple of TILE_CHUNK (one block of threads, the
// boxes in the order of their blocks): the pair kernel's warp assignments then never mix boxes,
// and a box's partial sums are grouped as when it is alone.
__global__ void k_box_pad(SystemDev s, NbListDev nb) {
  if (!nb.ctl[1]) return;
  const int per = (nb.nbox + (int)blockDim.x - 1) / (int)blockDim.x;
  const int k0 = min(nb.nbox, (int)threadIdx.x * per), k1 = min(nb.nbox, k0 + per);
  auto pad = [&](int b) {
    const BoxDev &bx = s.box[b];
    const int tot = nb.tile_off[bx.blk0 + bx.nblk] - nb.tile_off[bx.blk0];
    return (TILE_CHUNK - tot % TILE_CHUNK) % TILE_CHUNK;
  };
  int acc = 0;
  for (int k = k0; k < k1; k++) acc += pad(nb.box_order[k]);
  int tot;
  int ex = block_exclusive_scan(acc, &tot);
  for (int k = k0; k < k1; k++) {
    const int b = nb.box_order[k];
    nb.box_shift[b] = ex;
    ex += pad(b);
  }
  if (threadIdx.x == 0) nb.tile_start[nb.nblk_total] = nb.tile_off[nb.nblk_total] + tot;
}

// One warp per block: its first tile and its tiles' (block, index) entries, written by
// consecutive lanes; a box's last block also writes the box's empty padding tiles.
__global__ void k_tile_map(SystemDev s, NbListDev nb) {
  if (!nb.ctl[1]) return;
  const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (I >= nb.nblk_total) return;
  const int b = nb.blk_box[I];
  const BoxDev &bx = s.box[b];
  const int shift = nb.box_shift[b];
  const int off = nb.tile_off[I] + shift, cnt = nb.jcount[I];
  int end = off + cnt;
  if (I == bx.blk0 + bx.nblk - 1) {
    const int start = nb.tile_off[bx.blk0] + shift;
    end = start + (end - start + TILE_CHUNK - 1) / TILE_CHUNK * TILE_CHUNK;
  }
  if (lane == 0) nb.tile_start[I] = off;
  if (end > nb.tile_cap) {
    if (lane == 0) atomicExch(&nb.status[1], 1);
    return;
  }
  for (int k = lane; k < end - off; k += 32) {
    nb.tile_blk[off + k] = k < cnt ? I : -1;
    nb.tile_k[off + k] = k;
  }
}

int scan_exclusive(const int *in, int *out, int n, int *tmp, cudaStream_t st, const unsigned *go) {
  int nchunk = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  if (nchunk < 1) nchunk = 1;
  k_scan_reduce<<<nchunk, 1024, 0, st>>>(in, n, tmp, go);
  k_scan_chunks<<<1, 1024, 0, st>>>(tmp, nchunk, go);
  k_scan_apply<<<nchunk, 1024, 0, st>>>(in, n, tmp, out, go);
  return 0;
}

}  // namespace

// First half of a build: displacement check, sort into slots and the slot records of this step's
// positions (the PME kernels need no more than these).
int nblist_sort(const SystemDev &s, NbListDev &nb, cudaStream_t st) {
  const int T = 256;
  int na = s.natoms;
  if (na <= 0) return 0;
  // every kernel after the displacement check exits at once unless ctl[1] asks for a rebuild
  // (inside a CUDA graph such a launch costs about a microsecond)
  k_disp_check<<<(na + T - 1) / T, T, 0, st>>>(s, nb);
  k_zero_bins<<<(nb.nkeys + T) / T, T, 0, st>>>(nb.bin_count, nb.nkeys, nb.ctl);
  k_bin<<<(na + T - 1) / T, T, 0, st>>>(s, nb.key, nb.rank, nb.bin_count, nb.ctl, nb.box_rb);
  scan_exclusive(nb.bin_count, nb.bin_start, nb.nkeys, nb.scan_tmp, st, nb.ctl);
  k_scatter<<<(na + T - 1) / T, T, 0, st>>>(s, nb.key, nb.rank, nb.bin_start, nb.slot_orig, nb.ctl, nb.box_rb);
  k_sort_bins<<<(nb.nkeys + T - 1) / T, T, 0, st>>>(s, nb.bin_box, nb.bin_start, nb.bin_count,
                                                   nb.nkeys, nb.slot_orig, nb.ctl);
  k_pack<<<(nb.nslot + T - 1) / T, T, 0, st>>>(s, nb, nb.want_fp64);
  return 0;
}

// Second half: cluster boxes, the cluster j-lists and the tile map of the pair kernel.
int nblist_lists(const SystemDev &s, NbListDev &nb, double list_cutoff, cudaStream_t st) {
  const int T = 256;
  if (s.natoms <= 0) return 0;
  const int wthreads = nb.nblk_total * 32;
  k_block_bbox<<<(nb.nslot + T - 1) / T, T, 0, st>>>(nb);
  k_superblock_bbox<<<(nb.nsblk * 32 + T - 1) / T, T, 0, st>>>(nb);
  k_build_lists<<<(wthreads + BL_THREADS - 1) / BL_THREADS, BL_THREADS, 0, st>>>(s, nb, list_cutoff * list_cutoff);
  scan_exclusive(nb.jcount, nb.tile_off, nb.nblk_total, nb.scan_tmp, st, nb.ctl);
  k_box_pad<<<1, 1024, 0, st>>>(s, nb);
  k_tile_map<<<(wthreads + T - 1) / T, T, 0, st>>>(s, nb);
  return 0;
}

}  // namespace pmb
