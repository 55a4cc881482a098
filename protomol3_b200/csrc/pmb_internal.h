// Host-side declarations shared by the .cu translation units of libpmb200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "pmb_common.cuh"

namespace pmb {

void set_error(const std::string &msg);

#define PMB_CUDA(expr)                                                                   \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      ::pmb::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));              \
      return PMB_ERR_CUDA;                                                               \
    }                                                                                    \
  } while (0)

enum {
  PMB_OK_ = 0,
};

// Index of the current device for per-device one-time settings (a kernel's attributes, such as
// its dynamic shared-memory limit, belong to the device they were set on).
constexpr int PMB_MAX_DEVICES = 64;
inline int device_slot() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= PMB_MAX_DEVICES) d = 0;
  return d;
}

// ------------------------------------------------------------------ neighbour list (nblist.cu)
struct NbListDev {
  // per block
  int nblk_total;
  const int *blk_box;          // [nblk]
  float4 *blk_center;          // [nblk] fractional-fixed centre (as uint bits) and count
  uint4 *blk_lo, *blk_hi;      // [nblk] fixed-point extents (x, y, z)
  uint4 *blk_c, *blk_h;        // [nblk] the same as centre (.w = atoms) and half extent
  int nsblk;                   // superblocks: runs of 32 consecutive blocks
  uint4 *sblk_lo, *sblk_hi;    // [nsblk] union of their blocks' extents, .w = atoms
  uint4 *sblk_c, *sblk_h;      // [nsblk] the same as centre (.w = atoms) and half extent
  int *jcap_off;               // [nblk+1] offset of each block's j-slot list region
  int *jcount;                 // [nblk] tiles per block (its j-list, own slots first, in 32s)
  int *jlist;                  // [jcap_off[nblk]] j slots (-1 padding), JSAME flag bit
  int *tile_off;               // [nblk+1] exclusive scan of jcount
  int *tile_start;             // [nblk+1] first tile of each block: tile_off moved on so that
                               // each box's tiles start at a multiple of TILE_CHUNK (a box's
                               // last block is followed by up to TILE_CHUNK - 1 empty tiles)
  int *tile_blk;               // [tile_cap] block of each tile (-1: empty)
  int *tile_k;                 // [tile_cap] tile index within the block
  int tile_cap;
  int *status;                 // [4]: list / tile overflow, non-finite position, vacuum extent
  // per slot
  int nslot;
  int *slot_orig;              // [nslot] original atom index or -1
  uint4 *slot_fx;              // [nslot] fractional fixed-point x, y, z (2^32 per edge) + q bits
  double4 *slot_pq;            // [nslot] raw double position + q (FP64 path)
  int4 *slot_meta;             // [nslot] orig, molecule, type, box
  long long *fslot;            // [3][nslot] pair forces by slot (component-major), fixed point;
                               // folded into facc and cleared after the pair kernels
  // sort
  int nkeys;
  int *key;                    // [natoms]
  int *rank;                   // [natoms]
  int *bin_count;              // [nkeys + 1]
  int *bin_start;              // [nkeys + 1]
  int *scan_tmp;               // scratch for scans
  const int *bin_box;          // [nkeys] box of each sort bin
  int want_fp64;               // also pack raw double positions
  // list reuse: the list is built with cutoff + skin and rebuilt only once some atom moved more
  // than skin/2 since the last build (decided on the device, every step)
  double *xref;                // [3 natoms] positions at the last build
  unsigned *ctl;               // [8] max displacement^2 (float bits), rebuild flag, block counter,
                               // force flag, list builds (64-bit counter in [4..5]), the pair
                               // kernel's next chunk and finished warps ([6], [7]; zero between launches)
  float half_skin2;
  // per box: rebuilds are decided box by box (a box's list, slot order and therefore its
  // rounding do not depend on the other boxes of the system); ctl[1] says whether any box rebuilds
  int nbox;
  unsigned *box_d2;            // [nbox] max displacement^2 since the box's last build (float bits)
  unsigned *box_rb;            // [nbox] 1: the box rebuilds this step
  const int *box_order;        // [nbox] the boxes in ascending order of their first block
  int *box_shift;              // [nbox] tiles of padding before the box's first tile
  int *vext;                   // [6 nbox] vacuum extent per box: smallest and largest x, y, z as
                               // order-preserving int images of their float values (ctl[10] on)
};

struct SystemDev {
  int nbox, natoms;
  const BoxDev *box;           // [nbox]
  const int *atom_box;         // [natoms]
  const double *pos;           // [3 natoms] caller order
  const double *charge;        // [natoms]
  const int *type, *molecule;  // [natoms]
  const int *excl_start, *excl_partner, *excl_kind;  // CSR by atom
  long long *facc;             // [3 natoms]
  long long *eacc;             // [nbox * ACC_PER_BOX]
};

int nblist_sort(const SystemDev &s, NbListDev &nb, cudaStream_t st);
int nblist_lists(const SystemDev &s, NbListDev &nb, double list_cutoff, cudaStream_t st);
int fp32_peak_probe(double *tflops);

// ------------------------------------------------------------------ pair kernel (pair.cu)
struct PairLaunch {
  int precision;                  // 0 fp64, 1 mixed
  int do_lj, coul_mode, virial;
  const double *lj;               // [ntypes*ntypes*4] device
  const float *ljf;               // float copy
  const double *lattice;          // [nlat_total*3]
  int multi;                      // some box needs Ewald lattice images
  int ctas_per_sm;                // resident CTAs per SM of the persistent kernel (0: all that fit)
  int blk_lo, blk_hi;             // the blocks whose tiles this launch evaluates
  int wslot;                      // which chunk counter of the list's ctl words it uses (0 or 1)
  PairParams p;
};
int pair_launch(const SystemDev &s, const NbListDev &nb, const PairLaunch &pl, cudaStream_t st);
int pair_fold(const SystemDev &s, const NbListDev &nb, cudaStream_t st);

// Allocation-free all-pairs variant (FP64): energy/virial accumulators in a static device array
// of STATIC_MAX_BOXES boxes.  static_eacc_address looks the array up once per device (current
// device); pair_allpairs_launch zeroes s.nbox boxes of it on st, then writes fout [3 natoms].
constexpr int STATIC_MAX_BOXES = 1024;
cudaError_t static_eacc_address(long long **out);
cudaError_t pair_allpairs_launch(const SystemDev &s, const PairParams &p, const double *ljd,
                                 const double *pos, double *fout, long long *eacc,
                                 int max_box_atoms, cudaStream_t st);

// ------------------------------------------------------------------ PME (pme.cu)
struct PmeBoxPlan {
  int n[3];
  long long grid0;    // offset of this box's real/fixed grid (elements)
  long long cgrid0;   // offset of this box's half-complex grid (elements)
  int tw0[3];         // offsets of twiddle tables (complex elements)
  int inf0[3];        // offsets of influence tables
  int rad0[3], nrad[3];
  double hr[3];       // n / L
  double mr[3];       // 1 / L
  double piVr, fac;   // 1/(pi V), pi^2 / alpha^2
};

struct PmeDev {
  int nbox, order, precision;
  const PmeBoxPlan *plan;     // [nbox] device
  long long *qgrid;           // fixed-point charge grid
  void *cgrid;                // half-complex grid (float2 or double2), layout [kz][x][y]
  void *rgrid;                // real potential grid (float or double), layout [x][y][z]
  const double2 *twiddle;     // per dim tables exp(-2 pi i k / n)
  const float2 *twiddlef;
  const double *infl;         // per dim influence factor B(m) exp(-pi^2 m^2/alpha^2)
  const void *theta;          // influence function per half-spectrum point (float / double,
                              // layout as cgrid), 0 at m = 0
  const int *radix;           // radices per dim
  const int4 *zwork;          // z-pass work items: box, x, y0, count
  int nzwork;
  const int4 *ywork;          // y-line work items: box, kz, x0, rows
  int nywork;
  const int4 *xwork;          // x-line work items: box, kz, y0, columns
  int nxwork;
  int zbuf, lbuf;             // complex elements per ping-pong buffer of the z / line kernels
  int wz, wy, wx;             // R > 0: every box's z (y, x) lines have 32 R points and the inverse
                              // z pass (the y passes, the x pass) run the warp-shuffle transforms;
                              // 0: the shared-memory ones
  double alpha, a2pi;
  int virial;
};
// Block size of the warp-transform x kernel (one column per warp).
#ifndef PME_WX_THREADS
#define PME_WX_THREADS 256
#endif
// Optional stage marker (profiling): called on the host between kernel launches.
typedef void (*StageMark)(void *ctx, const char *stage);
int pme_recip_launch(const SystemDev &s, const NbListDev &nb, const PmeDev &pm, cudaStream_t st,
                     StageMark mark = nullptr, void *mark_ctx = nullptr);
int pme_line_capacity();
// Exact Ewald reciprocal sum of one box (pmb_ewald.cu): S, C [nk] and the box's forces in fout.
int ewald_recip_launch(const double *pos, const double *charge, int atom0, int n, const double3 *kv,
                       const double *a, int nk, double *S, double *Cc, double *fout, cudaStream_t st);
int pme_correction_launch(const SystemDev &s, const PmeDev &pm, const int *excl_pairs,
                          const int *excl_kind, int nexcl, double coulomb_scaling, cudaStream_t st);

// ------------------------------------------------------------------ bonded / integrator (md.cu)
struct BondedDev {
  int nbonds, nangles;
  const int *bonds;
  const double *bond_k, *bond_r0;
  const int *angles;
  const double *angle_k, *angle_theta0, *ub_k, *ub_r0;
  int virial;
};
int bonded_launch(const SystemDev &s, const BondedDev &b, cudaStream_t st);
// out = base + the accumulated forces (base may be null)
int forces_to_double(const SystemDev &s, double *out, cudaStream_t st, const double *base = nullptr);
int energies_to_double(const SystemDev &s, const double *const_e, double *out, cudaStream_t st);
int zero_accumulators(const SystemDev &s, cudaStream_t st);

struct IntegratorDev {
  int kind;            // 0 leapfrog, 1 Langevin
  double h;            // dt * INV_TIMEFACTOR
  double gamma, kT;    // Langevin (internal units)
  unsigned long long seed;
  // per box: the noise seed and the offset of the box's step count from the run's (a box that
  // joined the run part-way); an atom's noise is keyed by its box's seed, its index within the
  // box and its box's step, so a box draws the same numbers alone and beside other boxes
  const unsigned long long *box_seed;  // [nbox]
  const long long *box_step0;          // [nbox]
  const double *mass;  // [natoms]
  double *pos, *vel;
  long long *step;     // device step counter
};
// SHAKE / RATTLE bond constraints, one thread per connected group of constraints (a rigid water:
// 3 constraints on 3 atoms).  A group's constraints keep their order in the reference's list.
constexpr int CON_MAX_ATOMS = 8;    // atoms of one group
constexpr int CON_MAX_CONS = 16;    // constraints of one group
constexpr double CON_ERR_SCALE = 1099511627776.0;  // 2^40: fixed point of the per-sweep error sums
struct ConstraintDev {
  int ngroup, ncons;
  int max_atoms, max_cons;  // largest group (selects the kernel: rigid waters have 3 and 3)
  const int *group_con;    // [ngroup + 1] constraint offsets of each group
  const int *group_atom;   // [ngroup + 1] offsets into atoms
  const int *atoms;        // group atoms (global indices), each group's first-use order
  const int2 *con_local;   // [ncons] the two atoms of a constraint as indices into its group
  const double *len;       // [ncons] rest lengths
  double *rab;             // [3 ncons] SHAKE reference vectors x[a1] - x[a2] of the last SHAKE
  long long *err;          // [2][CON_ERR_BLOCK]: per modifier, the per-sweep error sums of the
                           // two rounds and the hand-over words (continue flag, first-round sweeps)
  int *sweeps;             // [2] sweeps of the last SHAKE and RATTLE (the next first round scans
                           // up to two more)
  double *win;             // [CON_WINDOW][6][max_atoms][ngroup] group states at the sweep counts
                           // around the last one, written by the first scan
  double clamp;            // largest group error added to a sum (keeps the int64 sums in range)
  double dt;               // timestep / TIMEFACTOR, as the modifiers use it
  double shake_eps, rattle_eps;
  int shake_max, rattle_max;
  // RATTLE's constraint virial (ModifierRattle.cpp:58), added to the box accumulators when set
  int virial;
  long long *eacc;
  const int *atom_box;
};
constexpr int CON_MAX_SWEEPS = 256;  // max_iter + 1 bound
constexpr int CON_ERR_BLOCK = 2 * (CON_MAX_SWEEPS + 1) + 2;
constexpr int CON_WINDOW = 3;
int constraints_init(const ConstraintDev &c, const IntegratorDev &in, cudaStream_t st);
int constraints_apply(const ConstraintDev &c, const IntegratorDev &in, int rattle, cudaStream_t st);
int integrate_kick_drift(const SystemDev &s, const IntegratorDev &in, double kick, cudaStream_t st);
int integrate_half_kick(const SystemDev &s, const IntegratorDev &in, cudaStream_t st);
int kinetic_energy(const SystemDev &s, const IntegratorDev &in, double *out_per_box, cudaStream_t st);

}  // namespace pmb
