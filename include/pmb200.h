/*
 * libpmb200 -- B200 (sm_100a) implementation of ProtoMol 3's nonbonded force path behind a
 * plain C ABI: cell-list cutoff Lennard-Jones + Coulomb with C1/C2 switching, and particle-mesh
 * Ewald (B-spline spreading, 3-D FFT, influence function, gather, Ewald real-space, self and
 * exclusion corrections), with the bonded water terms and leapfrog / Langevin integrators that
 * the ns/day metric needs.
 *
 * Every entry point returns 0 (PMB_OK) or a PMB_ERR_* status; pmb_last_error() gives the message
 * (thread local).  Handles are not re-entrant: one host thread drives a system at a time, as
 * ProtoMol drives SystemForce::evaluate.  A system, its forces, MD runs and trajectories belong
 * to the CUDA device that was current when the system was created; calls on them are made with
 * that device current (as for its streams and memory).
 *
 * A system is a batch of one or more independent periodic boxes.  Per-atom host arrays are the
 * concatenation of the boxes' atoms in box order; per-box outputs are PMB_E_STRIDE doubles each:
 *   [PMB_E_COULOMB, PMB_E_LJ, PMB_E_BOND, PMB_E_ANGLE, PMB_E_VIRIAL + 0..8 (row-major 3x3), pad]
 * matching ProtoMol's ScalarStructure slots COULOMB, LENNARDJONES, BOND, ANGLE, VIRIALXX..ZZ
 * (type/ScalarStructure.h:26-54).
 */
#ifndef PMB200_H
#define PMB200_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define PMB_OK 0
#define PMB_ERR_ARG 1         /* invalid argument (ProtoMol: report << error, doMake -> NULL) */
#define PMB_ERR_CUDA 2        /* CUDA runtime error or no device */
#define PMB_ERR_CAPACITY 3    /* a neighbour or tile list overflowed its buffer */
#define PMB_ERR_UNSUPPORTED 4 /* configuration outside what this build implements */
#define PMB_ERR_STATE 5       /* call out of order (e.g. run before set_state) */
#define PMB_ERR_NUMERIC 6     /* non-finite input or result */

enum { PMB_FP64 = 0, PMB_MIXED = 1 };
enum { PMB_SWITCH_CUTOFF = 0, PMB_SWITCH_C1 = 1, PMB_SWITCH_C2 = 2 };
enum { PMB_FORCE_CUTOFF = 1, PMB_FORCE_PME = 2, PMB_FORCE_BONDED = 3 };
enum { PMB_LEAPFROG = 0, PMB_LANGEVIN = 1 };
enum {
  PMB_E_COULOMB = 0,
  PMB_E_LJ = 1,
  PMB_E_BOND = 2,
  PMB_E_ANGLE = 3,
  PMB_E_VIRIAL = 4,
  PMB_E_STRIDE = 16
};

typedef struct pmb_system pmb_system;
typedef struct pmb_force pmb_force;
typedef struct pmb_md pmb_md;

/* One periodic box: the parts of ProtoMol's GenericTopology the force path reads
 * (topology/GenericTopology.h:142-164) plus its PeriodicBoundaryConditions. */
typedef struct {
  int n_atoms, n_types;
  const double *charge;   /* [n_atoms] scaled charge = e * 18.2226123264 (Atom::scaledCharge) */
  const double *mass;     /* [n_atoms] (Atom::scaledMass); integrators only, may be NULL */
  const int *type;        /* [n_atoms] LJ type index (Atom::type) */
  const int *molecule;    /* [n_atoms] (Atom::molecule) */
  const double *lj;       /* [n_types * n_types * 4] {A, B, A14, B14} (LennardJonesParameterTable) */
  int n_excl;             /* ExclusionTable::getTable() */
  const int *excl_pairs;  /* [2 * n_excl] atom indices within the box */
  const int *excl_kind;   /* [n_excl] 1 = EXCLUSION_MODIFIED, 2 = EXCLUSION_FULL */
  int n_bonds;
  const int *bonds;       /* [2 * n_bonds] */
  const double *bond_k, *bond_r0;
  int n_angles;
  const int *angles;      /* [3 * n_angles] */
  const double *angle_k, *angle_theta0, *ub_k, *ub_r0;
  double box[3];          /* orthogonal box edges (cellBasisVector1..3) */
  double coulomb_scaling; /* GenericTopology::coulombScalingFactor */
} pmb_box_desc;

/* One force term.  PMB_FORCE_CUTOFF replaces NonbondedCutoffSystemForce with
 * OneAtomPair(Two)<PBC, Switch, LennardJonesForce [, Switch, CoulombForce]>
 * (force/nonbonded/NonbondedCutoffSystemForce.h:45-55); PMB_FORCE_PME replaces
 * NonbondedPMEwaldSystemForce<PBC, CubicCellManager, real, reciprocal, correction, BSpline,
 * Cutoff|C1> (mdl/interface/force/nonbonded/NonbondedPMEwaldSystemForce.h:245-319) with the
 * parameters of its getParameters() (:1003-1014); PMB_FORCE_BONDED replaces BondSystemForce +
 * AngleSystemForce. */
typedef struct {
  int kind;
  /* cutoff: -switchingFunction, -switchon, -cutoff per potential */
  int lj, lj_switch;
  double lj_switchon, lj_cutoff;
  int coulomb, coulomb_switch;
  double coulomb_switchon, coulomb_cutoff;
  /* PME: -gridsize nx ny nz, -cutoff, -order, -accuracy, -alpha (<= 0: bisection) */
  int grid[3];
  const int *box_grids;   /* optional [3 * n_boxes] per-box grid sizes (batched systems) */
  int order;
  double cutoff, accuracy, alpha;
  int real_switch;        /* PMB_SWITCH_CUTOFF or PMB_SWITCH_C1 */
  int real, reciprocal, correction;
} pmb_force_desc;

typedef struct {
  int kind;                 /* PMB_LEAPFROG or PMB_LANGEVIN */
  double timestep_fs;
  double temperature;       /* Langevin temperature (K) */
  double gamma_ps;          /* Langevin friction (1/ps) */
  unsigned long long seed;  /* Langevin noise seed */
} pmb_integrator_desc;

const char *pmb_last_error(void);
int pmb_device_count(void);

/* Systems ------------------------------------------------------------------------------------ */
pmb_system *pmb_system_create(const pmb_box_desc *boxes, int n_boxes, int precision);
int pmb_system_destroy(pmb_system *sys);
int pmb_system_set_stream(pmb_system *sys, void *cuda_stream);
int pmb_system_n_atoms(const pmb_system *sys);
int pmb_system_n_boxes(const pmb_system *sys);
/* Verlet skin (A, default 0.8): the cell/neighbour list is built for cutoff + skin and rebuilt
 * on the device only when some atom moved more than skin/2 since the last build; 0 rebuilds at
 * every evaluation like Topology::updateCellLists.  The pair set evaluated is the same either
 * way (every pair within the cutoff). */
int pmb_system_set_skin(pmb_system *sys, double skin);
/* Knobs that change the speed of a system's evaluations but not which pairs are evaluated, set
 * by the autotuner (protomol3_b200/autotune.py) per workload; no counterpart in the reference.
 *   skin: as pmb_system_set_skin;
 *   sort_cell: smallest edge (A) of the sort cells that order atoms along a Hilbert curve before
 *     they are grouped into 8-atom clusters (default 2.4; cells per axis are powers of two);
 *   pair_ctas_per_sm: resident CTAs per SM of the persistent pair kernel (0: as many as fit).
 * A change of skin or sort_cell re-sizes the neighbour list; after a change of any knob, MD runs
 * and host-pointer evaluations capture their step again.
 * Results differ only in the rounding order of the FP32 / FP64 partial sums. */
typedef struct {
  double skin;
  double sort_cell;
  int pair_ctas_per_sm;
} pmb_tuning;
int pmb_system_set_tuning(pmb_system *sys, const pmb_tuning *tuning);
int pmb_system_get_tuning(const pmb_system *sys, pmb_tuning *tuning);
/* Vacuum (VacuumBoundaryConditions, topology/VacuumBoundaryConditions.h: the plain difference,
 * no images; cell pairs of CellListEnumerator_standard) for the cutoff forces: a box whose edges
 * are more than twice the extent of its atoms stands in for vacuum, because every minimal-image
 * difference is then the plain difference.  pmb_vacuum_box gives such edges for positions
 * [3 n_atoms]: 2 (extent + margin) + 1 per axis (margin: room for the atoms to move, e.g. the
 * list radius).  With pmb_system_set_vacuum on, pmb_evaluate and pmb_force_evaluate check the
 * extent of every box's atoms and return PMB_ERR_STATE once it reaches half an edge; evaluations
 * of device positions and MD runs check it on the device (the list's displacement check, for
 * force sets with a pair term), reported by pmb_system_check and the MD calls that wait for the
 * stream (pmb_md_get_state, pmb_md_energies, ...). */
int pmb_vacuum_box(const double *positions, int n_atoms, double margin, double edges[3]);
/* Exact Ewald reciprocal sum, the check path for the PME reciprocal term: what
 * NonbondedFullEwaldSystemForce with only -reciprocal adds (reciprocalTerm,
 * force/nonbonded/NonbondedFullEwaldSystemForce.h:873-1083), over the k-vectors |k| < kc of its
 * initialize (:590-660): kc = 2 alpha sqrt(-ln accuracy), alpha <= 0 takes the reference's
 * default sqrt(pi) (5.5 N / V^2)^(1/6) per box.  Host positions [3 N]; forces +=, energies +=
 * (PMB_E_COULOMB and, with virial, the virial slots of each box).  Allocates its k-vector
 * scratch per call; cost N x (number of k-vectors) per box. */
int pmb_ewald_reciprocal(pmb_system *sys, const double *positions, double alpha, double accuracy, double *forces,
                         double *energies, int virial);
int pmb_system_set_vacuum(pmb_system *sys, int on);
/* Waits for the system's stream and reports whether a neighbour list overflowed since the last
 * check: PMB_ERR_CAPACITY, with the list storage enlarged so that the next evaluation fits; or
 * whether an evaluation met a non-finite position (device evaluations, MD runs that blew up):
 * PMB_ERR_NUMERIC.  The
 * host-pointer entry points check by themselves and retry; pmb_evaluate_device does not
 * synchronise, so its callers call this after their evaluations and repeat one that overflowed. */
int pmb_system_check(pmb_system *sys);
/* Neighbour-list builds so far (the first evaluation builds; later ones rebuild once an atom has
 * moved more than half the skin).  Synchronises the system stream.  No counterpart in the
 * reference, which rebuilds its cell lists at every evaluation. */
int pmb_system_list_builds(pmb_system *sys, long long *n);
/* Size of the current neighbour list in pair-kernel tiles: each tile is 8 i-atoms against 32
 * listed j-atoms (256 pair slots), padding included, so 256 tiles over the pairs within the
 * cutoff is the share of the evaluated pairs that count.  Synchronises the system stream.  No
 * counterpart in the reference (its cell lists have no tiles). */
int pmb_system_list_tiles(pmb_system *sys, long long *tiles);
/* Host time of the last pmb_evaluate / pmb_force_evaluate, in ms: [0] checks and enqueueing
 * (the position upload and every launch), [1] waiting for the device's first results (status
 * and energies), [2] adding the forces into the caller's array while their device->host copies
 * land piece by piece (a page-locked force array: waiting for the sum to land in it).  No
 * counterpart in the reference (TimerStatistic times whole forces). */
int pmb_system_evaluate_times(const pmb_system *sys, double ms[3]);

/* Forces ------------------------------------------------------------------------------------- */
pmb_force *pmb_force_create(pmb_system *sys, const pmb_force_desc *desc);
int pmb_force_destroy(pmb_force *f);
/* Ewald splitting parameter in use (NonbondedPMEwaldSystemForce::initialize, :520-537). */
int pmb_force_alpha(const pmb_force *f, double *alpha);

/* SystemForce::evaluate(topology, positions, forces, energies) for one force: host positions
 * [3 N], forces += [3 N], energies += [n_boxes * PMB_E_STRIDE]; virial != 0 also fills the
 * virial slots (ScalarStructure::virial()). */
int pmb_force_evaluate(pmb_force *f, const double *positions, double *forces, double *energies,
                       int virial);
/* Several forces of one system in one device pass (ForceGroup::evaluateSystemForces).  A
 * non-finite position gives PMB_ERR_NUMERIC with forces and energies untouched (detected on the
 * device by the list kernels, on the host for force sets that need no list).  A page-locked
 * forces_out (cudaMallocHost, cudaHostAlloc, cudaHostRegister) is uploaded beside the force
 * kernels, added to on the device and copied back into directly, with no host pass over it; a
 * pageable one is added to on the host.  Both give the same doubles.  With page-locked positions
 * as well, the copies are part of the evaluation's CUDA graph (kept per pair of host arrays), so
 * a call enqueues one graph launch. */
int pmb_evaluate(pmb_system *sys, pmb_force *const *forces, int n_forces, const double *positions,
                 double *forces_out, double *energies, int virial);
/* Same, with device pointers and no host synchronisation: d_forces and d_energies are
 * overwritten (not accumulated), on the system's stream.  d_positions NULL reuses the positions
 * of the last evaluation (PMB_ERR_STATE if there was none). */
int pmb_evaluate_device(pmb_system *sys, pmb_force *const *forces, int n_forces,
                        const double *d_positions, double *d_forces, double *d_energies,
                        int virial);

/* Device-resident MD (the integrator owns the step; one CUDA graph per step) ----------------- */
pmb_md *pmb_md_create(pmb_system *sys, pmb_force *const *forces, int n_forces,
                      const pmb_integrator_desc *desc);
int pmb_md_destroy(pmb_md *md);
/* Host state in; computes the initial forces (StandardIntegrator::initializeForces). */
int pmb_md_set_state(pmb_md *md, const double *positions, const double *velocities);
/* Checkpoint of the run's resident state, exact (the checkpoint's content of OutputCheckpoint,
 * output/OutputCheckpoint.cpp:58-70, 137-178, without its text rounding): positions and
 * velocities [3 N], the neighbour list's reference positions [3 N] (those of its last build;
 * NULL skips them) and the steps taken since the state was set (the Langevin noise counter).
 * Waits for the system's stream. */
int pmb_md_get_checkpoint(pmb_md *md, double *positions, double *velocities, double *list_reference,
                          long long *step);
/* Restores a checkpoint into this run, which may belong to another system made from the same
 * boxes and forces (a segment moved to another slot or device), and computes the initial forces
 * as pmb_md_set_state does (CheckpointModule::read / postBuild, module/CheckpointModule.cpp:30-48).
 * With list_reference the neighbour list is first built at those positions, so that the run
 * continues bit for bit as the run the checkpoint came from; without it (NULL) the list is built
 * at the positions and the continuation agrees to the rounding of the arithmetic.  velocities
 * NULL: zero.  pmb_md_set_state is this call with no list reference and step 0. */
int pmb_md_set_checkpoint(pmb_md *md, const double *positions, const double *velocities,
                          const double *list_reference, long long step);
/* Per-box Langevin noise streams.  An atom's noise is keyed by its box's seed, its index within
 * the box and its box's step count, so a box draws the same numbers alone and beside other boxes.
 * seeds[n_boxes] (NULL keeps them; a run made with seed s starts box b at s + b) and steps[n_boxes],
 * each box's own step count at the run's current step (NULL keeps them; by default the run's):
 * a box restored from another run continues that run's noise.  No counterpart in the reference
 * (one serial generator per run, base/MathUtilities.cpp:206-238). */
int pmb_md_set_box_noise(pmb_md *md, const unsigned long long *seeds, const long long *steps);
int pmb_md_get_box_noise(const pmb_md *md, unsigned long long *seeds, long long *steps);
/* Writes a checkpoint in the reference's files (OutputCheckpoint::doIt, :58-70): positions to
 * pos_base + id + ".pos" and velocities to vel_base + id + ".vel" as XYZWriter writes them
 * (io/XYZWriter.cpp:28-53; names: one string per atom), then the checkpoint file config_path
 * (written to config_path + ".tmp" and renamed, as WriteConfig does) in CheckpointConfigWriter's
 * layout (io/CheckpointConfigWriter.cpp:11-25): "!Checkpoint File!", #ID, #Step (first_step +
 * the steps taken), #Random and #Integrator.  #Random holds this library's noise state,
 * "philox4x32-10 <seed> <half kicks drawn>" of the first box (every box's stream:
 * pmb_md_get_box_noise), in place of the reference's serial generator;
 * #Integrator is empty, as the leapfrog and Langevin integrators write nothing there.  The files
 * of checkpoint id - 1 are removed, as the reference removes them. */
int pmb_md_write_checkpoint(pmb_md *md, const char *config_path, int id, long long first_step,
                            const char *pos_base, const char *vel_base, const char *const *names);
int pmb_md_get_state(pmb_md *md, double *positions, double *velocities);
int pmb_md_get_forces(pmb_md *md, double *forces);
/* LeapfrogIntegrator::run(n) / StandardIntegrator::run(n) semantics. */
int pmb_md_run(pmb_md *md, int n_steps);
/* Energies of the last force evaluation [n_boxes * PMB_E_STRIDE] and kinetic energy per box. */
int pmb_md_energies(pmb_md *md, double *energies, double *kinetic);
int pmb_md_use_graph(pmb_md *md, int enable);
/* The virial in the MD run's energies (ScalarStructure::virial() on): every step evaluates the
 * force virial, and RATTLE adds its constraint terms (2 dp) x rab (modifier/ModifierRattle.cpp:58).
 * pmb_md_energies then fills the virial slots: after run(n), those of the last evaluation plus the
 * last RATTLE application, what the reference's energies hold then (the SHAKE terms of
 * modifier/ModifierShake.cpp:65-68 are cleared by the force evaluation after each drift,
 * integrator/STSIntegrator.cpp:34-46, so they never reach an output).  Off by default. */
int pmb_md_set_virial(pmb_md *md, int on);
/* Runs n_steps (pmb_md_run) between two CUDA events on the system's stream and returns the mean
 * device time per step in ms (the autotuner's clock). */
int pmb_md_time(pmb_md *md, int n_steps, double *ms_per_step);
/* Bond constraints of a leapfrog or Langevin run (replaces ModifierShake / ModifierRattle as
 * module/ModifierModule.cpp:106-128 installs them): SHAKE after every drift, RATTLE after every
 * step, on a constraint list in the reference's order (topology/TopologyUtilities.cpp:695-775,
 * buildRattleShakeBondConstraintList).  A modifier is on when its flag is set, epsilon > 0 and
 * max_iter > 0 (the reference's defaults: 1e-5 and 30).  Each application sweeps the list as the
 * reference does until the mean error is at most epsilon, at most max_iter + 1 sweeps; the
 * constraint virial enters the energies with pmb_md_set_virial.  Constrained groups (atoms linked by constraints) hold at
 * most 8 atoms and 16 constraints; max_iter below 256.  The SHAKE reference positions are the
 * positions at pmb_md_set_state, or the current ones when this is called after it.  With the
 * Langevin integrator the modifiers sit where StandardIntegrator::run calls them
 * (integrator/StandardIntegrator.cpp:27-37; STSIntegrator::doDriftOrNextIntegrator): SHAKE after
 * the drift, RATTLE after the step's closing half kick. */
typedef struct {
  int n_constraints;
  const int *atom1, *atom2;   /* [n_constraints] */
  const double *rest_length;  /* [n_constraints] A */
  int shake;
  double shake_epsilon;
  int shake_max_iter;
  int rattle;
  double rattle_epsilon;
  int rattle_max_iter;
} pmb_constraint_desc;
int pmb_md_set_constraints(pmb_md *md, const pmb_constraint_desc *desc);
/* Sweeps of the last SHAKE and RATTLE application (max_iter + 1: not converged). */
int pmb_md_constraint_sweeps(pmb_md *md, int *shake_sweeps, int *rattle_sweeps);

/* Trajectory output -------------------------------------------------------------------------- */
typedef struct pmb_traj pmb_traj;
/* A DCD trajectory in the format of DCDTrajectoryWriter (io/DCDTrajectoryWriter.cpp:75-233), as
 * OutputDCDTrajectory opens it (output/OutputDCDTrajectory.cpp:27-43; the reference passes
 * timestep 1.0): header written with the first frame, frame count updated with every frame,
 * float32 coordinates.  little_endian selects the byte order of the file.  The first title line
 * names the file and this library's build, like the reference's. */
pmb_traj *pmb_traj_open_dcd(const char *path, int n_atoms, double timestep, int first_step, int little_endian,
                            const char *comment);
/* An XYZ file in the format of XYZWriter::write (io/XYZWriter.cpp:28-53); every frame rewrites
 * it (final positions, as OutputFinalXYZPos).  names: one string per atom. */
pmb_traj *pmb_traj_open_xyz(const char *path, int n_atoms, const char *const *names);
/* An XYZ trajectory in the format of XYZTrajectoryWriter (io/XYZTrajectoryWriter.cpp:64-160): a
 * first line holding the frame count in 19 characters, rewritten with every frame, then per frame
 * the atom count and per atom the name and three coordinates as XYZWriter writes them.
 * OutputXYZTrajectoryForce (output/OutputXYZTrajectoryForce.cpp:39-44) writes the integrator's
 * forces into such a file: pmb_md_write_force_frame. */
pmb_traj *pmb_traj_open_xyz_trajectory(const char *path, int n_atoms, const char *const *names);
/* Minimal-image output for a DCD trajectory (OutputDCDTrajectory with minimalImage,
 * output/OutputDCDTrajectory.cpp:67, through OutputCache::getMinimalPositions and
 * SemiGenericTopology::minimalImage, topology/SemiGenericTopology.h:127-150): every frame is
 * written after, per molecule, each bonded pair's second atom is moved by lattice vectors to the
 * image nearest its first atom (pairs in ascending (first, second) order, as the topology builder
 * sorts them), and the molecule by lattice vectors so that its centre of mass (masses [n_atoms],
 * Kahan sum) lies in the box around origin.  molecule [n_atoms] as in pmb_box_desc, pairs
 * [2 n_pairs] the bonds, box the orthogonal edges.  Host positions and device frames alike. */
int pmb_traj_set_minimal_image(pmb_traj *t, const double *mass, const int *molecule, int n_pairs,
                               const int *pairs, const double box[3], const double origin[3]);
/* A frame from host positions [3 n_atoms]; written before the call returns. */
int pmb_traj_write_host(pmb_traj *t, const double *positions);
/* A frame of the MD run's current positions, taken without stopping the device: a device
 * snapshot on the system's stream, its copy into one of three pinned host buffers on a stream of
 * the trajectory's own, and a writer thread that appends the frame once the copy has landed
 * (OutputDCDTrajectory::doRun without the synchronisation).  Waits only when all three buffers
 * are in flight; the first frame allocates the buffers.  Not during a stream capture. */
int pmb_md_write_frame(pmb_md *md, pmb_traj *t);
/* A frame of the MD run's forces (those of its last evaluation, as the integrator's getForces()
 * holds them after a step), taken like pmb_md_write_frame: the conversion to FP64 on the
 * system's stream, the host copy on the trajectory's stream. */
int pmb_md_write_force_frame(pmb_md *md, pmb_traj *t);
/* Waits until every frame handed over is in the file; the first write error, if any. */
int pmb_traj_flush(pmb_traj *t);
int pmb_traj_frames(pmb_traj *t, long long *frames);
/* Flushes, closes the file and frees the trajectory. */
int pmb_traj_close(pmb_traj *t);
/* Kernel launches in one captured MD step (0 before the first graph run); the list-rebuild
 * kernels are launched every step and return at once when no rebuild is due. */
int pmb_md_kernels_per_step(pmb_md *md, int *n);
/* Device memory held for this MD run: its system (atoms, neighbour lists, accumulators), its
 * forces (PME grids and tables) and the integrator state, in bytes (for admission by memory
 * budget; the lists are sized at the first evaluation, pmb_md_set_state). */
int pmb_md_device_bytes(const pmb_md *md, unsigned long long *bytes);

/* Diagnostics -------------------------------------------------------------------------------- */
/* Runs the force set nrep times with CUDA events between pipeline stages (TimerStatistic /
 * DEBUG_PME_TIMING of the reference, as device times); flush_l2 writes a 256 MB buffer before
 * each repetition.  positions [3 N] (host) are uploaded first; NULL reuses the positions of the
 * last evaluation (PMB_ERR_STATE if there was none).  stage_ms[i] is the mean time of stage i,
 * names receives the comma-separated stage names. */
int pmb_profile(pmb_system *sys, const double *positions, pmb_force *const *forces, int n_forces,
                int nrep, int flush_l2, double *stage_ms, int max_stages, int *n_stages,
                char *names, int names_len);
/* Measured FP32 FMA issue rate of the device (TFLOP/s), the roofline of the pair kernel. */
int pmb_fp32_peak(double *tflops);

/* Allocation-free cutoff evaluation (no counterpart in the reference) ------------------------ */
#define PMB_STATIC_MAX_BOXES 1024
/* pmb_evaluate_device for one NonbondedCutoff force, for callers that may not allocate device
 * memory: callers whose HBM is reserved up front (a serving loop that admits boxes against a
 * fixed memory budget, a host framework whose caching allocator owns the device) and callers
 * that cannot take the device-wide synchronisation of cudaFree.  pmb_evaluate_device allocates
 * the neighbour list on its first call and whenever a larger cutoff needs more room; this entry
 * point makes no cudaMalloc, cudaFree or other allocating call.  It visits all pairs of each box
 * in FP64 whatever the system's precision (no neighbour list; cost grows as the square of the
 * atoms per box), so its results equal pmb_evaluate_device's within FP64 rounding.
 * Scratch: one static device array of fixed-point energy/virial accumulators per device,
 * PMB_STATIC_MAX_BOXES boxes x PMB_E_STRIDE int64 (128 KiB); a system with more boxes gets
 * PMB_ERR_CAPACITY and nothing runs.  The call zeroes the scratch itself (cudaMemsetAsync on
 * the system's stream) before using it, so nothing has to start at zero.
 * d_positions [3 N], d_forces [3 N] (overwritten) and d_energies [n_boxes * PMB_E_STRIDE]
 * (overwritten; may be NULL) are device pointers; work is enqueued on the system's stream with
 * no host synchronisation.  The first call on a device (the current device), and the first in
 * a new context of that device (after cudaDeviceReset), looks the scratch up with
 * cudaGetSymbolAddress, which may load the module: make that first call before any stream
 * capture.  Calls whose executions overlap on one device (other streams, systems or host
 * threads) share the scratch and race on it: order them on one stream or synchronise between. */
int pmb_cutoff_evaluate_static(pmb_force *f, const double *d_positions, double *d_forces,
                               double *d_energies, int virial);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* PMB200_H */
