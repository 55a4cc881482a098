/*
 * CPU oracle for the nonbonded cutoff / PME force path: a plain-C, FP64 restatement of
 * ProtoMol 3's algorithms, used ONLY as the checker by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py.  The product path never links or calls this code.
 *
 * Parity of this restatement is pinned against the reference's own regression data
 * (tests/golden/*.npz, generated from test/tests/expected/water_CHARMM_PERIODIC_L.* and
 * protomol-test/ConfigTests/data/EnergiesTest.energies.orig) and against the reference's own
 * C++ code compiled from its sources into oracle/_ref (see oracle/Makefile).
 */
#ifndef PM_ORACLE_H
#define PM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Switching-function kinds (protomol/switch/*.h). */
enum { ORC_SWITCH_CUTOFF = 0, ORC_SWITCH_C1 = 1, ORC_SWITCH_C2 = 2 };

/* Energy slots, in the order of ScalarStructure::Index (type/ScalarStructure.h:26-54). */
enum { ORC_E_COULOMB = 0, ORC_E_LJ = 1, ORC_E_BOND = 2, ORC_E_ANGLE = 3, ORC_E_COUNT = 4 };

typedef struct {
  int n;                    /* atoms */
  int ntypes;               /* LJ atom types */
  const double *charge;     /* [n] scaled charge, e * 18.2226123264 */
  const double *mass;       /* [n] (integrator only) */
  const int *type;          /* [n] */
  const int *molecule;      /* [n] */
  const double *lj;         /* [ntypes*ntypes*4] {A, B, A14, B14} */
  int nexcl;
  const int *excl_pairs;    /* [2*nexcl] */
  const int *excl_kind;     /* [nexcl] 1 = MODIFIED, 2 = FULL */
  int nbonds;
  const int *bonds;         /* [2*nbonds] */
  const double *bond_k, *bond_r0;
  int nangles;
  const int *angles;        /* [3*nangles] */
  const double *angle_k, *angle_theta0, *ub_k, *ub_r0;
  double box[3];            /* orthogonal periodic box edges */
  double coulomb_scaling;   /* coulombScalingFactor for MODIFIED pairs */
} orc_system;

typedef struct {
  int do_lj, lj_switch;
  double lj_switchon, lj_cutoff;
  int do_coul, coul_switch;
  double coul_switchon, coul_cutoff;
} orc_cutoff_params;

typedef struct {
  int nx, ny, nz, order;
  double cutoff, accuracy, alpha;   /* alpha <= 0: bisection on erfc(alpha rc)/rc = accuracy */
  int real_switch;                  /* ORC_SWITCH_CUTOFF or ORC_SWITCH_C1 */
  int do_real, do_recip, do_corr;
} orc_pme_params;

/* Cell-list cutoff LJ and/or Coulomb, each with its own switching function.
 * forces += (AoS xyz), energies[ORC_E_*] +=, virial[9] += (row-major xx xy xz yx ...). */
int orc_cutoff(const orc_system *s, const double *pos, const orc_cutoff_params *p,
               double *forces, double *energies, double *virial);

/* Particle-mesh Ewald: real + reciprocal + correction/self/charged terms.
 * terms_out (optional, 5 doubles): real, reciprocal, intra-molecular, self, charged. */
int orc_pme(const orc_system *s, const double *pos, const orc_pme_params *p,
            double *forces, double *energies, double *virial, double *alpha_out,
            double *terms_out);

/* Harmonic bonds and angles (with Urey-Bradley). */
int orc_bonded(const orc_system *s, const double *pos, double *forces, double *energies,
               double *virial);

/* Ewald splitting parameter exactly as NonbondedPMEwaldSystemForce::initialize. */
double orc_pme_alpha(double cutoff, double accuracy);

/* Leapfrog run(nsteps) with bonded + cutoff (+ optional PME) forces.  pos/vel are updated in
 * place; forces_out receives the forces of the last evaluation; energies_out the energies of
 * the last evaluation.  pme may be NULL. */
int orc_leapfrog(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                 int do_bonded, double dt_fs, int nsteps, double *pos, double *vel,
                 double *forces_out, double *energies_out);

/* LangevinLeapfrogIntegrator run(nsteps) (integrator/base/LangevinLeapfrogIntegrator.cpp:44-71
 * through integrator/StandardIntegrator.cpp:27-37) with bonded + cutoff (+ optional PME) forces,
 * temperature in K and gamma in 1/ps as the reference's parameters.  The Gaussian numbers are the
 * device integrator's counter-based stream (orc_gauss3), first_step = steps already taken since
 * the state was set (half kick j uses stream j).  pos/vel updated in place; forces_out and
 * energies_out as orc_leapfrog. */
int orc_langevin(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                 int do_bonded, double dt_fs, double temperature, double gamma_ps,
                 unsigned long long seed, long long first_step, int nsteps, double *pos, double *vel,
                 double *forces_out, double *energies_out);
/* Three standard normals of the device's Langevin noise for (atom, stream). */
void orc_gauss3(unsigned long long seed, int atom, long long stream, double g[3]);

/* SHAKE / RATTLE bond constraints (modifier/ModifierShake.cpp, ModifierRattle.cpp): the
 * constraint list in the reference's order (topology/TopologyUtilities.cpp:695-775).  A sweep
 * applies every constraint in list order (Gauss-Seidel); sweeps repeat while the mean error over
 * all constraints exceeds epsilon, at most max_iter + 1 of them.  epsilon <= 0 or max_iter <= 0
 * switches a modifier off (ModifierModule.cpp:111, 124). */
typedef struct {
  int n;
  const int *a1, *a2;
  const double *len;
  double shake_eps;
  int shake_maxiter;
  double rattle_eps;
  int rattle_maxiter;
} orc_constraints;

/* One SHAKE application after a drift: moves pos and vel, then last_pos = pos.  Returns the
 * number of sweeps (ModifierShake::doExecute). */
int orc_shake(const orc_constraints *c, const double *mass, int n_atoms, double dt_fs, double *pos,
              double *vel, double *last_pos);
/* One RATTLE application (velocities only; ModifierRattle::doExecute).  Returns the sweeps. */
int orc_rattle(const orc_constraints *c, const double *mass, double dt_fs, const double *pos,
               double *vel);

/* LeapfrogIntegrator::run(nsteps) with SHAKE as a post-drift modifier and RATTLE as a post-step
 * modifier (LeapfrogIntegrator.cpp:56-87,89-102; ModifierModule.cpp:106-128).  last_pos holds
 * the SHAKE reference positions (the initial positions before the first run).  cp/pme may be
 * NULL; with no force terms the forces are zero.  rattle_virial (9 doubles, may be NULL): the
 * virial the last RATTLE application adds, what the reference's energies hold of the modifiers
 * after run(n) (the SHAKE terms are cleared by the next force evaluation). */
int orc_leapfrog_constrained(const orc_system *s, const orc_cutoff_params *cp,
                             const orc_pme_params *pme, int do_bonded, const orc_constraints *c,
                             double dt_fs, int nsteps, double *pos, double *vel, double *last_pos,
                             double *forces_out, double *energies_out, double *rattle_virial);

/* LangevinLeapfrogIntegrator::run with SHAKE (post-drift) and RATTLE (post-step), the half kicks
 * and noise as orc_langevin, the modifiers as orc_leapfrog_constrained. */
int orc_langevin_constrained(const orc_system *s, const orc_cutoff_params *cp, const orc_pme_params *pme,
                             int do_bonded, const orc_constraints *c, double dt_fs, double temperature,
                             double gamma_ps, unsigned long long seed, long long first_step, int nsteps,
                             double *pos, double *vel, double *last_pos, double *forces_out,
                             double *energies_out, double *rattle_virial);

#ifdef __cplusplus
}
#endif
#endif
