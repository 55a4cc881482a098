// Test-infrastructure harness: ProtoMol 3's own leapfrog and Langevin leapfrog integrators with
// its SHAKE and RATTLE modifiers, compiled from the reference sources by oracle/Makefile, run on a
// topology built in
// memory with no force terms (the forces are exactly zero), so that the constrained drift, the
// constraint list and every SHAKE/RATTLE sweep are the reference's own.  Tests compare the CPU
// restatement (orc_leapfrog_constrained in pm_oracle.c) and the CUDA path against it.
//
// What is run (all reference code):
//   LeapfrogIntegrator::run (integrator/leapfrog/LeapfrogIntegrator.cpp:89-102), or
//   LangevinLeapfrogIntegrator through StandardIntegrator::run (integrator/StandardIntegrator.cpp:
//   27-37) at temperature 0 (its noise term vanishes)
//   ModifierShake as a post-drift modifier, ModifierRattle as a post-step modifier, with the
//   placement ModifierModule::addModifiers gives them (module/ModifierModule.cpp:106-128)
//   buildRattleShakeBondConstraintList (topology/TopologyUtilities.cpp:695-775), reached through
//   ModifierMetaRattleShake::doInitialize
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/ProtoMolApp.h>
#include <protomol/force/ForceGroup.h>
#include <protomol/integrator/base/LangevinLeapfrogIntegrator.h>
#include <protomol/integrator/leapfrog/LeapfrogIntegrator.h>
#include <protomol/modifier/ModifierRattle.h>
#include <protomol/modifier/ModifierShake.h>
#include <protomol/module/MainModule.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/ScalarStructure.h>

#include <cstring>

using namespace ProtoMol;

typedef PeriodicBoundaryConditions PBC;
typedef Topology<PBC, CubicCellManager> Topo;

#include "ref_topology.h"

// The three input keywords the compiled integrator and output sources refer to; their home,
// module/MainModule.cpp, is not compiled here (same names and strings as there, lines 18, 20, 33).
namespace ProtoMol {
defineInputValue(InputFirststep, "firststep")
defineInputValue(InputNumsteps, "numsteps")
defineInputValue(InputOutputfreq, "outputfreq")
}

// elem[i]: first letter of atom i's name ('O', 'H', ...), which is all the constraint builder
// reads of a name.  On return: pos/vel after run(nsteps); cons[3k..3k+2] = atom1, atom2 and
// rest_len[k] of the first max_cons constraints of the reference's list; *n_cons its length.
// kind 0: LeapfrogIntegrator(dt); kind 1: LangevinLeapfrogIntegrator(dt, temperature, gamma_ps,
// seed), its half kicks and drift with the modifiers where StandardIntegrator::run places them.
static int run_constrained(const ref_input *in, const char *elem, int shake, double shake_eps,
                           int shake_maxiter, int rattle, double rattle_eps, int rattle_maxiter, int all,
                           int kind, double dt_fs, double temperature, double gamma_ps, int seed,
                           int nsteps, double *pos, double *vel, int *n_cons, int *cons, double *rest_len,
                           int max_cons, double *virial) {
  Topo *t = make_topo(in);
  for (int i = 0; i < in->n; i++) t->atoms[i].name = std::string(1, elem[i]);
  // what the topology builder sets besides: each atom's bond list and each molecule's atoms
  for (unsigned int k = 0; k < t->bonds.size(); k++) {
    t->atoms[t->bonds[k].atom1].mybonds.push_back((int)k);
    t->atoms[t->bonds[k].atom2].mybonds.push_back((int)k);
  }
  for (int i = 0; i < in->n; i++) {
    t->molecules[in->molecule[i]].atoms.push_back(i);
    t->molecules[in->molecule[i]].mass += t->atoms[i].scaledMass;
  }
  // the application object is left alive: its destructor lives in ProtoMolApp.cpp, which is not
  // compiled here
  ProtoMolApp *app = new ProtoMolApp();
  app->topology = t;
  app->positions.resize(in->n);
  app->velocities.resize(in->n);
  for (int i = 0; i < in->n; i++)
    for (int c = 0; c < 3; c++) {
      app->positions[i][c] = pos[3 * i + c];
      app->velocities[i][c] = vel[3 * i + c];
    }
  STSIntegrator *li;
  if (kind == 1)
    li = new LangevinLeapfrogIntegrator(dt_fs, temperature, gamma_ps, seed, new ForceGroup());
  else
    li = new LeapfrogIntegrator(dt_fs, new ForceGroup());
  app->energies.virial(virial != 0);
  app->energies.molecularVirial(false);
  li->initialize(app);
  if (shake) li->adoptPostDriftOrNextModifier(new ModifierShake(shake_eps, shake_maxiter, all != 0));
  if (rattle) li->adoptPostStepModifier(new ModifierRattle(rattle_eps, rattle_maxiter, all != 0));
  li->run(nsteps);
  // with no force terms what the energies hold after run(n) is the last RATTLE's virial (SHAKE's
  // terms are cleared by the force evaluation that follows each drift)
  if (virial)
    for (int k = 0; k < 9; k++) virial[k] = app->energies[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
  for (int i = 0; i < in->n; i++)
    for (int c = 0; c < 3; c++) {
      pos[3 * i + c] = app->positions[i][c];
      vel[3 * i + c] = app->velocities[i][c];
    }
  const std::vector<Bond::Constraint> &cl = t->bondRattleShakeConstraints;
  *n_cons = (int)cl.size();
  for (int k = 0; k < (int)cl.size() && k < max_cons; k++) {
    cons[3 * k] = cl[k].atom1;
    cons[3 * k + 1] = cl[k].atom2;
    cons[3 * k + 2] = 0;
    rest_len[k] = cl[k].restLength;
  }
  return 0;
}

extern "C" int ref_leapfrog_constrained(const ref_input *in, const char *elem, int shake,
                                        double shake_eps, int shake_maxiter, int rattle,
                                        double rattle_eps, int rattle_maxiter, int all,
                                        double dt_fs, int nsteps, double *pos, double *vel,
                                        int *n_cons, int *cons, double *rest_len, int max_cons,
                                        double *virial) {
  return run_constrained(in, elem, shake, shake_eps, shake_maxiter, rattle, rattle_eps, rattle_maxiter, all, 0,
                         dt_fs, 0.0, 0.0, 0, nsteps, pos, vel, n_cons, cons, rest_len, max_cons, virial);
}

// The same with the LangevinLeapfrogIntegrator (temperature 0 makes its noise term vanish).
extern "C" int ref_langevin_constrained(const ref_input *in, const char *elem, int shake,
                                        double shake_eps, int shake_maxiter, int rattle,
                                        double rattle_eps, int rattle_maxiter, int all, double dt_fs,
                                        double temperature, double gamma_ps, int seed, int nsteps,
                                        double *pos, double *vel, int *n_cons, int *cons,
                                        double *rest_len, int max_cons, double *virial) {
  return run_constrained(in, elem, shake, shake_eps, shake_maxiter, rattle, rattle_eps, rattle_maxiter, all, 1,
                         dt_fs, temperature, gamma_ps, seed, nsteps, pos, vel, n_cons, cons, rest_len,
                         max_cons, virial);
}
