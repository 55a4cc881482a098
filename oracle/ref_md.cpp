// Test-infrastructure harness: ProtoMol 3's own integrators with force terms, compiled from the
// reference sources by oracle/Makefile, stepped one step per call of run(1) as ProtoMolApp does
// with outputfreq 1, recording what every step ends with: the energies of the force evaluation at
// the step's new positions, the forces, and optionally positions and velocities.
//
// What is run (all reference code):
//   LeapfrogIntegrator::run (integrator/leapfrog/LeapfrogIntegrator.cpp:89-102), or
//   LangevinLeapfrogIntegrator through StandardIntegrator::run (integrator/StandardIntegrator.cpp:
//   27-37) with its doHalfKick / doDrift (integrator/base/LangevinLeapfrogIntegrator.cpp:36-71);
//   a ForceGroup (force/ForceGroup.cpp:54-75) holding BondSystemForce, AngleSystemForce, the
//   NonbondedCutoffSystemForce and the NonbondedPMEwaldSystemForce of ref_harness.cpp.
// With temperature 0 the Langevin noise term is exactly zero (its scale is sqrt(2 kB T gamma / m)),
// so the run is deterministic and independent of the reference's serial random generator.
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/ProtoMolApp.h>
#include <protomol/force/ForceGroup.h>
#include <protomol/topology/SemiGenericTopology.h>
#include <protomol/force/bonded/AngleSystemForce.h>
#include <protomol/force/bonded/BondSystemForce.h>
#include <protomol/io/DCDTrajectoryWriter.h>
#include <protomol/integrator/base/LangevinLeapfrogIntegrator.h>
#include <protomol/integrator/leapfrog/LeapfrogIntegrator.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/ScalarStructure.h>

using namespace ProtoMol;

typedef PeriodicBoundaryConditions PBC;
typedef Topology<PBC, CubicCellManager> Topo;

#include "ref_topology.h"

#include <algorithm>

SystemForce *ref_new_cutoff_force(const ref_cutoff *c);
SystemForce *ref_new_pme_force(const ref_pme *p);

static void read_out(ProtoMolApp *app, Integrator *it, int n, int k, double *energies,
                     double *pos, double *vel, double *forces) {
  const ScalarStructure &e = app->energies;
  energies[4 * k + 0] = e[ScalarStructure::COULOMB];
  energies[4 * k + 1] = e[ScalarStructure::LENNARDJONES];
  energies[4 * k + 2] = e[ScalarStructure::BOND];
  energies[4 * k + 3] = e[ScalarStructure::ANGLE];
  const Vector3DBlock *f = it->getForces();
  for (int i = 0; i < n; i++)
    for (int c = 0; c < 3; c++) {
      size_t o = 3 * ((size_t)k * n + i) + c;
      if (pos) pos[o] = app->positions[i][c];
      if (vel) vel[o] = app->velocities[i][c];
      if (forces) forces[o] = (*f)[i][c];
    }
}

// kind 0: LeapfrogIntegrator(dt); kind 1: LangevinLeapfrogIntegrator(dt, temperature, gamma_ps,
// seed).  c / p may be NULL; bonded adds the bond and angle forces.  Row k of every output
// (k = 0 .. nsteps) holds the state after k calls of run(1) (row 0: after initialize, which
// evaluates the initial forces).  energies [nsteps+1][4] (Coulomb, LJ, bond, angle); pos, vel,
// forces [nsteps+1][n][3] or NULL.  The initial positions and velocities are in->pos and vel0.
extern "C" int ref_md_run(const ref_input *in, const ref_cutoff *c, const ref_pme *p, int bonded,
                          int kind, double dt_fs, double temperature, double gamma_ps, int seed,
                          const double *vel0, int nsteps, double *energies, double *pos,
                          double *vel, double *forces) {
  Topo *t = make_topo(in);
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
    for (int q = 0; q < 3; q++) {
      app->positions[i][q] = in->pos[3 * i + q];
      app->velocities[i][q] = vel0[3 * i + q];
    }
  app->energies.clear();
  app->energies.molecularVirial(false);
  app->energies.virial(false);
  ForceGroup *fg = new ForceGroup();
  if (bonded) {
    fg->addSystemForce(new BondSystemForce<PBC>());
    fg->addSystemForce(new AngleSystemForce<PBC>());
  }
  if (c) {
    SystemForce *f = ref_new_cutoff_force(c);
    if (f) fg->addSystemForce(f);
  }
  if (p) fg->addSystemForce(ref_new_pme_force(p));
  STSIntegrator *it;
  if (kind == 1)
    it = new LangevinLeapfrogIntegrator(dt_fs, temperature, gamma_ps, seed, fg);
  else
    it = new LeapfrogIntegrator(dt_fs, fg);
  it->initialize(app);
  read_out(app, it, in->n, 0, energies, pos, vel, forces);
  for (int k = 1; k <= nsteps; k++) {
    it->run(1);
    read_out(app, it, in->n, k, energies, pos, vel, forces);
  }
  delete it;  // deletes its force group
  return 0;
}

// DCD frames in minimal image as OutputDCDTrajectory with minimalImage writes them
// (output/OutputDCDTrajectory.cpp:64-70 through OutputCache::getMinimalPositions,
// output/OutputCache.cpp:226-235): SemiGenericTopology::minimalImage on a copy of each frame.
// The topology's molecules are the atoms of each molecule index with the given bonded pairs,
// (first, second) with first < second, in ascending order as the topology builder leaves them
// (topology/BuildTopology.cpp:1034-1050); the box origin is in->origin.
extern "C" int ref_write_dcd_minimal(const ref_input *in, int n_pairs, const int *pairs, int n_frames,
                                     const double *frames, const char *path) {
  Topo *t = make_topo(in);
  for (int i = 0; i < in->n; i++) {
    t->molecules[in->molecule[i]].atoms.push_back(i);
    t->molecules[in->molecule[i]].mass += t->atoms[i].scaledMass;
  }
  for (int k = 0; k < n_pairs; k++) {
    int a = pairs[2 * k], b = pairs[2 * k + 1];
    if (a > b) std::swap(a, b);
    t->molecules[in->molecule[a]].pairs.push_back(PairInt(a, b));
  }
  for (unsigned int m = 0; m < t->molecules.size(); m++)
    std::sort(t->molecules[m].pairs.begin(), t->molecules[m].pairs.end());
  DCDTrajectoryWriter w(std::string(path), 1.0, 0u);
  if (!w.open()) return 1;
  Vector3DBlock v(in->n);
  for (int f = 0; f < n_frames; f++) {
    for (int i = 0; i < in->n; i++)
      for (int c = 0; c < 3; c++) v[i][c] = frames[3 * ((size_t)f * in->n + i) + c];
    t->minimalImage(v);
    if (!w.write(v)) return 2;
  }
  w.close();
  delete t;
  return 0;
}
