// Test-infrastructure harness: runs ProtoMol 3's own force classes, compiled from the reference
// sources by oracle/Makefile, on a topology built in memory, and returns forces, energies and
// virial through a C ABI so tests can compare the CPU restatement (oracle/pm_oracle.c) and the
// CUDA path against the reference itself.
//
// The forces instantiated here are exactly the ones the reference registers:
//   NonbondedCutoffSystemForce<CubicCellManager, OneAtomPairTwo<PBC, Switch, LennardJonesForce,
//       Switch, CoulombForce>>          (module/NonbondedCutoffForceModule.cpp:58-88)
//   NonbondedCutoffSystemForce<CubicCellManager, OneAtomPair<PBC, Switch, LennardJonesForce>>
//   NonbondedPMEwaldSystemForce<PBC, CubicCellManager, true, true, true, BSpline, Cutoff|C1>
//       (mdl/interface/force/nonbonded/PMEForce.i:82-115)
//   BondSystemForce<PBC>, AngleSystemForce<PBC> (module/BondedForcesModule.cpp:30-31)
#include <protomol/base/Report.h>
using namespace ProtoMol::Report;

#include <protomol/force/CoulombForce.h>
#include <protomol/force/LennardJonesForce.h>
#include <protomol/force/OneAtomPair.h>
#include <protomol/force/OneAtomPairTwo.h>
#include <protomol/force/bonded/AngleSystemForce.h>
#include <protomol/force/bonded/BondSystemForce.h>
#include <protomol/force/nonbonded/NonbondedCutoffSystemForce.h>
#include <protomol/switch/C1SwitchingFunction.h>
#include <protomol/switch/C2SwitchingFunction.h>
#include <protomol/switch/CutoffSwitchingFunction.h>
#include <protomol/topology/CellListEnumeratorPeriodicBoundaries.h>
#include <protomol/topology/CubicCellManager.h>
#include <protomol/topology/PeriodicBoundaryConditions.h>
#include <protomol/topology/Topology.h>
#include <protomol/type/ScalarStructure.h>
#include <protomol/type/Vector3DBlock.h>

#include "BSpline.h"
#include "NonbondedPMEwaldSystemForce.h"

#include <cstring>

using namespace ProtoMol;

typedef PeriodicBoundaryConditions PBC;
typedef Topology<PBC, CubicCellManager> Topo;

#include "ref_topology.h"

static void run_force(SystemForce *f, Topo *t, const ref_input *in, double *forces,
                      double *energies, double *virial) {
  Vector3DBlock pos(in->n), frc(in->n);
  for (int i = 0; i < in->n; i++) {
    pos[i] = Vector3D(in->pos[3 * i], in->pos[3 * i + 1], in->pos[3 * i + 2]);
    frc[i] = Vector3D(0, 0, 0);
  }
  ScalarStructure e;
  e.clear();
  e.molecularVirial(false);
  e.virial(virial != 0);
  t->uncacheCellList();
  f->evaluate(t, &pos, &frc, &e);
  for (int i = 0; i < in->n; i++)
    for (int k = 0; k < 3; k++) forces[3 * i + k] += frc[i].c[k];
  energies[0] += e[ScalarStructure::COULOMB];
  energies[1] += e[ScalarStructure::LENNARDJONES];
  energies[2] += e[ScalarStructure::BOND];
  energies[3] += e[ScalarStructure::ANGLE];
  if (virial)
    for (int k = 0; k < 9; k++) virial[k] += e[(ScalarStructure::Index)(ScalarStructure::VIRIALXX + k)];
}

template <class SA, class SB>
static SystemForce *make_two(const ref_cutoff *c, SA sa, SB sb) {
  typedef OneAtomPairTwo<PBC, SA, LennardJonesForce, SB, CoulombForce> OAP;
  double rc = c->lj_cutoff > c->coul_cutoff ? c->lj_cutoff : c->coul_cutoff;
  return new NonbondedCutoffSystemForce<CubicCellManager, OAP>(
      rc, OAP(LennardJonesForce(), sa, CoulombForce(), sb));
}

template <class S, class F>
static SystemForce *make_one(double rc, S s) {
  typedef OneAtomPair<PBC, S, F> OAP;
  return new NonbondedCutoffSystemForce<CubicCellManager, OAP>(rc, OAP(F(), s));
}

template <class S>
static SystemForce *with_coul(const ref_cutoff *c, S sa) {
  switch (c->coul_switch) {
    case 1: return make_two(c, sa, C1SwitchingFunction(c->coul_cutoff));
    case 2: return make_two(c, sa, C2SwitchingFunction(c->coul_switchon, c->coul_cutoff));
    default: return make_two(c, sa, CutoffSwitchingFunction(c->coul_cutoff));
  }
}

// The reference's cutoff force for c (NULL when c selects no potential); also used by the MD
// harness (ref_md.cpp), which puts it in a ForceGroup.
SystemForce *ref_new_cutoff_force(const ref_cutoff *c) {
  SystemForce *f = 0;
  if (c->do_lj && c->do_coul) {
    switch (c->lj_switch) {
      case 1: f = with_coul(c, C1SwitchingFunction(c->lj_cutoff)); break;
      case 2: f = with_coul(c, C2SwitchingFunction(c->lj_switchon, c->lj_cutoff)); break;
      default: f = with_coul(c, CutoffSwitchingFunction(c->lj_cutoff)); break;
    }
  } else if (c->do_lj) {
    if (c->lj_switch == 2)
      f = make_one<C2SwitchingFunction, LennardJonesForce>(
          c->lj_cutoff, C2SwitchingFunction(c->lj_switchon, c->lj_cutoff));
    else if (c->lj_switch == 1)
      f = make_one<C1SwitchingFunction, LennardJonesForce>(c->lj_cutoff, C1SwitchingFunction(c->lj_cutoff));
    else
      f = make_one<CutoffSwitchingFunction, LennardJonesForce>(c->lj_cutoff, CutoffSwitchingFunction(c->lj_cutoff));
  } else if (c->do_coul) {
    if (c->coul_switch == 2)
      f = make_one<C2SwitchingFunction, CoulombForce>(
          c->coul_cutoff, C2SwitchingFunction(c->coul_switchon, c->coul_cutoff));
    else if (c->coul_switch == 1)
      f = make_one<C1SwitchingFunction, CoulombForce>(c->coul_cutoff, C1SwitchingFunction(c->coul_cutoff));
    else
      f = make_one<CutoffSwitchingFunction, CoulombForce>(c->coul_cutoff, CutoffSwitchingFunction(c->coul_cutoff));
  }
  return f;
}

extern "C" int ref_cutoff_eval(const ref_input *in, const ref_cutoff *c, double *forces,
                               double *energies, double *virial) {
  Topo *t = make_topo(in);
  SystemForce *f = ref_new_cutoff_force(c);
  if (f) run_force(f, t, in, forces, energies, virial);
  delete f;
  delete t;
  return 0;
}

// The reference's PME force for p (with the real, reciprocal and correction terms).
SystemForce *ref_new_pme_force(const ref_pme *p) {
  SystemForce *f;
  if (p->real_switch == 1)
    f = new NonbondedPMEwaldSystemForce<PBC, CubicCellManager, true, true, true, BSpline,
                                        C1SwitchingFunction>(p->nx, p->ny, p->nz, p->order,
                                                             p->cutoff, p->accuracy, p->alpha, 3.0);
  else
    f = new NonbondedPMEwaldSystemForce<PBC, CubicCellManager, true, true, true, BSpline,
                                        CutoffSwitchingFunction>(p->nx, p->ny, p->nz, p->order,
                                                                 p->cutoff, p->accuracy, p->alpha, 3.0);
  return f;
}

extern "C" int ref_pme_eval(const ref_input *in, const ref_pme *p, double *forces,
                            double *energies, double *virial) {
  Topo *t = make_topo(in);
  SystemForce *f = ref_new_pme_force(p);
  run_force(f, t, in, forces, energies, virial);
  delete f;
  delete t;
  return 0;
}

extern "C" int ref_bonded_eval(const ref_input *in, double *forces, double *energies,
                               double *virial) {
  Topo *t = make_topo(in);
  BondSystemForce<PBC> b;
  AngleSystemForce<PBC> a;
  run_force(&b, t, in, forces, energies, virial);
  run_force(&a, t, in, forces, energies, virial);
  delete t;
  return 0;
}

// Repeated evaluation of one force on the same topology, for CPU timing (the force object and
// topology are built once, as in a ProtoMol run; each call evaluates nrep times).
extern "C" int ref_time_step(const ref_input *in, const ref_cutoff *c, const ref_pme *p,
                             int nrep, double *forces, double *energies) {
  Topo *t = make_topo(in);
  SystemForce *lj = 0, *pme = 0;
  if (c) lj = make_one<C2SwitchingFunction, LennardJonesForce>(
                 c->lj_cutoff, C2SwitchingFunction(c->lj_switchon, c->lj_cutoff));
  if (p)
    pme = new NonbondedPMEwaldSystemForce<PBC, CubicCellManager, true, true, true, BSpline,
                                          CutoffSwitchingFunction>(p->nx, p->ny, p->nz, p->order,
                                                                   p->cutoff, p->accuracy, p->alpha, 3.0);
  for (int r = 0; r < nrep; r++) {
    for (int i = 0; i < 3 * in->n; i++) forces[i] = 0.0;
    for (int k = 0; k < 4; k++) energies[k] = 0.0;
    if (lj) run_force(lj, t, in, forces, energies, 0);
    if (pme) run_force(pme, t, in, forces, energies, 0);
  }
  delete lj;
  delete pme;
  delete t;
  return 0;
}
